// Selected-region estimates shared by the batch planner and the expansion
// loop: vertices of a tile set and edges whose endpoints both lie in it, the
// quantities of the reference's SelectedRegionIndex
// (src/selected_region_index.cpp:112-141), from per-tile destination-tile
// edge counts built once from the CSR runs.
#pragma once

#include "bfx.h"
#include "bfx_host.h"
#include "bfx_internal.hpp"

#include <algorithm>
#include <cstdint>
#include <utility>
#include <vector>

namespace bfx {

struct RegionIndex {
  std::uint32_t T{};
  std::vector<std::uint64_t> vertex_counts;
  std::vector<std::uint32_t> adj_offsets;
  std::vector<std::uint32_t> adj_tiles;
  std::vector<std::uint64_t> adj_edges;

  std::uint64_t vertices(const std::vector<std::uint32_t>& tiles) const {
    std::uint64_t n = 0;
    for (std::uint32_t t : tiles) n += vertex_counts[t];
    return n;
  }
  // Edges whose endpoints both lie in the tile set marked in `member`.
  std::uint64_t edges(const std::vector<std::uint32_t>& tiles, const std::vector<std::uint8_t>& member) const {
    std::uint64_t n = 0;
    for (std::uint32_t t : tiles) {
      for (std::uint32_t k = adj_offsets[t]; k < adj_offsets[t + 1]; ++k) {
        if (member[adj_tiles[k]]) n += adj_edges[k];
      }
    }
    return n;
  }
};

// Built per source tile in parallel: a tile's vertices are one contiguous
// span (the layout orders vertices by tile), and their CSR runs name the
// destination tiles.  A tile's runs reach few distinct tiles (its own and
// its neighbours), so their edge counts are accumulated by a linear search
// of the short list of tiles seen so far and the list is sorted once; a
// tile that reaches more than kLinear tiles falls back to sorting all its
// (destination tile, edge count) pairs.
inline RegionIndex make_region_index(const bfx_device_graph_layout32& g) {
  RegionIndex r;
  r.T = g.tile_count;
  r.vertex_counts.assign(r.T, 0U);
  for (std::uint32_t v = 0; v < g.vertex_count; ++v) ++r.vertex_counts[g.owner_tiles[v]];
  std::vector<std::uint32_t> first(r.T + 1, 0U);
  for (std::uint32_t t = 0; t < r.T; ++t) first[t + 1] = first[t] + static_cast<std::uint32_t>(r.vertex_counts[t]);
  std::vector<std::vector<std::pair<std::uint32_t, std::uint64_t>>> per(r.T);
  constexpr std::size_t kLinear = 64;
  parallel_for(r.T, 0, [&](std::uint64_t tb, std::uint64_t te) {
    std::vector<std::pair<std::uint32_t, std::uint64_t>> lst;
    for (std::uint64_t t = tb; t < te; ++t) {
      auto& merged = per[t];
      bool wide = false;
      std::size_t hint = 0;
      for (std::uint32_t v = first[t]; v < first[t + 1] && !wide; ++v) {
        for (std::uint32_t run = g.csr_row_run_offsets[v]; run < g.csr_row_run_offsets[v + 1]; ++run) {
          const std::uint32_t dt = g.csr_run_destination_tiles[run];
          const std::uint64_t n = g.csr_run_edge_offsets[run + 1] - g.csr_run_edge_offsets[run];
          if (hint < merged.size() && merged[hint].first == dt) {
            merged[hint].second += n;
            continue;
          }
          std::size_t i = 0;
          while (i < merged.size() && merged[i].first != dt) ++i;
          if (i == merged.size()) {
            if (merged.size() == kLinear) {
              wide = true;
              break;
            }
            merged.emplace_back(dt, 0U);
          }
          merged[i].second += n;
          hint = i;
        }
      }
      if (!wide) {
        std::sort(merged.begin(), merged.end());
        continue;
      }
      // many destination tiles: all pairs of the tile, sorted and merged
      merged.clear();
      lst.clear();
      for (std::uint32_t v = first[t]; v < first[t + 1]; ++v) {
        for (std::uint32_t run = g.csr_row_run_offsets[v]; run < g.csr_row_run_offsets[v + 1]; ++run) {
          lst.emplace_back(g.csr_run_destination_tiles[run],
                           g.csr_run_edge_offsets[run + 1] - g.csr_run_edge_offsets[run]);
        }
      }
      std::sort(lst.begin(), lst.end());
      for (const auto& q : lst) {
        if (!merged.empty() && merged.back().first == q.first) {
          merged.back().second += q.second;
        } else {
          merged.push_back(q);
        }
      }
    }
  });
  r.adj_offsets.assign(r.T + 1, 0U);
  for (std::uint32_t t = 0; t < r.T; ++t) {
    r.adj_offsets[t + 1] = r.adj_offsets[t] + static_cast<std::uint32_t>(per[t].size());
  }
  r.adj_tiles.resize(r.adj_offsets[r.T]);
  r.adj_edges.resize(r.adj_offsets[r.T]);
  for (std::uint32_t t = 0; t < r.T; ++t) {
    std::uint32_t k = r.adj_offsets[t];
    for (const auto& q : per[t]) {
      r.adj_tiles[k] = q.first;
      r.adj_edges[k] = q.second;
      ++k;
    }
  }
  return r;
}

// bfx_plan_build with a region index the caller already holds for the same
// graph (the expansion loop plans every pass against one index).  Throws on
// invalid input like bfx_plan_build reports it.
bfx_plan* plan_build_with_region(const bfx_device_graph_layout32& g, const std::uint32_t* tile_vertex_offsets,
                                 std::uint32_t query_count, const bfx_route_query* queries,
                                 const bfx_planner_policy& policy, const RegionIndex& region);

}  // namespace bfx
