// Selected-region estimates shared by the batch planner and the expansion
// loop: vertices of a tile set and edges whose endpoints both lie in it, the
// quantities of the reference's SelectedRegionIndex
// (src/selected_region_index.cpp:112-141), from per-tile destination-tile
// edge counts built once from the CSR runs.
#pragma once

#include "bfx.h"

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

inline RegionIndex make_region_index(const bfx_device_graph_layout32& g) {
  RegionIndex r;
  r.T = g.tile_count;
  r.vertex_counts.assign(r.T, 0U);
  for (std::uint32_t v = 0; v < g.vertex_count; ++v) ++r.vertex_counts[g.owner_tiles[v]];
  std::vector<std::vector<std::pair<std::uint32_t, std::uint64_t>>> per(r.T);
  for (std::uint32_t v = 0; v < g.vertex_count; ++v) {
    const std::uint32_t st = g.owner_tiles[v];
    for (std::uint32_t run = g.csr_row_run_offsets[v]; run < g.csr_row_run_offsets[v + 1]; ++run) {
      per[st].emplace_back(g.csr_run_destination_tiles[run],
                           g.csr_run_edge_offsets[run + 1] - g.csr_run_edge_offsets[run]);
    }
  }
  r.adj_offsets.assign(r.T + 1, 0U);
  for (std::uint32_t t = 0; t < r.T; ++t) {
    auto& lst = per[t];
    std::sort(lst.begin(), lst.end());
    std::vector<std::pair<std::uint32_t, std::uint64_t>> merged;
    for (const auto& p : lst) {
      if (!merged.empty() && merged.back().first == p.first) {
        merged.back().second += p.second;
      } else {
        merged.push_back(p);
      }
    }
    r.adj_offsets[t + 1] = r.adj_offsets[t] + static_cast<std::uint32_t>(merged.size());
    for (const auto& p : merged) {
      r.adj_tiles.push_back(p.first);
      r.adj_edges.push_back(p.second);
    }
  }
  return r;
}

}  // namespace bfx
