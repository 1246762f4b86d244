// Host builder for the spatially ordered graph and its checked 32-bit device
// image (the input side of the batched relaxation path).
//
// The result is defined by the reference and must be identical to it array
// for array, because stable edge ids decide predecessor ties:
//   * canonical logical edge ids: edges sorted by (source, destination,
//     canonical weight bits, provenance domain, kind, record); the id is the
//     sorted position (src/graph_builder.cpp:49-58, 197-214).  InputGraph
//     canonicalises -0.0 weights to +0.0 on construction (graph_builder.cpp:169).
//   * vertex order: located vertices by (tile_y, tile_x, resource class,
//     Morton(local x, local y), original id), then unlocated vertices by
//     (resource class, original id) in one trailing spill tile
//     (src/reorder.cpp:151-245).  Tiles are dense ids in (tile_y, tile_x)
//     order; tile = floor((coord - origin) / tile_size) (reorder.cpp:75-98).
//   * CSR rows sorted by (owner tile of destination, destination, edge id);
//     CSC columns by (owner tile of source, source, edge id)
//     (reorder.cpp:282-351).
//   * maximal per-row destination-tile runs and per-column source-tile runs
//     (src/device_layout.cpp:186-251).
//
// The construction here is our own: bucketing by source / tile / column with
// small per-bucket sorts (O(E) plus tiny sorts) instead of the reference's
// global comparison sorts, a dense tile grid when the located tiles fill their
// bounding box, and host threads over rows.  That keeps the 168M-edge graph
// build to seconds.
#include "bfx_host.h"
#include "bfx_internal.hpp"

#include <algorithm>
#include <bit>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <numeric>
#include <tuple>
#include <vector>

namespace bfx {

struct HostLayout {
  std::uint32_t V{}, E{}, T{};
  std::vector<std::uint32_t> owner_tiles;
  std::vector<std::uint32_t> csr_row_offsets, csr_destinations, csr_edge_ids;
  std::vector<float> csr_weights;
  std::vector<std::uint32_t> csr_row_run_offsets, csr_run_edge_offsets, csr_run_destination_tiles;
  std::vector<std::uint32_t> csc_column_offsets, csc_sources, csc_edge_ids;
  std::vector<float> csc_weights;
  std::vector<std::uint32_t> csc_column_run_offsets, csc_run_edge_offsets, csc_run_source_tiles;
  std::vector<std::int64_t> tile_xy;
  std::vector<std::uint8_t> tile_has_location;
  std::vector<std::uint32_t> tile_vertex_offsets;
  std::vector<std::uint32_t> new_to_old;
};

namespace {

std::uint32_t weight_bits(float w) {
  const float c = (w == 0.0F) ? 0.0F : w;
  return std::bit_cast<std::uint32_t>(c);
}

std::uint64_t spread_bits(std::uint32_t v) {
  std::uint64_t x = v;
  x = (x | (x << 16U)) & 0x0000FFFF0000FFFFULL;
  x = (x | (x << 8U)) & 0x00FF00FF00FF00FFULL;
  x = (x | (x << 4U)) & 0x0F0F0F0F0F0F0F0FULL;
  x = (x | (x << 2U)) & 0x3333333333333333ULL;
  x = (x | (x << 1U)) & 0x5555555555555555ULL;
  return x;
}

std::int64_t floor_div(std::int64_t n, std::uint32_t d) {
  const std::int64_t dd = static_cast<std::int64_t>(d);
  std::int64_t q = n / dd;
  if (n % dd < 0) --q;
  return q;
}

std::uint32_t checked32(std::uint64_t v, const char* what) {
  if (v > std::numeric_limits<std::uint32_t>::max()) throw std::overflow_error(what);
  return static_cast<std::uint32_t>(v);
}

// Exclusive prefix sum of counts[0..n) into offsets[0..n] (64-bit checked).
void prefix(const std::vector<std::uint32_t>& counts, std::vector<std::uint32_t>& offsets,
            const char* what) {
  offsets.assign(counts.size() + 1, 0U);
  std::uint64_t acc = 0;
  for (std::size_t i = 0; i < counts.size(); ++i) {
    offsets[i] = static_cast<std::uint32_t>(acc);
    acc += counts[i];
    if (acc > std::numeric_limits<std::uint32_t>::max()) throw std::overflow_error(what);
  }
  offsets[counts.size()] = static_cast<std::uint32_t>(acc);
}

// Runs of equal tile over each bucket of `keys` (offsets per bucket).
void build_runs(std::uint32_t V, const std::vector<std::uint32_t>& bucket_offsets,
                const std::vector<std::uint32_t>& endpoint, const std::vector<std::uint32_t>& owner,
                unsigned threads, std::vector<std::uint32_t>& bucket_run_offsets,
                std::vector<std::uint32_t>& run_edge_offsets, std::vector<std::uint32_t>& run_tiles) {
  std::vector<std::uint32_t> runs_per(V, 0U);
  parallel_for(V, threads, [&](std::uint64_t b, std::uint64_t e) {
    for (std::uint64_t v = b; v < e; ++v) {
      std::uint32_t n = 0, prev = 0;
      for (std::uint32_t p = bucket_offsets[v]; p < bucket_offsets[v + 1]; ++p) {
        const std::uint32_t t = owner[endpoint[p]];
        if (p == bucket_offsets[v] || t != prev) ++n;
        prev = t;
      }
      runs_per[v] = n;
    }
  });
  prefix(runs_per, bucket_run_offsets, "run count exceeds 32 bits");
  const std::uint32_t R = bucket_run_offsets[V];
  run_edge_offsets.assign(static_cast<std::size_t>(R) + 1U, 0U);
  run_tiles.assign(R, 0U);
  parallel_for(V, threads, [&](std::uint64_t b, std::uint64_t e) {
    for (std::uint64_t v = b; v < e; ++v) {
      std::uint32_t r = bucket_run_offsets[v];
      const std::uint32_t beg = bucket_offsets[v], end = bucket_offsets[v + 1];
      std::uint32_t p = beg;
      while (p < end) {
        const std::uint32_t t = owner[endpoint[p]];
        ++p;
        while (p < end && owner[endpoint[p]] == t) ++p;
        run_tiles[r] = t;
        run_edge_offsets[r + 1] = p;
        ++r;
      }
    }
  });
}

std::unique_ptr<HostLayout> build_layout(const bfx_input_graph& in, const bfx_spatial_order_config& cfg,
                                         unsigned threads) {
  require(cfg.tile_width > 0 && cfg.tile_height > 0, "tile width and height must both be positive");
  require(in.vertex_count == 0 || (in.x && in.y && in.has_location && in.resource_class),
          "vertex arrays must be non-null");
  require(in.edge_count == 0 || (in.edge_source && in.edge_destination && in.edge_weight &&
                                 in.provenance_domain && in.provenance_kind && in.provenance_record),
          "edge arrays must be non-null");
  const std::uint32_t V = in.vertex_count;
  const std::uint64_t E64 = in.edge_count;
  const std::uint32_t E = checked32(E64, "graph counts do not fit the 32-bit device layout");

  // Input validation in the order of validate_graph_input (graph_builder.cpp:108-136).
  for (std::uint64_t e = 0; e < E64; ++e) {
    const float w = in.edge_weight[e];
    if (!std::isfinite(w)) throw std::invalid_argument("edge weight must be finite");
    if (w < 0.0F) throw std::invalid_argument("edge weight must be nonnegative");
    if (in.edge_source[e] >= V) throw std::out_of_range("edge source is outside the vertex range");
    if (in.edge_destination[e] >= V) throw std::out_of_range("edge destination is outside the vertex range");
  }

  auto L = std::make_unique<HostLayout>();
  L->V = V;
  L->E = E;

  // ---- canonical edge ids: bucket by original source, sort each row by the
  // remaining key.  can_* arrays are indexed by edge id.
  std::vector<std::uint32_t> old_row_offsets;
  {
    std::vector<std::uint32_t> deg(V, 0U);
    for (std::uint64_t e = 0; e < E64; ++e) ++deg[in.edge_source[e]];
    prefix(deg, old_row_offsets, "edge count exceeds 32 bits");
  }
  std::vector<std::uint32_t> perm(E);
  {
    std::vector<std::uint32_t> cursor(old_row_offsets.begin(), old_row_offsets.end() - 1);
    for (std::uint32_t e = 0; e < E; ++e) perm[cursor[in.edge_source[e]]++] = e;
  }
  parallel_for(V, threads, [&](std::uint64_t b, std::uint64_t end) {
    for (std::uint64_t s = b; s < end; ++s) {
      auto first = perm.begin() + old_row_offsets[s];
      auto last = perm.begin() + old_row_offsets[s + 1];
      if (last - first < 2) continue;
      std::sort(first, last, [&](std::uint32_t a, std::uint32_t c) {
        return std::tuple(in.edge_destination[a], weight_bits(in.edge_weight[a]), in.provenance_domain[a],
                          in.provenance_kind[a], in.provenance_record[a]) <
               std::tuple(in.edge_destination[c], weight_bits(in.edge_weight[c]), in.provenance_domain[c],
                          in.provenance_kind[c], in.provenance_record[c]);
      });
    }
  });
  std::vector<std::uint32_t> can_dst(E);
  std::vector<float> can_w(E);
  parallel_for(E, threads, [&](std::uint64_t b, std::uint64_t end) {
    for (std::uint64_t k = b; k < end; ++k) {
      const std::uint32_t e = perm[k];
      can_dst[k] = in.edge_destination[e];
      can_w[k] = std::bit_cast<float>(weight_bits(in.edge_weight[e]));
    }
  });
  perm.clear();
  perm.shrink_to_fit();

  // ---- tiles and vertex order.
  std::vector<std::int64_t> vtx(V), vty(V);
  std::vector<std::uint64_t> morton(V, 0U);
  bool any_located = false, any_unlocated = false;
  std::int64_t minx = 0, maxx = 0, miny = 0, maxy = 0;
  for (std::uint32_t v = 0; v < V; ++v) {
    if (!in.has_location[v]) {
      any_unlocated = true;
      continue;
    }
    const std::int64_t dx = static_cast<std::int64_t>(in.x[v]) - cfg.origin_x;
    const std::int64_t dy = static_cast<std::int64_t>(in.y[v]) - cfg.origin_y;
    const std::int64_t tx = floor_div(dx, cfg.tile_width);
    const std::int64_t ty = floor_div(dy, cfg.tile_height);
    const std::int64_t lx = dx - tx * static_cast<std::int64_t>(cfg.tile_width);
    const std::int64_t ly = dy - ty * static_cast<std::int64_t>(cfg.tile_height);
    vtx[v] = tx;
    vty[v] = ty;
    morton[v] = spread_bits(static_cast<std::uint32_t>(lx)) | (spread_bits(static_cast<std::uint32_t>(ly)) << 1U);
    if (!any_located) {
      minx = maxx = tx;
      miny = maxy = ty;
      any_located = true;
    } else {
      minx = std::min(minx, tx);
      maxx = std::max(maxx, tx);
      miny = std::min(miny, ty);
      maxy = std::max(maxy, ty);
    }
  }
  std::vector<std::uint32_t> owner(V, 0U);
  std::uint32_t located_tiles = 0;
  const unsigned __int128 box = any_located
      ? static_cast<unsigned __int128>(maxx - minx + 1) * static_cast<unsigned __int128>(maxy - miny + 1)
      : 0;
  if (any_located && box <= static_cast<unsigned __int128>(4U) * V + 1024U) {
    // Dense grid: occupancy table in (tile_y, tile_x) order.
    const std::uint64_t W = static_cast<std::uint64_t>(maxx - minx + 1);
    std::vector<std::uint32_t> dense(static_cast<std::size_t>(box), 0U);
    for (std::uint32_t v = 0; v < V; ++v) {
      if (in.has_location[v]) dense[static_cast<std::size_t>((vty[v] - miny) * W + (vtx[v] - minx))] = 1U;
    }
    for (std::size_t i = 0; i < dense.size(); ++i) {
      if (dense[i]) {
        dense[i] = located_tiles++ + 1U;  // 1-based
        L->tile_xy.push_back(minx + static_cast<std::int64_t>(i % W));
        L->tile_xy.push_back(miny + static_cast<std::int64_t>(i / W));
      }
    }
    for (std::uint32_t v = 0; v < V; ++v) {
      if (in.has_location[v]) owner[v] = dense[static_cast<std::size_t>((vty[v] - miny) * W + (vtx[v] - minx))] - 1U;
    }
  } else if (any_located) {
    std::vector<std::pair<std::int64_t, std::int64_t>> keys;
    keys.reserve(V);
    for (std::uint32_t v = 0; v < V; ++v) {
      if (in.has_location[v]) keys.emplace_back(vty[v], vtx[v]);
    }
    std::sort(keys.begin(), keys.end());
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    located_tiles = checked32(keys.size(), "tile count exceeds 32 bits");
    for (const auto& k : keys) {
      L->tile_xy.push_back(k.second);
      L->tile_xy.push_back(k.first);
    }
    for (std::uint32_t v = 0; v < V; ++v) {
      if (!in.has_location[v]) continue;
      const auto it = std::lower_bound(keys.begin(), keys.end(), std::make_pair(vty[v], vtx[v]));
      owner[v] = static_cast<std::uint32_t>(it - keys.begin());
    }
  }
  const std::uint32_t spill = located_tiles;
  L->T = located_tiles + 1U;
  L->tile_has_location.assign(L->T, 1U);
  L->tile_has_location[spill] = 0U;
  L->tile_xy.push_back(0);
  L->tile_xy.push_back(0);
  (void)any_unlocated;
  for (std::uint32_t v = 0; v < V; ++v) {
    if (!in.has_location[v]) owner[v] = spill;
  }

  // Bucket vertices by tile, then order inside each tile.
  std::vector<std::uint32_t> tile_counts(L->T, 0U);
  for (std::uint32_t v = 0; v < V; ++v) ++tile_counts[owner[v]];
  prefix(tile_counts, L->tile_vertex_offsets, "vertex count exceeds 32 bits");
  L->new_to_old.assign(V, 0U);
  {
    std::vector<std::uint32_t> cursor(L->tile_vertex_offsets.begin(), L->tile_vertex_offsets.end() - 1);
    for (std::uint32_t v = 0; v < V; ++v) L->new_to_old[cursor[owner[v]]++] = v;
  }
  parallel_for(L->T, threads, [&](std::uint64_t b, std::uint64_t end) {
    for (std::uint64_t t = b; t < end; ++t) {
      auto first = L->new_to_old.begin() + L->tile_vertex_offsets[t];
      auto last = L->new_to_old.begin() + L->tile_vertex_offsets[t + 1];
      if (t == spill) {
        std::sort(first, last, [&](std::uint32_t a, std::uint32_t c) {
          return std::tuple(in.resource_class[a], a) < std::tuple(in.resource_class[c], c);
        });
      } else {
        std::sort(first, last, [&](std::uint32_t a, std::uint32_t c) {
          return std::tuple(in.resource_class[a], morton[a], a) < std::tuple(in.resource_class[c], morton[c], c);
        });
      }
    }
  });
  std::vector<std::uint32_t> old_to_new(V);
  for (std::uint32_t n = 0; n < V; ++n) old_to_new[L->new_to_old[n]] = n;
  L->owner_tiles.assign(V, 0U);
  for (std::uint32_t t = 0; t < L->T; ++t) {
    for (std::uint32_t n = L->tile_vertex_offsets[t]; n < L->tile_vertex_offsets[t + 1]; ++n) L->owner_tiles[n] = t;
  }
  vtx.clear(); vtx.shrink_to_fit();
  vty.clear(); vty.shrink_to_fit();
  morton.clear(); morton.shrink_to_fit();
  owner.clear(); owner.shrink_to_fit();

  // ---- CSR in reordered ids.
  {
    std::vector<std::uint32_t> deg(V);
    for (std::uint32_t n = 0; n < V; ++n) {
      const std::uint32_t s = L->new_to_old[n];
      deg[n] = old_row_offsets[s + 1] - old_row_offsets[s];
    }
    prefix(deg, L->csr_row_offsets, "edge count exceeds 32 bits");
  }
  L->csr_destinations.assign(E, 0U);
  L->csr_weights.assign(E, 0.0F);
  L->csr_edge_ids.assign(E, 0U);
  const std::vector<std::uint32_t>& own = L->owner_tiles;
  parallel_for(V, threads, [&](std::uint64_t b, std::uint64_t end) {
    std::vector<std::uint32_t> idx;
    for (std::uint64_t n = b; n < end; ++n) {
      const std::uint32_t s = L->new_to_old[n];
      const std::uint32_t ob = old_row_offsets[s], oe = old_row_offsets[s + 1];
      idx.resize(oe - ob);
      for (std::uint32_t k = ob; k < oe; ++k) idx[k - ob] = k;
      std::sort(idx.begin(), idx.end(), [&](std::uint32_t a, std::uint32_t c) {
        const std::uint32_t da = old_to_new[can_dst[a]], dc = old_to_new[can_dst[c]];
        return std::tuple(own[da], da, a) < std::tuple(own[dc], dc, c);
      });
      std::uint32_t p = L->csr_row_offsets[n];
      for (const std::uint32_t k : idx) {
        L->csr_destinations[p] = old_to_new[can_dst[k]];
        L->csr_weights[p] = can_w[k];
        L->csr_edge_ids[p] = k;
        ++p;
      }
    }
  });
  can_dst.clear(); can_dst.shrink_to_fit();
  can_w.clear(); can_w.shrink_to_fit();

  // ---- CSC: bucket by destination, sort each column.
  {
    std::vector<std::uint32_t> indeg(V, 0U);
    for (std::uint32_t p = 0; p < E; ++p) ++indeg[L->csr_destinations[p]];
    prefix(indeg, L->csc_column_offsets, "edge count exceeds 32 bits");
  }
  L->csc_sources.assign(E, 0U);
  L->csc_weights.assign(E, 0.0F);
  L->csc_edge_ids.assign(E, 0U);
  {
    std::vector<std::uint32_t> cursor(L->csc_column_offsets.begin(), L->csc_column_offsets.end() - 1);
    for (std::uint32_t n = 0; n < V; ++n) {
      for (std::uint32_t p = L->csr_row_offsets[n]; p < L->csr_row_offsets[n + 1]; ++p) {
        const std::uint32_t q = cursor[L->csr_destinations[p]]++;
        L->csc_sources[q] = n;
        L->csc_weights[q] = L->csr_weights[p];
        L->csc_edge_ids[q] = L->csr_edge_ids[p];
      }
    }
  }
  parallel_for(V, threads, [&](std::uint64_t b, std::uint64_t end) {
    std::vector<std::uint32_t> idx;
    std::vector<std::uint32_t> src, eid;
    std::vector<float> w;
    for (std::uint64_t n = b; n < end; ++n) {
      const std::uint32_t cb = L->csc_column_offsets[n], ce = L->csc_column_offsets[n + 1];
      const std::uint32_t m = ce - cb;
      if (m < 2) continue;
      idx.resize(m);
      std::iota(idx.begin(), idx.end(), cb);
      std::sort(idx.begin(), idx.end(), [&](std::uint32_t a, std::uint32_t c) {
        const std::uint32_t sa = L->csc_sources[a], sc = L->csc_sources[c];
        return std::tuple(own[sa], sa, L->csc_edge_ids[a]) < std::tuple(own[sc], sc, L->csc_edge_ids[c]);
      });
      src.resize(m);
      eid.resize(m);
      w.resize(m);
      for (std::uint32_t i = 0; i < m; ++i) {
        src[i] = L->csc_sources[idx[i]];
        eid[i] = L->csc_edge_ids[idx[i]];
        w[i] = L->csc_weights[idx[i]];
      }
      std::copy(src.begin(), src.end(), L->csc_sources.begin() + cb);
      std::copy(eid.begin(), eid.end(), L->csc_edge_ids.begin() + cb);
      std::copy(w.begin(), w.end(), L->csc_weights.begin() + cb);
    }
  });

  // ---- tile runs.
  build_runs(V, L->csr_row_offsets, L->csr_destinations, own, threads, L->csr_row_run_offsets,
             L->csr_run_edge_offsets, L->csr_run_destination_tiles);
  build_runs(V, L->csc_column_offsets, L->csc_sources, own, threads, L->csc_column_run_offsets,
             L->csc_run_edge_offsets, L->csc_run_source_tiles);
  return L;
}

}  // namespace

void fill_view(const HostLayout& L, bfx_device_graph_layout32& v) {
  std::memset(&v, 0, sizeof(v));
  v.vertex_count = L.V;
  v.edge_count = L.E;
  v.tile_count = L.T;
  v.csr_run_count = static_cast<std::uint32_t>(L.csr_run_destination_tiles.size());
  v.csc_run_count = static_cast<std::uint32_t>(L.csc_run_source_tiles.size());
  v.owner_tiles = L.owner_tiles.data();
  v.csr_row_offsets = L.csr_row_offsets.data();
  v.csr_destinations = L.csr_destinations.data();
  v.csr_weights = L.csr_weights.data();
  v.csr_row_run_offsets = L.csr_row_run_offsets.data();
  v.csr_run_edge_offsets = L.csr_run_edge_offsets.data();
  v.csr_run_destination_tiles = L.csr_run_destination_tiles.data();
  v.csc_column_offsets = L.csc_column_offsets.data();
  v.csc_sources = L.csc_sources.data();
  v.csc_weights = L.csc_weights.data();
  v.csc_edge_ids = L.csc_edge_ids.data();
  v.csc_column_run_offsets = L.csc_column_run_offsets.data();
  v.csc_run_edge_offsets = L.csc_run_edge_offsets.data();
  v.csc_run_source_tiles = L.csc_run_source_tiles.data();
  v.csr_edge_ids = L.csr_edge_ids.data();
}

const HostLayout& layout_ref(const bfx_layout* layout) {
  if (!layout) throw std::invalid_argument("layout must be non-null");
  return *reinterpret_cast<const HostLayout*>(layout);
}

}  // namespace bfx

extern "C" {

int bfx_layout_build(const bfx_input_graph* input, const bfx_spatial_order_config* config,
                     uint32_t threads, bfx_layout** out) {
  return bfx::guarded([&] {
    bfx::require(input && config && out, "null argument");
    *out = nullptr;
    auto L = bfx::build_layout(*input, *config, threads);
    *out = reinterpret_cast<bfx_layout*>(L.release());
  });
}

int bfx_layout_destroy(bfx_layout* layout) {
  return bfx::guarded([&] { delete reinterpret_cast<bfx::HostLayout*>(layout); });
}

int bfx_layout_view(const bfx_layout* layout, bfx_device_graph_layout32* view) {
  return bfx::guarded([&] {
    bfx::require(view != nullptr, "null view");
    bfx::fill_view(bfx::layout_ref(layout), *view);
  });
}

int bfx_layout_tiles(const bfx_layout* layout, int64_t* tile_xy, uint8_t* has_location,
                     uint32_t* tile_vertex_offsets) {
  return bfx::guarded([&] {
    const bfx::HostLayout& L = bfx::layout_ref(layout);
    if (tile_xy) std::copy(L.tile_xy.begin(), L.tile_xy.end(), tile_xy);
    if (has_location) std::copy(L.tile_has_location.begin(), L.tile_has_location.end(), has_location);
    if (tile_vertex_offsets) std::copy(L.tile_vertex_offsets.begin(), L.tile_vertex_offsets.end(), tile_vertex_offsets);
  });
}

int bfx_layout_new_to_old(const bfx_layout* layout, uint32_t* new_to_old) {
  return bfx::guarded([&] {
    const bfx::HostLayout& L = bfx::layout_ref(layout);
    bfx::require(new_to_old != nullptr, "null output");
    std::copy(L.new_to_old.begin(), L.new_to_old.end(), new_to_old);
  });
}

}  // extern "C"
