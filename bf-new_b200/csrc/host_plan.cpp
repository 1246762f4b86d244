// Host batch planning and batch descriptions: the per-batch input of the
// device engines.
//
// The planner restates the reference's greedy overlap planner
// (src/batch_plan.cpp:404-543): anchors in order of (selected edges desc,
// selected vertices desc, selected tile count desc, generation asc, query id
// asc); each batch grows from its anchor by repeatedly adding the unassigned
// query that passes Jaccard >= policy minimum and projected union inflation
// <= policy maximum and ranks first by (Jaccard desc, terminal-tile overlap
// desc, inflation asc, projected union edges, projected union vertices, new
// tiles, |generation diff|, |source-count diff|, |target-count diff|, query
// id) (batch_plan.cpp:271-402).  Query features follow
// make_batch_query_features (batch_plan.cpp:578-625, sorted by query id) and
// the region estimates follow SelectedRegionIndex (src/selected_region_index.cpp).
//
// Our implementation evaluates the expensive union-edge tie-breakers only for
// candidates that tie on the first three keys, keeps the union as a tile
// bitmap and, with a positive minimum Jaccard, meets only the candidates that
// share a tile with the union (a tile -> queries index), which yields the
// same plan in far less time on 256+ query sets.
//
// Descriptions follow prepare_batch_device_description
// (src/batch_layout.cpp:1056-1296) with device-materialized run masks: lane
// terminal slices, dense tile lane masks and one vertex range per union tile.
#include "bfx_host.h"
#include "bfx_internal.hpp"
#include "host_region.hpp"

#include <algorithm>
#include <bit>
#include <cstring>
#include <limits>
#include <memory>
#include <numeric>
#include <tuple>
#include <vector>

namespace bfx {

namespace {

using u32 = std::uint32_t;
using u64 = std::uint64_t;

struct Fraction {
  u64 num{0}, den{1};
};

int compare(const Fraction& a, const Fraction& b) {
  const unsigned __int128 l = static_cast<unsigned __int128>(a.num) * b.den;
  const unsigned __int128 r = static_cast<unsigned __int128>(b.num) * a.den;
  return l < r ? -1 : (l > r ? 1 : 0);
}

struct Feature {
  u32 query_index{};  // index into the caller's query array
  u32 query_id{};
  u32 generation{};
  u32 source_count{}, target_count{};
  std::vector<u32> source_tiles, target_tiles, selected_tiles;
  u64 selected_vertices{}, selected_edges{};
};

std::vector<u32> sorted_unique(std::vector<u32> v) {
  std::sort(v.begin(), v.end());
  v.erase(std::unique(v.begin(), v.end()), v.end());
  return v;
}

u64 intersection(const std::vector<u32>& a, const std::vector<u32>& b) {
  std::size_t i = 0, j = 0;
  u64 n = 0;
  while (i < a.size() && j < b.size()) {
    if (a[i] < b[j]) {
      ++i;
    } else if (b[j] < a[i]) {
      ++j;
    } else {
      ++n;
      ++i;
      ++j;
    }
  }
  return n;
}

std::vector<u32> set_union(const std::vector<u32>& a, const std::vector<u32>& b) {
  std::vector<u32> r;
  r.reserve(a.size() + b.size());
  std::set_union(a.begin(), a.end(), b.begin(), b.end(), std::back_inserter(r));
  return r;
}

bool canonical(const std::vector<u32>& t, u32 T) {
  for (std::size_t i = 0; i < t.size(); ++i) {
    if (t[i] >= T || (i > 0 && t[i] <= t[i - 1])) return false;
  }
  return true;
}

u32 absdiff(u32 a, u32 b) { return a > b ? a - b : b - a; }

struct Batch {
  u32 lane_width{};
  u32 valid_mask{};
  std::vector<u32> feature_by_lane;  // feature indices of valid lanes
  std::vector<u32> union_tiles;
  std::vector<u32> union_masks;
  u64 union_vertices{}, union_edges{}, lane_vertices{}, lane_edges{};
};

}  // namespace

struct HostPlan {
  std::vector<Feature> features;
  std::vector<Batch> batches;
  // Per-batch description storage.
  std::vector<std::vector<u32>> source_offsets, sources, target_offsets, targets, union_tiles, tile_masks;
  std::vector<std::vector<bfx_batch_vertex_range>> ranges;
  std::vector<bfx_batch_description> descriptions;
};

namespace {

std::unique_ptr<HostPlan> build_plan(const bfx_device_graph_layout32& g, const std::vector<u32>& tile_offsets,
                                     u32 nq, const bfx_route_query* queries, const bfx_planner_policy& policy,
                                     const RegionIndex* shared_region = nullptr) {
  const u32 W = policy.lane_width;
  require(W == 1 || W == 8 || W == 16 || W == 32, "batch planner policy is invalid");
  require(policy.minimum_jaccard_denominator != 0 &&
              policy.minimum_jaccard_numerator <= policy.minimum_jaccard_denominator,
          "batch planner policy is invalid");
  require(policy.maximum_union_inflation_denominator != 0 &&
              policy.maximum_union_inflation_numerator >= policy.maximum_union_inflation_denominator,
          "batch planner policy is invalid");
  require(nq > 0, "batch planning requires at least one query");
  const u32 T = g.tile_count;
  RegionIndex own;
  if (shared_region == nullptr) own = make_region_index(g);
  const RegionIndex& region = shared_region != nullptr ? *shared_region : own;

  auto plan = std::make_unique<HostPlan>();
  auto& F = plan->features;
  F.resize(nq);
  std::vector<std::uint8_t> member(T, 0U);
  for (u32 q = 0; q < nq; ++q) {
    const bfx_route_query& r = queries[q];
    require(r.source_count > 0 && r.target_count > 0, "route queries require sources and targets");
    require(r.sources && r.targets && r.selected_tiles, "null query array");
    Feature& f = F[q];
    f.query_index = q;
    f.query_id = r.query_id;
    f.generation = r.expansion_generation;
    f.source_count = r.source_count;
    f.target_count = r.target_count;
    std::vector<u32> st, tt;
    for (u32 i = 0; i < r.source_count; ++i) {
      if (r.sources[i] >= g.vertex_count) throw std::out_of_range("query terminal is outside the graph");
      if (i > 0 && r.sources[i] <= r.sources[i - 1]) throw std::invalid_argument("noncanonical sources");
      st.push_back(g.owner_tiles[r.sources[i]]);
    }
    for (u32 i = 0; i < r.target_count; ++i) {
      if (r.targets[i] >= g.vertex_count) throw std::out_of_range("query terminal is outside the graph");
      if (i > 0 && r.targets[i] <= r.targets[i - 1]) throw std::invalid_argument("noncanonical targets");
      tt.push_back(g.owner_tiles[r.targets[i]]);
    }
    f.source_tiles = sorted_unique(std::move(st));
    f.target_tiles = sorted_unique(std::move(tt));
    f.selected_tiles.assign(r.selected_tiles, r.selected_tiles + r.selected_tile_count);
    require(!f.selected_tiles.empty() && canonical(f.selected_tiles, T), "noncanonical selected tiles");
    require(std::includes(f.selected_tiles.begin(), f.selected_tiles.end(), f.source_tiles.begin(),
                          f.source_tiles.end()) &&
                std::includes(f.selected_tiles.begin(), f.selected_tiles.end(), f.target_tiles.begin(),
                              f.target_tiles.end()),
            "terminal owner tile not selected");
    for (u32 t : f.selected_tiles) member[t] = 1U;
    f.selected_vertices = region.vertices(f.selected_tiles);
    f.selected_edges = region.edges(f.selected_tiles, member);
    for (u32 t : f.selected_tiles) member[t] = 0U;
    require(f.selected_vertices != 0, "batch planner query features are invalid");
  }
  std::sort(F.begin(), F.end(), [](const Feature& a, const Feature& b) { return a.query_id < b.query_id; });
  for (u32 i = 1; i < nq; ++i) require(F[i].query_id != F[i - 1].query_id, "batch query IDs must be unique");

  std::vector<u32> anchors(nq);
  std::iota(anchors.begin(), anchors.end(), 0U);
  std::sort(anchors.begin(), anchors.end(), [&](u32 a, u32 b) {
    const Feature& l = F[a];
    const Feature& r = F[b];
    if (l.selected_edges != r.selected_edges) return l.selected_edges > r.selected_edges;
    if (l.selected_vertices != r.selected_vertices) return l.selected_vertices > r.selected_vertices;
    if (l.selected_tiles.size() != r.selected_tiles.size()) return l.selected_tiles.size() > r.selected_tiles.size();
    if (l.generation != r.generation) return l.generation < r.generation;
    return l.query_id < r.query_id;
  });

  const Fraction min_j{policy.minimum_jaccard_numerator, policy.minimum_jaccard_denominator};
  const Fraction max_i{policy.maximum_union_inflation_numerator, policy.maximum_union_inflation_denominator};
  std::vector<std::uint8_t> assigned(nq, 0U);
  std::vector<std::uint8_t> in_union(T, 0U), scratch(T, 0U);
  u32 assigned_count = 0;
  std::size_t anchor_cursor = 0;

  // With a positive minimum Jaccard only a query that shares a tile with the
  // batch's union can join it, so the candidates of a growing batch are
  // found through a tile -> queries index, and each one's overlap with the
  // union is counted as tiles join the union (shared[c] = |tiles(c) & U|)
  // instead of rescanning every query's tiles for every lane.  The choice
  // does not depend on the order candidates are met in (the last
  // tie-breaker is the unique query id), so the plan is the same.
  const bool indexed = policy.minimum_jaccard_numerator > 0;
  std::vector<u32> tile_q_off, tile_q, shared, touched;
  if (indexed) {
    tile_q_off.assign(T + 1U, 0U);
    for (u32 c = 0; c < nq; ++c) {
      for (u32 t : F[c].selected_tiles) ++tile_q_off[t + 1U];
    }
    for (u32 t = 0; t < T; ++t) tile_q_off[t + 1U] += tile_q_off[t];
    tile_q.resize(tile_q_off[T]);
    std::vector<u32> fill(tile_q_off.begin(), tile_q_off.end() - 1);
    for (u32 c = 0; c < nq; ++c) {
      for (u32 t : F[c].selected_tiles) tile_q[fill[t]++] = c;
    }
    shared.assign(nq, 0U);
  }
  const auto union_gains = [&](u32 t) {  // tile t joins the union
    for (u32 k = tile_q_off[t]; k < tile_q_off[t + 1U]; ++k) {
      const u32 c = tile_q[k];
      if (shared[c]++ == 0U) touched.push_back(c);
    }
  };

  struct Cand {
    u32 idx;
    Fraction jac;
    u64 overlap;
    Fraction infl;
    u64 union_size;
  };

  while (assigned_count < nq) {
    while (assigned[anchors[anchor_cursor]]) ++anchor_cursor;
    const u32 a = anchors[anchor_cursor];
    const Feature& anchor = F[a];
    Batch b;
    b.lane_width = W;
    b.feature_by_lane.push_back(a);
    assigned[a] = 1U;
    ++assigned_count;
    std::vector<u32> U = anchor.selected_tiles;
    std::vector<u32> US = anchor.source_tiles, UT = anchor.target_tiles;
    for (u32 t : U) in_union[t] = 1U;
    if (indexed) {
      for (u32 c : touched) shared[c] = 0U;
      touched.clear();
      for (u32 t : U) union_gains(t);
    }
    u64 lane_tiles = anchor.selected_tiles.size();

    while (b.feature_by_lane.size() < W) {
      std::vector<Cand> top;
      const u32 ncand = indexed ? static_cast<u32>(touched.size()) : nq;
      for (u32 ci = 0; ci < ncand; ++ci) {
        const u32 c = indexed ? touched[ci] : ci;
        if (assigned[c]) continue;
        const Feature& f = F[c];
        u64 inter = 0;
        if (indexed) {
          inter = shared[c];
        } else {
          for (u32 t : f.selected_tiles) inter += in_union[t];
        }
        const u64 usize = U.size() + f.selected_tiles.size() - inter;
        Cand cd;
        cd.idx = c;
        cd.jac = usize == 0 ? Fraction{1, 1} : Fraction{inter, usize};
        cd.overlap = intersection(US, f.source_tiles) + intersection(UT, f.target_tiles);
        cd.infl = Fraction{(b.feature_by_lane.size() + 1U) * usize, lane_tiles + f.selected_tiles.size()};
        cd.union_size = usize;
        if (compare(cd.jac, min_j) < 0 || compare(cd.infl, max_i) > 0) continue;
        if (top.empty()) {
          top.push_back(cd);
          continue;
        }
        const Cand& best = top.front();
        int o = compare(cd.jac, best.jac);
        if (o == 0) o = (cd.overlap > best.overlap) - (cd.overlap < best.overlap);
        if (o == 0) o = -compare(cd.infl, best.infl);
        if (o > 0) {
          top.clear();
          top.push_back(cd);
        } else if (o == 0) {
          top.push_back(cd);
        }
      }
      if (top.empty()) break;
      u32 chosen = top.front().idx;
      if (top.size() > 1) {
        // Remaining keys, evaluated only for the tied group.
        using Key = std::tuple<u64, u64, u64, u32, u32, u32, u32>;
        Key best_key{};
        bool have = false;
        for (const Cand& cd : top) {
          const Feature& f = F[cd.idx];
          std::vector<u32> pu = set_union(U, f.selected_tiles);
          for (u32 t : pu) scratch[t] = 1U;
          const u64 ue = region.edges(pu, scratch);
          for (u32 t : pu) scratch[t] = 0U;
          const Key k{ue, region.vertices(pu), pu.size() - U.size(), absdiff(f.generation, anchor.generation),
                      absdiff(f.source_count, anchor.source_count), absdiff(f.target_count, anchor.target_count),
                      f.query_id};
          if (!have || k < best_key) {
            best_key = k;
            chosen = cd.idx;
            have = true;
          }
        }
      }
      const Feature& s = F[chosen];
      b.feature_by_lane.push_back(chosen);
      assigned[chosen] = 1U;
      ++assigned_count;
      lane_tiles += s.selected_tiles.size();
      U = set_union(U, s.selected_tiles);
      for (u32 t : s.selected_tiles) {
        if (indexed && !in_union[t]) union_gains(t);
        in_union[t] = 1U;
      }
      US = set_union(US, s.source_tiles);
      UT = set_union(UT, s.target_tiles);
    }

    const u32 lanes = static_cast<u32>(b.feature_by_lane.size());
    b.valid_mask = lanes == 32 ? 0xFFFFFFFFu : ((1u << lanes) - 1u);
    b.union_tiles = U;
    b.union_masks.assign(U.size(), 0U);
    for (u32 lane = 0; lane < lanes; ++lane) {
      const Feature& f = F[b.feature_by_lane[lane]];
      b.lane_vertices += f.selected_vertices;
      b.lane_edges += f.selected_edges;
      std::size_t i = 0;
      for (u32 t : f.selected_tiles) {
        while (b.union_tiles[i] < t) ++i;
        b.union_masks[i] |= 1u << lane;
      }
    }
    b.union_vertices = region.vertices(U);
    b.union_edges = region.edges(U, in_union);
    for (u32 t : U) in_union[t] = 0U;
    if (policy.narrow_lanes) {
      b.lane_width = lanes == 1 ? 1U : (lanes <= 8 ? 8U : (lanes <= 16 ? 16U : 32U));
    }
    plan->batches.push_back(std::move(b));
  }

  // Descriptions.
  const std::size_t nb = plan->batches.size();
  plan->source_offsets.resize(nb);
  plan->sources.resize(nb);
  plan->target_offsets.resize(nb);
  plan->targets.resize(nb);
  plan->union_tiles.resize(nb);
  plan->tile_masks.resize(nb);
  plan->ranges.resize(nb);
  plan->descriptions.resize(nb);
  for (std::size_t bi = 0; bi < nb; ++bi) {
    const Batch& b = plan->batches[bi];
    auto& so = plan->source_offsets[bi];
    auto& sv = plan->sources[bi];
    auto& to = plan->target_offsets[bi];
    auto& tv = plan->targets[bi];
    so.assign(b.lane_width + 1U, 0U);
    to.assign(b.lane_width + 1U, 0U);
    for (u32 lane = 0; lane < b.lane_width; ++lane) {
      if (lane < b.feature_by_lane.size()) {
        const bfx_route_query& r = queries[F[b.feature_by_lane[lane]].query_index];
        sv.insert(sv.end(), r.sources, r.sources + r.source_count);
        tv.insert(tv.end(), r.targets, r.targets + r.target_count);
      }
      so[lane + 1] = static_cast<u32>(sv.size());
      to[lane + 1] = static_cast<u32>(tv.size());
    }
    plan->union_tiles[bi] = b.union_tiles;
    auto& tm = plan->tile_masks[bi];
    tm.assign(T, 0U);
    auto& rg = plan->ranges[bi];
    for (std::size_t i = 0; i < b.union_tiles.size(); ++i) {
      const u32 t = b.union_tiles[i];
      tm[t] = b.union_masks[i];
      rg.push_back(bfx_batch_vertex_range{tile_offsets[t], tile_offsets[t + 1], b.union_masks[i]});
    }
    bfx_batch_description& d = plan->descriptions[bi];
    std::memset(&d, 0, sizeof(d));
    d.lane_width = b.lane_width;
    d.valid_lane_mask = b.valid_mask;
    d.source_offsets = so.data();
    d.sources = sv.data();
    d.target_offsets = to.data();
    d.targets = tv.data();
    d.union_tile_count = static_cast<u32>(b.union_tiles.size());
    d.tile_count = T;
    d.union_tiles = plan->union_tiles[bi].data();
    d.tile_lane_masks = tm.data();
    d.range_count = static_cast<u32>(rg.size());
    d.selected_vertex_ranges = rg.data();
  }
  return plan;
}

const HostPlan& plan_ref(const bfx_plan* p) {
  if (!p) throw std::invalid_argument("plan must be non-null");
  return *reinterpret_cast<const HostPlan*>(p);
}

}  // namespace
}  // namespace bfx

namespace bfx {

bfx_plan* plan_build_with_region(const bfx_device_graph_layout32& g, const std::uint32_t* tile_vertex_offsets,
                                 std::uint32_t query_count, const bfx_route_query* queries,
                                 const bfx_planner_policy& policy, const RegionIndex& region) {
  require(tile_vertex_offsets && queries, "null argument");
  require(region.T == g.tile_count, "region index does not match the graph");
  std::vector<std::uint32_t> offsets(tile_vertex_offsets, tile_vertex_offsets + g.tile_count + 1U);
  return reinterpret_cast<bfx_plan*>(build_plan(g, offsets, query_count, queries, policy, &region).release());
}

}  // namespace bfx

extern "C" {

int bfx_plan_build(const bfx_device_graph_layout32* layout, const uint32_t* tile_vertex_offsets,
                   uint32_t query_count, const bfx_route_query* queries, const bfx_planner_policy* policy,
                   bfx_plan** out) {
  return bfx::guarded([&] {
    bfx::require(layout && tile_vertex_offsets && queries && policy && out, "null argument");
    bfx::require(layout->owner_tiles && layout->csr_row_run_offsets && layout->csr_run_edge_offsets &&
                     layout->csr_run_destination_tiles,
                 "planner needs owner tiles and CSR runs");
    *out = nullptr;
    std::vector<std::uint32_t> offsets(tile_vertex_offsets, tile_vertex_offsets + layout->tile_count + 1U);
    auto p = bfx::build_plan(*layout, offsets, query_count, queries, *policy);
    *out = reinterpret_cast<bfx_plan*>(p.release());
  });
}

int bfx_plan_destroy(bfx_plan* plan) {
  return bfx::guarded([&] { delete reinterpret_cast<bfx::HostPlan*>(plan); });
}

int bfx_plan_batch_count(const bfx_plan* plan, uint32_t* count) {
  return bfx::guarded([&] {
    bfx::require(count != nullptr, "null output");
    *count = static_cast<uint32_t>(bfx::plan_ref(plan).batches.size());
  });
}

int bfx_plan_description(const bfx_plan* plan, uint32_t batch, bfx_batch_description* out) {
  return bfx::guarded([&] {
    const bfx::HostPlan& p = bfx::plan_ref(plan);
    bfx::require(out != nullptr, "null output");
    if (batch >= p.descriptions.size()) throw std::out_of_range("batch index");
    *out = p.descriptions[batch];
  });
}

int bfx_plan_descriptions(const bfx_plan* plan, const bfx_batch_description** out) {
  return bfx::guarded([&] {
    bfx::require(out != nullptr, "null output");
    *out = bfx::plan_ref(plan).descriptions.data();
  });
}

int bfx_plan_batch_info(const bfx_plan* plan, uint32_t batch, uint32_t* query_index_by_lane,
                        uint64_t estimates[4]) {
  return bfx::guarded([&] {
    const bfx::HostPlan& p = bfx::plan_ref(plan);
    if (batch >= p.batches.size()) throw std::out_of_range("batch index");
    const auto& b = p.batches[batch];
    if (query_index_by_lane) {
      for (std::uint32_t l = 0; l < b.lane_width; ++l) {
        query_index_by_lane[l] =
            l < b.feature_by_lane.size() ? p.features[b.feature_by_lane[l]].query_index : 0xFFFFFFFFu;
      }
    }
    if (estimates) {
      estimates[0] = b.union_vertices;
      estimates[1] = b.union_edges;
      estimates[2] = b.lane_vertices;
      estimates[3] = b.lane_edges;
    }
  });
}

}  // extern "C"
