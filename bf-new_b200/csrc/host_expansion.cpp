// Expansion loop over the batched engines (bfx_expansion.h).
//
// Restates the reference's orchestration (src/batched_expansion.cpp:888-1679)
// per query: states ordered by query id, one planning pass per round of
// retries, per-lane classification of each batch status (clean convergence
// with the lane reached -> reached; non-clean -> engine_failure, never
// expanded; clean miss -> retry decision), and the retry decision of
// advance_failed_query (:685-770): full region or fallback already used ->
// unreachable_in_full_region; otherwise advance the margin cursor by the
// schedule (advance_margin_cursor, :307-365), grow the region to every located
// tile inside the anchor box widened by the margins (expanded_tiles,
// :367-427, spill tile only through an actual edge from a selected located
// tile), and restart with generation + 1; a region that did not grow is
// stalled (explicit-failure policy) or falls back to the full region once.
//
// bfx runs all batches of a pass through one runner call -- one relaxation
// launch on the GPU -- instead of one engine run per batch.
#include "bfx_expansion.h"
#include "bfx_internal.hpp"
#include "host_region.hpp"

#include <algorithm>
#include <bit>
#include <cstring>
#include <limits>
#include <memory>
#include <vector>

namespace bfx {
namespace {

using u32 = std::uint32_t;
using u64 = std::uint64_t;
using i64 = std::int64_t;

struct Bounds {
  bool present{};
  i64 min_x{}, min_y{}, max_x{}, max_y{};
};

struct State {
  u32 query_id{};
  u32 generation{};
  std::vector<u32> sources, targets, tiles;
  Bounds anchor{};
  u64 margin_x{}, margin_y{};
  u32 attempts{}, scheduled{}, total{};
  bool fallback{}, terminal{};
  u32 disposition{BFX_EXPANSION_ENGINE_FAILURE};
  u32 stop_reason{}, error_bits{};
};

struct Geometry {
  u32 T{};
  u32 spill{};
  std::vector<i64> x, y;
  std::vector<std::uint8_t> located;
  // tiles joined to the spill tile by an edge in either direction
  std::vector<std::uint8_t> spill_neighbor;
};

}  // namespace

struct ExpansionResult {
  std::vector<bfx_expansion_outcome> outcomes;
  std::vector<std::vector<u32>> final_tiles;
  bfx_expansion_metrics metrics{};
  std::vector<u64> histogram;
};

namespace {

void validate(const bfx_expansion_options& o, bool gpu) {
  const bfx_gpu_run_options& r = o.run_options;
  const auto bad = [](const char* m) { throw std::invalid_argument(m); };
  // validate_gpu_run_options (src/gpu_api.cpp:71-105)
  if (r.engine > 2u) bad(gpu ? "expansion needs a fixed engine" : "invalid engine");
  if (r.control_mode > 2u || r.rounds_per_chunk == 0u || r.block_size == 0u || r.block_size % 32u != 0u ||
      r.grid_policy > 1u || (r.grid_policy == 1u) != (r.blocks_per_wgp != 0u) || r.instrumentation > 2u ||
      r.maximum_rounds == 0u || r.enable_per_lane_convergence > 1u)
    bad("batched expansion options are invalid: run options");
  const bfx_planner_policy& p = o.planner_policy;
  if (!(p.lane_width == 1 || p.lane_width == 8 || p.lane_width == 16 || p.lane_width == 32) ||
      p.minimum_jaccard_denominator == 0 || p.minimum_jaccard_numerator > p.minimum_jaccard_denominator ||
      p.maximum_union_inflation_denominator == 0 ||
      p.maximum_union_inflation_numerator < p.maximum_union_inflation_denominator || p.narrow_lanes > 1u)
    bad("batched expansion options are invalid: planner policy");
  switch (o.schedule_kind) {
    case BFX_EXPANSION_ONE_RING:
    case BFX_EXPANSION_DOUBLING:
      if (o.fixed_ring_size != 0u || o.hybrid_small_expansion_count != 0u) bad("invalid schedule parameters");
      break;
    case BFX_EXPANSION_FIXED_RING:
      if (o.fixed_ring_size < 2u || o.hybrid_small_expansion_count != 0u) bad("invalid schedule parameters");
      break;
    case BFX_EXPANSION_HYBRID:
      if (o.fixed_ring_size != 0u || o.hybrid_small_expansion_count == 0u) bad("invalid schedule parameters");
      break;
    default:
      bad("unspecified or invalid expansion schedule");
  }
  if (o.terminal_policy > BFX_EXPANSION_EXPLICIT_FAILURE) bad("invalid terminal policy");
}

Geometry make_geometry(const bfx_device_graph_layout32& g, const bfx_tile_geometry& tg) {
  require(tg.tile_count == g.tile_count && tg.tile_count >= 1 && tg.tile_xy && tg.has_location &&
              tg.tile_vertex_offsets,
          "tile geometry does not match the graph");
  require(g.csr_row_offsets && g.csr_destinations && g.csc_column_offsets && g.csc_sources && g.owner_tiles,
          "expansion needs CSR, CSC and owner tiles");
  Geometry geo;
  geo.T = tg.tile_count;
  geo.spill = tg.tile_count - 1u;
  geo.x.resize(geo.T);
  geo.y.resize(geo.T);
  geo.located.resize(geo.T);
  for (u32 t = 0; t < geo.T; ++t) {
    geo.x[t] = tg.tile_xy[2 * size_t{t}];
    geo.y[t] = tg.tile_xy[2 * size_t{t} + 1];
    geo.located[t] = tg.has_location[t] ? 1u : 0u;
  }
  // src/tiled_graph.cpp:143-154: cross edges touching the spill tile make
  // both end tiles neighbours of each other.
  geo.spill_neighbor.assign(geo.T, 0u);
  for (u32 v = tg.tile_vertex_offsets[geo.spill]; v < tg.tile_vertex_offsets[geo.spill + 1]; ++v) {
    for (u32 e = g.csr_row_offsets[v]; e < g.csr_row_offsets[v + 1]; ++e) {
      const u32 t = g.owner_tiles[g.csr_destinations[e]];
      if (t != geo.spill) geo.spill_neighbor[t] = 1u;
    }
    for (u32 e = g.csc_column_offsets[v]; e < g.csc_column_offsets[v + 1]; ++e) {
      const u32 t = g.owner_tiles[g.csc_sources[e]];
      if (t != geo.spill) geo.spill_neighbor[t] = 1u;
    }
  }
  return geo;
}

Bounds located_bounds(const Geometry& geo, const std::vector<u32>& tiles) {
  Bounds b;
  for (u32 t : tiles) {
    if (!geo.located[t]) continue;
    if (!b.present) {
      b = Bounds{true, geo.x[t], geo.y[t], geo.x[t], geo.y[t]};
      continue;
    }
    b.min_x = std::min(b.min_x, geo.x[t]);
    b.min_y = std::min(b.min_y, geo.y[t]);
    b.max_x = std::max(b.max_x, geo.x[t]);
    b.max_y = std::max(b.max_y, geo.y[t]);
  }
  return b;
}

i64 sat_sub(i64 v, u64 a) {
  constexpr i64 lo = std::numeric_limits<i64>::min();
  if (a > static_cast<u64>(std::numeric_limits<i64>::max())) return lo;
  const i64 n = static_cast<i64>(a);
  return v < lo + n ? lo : v - n;
}

i64 sat_add(i64 v, u64 a) {
  constexpr i64 hi = std::numeric_limits<i64>::max();
  if (a > static_cast<u64>(hi)) return hi;
  const i64 n = static_cast<i64>(a);
  return v > hi - n ? hi : v + n;
}

bool add_u64(u64 a, u64 b, u64& out) {
  if (a > std::numeric_limits<u64>::max() - b) return false;
  out = a + b;
  return true;
}

bool double_u64(u64 a, u64& out) {
  if (a > std::numeric_limits<u64>::max() / 2u) return false;
  out = a * 2u;
  return true;
}

// One step of the margin schedule; false on counter overflow.
bool advance_margins(State& s, const bfx_expansion_options& o) {
  u64 nx = s.margin_x, ny = s.margin_y;
  const auto ring = [&](u64 k) { return add_u64(nx, k, nx) && add_u64(ny, k, ny); };
  const auto dbl = [&] {
    if (nx == 0u) {
      nx = 1u;
    } else if (!double_u64(nx, nx)) {
      return false;
    }
    if (ny == 0u) {
      ny = 1u;
    } else if (!double_u64(ny, ny)) {
      return false;
    }
    return true;
  };
  bool ok = false;
  switch (o.schedule_kind) {
    case BFX_EXPANSION_ONE_RING: ok = ring(1u); break;
    case BFX_EXPANSION_FIXED_RING: ok = ring(o.fixed_ring_size); break;
    case BFX_EXPANSION_DOUBLING: ok = dbl(); break;
    case BFX_EXPANSION_HYBRID: ok = s.scheduled < o.hybrid_small_expansion_count ? ring(1u) : dbl(); break;
    default: ok = false;
  }
  if (!ok) return false;
  s.margin_x = nx;
  s.margin_y = ny;
  return true;
}

std::vector<u32> expanded_tiles(const Geometry& geo, State& s) {
  std::vector<u32> sel = s.tiles;
  if (!s.anchor.present) {
    // Spill-only region: its first expansion adds the located tiles joined
    // to the spill tile by an edge, which then anchor the box.
    if (std::binary_search(sel.begin(), sel.end(), geo.spill)) {
      for (u32 t = 0; t < geo.T; ++t) {
        if (t != geo.spill && geo.located[t] && geo.spill_neighbor[t]) sel.push_back(t);
      }
      std::sort(sel.begin(), sel.end());
      sel.erase(std::unique(sel.begin(), sel.end()), sel.end());
      s.anchor = located_bounds(geo, sel);
      s.margin_x = 0u;
      s.margin_y = 0u;
    }
    return sel;
  }
  const i64 lx = sat_sub(s.anchor.min_x, s.margin_x), ly = sat_sub(s.anchor.min_y, s.margin_y);
  const i64 ux = sat_add(s.anchor.max_x, s.margin_x), uy = sat_add(s.anchor.max_y, s.margin_y);
  for (u32 t = 0; t < geo.T; ++t) {
    if (geo.located[t] && geo.x[t] >= lx && geo.x[t] <= ux && geo.y[t] >= ly && geo.y[t] <= uy) sel.push_back(t);
  }
  std::sort(sel.begin(), sel.end());
  sel.erase(std::unique(sel.begin(), sel.end()), sel.end());
  if (!std::binary_search(sel.begin(), sel.end(), geo.spill)) {
    for (u32 t : sel) {
      if (geo.located[t] && geo.spill_neighbor[t]) {
        sel.push_back(geo.spill);
        std::sort(sel.begin(), sel.end());
        break;
      }
    }
  }
  return sel;
}

struct Counter {
  const RegionIndex& region;
  std::vector<std::uint8_t> member;
  explicit Counter(const RegionIndex& r) : region(r), member(r.T, 0u) {}
  u64 edges(const std::vector<u32>& tiles) {
    for (u32 t : tiles) member[t] = 1u;
    const u64 n = region.edges(tiles, member);
    for (u32 t : tiles) member[t] = 0u;
    return n;
  }
};

void set_terminal(State& s, u32 disposition, u32 stop_reason, u32 error_bits) {
  s.terminal = true;
  s.disposition = disposition;
  s.stop_reason = stop_reason;
  s.error_bits = error_bits;
}

bool clean(const bfx_device_run_status& st) {
  return st.converged == 1u && st.error_bits == 0u && st.stop_reason == BFX_STOP_CONVERGED;
}

// advance_failed_query: true = retry with the state's new region.
bool advance_failed(const Geometry& geo, Counter& count, const std::vector<u32>& full, const bfx_expansion_options& o,
                    State& s, bfx_expansion_metrics& m) {
  // synthetic clean-miss status of a geometric decision
  const u32 kStop = BFX_STOP_CONVERGED, kErr = 0u;
  if (s.fallback || s.tiles == full) {
    set_terminal(s, BFX_EXPANSION_UNREACHABLE_IN_FULL_REGION, kStop, kErr);
    return false;
  }
  const auto restart = [&](std::vector<u32> next, bool fallback) {
    if (s.generation == std::numeric_limits<u32>::max() || s.total == std::numeric_limits<u32>::max()) return false;
    m.repeated_selected_edge_estimate += count.edges(s.tiles);
    ++s.generation;
    ++s.total;
    s.tiles = std::move(next);
    if (fallback) {
      s.fallback = true;
      ++m.full_region_fallbacks;
    }
    return true;
  };
  if (s.scheduled < o.maximum_expansions) {
    if (!advance_margins(s, o)) {
      set_terminal(s, BFX_EXPANSION_IDENTITY_OR_COUNT_OVERFLOW, kStop, kErr);
      return false;
    }
    std::vector<u32> next = expanded_tiles(geo, s);
    if (next != s.tiles) {
      if (s.scheduled == std::numeric_limits<u32>::max() || !restart(std::move(next), false)) {
        set_terminal(s, BFX_EXPANSION_IDENTITY_OR_COUNT_OVERFLOW, kStop, kErr);
        return false;
      }
      ++s.scheduled;
      ++m.scheduled_expansions;
      return true;
    }
    if (o.terminal_policy == BFX_EXPANSION_EXPLICIT_FAILURE) {
      set_terminal(s, BFX_EXPANSION_REGION_STALLED, kStop, kErr);
      return false;
    }
  } else if (o.terminal_policy == BFX_EXPANSION_EXPLICIT_FAILURE) {
    set_terminal(s, BFX_EXPANSION_LIMIT, kStop, kErr);
    return false;
  }
  if (!restart(full, true)) {
    set_terminal(s, BFX_EXPANSION_IDENTITY_OR_COUNT_OVERFLOW, kStop, kErr);
    return false;
  }
  return true;
}

using Runner = int (*)(void*, u32, const bfx_batch_description*, bfx_device_run_status*);

std::unique_ptr<ExpansionResult> run(const bfx_device_graph_layout32& g, const bfx_tile_geometry& tg, u32 nq,
                                     const bfx_route_query* queries, const bfx_expansion_options& o, Runner runner,
                                     void* user) {
  const Geometry geo = make_geometry(g, tg);
  require(g.csr_row_run_offsets && g.csr_run_edge_offsets && g.csr_run_destination_tiles,
          "planner needs owner tiles and CSR runs");
  const RegionIndex region = make_region_index(g);
  Counter count(region);
  std::vector<u32> full(geo.T);
  for (u32 t = 0; t < geo.T; ++t) full[t] = t;

  auto out = std::make_unique<ExpansionResult>();
  bfx_expansion_metrics& m = out->metrics;
  m.input_queries = nq;
  std::vector<State> states(nq);
  for (u32 i = 0; i < nq; ++i) {
    const bfx_route_query& q = queries[i];
    require(q.sources && q.targets && q.selected_tiles, "null query array");
    State& s = states[i];
    s.query_id = q.query_id;
    s.generation = q.expansion_generation;
    s.sources.assign(q.sources, q.sources + q.source_count);
    s.targets.assign(q.targets, q.targets + q.target_count);
    s.tiles.assign(q.selected_tiles, q.selected_tiles + q.selected_tile_count);
    for (u32 t : s.tiles) require(t < geo.T, "selected tile out of range");
    s.anchor = located_bounds(geo, s.tiles);
  }
  std::sort(states.begin(), states.end(), [](const State& a, const State& b) { return a.query_id < b.query_id; });
  for (u32 i = 1; i < nq; ++i) {
    require(states[i].query_id != states[i - 1].query_id, "batched expansion query IDs must be unique");
  }

  std::vector<u32> active(nq);
  for (u32 i = 0; i < nq; ++i) active[i] = i;
  u32 pass = 0;
  std::vector<bfx_route_query> rq;
  std::vector<bfx_device_run_status> statuses;
  while (!active.empty()) {
    rq.assign(active.size(), bfx_route_query{});
    for (size_t k = 0; k < active.size(); ++k) {
      const State& s = states[active[k]];
      bfx_route_query& r = rq[k];
      r.query_id = s.query_id;
      r.expansion_generation = s.generation;
      r.source_count = static_cast<u32>(s.sources.size());
      r.target_count = static_cast<u32>(s.targets.size());
      r.sources = s.sources.data();
      r.targets = s.targets.data();
      r.selected_tile_count = static_cast<u32>(s.tiles.size());
      r.selected_tiles = s.tiles.data();
    }
    // every pass is planned against the loop's one region index
    bfx_plan* plan = plan_build_with_region(g, tg.tile_vertex_offsets, static_cast<u32>(rq.size()), rq.data(),
                                            o.planner_policy, region);
    std::unique_ptr<bfx_plan, int (*)(bfx_plan*)> plan_owner(plan, bfx_plan_destroy);
    u32 nb = 0;
    bfx_plan_batch_count(plan, &nb);
    const bfx_batch_description* descs = nullptr;
    bfx_plan_descriptions(plan, &descs);
    ++m.planning_passes;
    statuses.assign(nb, bfx_device_run_status{});
    if (runner(user, nb, descs, statuses.data()) != 0) {
      throw std::logic_error(std::string("expansion batch runner failed: ") + bfx_last_error());
    }
    std::vector<u32> failed;
    std::vector<u32> lane_query(32);
    for (u32 b = 0; b < nb; ++b) {
      u64 est[4];
      bfx_plan_batch_info(plan, b, lane_query.data(), est);
      const bfx_batch_description& d = descs[b];
      const bfx_device_run_status& st = statuses[b];
      ++m.batches_executed;
      if (pass == 0) {
        ++m.initial_batches_executed;
      } else {
        ++m.retry_batches_executed;
        m.retry_valid_lane_observations += static_cast<u64>(std::popcount(d.valid_lane_mask));
        m.retry_lane_capacity += d.lane_width;
      }
      m.attempted_selected_vertex_count += est[2];
      m.attempted_selected_edge_estimate += est[3];
      if (st.valid_lane_mask != d.valid_lane_mask) {
        throw std::logic_error("batch runner returned status for a different or invalid request");
      }
      const bool ok = clean(st);
      if (ok && ((st.reached_target_mask | st.bounding_box_miss_mask) != d.valid_lane_mask ||
                 (st.reached_target_mask & st.bounding_box_miss_mask) != 0u)) {
        throw std::logic_error("clean batch status does not partition valid lanes into reached/miss");
      }
      if (!ok && (st.reached_target_mask != 0u || st.bounding_box_miss_mask != 0u)) {
        throw std::logic_error("non-clean batch status must not classify reached or missed lanes");
      }
      if (ok && st.bounding_box_miss_mask != 0u) {
        m.failed_lane_observations += static_cast<u64>(std::popcount(st.bounding_box_miss_mask));
        m.failed_origin_valid_lane_observations += static_cast<u64>(std::popcount(d.valid_lane_mask));
      }
      for (u32 lane = 0; lane < d.lane_width; ++lane) {
        const u32 bit = 1u << lane;
        if ((d.valid_lane_mask & bit) == 0u) continue;
        require(lane_query[lane] < active.size(), "batch lane without a query");
        const u32 si = active[lane_query[lane]];
        State& s = states[si];
        if (s.terminal) throw std::logic_error("batch runner crossed query generation state");
        if (s.attempts == std::numeric_limits<u32>::max()) {
          set_terminal(s, BFX_EXPANSION_IDENTITY_OR_COUNT_OVERFLOW, st.stop_reason, st.error_bits);
          continue;
        }
        ++s.attempts;
        if (!ok) {
          set_terminal(s, BFX_EXPANSION_ENGINE_FAILURE, st.stop_reason, st.error_bits);
          continue;
        }
        if (st.reached_target_mask & bit) {
          set_terminal(s, BFX_EXPANSION_REACHED, st.stop_reason, st.error_bits);
          if (pass == 0) ++m.initial_reached_queries;
          continue;
        }
        failed.push_back(si);
      }
    }
    std::sort(failed.begin(), failed.end());  // state order = query-id order
    active.clear();
    for (u32 si : failed) {
      if (advance_failed(geo, count, full, o, states[si], m)) active.push_back(si);
    }
    if (!active.empty()) ++pass;
  }

  u32 largest = 0;
  out->outcomes.resize(nq);
  out->final_tiles.resize(nq);
  for (u32 i = 0; i < nq; ++i) {
    State& s = states[i];
    if (!s.terminal) throw std::logic_error("batched expansion omitted a terminal query outcome");
    bfx_expansion_outcome& r = out->outcomes[i];
    r.query_id = s.query_id;
    r.disposition = s.disposition;
    r.attempts = s.attempts;
    r.scheduled_expansions = s.scheduled;
    r.total_expansions = s.total;
    r.used_full_region_fallback = s.fallback ? 1u : 0u;
    r.expansion_generation = s.generation;
    r.final_tile_count = static_cast<u32>(s.tiles.size());
    r.selected_vertex_count = region.vertices(s.tiles);
    r.selected_edge_count = count.edges(s.tiles);
    r.terminal_stop_reason = s.stop_reason;
    r.terminal_error_bits = s.error_bits;
    largest = std::max(largest, s.total);
    switch (s.disposition) {
      case BFX_EXPANSION_REACHED: ++m.reached_queries; break;
      case BFX_EXPANSION_UNREACHABLE_IN_FULL_REGION: ++m.unreachable_full_region_queries; break;
      case BFX_EXPANSION_LIMIT: ++m.expansion_limit_queries; break;
      case BFX_EXPANSION_REGION_STALLED: ++m.stalled_region_queries; break;
      case BFX_EXPANSION_IDENTITY_OR_COUNT_OVERFLOW: ++m.identity_or_count_overflow_queries; break;
      default: ++m.engine_failure_queries; break;
    }
    m.final_selected_tile_count += s.tiles.size();
    m.final_selected_vertex_count += r.selected_vertex_count;
    m.final_selected_edge_count += r.selected_edge_count;
    out->final_tiles[i] = std::move(s.tiles);
  }
  out->histogram.assign(size_t{largest} + 1u, 0u);
  for (const auto& r : out->outcomes) ++out->histogram[r.total_expansions];
  return out;
}

struct GpuRunner {
  bfx_workspace* ws;
  const bfx_gpu_run_options* options;
  u64 launches{};
};

int gpu_runner(void* user, u32 count, const bfx_batch_description* batches, bfx_device_run_status* statuses) {
  auto* r = static_cast<GpuRunner*>(user);
  if (bfx_prepare_batches(r->ws, count, batches) != BFX_OK) return 1;
  if (bfx_execute(r->ws, r->options) != BFX_OK) return 1;
  if (bfx_fetch_statuses(r->ws, statuses, nullptr) != BFX_OK) return 1;
  ++r->launches;
  return 0;
}

const ExpansionResult& result_ref(const bfx_expansion_result* r) {
  require(r != nullptr, "null expansion result");
  return *reinterpret_cast<const ExpansionResult*>(r);
}

}  // namespace
}  // namespace bfx

extern "C" {

int bfx_expansion_run(bfx_workspace* ws, const bfx_device_graph_layout32* layout, const bfx_tile_geometry* tiles,
                      uint32_t query_count, const bfx_route_query* queries, const bfx_expansion_options* options,
                      bfx_expansion_result** out) {
  return bfx::guarded([&] {
    bfx::require(ws && layout && tiles && queries && options && out && query_count > 0, "null argument");
    *out = nullptr;
    bfx::validate(*options, true);
    bfx::GpuRunner r{ws, &options->run_options};
    auto res = bfx::run(*layout, *tiles, query_count, queries, *options, bfx::gpu_runner, &r);
    res->metrics.relaxation_launches = r.launches;
    *out = reinterpret_cast<bfx_expansion_result*>(res.release());
  });
}

int bfx_expansion_run_with_runner(const bfx_device_graph_layout32* layout, const bfx_tile_geometry* tiles,
                                  uint32_t query_count, const bfx_route_query* queries,
                                  const bfx_expansion_options* options, bfx_expansion_batch_runner runner,
                                  void* user, bfx_expansion_result** out) {
  return bfx::guarded([&] {
    bfx::require(layout && tiles && queries && options && runner && out && query_count > 0, "null argument");
    *out = nullptr;
    bfx::validate(*options, false);
    auto res = bfx::run(*layout, *tiles, query_count, queries, *options, runner, user);
    *out = reinterpret_cast<bfx_expansion_result*>(res.release());
  });
}

int bfx_expansion_destroy(bfx_expansion_result* result) {
  return bfx::guarded([&] { delete reinterpret_cast<bfx::ExpansionResult*>(result); });
}

int bfx_expansion_outcomes(const bfx_expansion_result* result, bfx_expansion_outcome* outcomes) {
  return bfx::guarded([&] {
    const auto& r = bfx::result_ref(result);
    bfx::require(outcomes != nullptr, "null argument");
    std::memcpy(outcomes, r.outcomes.data(), r.outcomes.size() * sizeof(bfx_expansion_outcome));
  });
}

int bfx_expansion_final_tiles(const bfx_expansion_result* result, uint32_t index, uint32_t* tiles) {
  return bfx::guarded([&] {
    const auto& r = bfx::result_ref(result);
    if (index >= r.final_tiles.size()) throw std::out_of_range("outcome index out of range");
    bfx::require(tiles != nullptr, "null argument");
    std::copy(r.final_tiles[index].begin(), r.final_tiles[index].end(), tiles);
  });
}

int bfx_expansion_metrics_get(const bfx_expansion_result* result, bfx_expansion_metrics* metrics) {
  return bfx::guarded([&] {
    const auto& r = bfx::result_ref(result);
    bfx::require(metrics != nullptr, "null argument");
    *metrics = r.metrics;
  });
}

int bfx_expansion_histogram(const bfx_expansion_result* result, uint32_t* count, uint64_t* histogram) {
  return bfx::guarded([&] {
    const auto& r = bfx::result_ref(result);
    bfx::require(count != nullptr, "null argument");
    *count = static_cast<uint32_t>(r.histogram.size());
    if (histogram) std::copy(r.histogram.begin(), r.histogram.end(), histogram);
  });
}

}  // extern "C"
