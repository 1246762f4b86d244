// Per-batch engine autotuner (a bfx component; the reference's engine
// shootout, src/engine_shootout.cpp, only catalogues configurations).
//
// Five phases, all timed on the device with the library's own CUDA events
// around the relaxation launch (best of `trials`):
//  1. In context: the whole set on frontier push with one near/far step for
//     every batch -- plain, and 1/2, 1, 2, 4, 8, 32, 128 mean edge weights -- as it
//     will run, in one launch; the fastest step wins.  (A batch timed alone
//     favours few rounds; in one launch with others the work matters.)  The
//     step, the phase-4 layout and the phase-5 pack are cached per set
//     class (graph, magnitudes of the batch count per lane width and of the
//     union size), so a later query set of the same class skips those
//     searches.
//  2. Per batch shape: Jacobi pull or dense chaotic push replaces frontier
//     push only where it is at least 1.5x faster on the batch alone.  Cached
//     by batch signature -- lane width, valid lanes, and the binary
//     magnitudes of the union vertex and tile counts.
//  3. In context again: the per-batch engines are kept only if the whole set
//     runs faster with them than all-frontier with the phase-1 step.
//  4. The work mapping (a workspace in the chunked or tiled frontier layout,
//     persistent control): in context, the other of the two layouts at the
//     chosen steps, kept if the whole set runs faster; under the tiled
//     layout, per batch shape, dense rounds as tile visits or as chunk-slot
//     warp items (timed alone, visits only where 1.1x faster; cached by
//     signature), the per-batch mix kept only if the whole set runs faster
//     than all-visits.
//  5. With either of those layouts: in context, 2, 4 or 8 chunk slots per
//     warp item, the fastest kept (cached per set class with the step and
//     the layout).
// The set is left prepared with its per-batch engines, steps and mappings, so
// an execute with engine == BFX_ENGINE_AUTO runs each batch on its own engine
// and mapping inside one launch.
#include "bfx.h"
#include "bfx_host.h"
#include "bfx_internal.hpp"

#include <algorithm>
#include <bit>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <vector>

namespace bfx {
namespace {

using Signature = std::tuple<std::uint32_t, std::uint32_t, std::uint32_t, std::uint32_t>;

struct Choice {
  std::uint32_t engine;
  float delta;  // near/far threshold step for frontier push; +inf = plain
};
constexpr float kPlain = __builtin_inff();

std::mutex g_tune_mutex;
std::map<Signature, Choice> g_tune_cache;
std::map<Signature, std::uint32_t> g_mapping_cache;  // tiled layout: BFX_MAPPING_* per batch shape

// A set's class: the graph (edge count and mean weight bits), and the binary
// magnitudes of the batch count, of the batch counts per lane width and of
// the total union vertices.  Two query sets of one workload fall into one
// class, so the second reuses the first's in-context choices.
using SetKey = std::tuple<std::uint64_t, std::uint32_t, std::uint32_t, std::uint32_t, std::uint32_t, std::uint32_t,
                          std::uint32_t, std::uint32_t, std::uint32_t>;
struct SetChoice {
  float step;           // phase 1
  std::uint32_t layout; // phase 4 (frontier layout kept)
  std::uint32_t pack;   // phase 5 (chunk slots per warp item)
};
std::map<SetKey, SetChoice> g_set_cache;

Signature signature(const bfx_batch_description& d) {
  std::uint64_t U = 0;
  for (std::uint32_t i = 0; i < d.range_count; ++i) U += d.selected_vertex_ranges[i].end - d.selected_vertex_ranges[i].begin;
  const auto log2u = [](std::uint64_t x) { return x ? 63U - static_cast<std::uint32_t>(std::countl_zero(x)) : 0U; };
  return {d.lane_width, static_cast<std::uint32_t>(std::popcount(d.valid_lane_mask)), log2u(U),
          log2u(d.union_tile_count)};
}

void check(int rc) {
  if (rc != BFX_OK) throw Error(rc, bfx_last_error());
}

SetKey set_key(const double stats[2], std::uint32_t count, const bfx_batch_description* batches,
               std::uint32_t layout) {
  const auto log2u = [](std::uint64_t x) { return x ? 64U - static_cast<std::uint32_t>(std::countl_zero(x)) : 0U; };
  std::uint64_t by_width[4] = {0, 0, 0, 0}, union_vertices = 0;
  for (std::uint32_t b = 0; b < count; ++b) {
    const bfx_batch_description& d = batches[b];
    by_width[d.lane_width == 1 ? 0 : d.lane_width == 8 ? 1 : d.lane_width == 16 ? 2 : 3] += 1;
    for (std::uint32_t i = 0; i < d.range_count; ++i) {
      union_vertices += d.selected_vertex_ranges[i].end - d.selected_vertex_ranges[i].begin;
    }
  }
  const float mean = static_cast<float>(stats[0]);
  std::uint32_t mean_bits;
  std::memcpy(&mean_bits, &mean, 4);
  // the chunked and tiled layouts are one family: phase 4 chooses between
  // them whichever the search starts from
  const std::uint32_t family = layout == BFX_FRONTIER_TILED ? static_cast<std::uint32_t>(BFX_FRONTIER_CHUNKED) : layout;
  return {static_cast<std::uint64_t>(stats[1]) << 32 | mean_bits, log2u(count), log2u(by_width[0]),
          log2u(by_width[1]), log2u(by_width[2]), log2u(by_width[3]), log2u(union_vertices), family, 0U};
}

}  // namespace
}  // namespace bfx

namespace bfx {
namespace {

// Best-of-`trials` relaxation time of the prepared set with `o`.
float time_set(bfx_workspace* ws, const bfx_gpu_run_options& o, std::uint32_t trials) {
  float best = 0.0f;
  for (std::uint32_t t = 0; t < trials; ++t) {
    check(bfx_execute(ws, &o));
    float ms[2];
    check(bfx_last_execute_timing(ws, ms));
    if (t == 0 || ms[0] < best) best = ms[0];
  }
  return best;
}

}  // namespace
}  // namespace bfx

extern "C" int bfx_autotune(bfx_workspace* ws, uint32_t count, const bfx_batch_description* batches,
                            const bfx_gpu_run_options* base, uint32_t trials, uint32_t* engines_out,
                            float* deltas_out, uint32_t* measured) {
  using bfx::Choice;
  using bfx::kPlain;
  return bfx::guarded([&] {
    bfx::require(ws && batches && base && engines_out && count > 0, "null argument");
    if (trials == 0) trials = 1;
    double stats[2];
    bfx::check(bfx_workspace_graph_stats(ws, stats));
    const float w = stats[0] > 0.0 ? static_cast<float>(stats[0]) : 1.0f;
    bfx_gpu_run_options o;
    std::memcpy(&o, base, sizeof(o));
    o.instrumentation = 0;

    // Phase 1, in context: every batch on frontier push with one step, the
    // whole set relaxed together as it will run; keep the fastest step.  A
    // set of a class tuned before reuses that class's step (timed once).
    std::uint32_t layout0 = 0;
    bfx::check(bfx_get_frontier_mapping(ws, &layout0, 0, nullptr));
    const bfx::SetKey key = bfx::set_key(stats, count, batches, layout0);
    bool set_cached = false;
    bfx::SetChoice set_choice{kPlain, layout0, 4U};
    {
      std::lock_guard<std::mutex> lock(bfx::g_tune_mutex);
      const auto it = bfx::g_set_cache.find(key);
      if (it != bfx::g_set_cache.end()) {
        set_cached = true;
        set_choice = it->second;
      }
    }
    const float steps[] = {kPlain, 0.5f * w, 1.0f * w, 2.0f * w, 4.0f * w, 8.0f * w, 32.0f * w, 128.0f * w};
    bfx::check(bfx_prepare_batches(ws, count, batches));
    o.engine = BFX_ENGINE_FRONTIER_PUSH;
    float best_step = kPlain, best_set = 0.0f;
    if (set_cached) {
      best_step = set_choice.step;
      const std::vector<float> d(count, best_step);
      bfx::check(bfx_set_batch_deltas(ws, count, d.data()));
      best_set = bfx::time_set(ws, o, trials);
    } else {
      for (std::size_t i = 0; i < sizeof(steps) / sizeof(steps[0]); ++i) {
        const std::vector<float> d(count, steps[i]);
        bfx::check(bfx_set_batch_deltas(ws, count, d.data()));
        const float t = bfx::time_set(ws, o, trials);
        if (i == 0 || t < best_set) {
          best_set = t;
          best_step = steps[i];
        }
      }
    }

    // Phase 2, per batch shape: Jacobi pull or dense push replaces frontier
    // push (with the chosen step) only where it is at least 1.5x faster on
    // the batch alone; choices are cached by batch signature.
    const Choice frontier{BFX_ENGINE_FRONTIER_PUSH, best_step};
    const Choice candidates[] = {frontier, {BFX_ENGINE_JACOBI_PULL, kPlain}, {BFX_ENGINE_DENSE_CHAOTIC_PUSH, kPlain}};
    std::vector<Choice> chosen(count, frontier);
    std::uint32_t n_measured = 0;
    for (std::uint32_t b = 0; b < count; ++b) {
      const bfx::Signature sig = bfx::signature(batches[b]);
      {
        std::lock_guard<std::mutex> lock(bfx::g_tune_mutex);
        const auto it = bfx::g_tune_cache.find(sig);
        if (it != bfx::g_tune_cache.end()) {
          chosen[b] = it->second.engine == BFX_ENGINE_FRONTIER_PUSH ? frontier : it->second;
          continue;
        }
      }
      bfx::check(bfx_prepare_batches(ws, 1, &batches[b]));
      float t_frontier = 0.0f, best = 0.0f;
      Choice pick = frontier;
      for (const Choice& c : candidates) {
        bfx::check(bfx_set_batch_deltas(ws, 1, &c.delta));
        bfx_gpu_run_options oc = o;
        oc.engine = c.engine;
        const float t = bfx::time_set(ws, oc, trials);
        if (c.engine == BFX_ENGINE_FRONTIER_PUSH) {
          t_frontier = best = t;
        } else if (t * 1.5f <= t_frontier && t < best) {
          best = t;
          pick = c;
        }
      }
      chosen[b] = pick;
      ++n_measured;
      std::lock_guard<std::mutex> lock(bfx::g_tune_mutex);
      bfx::g_tune_cache[sig] = pick;
    }

    // Phase 3, in context: keep the per-batch engines only if the whole set
    // runs faster with them than all-frontier with the chosen step.
    std::vector<std::uint32_t> engines(count);
    std::vector<float> deltas(count);
    for (std::uint32_t b = 0; b < count; ++b) {
      engines[b] = chosen[b].engine;
      deltas[b] = chosen[b].delta;
    }
    bfx::check(bfx_prepare_batches(ws, count, batches));
    bool mixed = false;
    for (std::uint32_t e : engines) mixed = mixed || e != BFX_ENGINE_FRONTIER_PUSH;
    if (mixed) {
      bfx::check(bfx_set_batch_engines(ws, count, engines.data()));
      bfx::check(bfx_set_batch_deltas(ws, count, deltas.data()));
      bfx_gpu_run_options oa = o;
      oa.engine = BFX_ENGINE_AUTO;
      if (bfx::time_set(ws, oa, trials) >= best_set) {
        std::fill(engines.begin(), engines.end(), static_cast<std::uint32_t>(BFX_ENGINE_FRONTIER_PUSH));
        std::fill(deltas.begin(), deltas.end(), best_step);
      }
    }
    for (std::uint32_t b = 0; b < count; ++b) {
      engines_out[b] = engines[b];
      if (deltas_out) deltas_out[b] = deltas[b];
    }
    bfx::check(bfx_set_batch_engines(ws, count, engines.data()));
    bfx::check(bfx_set_batch_deltas(ws, count, deltas.data()));

    // Phase 4: the work mapping.
    std::uint32_t layout = 0, pack = 0;
    bfx::check(bfx_get_frontier_mapping(ws, &layout, 0, nullptr));
    bfx::check(bfx_get_chunk_pack(ws, &pack));
    if ((layout == BFX_FRONTIER_CHUNKED || layout == BFX_FRONTIER_TILED) &&
        o.control_mode == BFX_CONTROL_PERSISTENT_COOPERATIVE && (o.block_size == 256 || o.block_size == 384)) {
      bfx_gpu_run_options oa = o;
      oa.engine = BFX_ENGINE_AUTO;
      bfx::check(bfx_set_batch_mappings(ws, 0, nullptr));
      float t_visits = 0.0f;
      if (set_cached) {
        // the class's layout, timed once (the baseline of the mapping mix)
        layout = set_choice.layout;
        bfx::check(bfx_set_frontier_layout(ws, layout));
        if (layout == BFX_FRONTIER_TILED) t_visits = bfx::time_set(ws, oa, trials);
      } else {
        const float t_here = bfx::time_set(ws, oa, trials);
        const std::uint32_t other = layout == BFX_FRONTIER_CHUNKED ? BFX_FRONTIER_TILED : BFX_FRONTIER_CHUNKED;
        bfx::check(bfx_set_frontier_layout(ws, other));
        const float t_other = bfx::time_set(ws, oa, trials);
        if (t_other < t_here) {
          layout = other;
        } else {
          bfx::check(bfx_set_frontier_layout(ws, layout));
        }
        t_visits = std::min(t_here, t_other);
      }
      if (layout == BFX_FRONTIER_TILED) {
        std::vector<std::uint32_t> mappings(count, BFX_MAPPING_TILE_VISITS);
        bool any_chunks = false;
        for (std::uint32_t b = 0; b < count; ++b) {
          if (engines[b] != BFX_ENGINE_FRONTIER_PUSH) continue;
          const bfx::Signature sig = bfx::signature(batches[b]);
          {
            std::lock_guard<std::mutex> lock(bfx::g_tune_mutex);
            const auto it = bfx::g_mapping_cache.find(sig);
            if (it != bfx::g_mapping_cache.end()) {
              mappings[b] = it->second;
              any_chunks |= it->second == BFX_MAPPING_CHUNKS;
              continue;
            }
          }
          bfx::check(bfx_prepare_batches(ws, 1, &batches[b]));
          bfx::check(bfx_set_batch_deltas(ws, 1, &deltas[b]));
          bfx_gpu_run_options of = o;
          of.engine = BFX_ENGINE_FRONTIER_PUSH;
          const std::uint32_t visit = BFX_MAPPING_TILE_VISITS, chunks = BFX_MAPPING_CHUNKS;
          bfx::check(bfx_set_batch_mappings(ws, 1, &visit));
          const float tv = bfx::time_set(ws, of, trials);
          bfx::check(bfx_set_batch_mappings(ws, 1, &chunks));
          const float tc = bfx::time_set(ws, of, trials);
          mappings[b] = tv * 1.1f <= tc ? BFX_MAPPING_TILE_VISITS : BFX_MAPPING_CHUNKS;
          any_chunks |= mappings[b] == BFX_MAPPING_CHUNKS;
          ++n_measured;
          std::lock_guard<std::mutex> lock(bfx::g_tune_mutex);
          bfx::g_mapping_cache[sig] = mappings[b];
        }
        bfx::check(bfx_prepare_batches(ws, count, batches));
        bfx::check(bfx_set_batch_engines(ws, count, engines.data()));
        bfx::check(bfx_set_batch_deltas(ws, count, deltas.data()));
        bfx::check(bfx_set_batch_mappings(ws, 0, nullptr));
        if (any_chunks) {
          bfx::check(bfx_set_batch_mappings(ws, count, mappings.data()));
          if (bfx::time_set(ws, oa, trials) >= t_visits) bfx::check(bfx_set_batch_mappings(ws, 0, nullptr));
        }
      }
      // Phase 5, in context: chunk slots per warp item, 2, 4 or 8 (the
      // class's choice when cached).
      if (set_cached) {
        pack = set_choice.pack;
        bfx::check(bfx_set_chunk_pack(ws, pack));
      } else {
        float t_best = bfx::time_set(ws, oa, trials);
        for (const std::uint32_t k : {2U, 4U, 8U}) {
          if (k == pack) continue;
          bfx::check(bfx_set_chunk_pack(ws, k));
          const float t = bfx::time_set(ws, oa, trials);
          if (t < t_best) {
            t_best = t;
            pack = k;
          }
        }
        bfx::check(bfx_set_chunk_pack(ws, pack));
      }
    }
    {
      std::lock_guard<std::mutex> lock(bfx::g_tune_mutex);
      bfx::g_set_cache[key] = bfx::SetChoice{best_step, layout, pack};
    }
    if (measured) *measured = n_measured;
  });
}

extern "C" int bfx_autotune_reset(void) {
  return bfx::guarded([&] {
    std::lock_guard<std::mutex> lock(bfx::g_tune_mutex);
    bfx::g_tune_cache.clear();
    bfx::g_mapping_cache.clear();
    bfx::g_set_cache.clear();
  });
}

extern "C" int bfx_autotune_policy(bfx_workspace* ws, const bfx_device_graph_layout32* layout,
                                   const uint32_t* tile_vertex_offsets, uint32_t query_count,
                                   const bfx_route_query* queries, uint32_t policy_count,
                                   const bfx_planner_policy* policies, const bfx_gpu_run_options* base,
                                   uint32_t trials, uint32_t* best, float* times_ms) {
  return bfx::guarded([&] {
    bfx::require(ws && layout && tile_vertex_offsets && queries && policies && base && best && query_count > 0 &&
                     policy_count > 0,
                 "null argument");
    if (trials == 0) trials = 1;
    bfx_gpu_run_options o;
    std::memcpy(&o, base, sizeof(o));
    o.instrumentation = 0;
    o.engine = BFX_ENGINE_AUTO;
    std::uint32_t best_i = 0;
    float best_t = 0.0f;
    // One candidate: plan, tune (engines and steps), time the whole set.
    const auto measure = [&](std::uint32_t i) -> float {
      bfx_plan* plan = nullptr;
      bfx::check(bfx_plan_build(layout, tile_vertex_offsets, query_count, queries, &policies[i], &plan));
      std::unique_ptr<bfx_plan, int (*)(bfx_plan*)> owner(plan, bfx_plan_destroy);
      std::uint32_t n = 0;
      bfx::check(bfx_plan_batch_count(plan, &n));
      const bfx_batch_description* descs = nullptr;
      bfx::check(bfx_plan_descriptions(plan, &descs));
      std::vector<std::uint32_t> engines(n);
      std::vector<float> deltas(n);
      bfx::check(bfx_autotune(ws, n, descs, base, trials, engines.data(), deltas.data(), nullptr));
      return bfx::time_set(ws, o, trials);
    };
    for (std::uint32_t i = 0; i < policy_count; ++i) {
      const float t = measure(i);
      if (times_ms) times_ms[i] = t;
      if (i == 0 || t < best_t) {
        best_t = t;
        best_i = i;
      }
    }
    // leave the workspace prepared and tuned with the winner (the engine
    // cache makes the second tuning pass cheap)
    if (best_i != policy_count - 1u) (void)measure(best_i);
    *best = best_i;
  });
}
