// Per-batch engine autotuner (a bfx component; the reference's engine
// shootout, src/engine_shootout.cpp, only catalogues configurations).
//
// For every batch of a set, the tuner runs the candidate configurations --
// frontier push (plain, and near/far with threshold steps of 1/2, 1, 2, 4, 8
// and 32 mean edge weights), Jacobi pull, dense chaotic push -- on that batch alone
// and keeps the fastest by device time (the library's own CUDA events around
// the relaxation launch, best of `trials`).  Choices are cached per batch
// signature -- lane width, valid lanes, and the binary magnitudes of the
// union vertex count and union tile count -- so later sets with batches of
// the same shape are tuned without measuring.  The set is prepared again at
// the end and its per-batch engines and steps are stored in the workspace, so an
// execute with engine == BFX_ENGINE_AUTO runs each batch on its own engine
// inside one launch.
#include "bfx.h"
#include "bfx_internal.hpp"

#include <algorithm>
#include <bit>
#include <cstring>
#include <map>
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
    // Candidates: the three engines; frontier push also with near/far
    // threshold steps of 1/2, 1, 2, 4, 8 and 32 mean edge weights.
    const Choice candidates[] = {{BFX_ENGINE_FRONTIER_PUSH, kPlain},       {BFX_ENGINE_FRONTIER_PUSH, 0.5f * w},
                                 {BFX_ENGINE_FRONTIER_PUSH, 1.0f * w},     {BFX_ENGINE_FRONTIER_PUSH, 2.0f * w},
                                 {BFX_ENGINE_FRONTIER_PUSH, 4.0f * w},     {BFX_ENGINE_FRONTIER_PUSH, 8.0f * w},
                                 {BFX_ENGINE_FRONTIER_PUSH, 32.0f * w},    {BFX_ENGINE_JACOBI_PULL, kPlain},
                                 {BFX_ENGINE_DENSE_CHAOTIC_PUSH, kPlain}};
    std::vector<Choice> chosen(count, Choice{BFX_ENGINE_FRONTIER_PUSH, kPlain});
    std::uint32_t n_measured = 0;
    for (std::uint32_t b = 0; b < count; ++b) {
      const bfx::Signature sig = bfx::signature(batches[b]);
      {
        std::lock_guard<std::mutex> lock(bfx::g_tune_mutex);
        const auto it = bfx::g_tune_cache.find(sig);
        if (it != bfx::g_tune_cache.end()) {
          chosen[b] = it->second;
          continue;
        }
      }
      bfx::check(bfx_prepare_batches(ws, 1, &batches[b]));
      float best = 0.0f;
      Choice best_choice{BFX_ENGINE_FRONTIER_PUSH, kPlain};
      bool have = false;
      for (const Choice& c : candidates) {
        bfx_gpu_run_options o;
        std::memcpy(&o, base, sizeof(o));
        o.engine = c.engine;
        o.instrumentation = 0;
        bfx::check(bfx_set_batch_deltas(ws, 1, &c.delta));
        float t_best = 0.0f;
        for (std::uint32_t t = 0; t < trials; ++t) {
          bfx::check(bfx_execute(ws, &o));
          float ms[2];
          bfx::check(bfx_last_execute_timing(ws, ms));
          if (t == 0 || ms[0] < t_best) t_best = ms[0];
        }
        if (!have || t_best < best) {
          best = t_best;
          best_choice = c;
          have = true;
        }
      }
      chosen[b] = best_choice;
      ++n_measured;
      std::lock_guard<std::mutex> lock(bfx::g_tune_mutex);
      bfx::g_tune_cache[sig] = best_choice;
    }
    bfx::check(bfx_prepare_batches(ws, count, batches));
    std::vector<std::uint32_t> engines(count);
    std::vector<float> deltas(count);
    for (std::uint32_t b = 0; b < count; ++b) {
      engines[b] = chosen[b].engine;
      deltas[b] = chosen[b].delta;
      engines_out[b] = chosen[b].engine;
      if (deltas_out) deltas_out[b] = chosen[b].delta;
    }
    bfx::check(bfx_set_batch_engines(ws, count, engines.data()));
    bfx::check(bfx_set_batch_deltas(ws, count, deltas.data()));
    if (measured) *measured = n_measured;
  });
}

extern "C" int bfx_autotune_reset(void) {
  return bfx::guarded([&] {
    std::lock_guard<std::mutex> lock(bfx::g_tune_mutex);
    bfx::g_tune_cache.clear();
  });
}
