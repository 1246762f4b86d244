// Compact path reconstruction on the device (the reference's
// ReusableCompactPathWorkspace::reconstruct, include/bfnew/hip/compact_path_results.hpp:99-127,
// whose kernel runs one serial depth-first search for every target on a
// single thread, src/hip/compact_path_results.hip.cpp:251-271).
//
// The relaxation labels already carry, per (vertex, lane), the smallest
// stable edge id among tight admitted in-edges -- the first candidate of the
// reference's search (tight_choices, src/compact_paths.cpp:98-129).  So a
// target's path is found by one thread walking predecessors, all targets of
// all lanes in parallel.  The walk equals the reference's search whenever it
// never revisits a vertex; a revisit needs an equal-distance (zero-weight)
// step, so the walk tracks runs of equal distances and hands a target to the
// exact backtracking search (reconstruct_target, src/compact_paths.cpp:131-211)
// when a run revisits a vertex or grows long.  Flagged targets are gathered
// into a list and searched in parallel, one thread per target over a bounded
// number of search slots (each with its own stacks and on-path marks sized by
// the largest union).
//
// Two passes as in the reference: summaries (status, source, distance,
// length), then, after a host prefix over the lengths, the payload (path
// vertices source-first, their labels, stable edge ids).
#include "bfx.h"
#include "bfx_internal.hpp"
#include "device_common.cuh"
#include "engine_types.cuh"

#include <cuda_runtime.h>

#include <cstring>
#include <vector>

namespace bfx {
namespace {

constexpr u32 kPlateau = 16;  // equal-distance run the walk checks itself
constexpr u32 kFallback = 0x80000000u;

struct PathArgs {
  DGraph g;
  const DBatch* batches;
  const bfx_device_run_status* status;
  u32 first_batch, batch_count;
  const u32* target_base;  // [batch_count+1] prefix of target counts
  bfx_compact_target_summary* summaries;
  u32* lengths;            // walk result | kFallback
  const u64* vertex_offsets;  // payload pass
  const u64* edge_offsets;
  u32* out_vertices;
  float* out_labels;
  u32* out_edges;
  // search scratch: `slots` search slots, each with its own stacks
  // (slot_stride words apart) and on-path bitmap (mark_stride words apart)
  u32* stack_v;
  u32* stack_c;
  u32* stack_e;
  u32* on_path;  // bitmap over compact vertices
  u32 max_union;
  u32 slots;
  u64 slot_stride;
  u64 mark_stride;
  u32* flagged;        // [targets] indices of the targets the walk handed over
  u32* flagged_count;  // [1]
};

__device__ __forceinline__ u32 lane_of(const u32* offsets, u32 W, u32 pos) {
  u32 lo = 0, hi = W;
  while (hi - lo > 1u) {
    const u32 mid = (lo + hi) >> 1;
    if (offsets[mid] <= pos) lo = mid; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ u32 find_b(const u32* prefix, u32 n, u32 x) {
  u32 lo = 0, hi = n;
  while (hi - lo > 1u) {
    const u32 mid = (lo + hi) >> 1;
    if (prefix[mid] <= x) lo = mid; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ u64 label(const DGraph& g, const DBatch& B, const u64* d, u32 v, u32 lane) {
  const uint2 t = B.tiles[g.owner[v]];
  if (((t.x >> lane) & 1u) == 0u) return dev::kUnreached;
  return d[(static_cast<u64>(v - t.y) << B.shift) + lane];
}

__device__ __forceinline__ bool clean(const bfx_device_run_status& s) {
  return s.stop_reason == BFX_STOP_CONVERGED && s.error_bits == 0u;
}

// Pass 1: one thread per target of the selected batches.
__global__ void summaries_kernel(PathArgs a) {
  const u32 total = a.target_base[a.batch_count];
  for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    const u32 bi = find_b(a.target_base, a.batch_count, i);
    const u32 b = a.first_batch + bi;
    const DBatch& B = a.batches[b];
    const bfx_device_run_status& st = a.status[b];
    const u32 pos = i - a.target_base[bi];
    const u32 lane = lane_of(B.tgt_off, B.W, pos);
    const u32 t = B.tgt[pos];
    bfx_compact_target_summary s;
    s.target = t;
    s.selected_source = 0u;
    s.distance = __uint_as_float(dev::kInfBits);
    s.path_length = 0u;
    s.reached = 0u;
    s.reconstruction = 2u;  // query_terminal_failure
    s.has_selected_source = 0u;
    u32 len = 0u;
    if (clean(st)) {
      const u64* d = B.dist[st.final_distance_slot];
      u64 w = label(a.g, B, d, t, lane);
      if (dev::hi(w) == dev::kInfBits) {
        s.reconstruction = 1u;  // unreachable
      } else {
        s.reached = 1u;
        s.distance = __uint_as_float(dev::hi(w));
        u32 v = t, pn = 0;
        u32 plateau[kPlateau];
        bool fallback = false;
        while (static_cast<u32>(w) != 0u) {
          const u32 e = static_cast<u32>(w) - 1u;
          if (e >= a.g.E) {
            fallback = true;
            break;
          }
          const u32 u = a.g.eid_src[e];
          const u64 wu = label(a.g, B, d, u, lane);
          if (dev::hi(wu) == dev::kInfBits) {  // inconsistent chain: let the search decide
            fallback = true;
            break;
          }
          if (dev::hi(wu) == dev::hi(w)) {
            if (pn == 0u) plateau[pn++] = v;
            for (u32 k = 0; k < pn; ++k) fallback |= plateau[k] == u;
            if (fallback || pn == kPlateau) {
              fallback = true;
              break;
            }
            plateau[pn++] = u;
          } else {
            pn = 0u;
          }
          ++len;
          if (len > B.U) {
            fallback = true;
            break;
          }
          v = u;
          w = wu;
        }
        if (fallback) {
          len = kFallback;
        } else {
          s.reconstruction = 0u;  // complete
          s.path_length = len;
          s.selected_source = v;
          s.has_selected_source = 1u;
        }
      }
    }
    a.lengths[i] = len;
    a.summaries[i] = s;
  }
}

// The reference's backtracking search for one target (reconstruct_target):
// candidates in stable-edge-id order, predecessors on the current path
// skipped, dead ends popped.  Returns the edge count (or ~0u if no path) and
// leaves the path on the stacks (stack_v[0] = target).
struct SearchSlot {
  u32* stack_v;
  u32* stack_c;
  u32* stack_e;
  u32* on_path;
};

__device__ __forceinline__ SearchSlot search_slot(const PathArgs& a, u32 slot) {
  return SearchSlot{a.stack_v + slot * a.slot_stride, a.stack_c + slot * a.slot_stride,
                    a.stack_e + slot * a.slot_stride, a.on_path + slot * a.mark_stride};
}

__device__ u32 search_target(const PathArgs& a, const SearchSlot& sl, const DBatch& B, const u64* d, u32 t,
                             u32 lane) {
  auto cv = [&](u32 v) { return v - B.tiles[a.g.owner[v]].y; };
  auto mark = [&](u32 v, bool on) {
    const u32 c = cv(v);
    if (on) sl.on_path[c >> 5] |= 1u << (c & 31u); else sl.on_path[c >> 5] &= ~(1u << (c & 31u));
  };
  auto marked = [&](u32 v) {
    const u32 c = cv(v);
    return (sl.on_path[c >> 5] >> (c & 31u)) & 1u;
  };
  int depth = 0;
  sl.stack_v[0] = t;
  sl.stack_c[0] = 0u;
  mark(t, true);
  u32 found = 0xFFFFFFFFu;
  while (depth >= 0) {
    const u32 v = sl.stack_v[depth];
    const u64 wv = label(a.g, B, d, v, lane);
    if (static_cast<u32>(wv) == 0u) {  // a source of this lane
      found = static_cast<u32>(depth);
      break;
    }
    const u32 dv = dev::hi(wv);
    u32 best = 0xFFFFFFFFu, bu = 0u;
    for (u32 q = a.g.csc_off[v]; q < a.g.csc_off[v + 1]; ++q) {
      const uint4 rec = a.g.csc[q];
      if (rec.z <= sl.stack_c[depth] || rec.z >= best) continue;
      const uint2 su = B.tiles[rec.w];
      if (((su.x >> lane) & 1u) == 0u) continue;
      const u32 du = dev::hi(d[(static_cast<u64>(rec.x - su.y) << B.shift) + lane]);
      if (du == dev::kInfBits) continue;
      if (__float_as_uint(__fadd_rn(__uint_as_float(du), __uint_as_float(rec.y))) != dv) continue;
      best = rec.z;
      bu = rec.x;
    }
    if (best == 0xFFFFFFFFu) {
      mark(v, false);
      --depth;
      continue;
    }
    sl.stack_c[depth] = best;
    if (marked(bu)) continue;
    ++depth;
    sl.stack_v[depth] = bu;
    sl.stack_c[depth] = 0u;
    sl.stack_e[depth] = best - 1u;
    mark(bu, true);
  }
  // clear the marks of the path that remained (popped vertices are clear)
  if (found != 0xFFFFFFFFu) {
    for (u32 k = 0; k <= found; ++k) mark(sl.stack_v[k], false);
  }
  return found;
}

// Gathers the indices of the targets the walk handed to the search.
__global__ void flag_list_kernel(PathArgs a) {
  const u32 total = a.target_base[a.batch_count];
  for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    if ((a.lengths[i] & kFallback) != 0u) a.flagged[atomicAdd(a.flagged_count, 1u)] = i;
  }
}

// The flagged targets (rare: zero-weight ties that revisit), one thread per
// target over `slots` search slots; each target's result depends only on
// the labels, so the order is free.  payload == false: fill summaries;
// true: write the payload.
__global__ void search_kernel(PathArgs a, bool payload) {
  const u32 slot = blockIdx.x * blockDim.x + threadIdx.x;
  if (slot >= a.slots) return;
  const SearchSlot sl = search_slot(a, slot);
  const u32 count = *a.flagged_count;
  for (u32 k = slot; k < count; k += a.slots) {
    const u32 i = a.flagged[k];
    const u32 bi = find_b(a.target_base, a.batch_count, i);
    const u32 b = a.first_batch + bi;
    const DBatch& B = a.batches[b];
    const u32 pos = i - a.target_base[bi];
    const u32 lane = lane_of(B.tgt_off, B.W, pos);
    const u64* d = B.dist[a.status[b].final_distance_slot];
    const u32 n = search_target(a, sl, B, d, B.tgt[pos], lane);
    if (!payload) {
      bfx_compact_target_summary& s = a.summaries[i];
      if (n == 0xFFFFFFFFu) {
        s.reconstruction = 3u;  // no_tight_path
      } else {
        s.reconstruction = 0u;
        s.path_length = n;
        s.selected_source = sl.stack_v[n];
        s.has_selected_source = 1u;
      }
    } else if (n != 0xFFFFFFFFu) {
      const u64 vo = a.vertex_offsets[i], eo = a.edge_offsets[i];
      for (u32 j = 0; j <= n; ++j) {
        const u32 v = sl.stack_v[n - j];
        a.out_vertices[vo + j] = v;
        a.out_labels[vo + j] = __uint_as_float(dev::hi(label(a.g, B, d, v, lane)));
        if (j < n) a.out_edges[eo + j] = sl.stack_e[n - j];
      }
    }
  }
}

// Pass 2: one thread per complete, walkable target writes its payload.
__global__ void payload_kernel(PathArgs a) {
  const u32 total = a.target_base[a.batch_count];
  for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    const u32 len = a.lengths[i];
    if ((len & kFallback) != 0u || a.summaries[i].reconstruction != 0u) continue;
    const u32 bi = find_b(a.target_base, a.batch_count, i);
    const u32 b = a.first_batch + bi;
    const DBatch& B = a.batches[b];
    const u32 pos = i - a.target_base[bi];
    const u32 lane = lane_of(B.tgt_off, B.W, pos);
    const u64* d = B.dist[a.status[b].final_distance_slot];
    const u64 vo = a.vertex_offsets[i], eo = a.edge_offsets[i];
    u32 v = B.tgt[pos];
    u64 w = label(a.g, B, d, v, lane);
    for (u32 k = 0;; ++k) {
      a.out_vertices[vo + len - k] = v;
      a.out_labels[vo + len - k] = __uint_as_float(dev::hi(w));
      if (k == len) break;
      const u32 e = static_cast<u32>(w) - 1u;
      a.out_edges[eo + len - 1u - k] = e;
      v = a.g.eid_src[e];
      w = label(a.g, B, d, v, lane);
    }
  }
}

// ---------------------------------------------------------------------------
// Edge-usage adjoint (no reference counterpart).  For L = sum_t g_t * d_t over
// the targets' shortest paths, dL/dw_e = sum of g_t over the targets whose
// path uses edge e.  Paths are recomputed from the final labels (predecessor
// walk, or the backtracking search for flagged targets); nothing per round is
// stored.  Contributions are summed exactly in per-edge fixed point (least
// significant bit 2^-63, four 32-bit digits in 64-bit atomics) and rounded
// once to float (nearest, ties to even), so the result does not depend on
// the order in which threads add -- and equals an exact CPU tree walk.
// Accepted upstream values: 0 or 2^-40 <= |g| < 2^40 (checked on the host).
// ---------------------------------------------------------------------------

__device__ __forceinline__ void exact_add(unsigned long long* acc, float g) {
  const u32 bits = __float_as_uint(g);
  const u32 ex = (bits >> 23) & 0xFFu;
  if (ex == 0u) return;
  const u64 m = static_cast<u64>((bits & 0x7FFFFFu) | 0x800000u);  // g = m * 2^(ex-150)
  const u32 b = ex - 87u;                                         // bit of m's lsb at 2^-63
  const u64 v = m << (b & 31u);
  u64 lo = v & 0xFFFFFFFFull, hi = v >> 32;
  if (bits >> 31) {
    lo = 0ull - lo;
    hi = 0ull - hi;
  }
  atomicAdd(acc + (b >> 5), lo);
  if (hi != 0ull) atomicAdd(acc + (b >> 5) + 1u, hi);
}

__device__ float exact_round(const unsigned long long* acc) {
  long long carry = 0;
  u32 dig[4];
  for (int d = 0; d < 4; ++d) {
    const long long x = static_cast<long long>(acc[d]) + carry;
    dig[d] = static_cast<u32>(x);
    carry = x >> 32;
  }
  const bool neg = carry < 0;
  u64 lo = (static_cast<u64>(dig[1]) << 32) | dig[0];
  u64 hi = (static_cast<u64>(dig[3]) << 32) | dig[2];
  if (neg) {
    lo = ~lo + 1ull;
    hi = ~hi + (lo == 0ull ? 1ull : 0ull);
  }
  if (hi == 0ull && lo == 0ull) return 0.0f;
  const int p = hi ? 127 - __clzll(static_cast<long long>(hi)) : 63 - __clzll(static_cast<long long>(lo));
  u64 mant;
  int shift = 0;
  if (p <= 23) {
    mant = lo;
  } else {
    shift = p - 23;
    // mant = bits [shift, shift + 24); guard = bit shift - 1; sticky = bits below.
    auto bit_range = [&](int from, int count) -> u64 {  // count <= 64
      u64 r;
      if (from >= 64) {
        r = hi >> (from - 64);
      } else if (from == 0) {
        r = lo;
      } else {
        r = (lo >> from) | (hi << (64 - from));
      }
      return count >= 64 ? r : (r & ((1ull << count) - 1ull));
    };
    mant = bit_range(shift, 24);
    const u64 guard = bit_range(shift - 1, 1);
    bool sticky = false;
    if (shift - 1 > 0) {
      const int n = shift - 1;
      sticky = n >= 64 ? (lo != 0ull || (hi & ((1ull << (n - 64)) - 1ull)) != 0ull)
                       : (lo & ((1ull << n) - 1ull)) != 0ull;
    }
    if (guard && (sticky || (mant & 1ull))) {
      ++mant;
      if (mant == (1ull << 24)) {
        mant >>= 1;
        ++shift;
      }
    }
  }
  const float r = ldexpf(static_cast<float>(mant), shift - 63);
  return neg ? -r : r;
}

__global__ void adjoint_walk_kernel(PathArgs a, const float* grads, unsigned long long* acc) {
  const u32 total = a.target_base[a.batch_count];
  for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    if ((a.lengths[i] & kFallback) != 0u || a.summaries[i].reconstruction != 0u) continue;
    const float g = grads[i];
    if (g == 0.0f) continue;
    const u32 bi = find_b(a.target_base, a.batch_count, i);
    const u32 b = a.first_batch + bi;
    const DBatch& B = a.batches[b];
    const u32 pos = i - a.target_base[bi];
    const u32 lane = lane_of(B.tgt_off, B.W, pos);
    const u64* d = B.dist[a.status[b].final_distance_slot];
    u64 w = label(a.g, B, d, B.tgt[pos], lane);
    while (static_cast<u32>(w) != 0u) {
      const u32 e = static_cast<u32>(w) - 1u;
      exact_add(acc + 4ull * e, g);
      w = label(a.g, B, d, a.g.eid_src[e], lane);
    }
  }
}

// The flagged targets' paths by search, one thread per target over the
// search slots (the exact accumulation makes the order free).
__global__ void adjoint_search_kernel(PathArgs a, const float* grads, unsigned long long* acc) {
  const u32 slot = blockIdx.x * blockDim.x + threadIdx.x;
  if (slot >= a.slots) return;
  const SearchSlot sl = search_slot(a, slot);
  const u32 count = *a.flagged_count;
  for (u32 k = slot; k < count; k += a.slots) {
    const u32 i = a.flagged[k];
    if (a.summaries[i].reconstruction != 0u || grads[i] == 0.0f) continue;
    const u32 bi = find_b(a.target_base, a.batch_count, i);
    const u32 b = a.first_batch + bi;
    const DBatch& B = a.batches[b];
    const u32 pos = i - a.target_base[bi];
    const u32 lane = lane_of(B.tgt_off, B.W, pos);
    const u64* d = B.dist[a.status[b].final_distance_slot];
    const u32 n = search_target(a, sl, B, d, B.tgt[pos], lane);
    for (u32 j = 1; j <= n && n != 0xFFFFFFFFu; ++j) exact_add(acc + 4ull * sl.stack_e[j], grads[i]);
  }
}

__global__ void adjoint_round_kernel(u32 E, const unsigned long long* acc, float* grad) {
  for (u32 e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x) {
    grad[e] = exact_round(acc + 4ull * e);
  }
}

void check_ready(bfx_workspace* ws) {
  require(ws != nullptr, "null workspace");
  require(ws->executed, "no executed batches");
}

// Layout of the workspace's path buffer for `targets` targets of
// `batch_count` batches whose largest union has `max_union` vertices:
// target prefix, summaries, walk lengths, payload offsets, the flagged list,
// then the search slots (stacks and on-path bitmaps).  The number of slots is
// what fits a 256 MB scratch budget (at least 1, at most 256).
struct PathLayout {
  size_t o_tb, o_sum, o_len, o_vo, o_eo, o_fl, o_fc, o_sv, o_sc, o_se, o_op, total;
  u32 slots;
  u64 slot_stride, mark_stride;
};

PathLayout path_layout(std::uint64_t T, std::uint32_t batch_count, std::uint32_t max_union) {
  PathLayout L{};
  L.slot_stride = align256((size_t{max_union} + 1) * 4) / 4;
  L.mark_stride = align256((size_t{max_union} / 32 + 1) * 4) / 4;
  const size_t per_slot = 3 * L.slot_stride * 4 + L.mark_stride * 4;
  L.slots = static_cast<u32>(std::max<size_t>(1, std::min<size_t>(256, (size_t{256} << 20) / per_slot)));
  L.o_tb = 0;
  L.o_sum = align256(L.o_tb + (batch_count + 1) * 4);
  L.o_len = align256(L.o_sum + T * sizeof(bfx_compact_target_summary));
  L.o_vo = align256(L.o_len + T * 4);
  L.o_eo = align256(L.o_vo + T * 8);
  L.o_fl = align256(L.o_eo + T * 8);
  L.o_fc = align256(L.o_fl + T * 4);
  L.o_sv = align256(L.o_fc + 4);
  L.o_sc = L.o_sv + size_t{L.slots} * L.slot_stride * 4;
  L.o_se = L.o_sc + size_t{L.slots} * L.slot_stride * 4;
  L.o_op = L.o_se + size_t{L.slots} * L.slot_stride * 4;
  L.total = align256(L.o_op + size_t{L.slots} * L.mark_stride * 4);
  return L;
}

PathArgs path_args_at(bfx_workspace* ws, const PathLayout& L, std::uint32_t first_batch, std::uint32_t batch_count,
                      std::uint32_t max_union) {
  char* base = static_cast<char*>(ws->paths.ptr);
  PathArgs a{};
  a.g = ws->graph->g;
  a.batches = ws->params.batches;
  a.status = ws->d_status;
  a.first_batch = first_batch;
  a.batch_count = batch_count;
  a.target_base = reinterpret_cast<const std::uint32_t*>(base + L.o_tb);
  a.summaries = reinterpret_cast<bfx_compact_target_summary*>(base + L.o_sum);
  a.lengths = reinterpret_cast<std::uint32_t*>(base + L.o_len);
  a.vertex_offsets = reinterpret_cast<const std::uint64_t*>(base + L.o_vo);
  a.edge_offsets = reinterpret_cast<const std::uint64_t*>(base + L.o_eo);
  a.flagged = reinterpret_cast<std::uint32_t*>(base + L.o_fl);
  a.flagged_count = reinterpret_cast<std::uint32_t*>(base + L.o_fc);
  a.stack_v = reinterpret_cast<std::uint32_t*>(base + L.o_sv);
  a.stack_c = reinterpret_cast<std::uint32_t*>(base + L.o_sc);
  a.stack_e = reinterpret_cast<std::uint32_t*>(base + L.o_se);
  a.on_path = reinterpret_cast<std::uint32_t*>(base + L.o_op);
  a.max_union = max_union;
  a.slots = L.slots;
  a.slot_stride = L.slot_stride;
  a.mark_stride = L.mark_stride;
  return a;
}

std::uint32_t largest_union(bfx_workspace* ws, std::uint32_t first_batch, std::uint32_t batch_count) {
  std::uint32_t m = 0;
  for (std::uint32_t i = 0; i < batch_count; ++i) m = std::max(m, ws->batches[first_batch + i].U);
  return m;
}

// PathArgs over the workspace's path buffer for the batches of the last
// summaries pass (same layout the summaries pass wrote).
PathArgs path_args(bfx_workspace* ws) {
  const std::uint32_t mu = largest_union(ws, ws->path_first_batch, ws->path_batch_count);
  return path_args_at(ws, path_layout(ws->path_targets, ws->path_batch_count, mu), ws->path_first_batch,
                      ws->path_batch_count, mu);
}

}  // namespace
}  // namespace bfx

extern "C" {

int bfx_compact_path_summaries(bfx_workspace* ws, uint32_t first_batch, uint32_t batch_count,
                               bfx_compact_target_summary* summaries, uint64_t sizes[3]) {
  return bfx::guarded([&] {
    bfx::check_ready(ws);
    bfx::require(summaries != nullptr, "null output");
    if (batch_count == 0 || first_batch >= ws->nb || batch_count > ws->nb - first_batch)
      throw std::out_of_range("batch range");
    BFX_CUDA(cudaSetDevice(ws->graph->device));
    std::vector<std::uint32_t> tbase(batch_count + 1, 0U);
    for (std::uint32_t i = 0; i < batch_count; ++i) tbase[i + 1] = tbase[i] + ws->batches[first_batch + i].tgt_count;
    const std::uint32_t max_union = bfx::largest_union(ws, first_batch, batch_count);
    const std::uint64_t T = tbase[batch_count];
    const bfx::PathLayout L = bfx::path_layout(T, batch_count, max_union);
    ws->paths.reserve(L.total, ws->graph->device);
    char* base = static_cast<char*>(ws->paths.ptr);
    BFX_CUDA(cudaMemcpyAsync(base + L.o_tb, tbase.data(), (batch_count + 1) * 4, cudaMemcpyHostToDevice, ws->stream));
    // every slot's on-path bitmap starts clear (a search leaves it clear)
    BFX_CUDA(cudaMemsetAsync(base + L.o_op, 0, size_t{L.slots} * L.mark_stride * 4, ws->stream));
    BFX_CUDA(cudaMemsetAsync(base + L.o_fc, 0, 4, ws->stream));
    const bfx::PathArgs a = bfx::path_args_at(ws, L, first_batch, batch_count, max_union);
    if (T > 0) {
      const int blocks = static_cast<int>(std::min<std::uint64_t>((T + 255) / 256, 4096));
      bfx::summaries_kernel<<<blocks, 256, 0, ws->stream>>>(a);
      BFX_CUDA(cudaGetLastError());
      bfx::flag_list_kernel<<<blocks, 256, 0, ws->stream>>>(a);
      BFX_CUDA(cudaGetLastError());
      bfx::search_kernel<<<(a.slots + 31) / 32, 32, 0, ws->stream>>>(a, false);
      BFX_CUDA(cudaGetLastError());
    }
    ws->paths_host.reserve(T * sizeof(bfx_compact_target_summary) + 256);
    BFX_CUDA(cudaMemcpyAsync(ws->paths_host.ptr, a.summaries, T * sizeof(bfx_compact_target_summary),
                             cudaMemcpyDeviceToHost, ws->stream));
    BFX_CUDA(cudaStreamSynchronize(ws->stream));
    std::memcpy(summaries, ws->paths_host.ptr, T * sizeof(bfx_compact_target_summary));
    // Payload offsets (checked host prefix, as the reference does).
    std::vector<std::uint64_t> vo(T), eo(T);
    std::uint64_t nv = 0, ne = 0;
    for (std::uint64_t i = 0; i < T; ++i) {
      vo[i] = nv;
      eo[i] = ne;
      if (summaries[i].reconstruction == 0u) {
        nv += std::uint64_t{summaries[i].path_length} + 1U;
        ne += summaries[i].path_length;
      }
    }
    BFX_CUDA(cudaMemcpyAsync(base + L.o_vo, vo.data(), T * 8, cudaMemcpyHostToDevice, ws->stream));
    BFX_CUDA(cudaMemcpyAsync(base + L.o_eo, eo.data(), T * 8, cudaMemcpyHostToDevice, ws->stream));
    BFX_CUDA(cudaStreamSynchronize(ws->stream));
    ws->path_first_batch = first_batch;
    ws->path_batch_count = batch_count;
    ws->path_targets = T;
    ws->path_vertices = nv;
    ws->path_edges = ne;
    ws->paths_ready = true;
    if (sizes) {
      sizes[0] = T;
      sizes[1] = nv;
      sizes[2] = ne;
    }
  });
}

int bfx_compact_path_payload(bfx_workspace* ws, uint32_t* vertices, float* distance_labels, uint32_t* edge_ids) {
  return bfx::guarded([&] {
    bfx::check_ready(ws);
    bfx::require(ws->paths_ready, "call bfx_compact_path_summaries first");
    bfx::require(vertices && distance_labels && (edge_ids || ws->path_edges == 0), "null output");
    BFX_CUDA(cudaSetDevice(ws->graph->device));
    const std::uint64_t T = ws->path_targets, nv = ws->path_vertices, ne = ws->path_edges;
    // Output arena: vertices, labels, edges in one device allocation.
    const size_t out_bytes = bfx::align256(nv * 4) * 2 + bfx::align256(ne * 4 + 4);
    char* dout = nullptr;
    BFX_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&dout), out_bytes, ws->stream));
    bfx::PathArgs a = bfx::path_args(ws);
    a.out_vertices = reinterpret_cast<std::uint32_t*>(dout);
    a.out_labels = reinterpret_cast<float*>(dout + bfx::align256(nv * 4));
    a.out_edges = reinterpret_cast<std::uint32_t*>(dout + 2 * bfx::align256(nv * 4));
    cudaError_t err = cudaSuccess;
    if (T > 0) {
      const int blocks = static_cast<int>(std::min<std::uint64_t>((T + 255) / 256, 4096));
      bfx::payload_kernel<<<blocks, 256, 0, ws->stream>>>(a);
      err = cudaGetLastError();
      if (err == cudaSuccess) {
        bfx::search_kernel<<<(a.slots + 31) / 32, 32, 0, ws->stream>>>(a, true);
        err = cudaGetLastError();
      }
    }
    if (err == cudaSuccess && nv) {
      cudaMemcpyAsync(vertices, a.out_vertices, nv * 4, cudaMemcpyDeviceToHost, ws->stream);
      cudaMemcpyAsync(distance_labels, a.out_labels, nv * 4, cudaMemcpyDeviceToHost, ws->stream);
    }
    if (err == cudaSuccess && ne) cudaMemcpyAsync(edge_ids, a.out_edges, ne * 4, cudaMemcpyDeviceToHost, ws->stream);
    cudaFreeAsync(dout, ws->stream);
    BFX_CUDA(err);
    BFX_CUDA(cudaStreamSynchronize(ws->stream));
  });
}

}  // extern "C"

extern "C" int bfx_edge_usage_adjoint(bfx_workspace* ws, const float* target_grads, float* edge_grads) {
  return bfx::guarded([&] {
    bfx::check_ready(ws);
    bfx::require(ws->paths_ready, "call bfx_compact_path_summaries first");
    bfx::require(edge_grads != nullptr && (target_grads != nullptr || ws->path_targets == 0), "null argument");
    const std::uint64_t T = ws->path_targets;
    const std::uint32_t E = ws->graph->g.E;
    for (std::uint64_t i = 0; i < T; ++i) {
      const float g = target_grads[i];
      const float a = g < 0 ? -g : g;
      bfx::require(g == 0.0f || (a >= 0x1p-40f && a < 0x1p40f),
                   "upstream gradients must be 0 or have magnitude in [2^-40, 2^40)");
    }
    BFX_CUDA(cudaSetDevice(ws->graph->device));
    const size_t o_acc = 0;
    const size_t o_g = bfx::align256(o_acc + size_t{E} * 32);
    const size_t o_out = bfx::align256(o_g + T * 4);
    const size_t total = bfx::align256(o_out + size_t{E} * 4);
    ws->adjoint.reserve(total, ws->graph->device);
    char* base = static_cast<char*>(ws->adjoint.ptr);
    auto* acc = reinterpret_cast<unsigned long long*>(base + o_acc);
    auto* g = reinterpret_cast<float*>(base + o_g);
    auto* out = reinterpret_cast<float*>(base + o_out);
    BFX_CUDA(cudaMemsetAsync(acc, 0, size_t{E} * 32, ws->stream));
    if (T) BFX_CUDA(cudaMemcpyAsync(g, target_grads, T * 4, cudaMemcpyHostToDevice, ws->stream));
    const bfx::PathArgs a = bfx::path_args(ws);
    if (T) {
      const int blocks = static_cast<int>(std::min<std::uint64_t>((T + 255) / 256, 4096));
      bfx::adjoint_walk_kernel<<<blocks, 256, 0, ws->stream>>>(a, g, acc);
      BFX_CUDA(cudaGetLastError());
      bfx::adjoint_search_kernel<<<(a.slots + 31) / 32, 32, 0, ws->stream>>>(a, g, acc);
      BFX_CUDA(cudaGetLastError());
    }
    bfx::adjoint_round_kernel<<<std::max(1, std::min<int>((E + 255) / 256, 8192)), 256, 0, ws->stream>>>(E, acc, out);
    BFX_CUDA(cudaGetLastError());
    BFX_CUDA(cudaMemcpyAsync(edge_grads, out, size_t{E} * 4, cudaMemcpyDeviceToHost, ws->stream));
    BFX_CUDA(cudaStreamSynchronize(ws->stream));
  });
}

namespace bfx {
namespace {

__global__ void set_weights_kernel(uint4* csr, uint4* csc, u32 E, const float* w) {
  for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < E; i += gridDim.x * blockDim.x) {
    csr[i].y = __float_as_uint(w[csr[i].z - 1u]);
    csc[i].y = __float_as_uint(w[csc[i].z - 1u]);
  }
}

}  // namespace
}  // namespace bfx

extern "C" int bfx_resident_graph_set_weights(bfx_resident_graph* graph, const float* weights_by_edge_id) {
  return bfx::guarded([&] {
    bfx::require(graph && weights_by_edge_id, "null argument");
    const std::uint32_t E = graph->g.E;
    std::vector<float> w(weights_by_edge_id, weights_by_edge_id + E);
    for (float& x : w) {
      if (!(x >= 0.0f) || x == __builtin_inff()) throw std::invalid_argument("edge weights must be finite and nonnegative");
      if (x == 0.0f) x = 0.0f;  // canonical +0 (InputGraph canonicalisation)
    }
    BFX_CUDA(cudaSetDevice(graph->device));
    float* d = nullptr;
    BFX_CUDA(cudaMalloc(reinterpret_cast<void**>(&d), size_t{E} * 4 + 4));
    cudaError_t err = cudaMemcpy(d, w.data(), size_t{E} * 4, cudaMemcpyHostToDevice);
    if (err == cudaSuccess && E) {
      bfx::set_weights_kernel<<<std::min<int>((E + 255) / 256, 8192), 256>>>(const_cast<uint4*>(graph->g.csr),
                                                                           const_cast<uint4*>(graph->g.csc), E, d);
      err = cudaGetLastError();
      if (err == cudaSuccess) err = cudaDeviceSynchronize();
    }
    cudaFree(d);
    BFX_CUDA(err);
  });
}
