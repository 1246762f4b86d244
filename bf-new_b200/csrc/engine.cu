// bfx batched relaxation engines for B200 (sm_100a).
//
// One launch relaxes any number of batches (planned query groups of 1, 8,
// 16 or 32 lanes, one query per lane) over the resident graph:
//   * frontier push  -- the reference's BatchedFrontierPushEngine
//                       (src/hip/batched_frontier_push.hip.cpp:710-906),
//   * Jacobi pull    -- BatchedJacobiPullEngine (src/hip/batched_jacobi.hip.cpp:466-694),
//   * dense chaotic  -- BatchedDenseChaoticPushEngine
//                       (src/hip/batched_dense_chaotic_push.hip.cpp:392-600).
// All three converge to the same labels: every label is the minimum over
// admitted paths of the left-folded float sum (float + is monotone), and the
// packed 64-bit label keeps the smallest stable edge id among tight
// in-edges.  The schedule is ours:
//   * labels live in compact union-tile storage per batch (vertex-major,
//     lanes contiguous), addressed through a dense per-tile {lane mask,
//     compact bias} table that doubles as the run admission test
//     (mask[src tile] & mask[dst tile], src/device_layout.cpp:762), so no run
//     masks are materialised;
//   * edges are 16-byte records {endpoint, weight bits, eid+1, endpoint tile}
//     read with 128-bit non-coherent loads;
//   * the frontier is a queue of 32-vertex chunks by default (frontier.cuh:
//     chunk bitmaps per round slot, pending lanes set with non-returning ORs,
//     near and far claims staged per warp and (round, batch)); a warp item
//     is a pack of up to 8 chunks whose pending vertices are compacted into
//     work lists of up to 32 vertices, each walked as a flat (lane, edge)
//     list, two items per thread in flight, and dense rounds take the chunk
//     slots in index order; the vertex-queue flat layout and the sub-warp group
//     layout remain options; improvements use a non-returning 64-bit min
//     after a coherent pre-read;
//   * persistent mode runs all rounds of all batches in one cooperative
//     launch with a grid barrier whose waits time out; host-poll modes run
//     CUDA-graph-captured chunks of rounds.
#include "bfx.h"
#include "bfx_host.h"
#include "bfx_internal.hpp"
#include "device_common.cuh"
#include "engine_types.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

namespace bfx {

namespace {
thread_local std::string g_last_error;
}

void set_last_error(const std::string& message) { g_last_error = message; }


// ---------------------------------------------------------------------------
// Small device helpers
// ---------------------------------------------------------------------------

__device__ __forceinline__ u32 lane_id() { return threadIdx.x & 31u; }

// Largest b with prefix[b] <= x (prefix strictly covering [0, prefix[nb])).
__device__ __forceinline__ u32 find_batch(const u32* prefix, u32 nb, u32 x) {
  u32 lo = 0, hi = nb;
  while (hi - lo > 1u) {
    const u32 mid = (lo + hi) >> 1;
    if (prefix[mid] <= x) {
      lo = mid;
    } else {
      hi = mid;
    }
  }
  return lo;
}

__device__ __forceinline__ u32 lane_of_position(const u32* offsets, u32 W, u32 pos) {
  u32 lo = 0, hi = W;
  while (hi - lo > 1u) {
    const u32 mid = (lo + hi) >> 1;
    if (offsets[mid] <= pos) {
      lo = mid;
    } else {
      hi = mid;
    }
  }
  return lo;
}

// Values of per-batch work that a round may pack: the chunk slots of a
// chunked near round carry this flag; their warp items are the slots
// divided by the round's pack (round_pack).
constexpr u32 kPackable = 0x80000000u;

// Chunk slots per warp item of the current round, set by block_prefix.
__shared__ u32 s_round_pack;

// Block-wide exclusive scan of per-batch work items into smem
// prefix[0..nb].  Each value is computed once (four batches per iteration,
// so their loads are in flight together) and parked in prefix[b].  Values
// flagged kPackable are chunk slots: the round's pack is the largest power
// of two up to `kmax` that still leaves at least two warp items per warp of
// the grid (slots / pack + the other items), so packing never starves the
// grid of items on a small frontier; the flagged slots then become
// ceil(slots / pack) items.  The second pass replaces each value by its
// exclusive sum.  Every block computes the same result from the same
// counters.
template <typename F>
__device__ void block_prefix(u32* prefix, u32 nb, F value, u32 kmax = 1u) {
  __shared__ u32 s_warp[33];
  __shared__ u64 s_tot[2][32];
  const u32 per = (nb + blockDim.x - 1) / blockDim.x;
  const u32 begin = threadIdx.x * per;
  const u32 warp = threadIdx.x >> 5;
  u64 slots = 0, other = 0;
#pragma unroll 4
  for (u32 i = 0; i < per; ++i) {
    const u32 b = begin + i;
    if (b < nb) {
      const u32 x = value(b);
      prefix[b] = x;
      if (x & kPackable) {
        slots += x & ~kPackable;
      } else {
        other += x;
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    slots += __shfl_down_sync(0xFFFFFFFFu, slots, o);
    other += __shfl_down_sync(0xFFFFFFFFu, other, o);
  }
  if (lane_id() == 0) {
    s_tot[0][warp] = slots;
    s_tot[1][warp] = other;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    u64 S = 0, O = 0;
    for (u32 w = 0; w < (blockDim.x >> 5); ++w) {
      S += s_tot[0][w];
      O += s_tot[1][w];
    }
    const u64 want = 2ull * gridDim.x * (blockDim.x >> 5);
    u32 k = kmax;
    while (k > 1u && S / k + O < want) k >>= 1;
    s_round_pack = k;
  }
  __syncthreads();
  const u32 k = s_round_pack;
  u32 local = 0;
  for (u32 i = 0; i < per; ++i) {
    const u32 b = begin + i;
    if (b < nb) {
      u32 x = prefix[b];
      if (x & kPackable) x = ((x & ~kPackable) + k - 1u) / k;
      prefix[b] = x;
      local += x;
    }
  }
  // inclusive warp scan
  u32 x = local;
  for (u32 o = 1; o < 32; o <<= 1) {
    const u32 y = __shfl_up_sync(0xFFFFFFFFu, x, o);
    if (lane_id() >= o) x += y;
  }
  if (lane_id() == 31) s_warp[warp] = x;
  __syncthreads();
  if (threadIdx.x == 0) {
    u32 acc = 0;
    const u32 nw = blockDim.x >> 5;
    for (u32 w = 0; w < nw; ++w) {
      const u32 t = s_warp[w];
      s_warp[w] = acc;
      acc += t;
    }
    s_warp[32] = acc;
  }
  __syncthreads();
  u32 run = s_warp[warp] + x - local;
  for (u32 i = 0; i < per; ++i) {
    const u32 b = begin + i;
    if (b < nb) {
      const u32 y = prefix[b];
      prefix[b] = run;
      run += y;
    }
  }
  if (threadIdx.x == 0) prefix[nb] = s_warp[32];
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Initialisation and seeding
// ---------------------------------------------------------------------------

// Grid-stride over all union vertices of all batches: compact->global map,
// +inf labels, clear masks; over tile tables: {mask, bias} for union tiles.
__global__ void init_kernel(LaunchParams p) {
  const u64 tid = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x;
  const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
  const u32 total_units = p.unit_base[p.nb];
  for (u64 u = tid; u < total_units; u += stride) {
    const u32 b = find_batch(p.unit_base, p.nb, static_cast<u32>(u));
    const DBatch& B = p.batches[b];
    const u32 cv = static_cast<u32>(u) - p.unit_base[b];
    // range containing cv
    u32 lo = 0, hi = B.range_count;
    while (hi - lo > 1u) {
      const u32 mid = (lo + hi) >> 1;
      if (B.range_off[mid] <= cv) lo = mid; else hi = mid;
    }
    const uint4 r = B.ranges[lo];
    B.c2g[cv] = r.y + (cv - B.range_off[lo]);
    B.mask[0][cv] = 0u;
    B.mask[1][cv] = 0u;
    B.fmask[cv] = 0u;
    B.fbound[cv] = 0xFFFFFFFFu;
    if (p.flat >= 2u) {
      if ((cv & 1023u) == 0u) {  // chunk bitmap words, one per 1,024 vertices (enough for any shift >= 5)
        B.cmask[0][cv >> 10] = 0u;
        B.cmask[1][cv >> 10] = 0u;
      }
      const u32 v = r.y + (cv - B.range_off[lo]);
      const u32 rb = p.g.csr_off[v];
      B.crow[cv] = make_uint2(rb, p.g.csr_off[v + 1u] - rb);
      if (p.flat == 3u) B.clrun[cv] = p.g.lrun[v];
    }
    for (u32 l = 0; l < B.W; ++l) {
      B.dist[0][(static_cast<u64>(cv) << B.shift) + l] = dev::kUnreached;
      if (engine_of(p, b) == BFX_ENGINE_JACOBI_PULL) B.dist[1][(static_cast<u64>(cv) << B.shift) + l] = dev::kUnreached;
    }
  }
  // Tile tables: clear every tile then write union tiles (a second pass in
  // the same kernel would race; clearing is done by the host-side memset).
  for (u32 b = 0; b < p.nb; ++b) {
    const DBatch& B = p.batches[b];
    for (u64 i = tid; i < B.range_count; i += stride) {
      const uint4 r = B.ranges[i];
      B.tiles[r.x] = make_uint2(r.w, r.y - B.range_off[i]);
    }
  }
  if (tid < p.nb) {
    DCtl& c = p.ctl[tid];
    c.count[0] = c.count[1] = c.count[2] = 0u;
    c.changed[0] = p.batches[tid].valid;
    c.fcount[0] = c.fcount[1] = c.fcount[2] = 0u;
    c.fmin[0] = c.fmin[1] = c.fmin[2] = 0xFFFFFFFFu;
    c.gen[0] = c.gen[1] = 0u;
    c.delta = p.deltas ? p.deltas[tid] : dev::kInfBits;
    c.tau[0] = c.tau[1] = c.delta;
    c.changed[1] = c.changed[2] = 0u;
    c.rounds = 0u;
    c.missing = 0u;
    c.active = 0u;
    c.error_bits = 0u;
  }
  if (tid == 0) {
    p.run->sync.arrive = 0u;
    p.run->sync.generation = 0u;
    p.run->sync.abort = 0u;
    p.run->round = 0u;
    p.run->done = 0u;
    p.run->stop = 0u;
    p.run->abort = 0u;
    for (int i = 0; i < 16; ++i) p.run->work[i] = 0u;
    for (int i = 0; i < 3; ++i) p.run->items[i] = 0u;
  }
}

// Sources: label (0, 0) in every lane that owns them; frontier engines also
// mark the lane bit and enqueue the vertex once (src/hip/batched_frontier_push.hip.cpp:495-559).
__global__ void seed_kernel(LaunchParams p, const u32* src_base) {
  const u64 tid = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x;
  const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
  const u32 total = src_base[p.nb];
  for (u64 i = tid; i < total; i += stride) {
    const u32 b = find_batch(src_base, p.nb, static_cast<u32>(i));
    const DBatch& B = p.batches[b];
    const u32 pos = static_cast<u32>(i) - src_base[b];
    const u32 lane = lane_of_position(B.src_off, B.W, pos);
    const u32 v = B.src[pos];
    const uint2 t = B.tiles[p.g.owner[v]];
    if (((t.x >> lane) & 1u) == 0u) {
      atomicOr(&p.ctl[b].error_bits, static_cast<u32>(BFX_DEVICE_ERROR_INVALID_CONTROLLER_STATE));
      continue;
    }
    const u32 cv = v - t.y;
    B.dist[0][(static_cast<u64>(cv) << B.shift) + lane] = dev::kSourceWord;
    const u32 eng = engine_of(p, b);
    if (eng == BFX_ENGINE_JACOBI_PULL) B.dist[1][(static_cast<u64>(cv) << B.shift) + lane] = dev::kSourceWord;
    if (eng == BFX_ENGINE_FRONTIER_PUSH && p.flat >= 2u) {
      // chunked / tiled frontier: pending lane, then the claim unit's bit;
      // the thread that sets the bit queues the unit
      atomicOr(&B.mask[0][cv], 1u << lane);
      const u32 chunk = cv >> p.cshift;
      const u32 bit = 1u << (chunk & 31u);
      if ((atomicOr(&B.cmask[0][chunk >> 5], bit) & bit) == 0u) {
        const u32 slot = atomicAdd(&p.ctl[b].count[0], 1u);
        if (slot < B.U) {
          B.queue[0][slot] = chunk;
        } else {
          atomicOr(&p.ctl[b].error_bits, static_cast<u32>(BFX_DEVICE_ERROR_QUEUE_OVERFLOW));
        }
      }
    } else if (eng == BFX_ENGINE_FRONTIER_PUSH) {
      const u32 old = atomicOr(&B.mask[0][cv], 1u << lane);
      if (old == 0u) {
        const u32 slot = atomicAdd(&p.ctl[b].count[0], 1u);
        if (slot < B.U) {
          B.queue[0][slot] = static_cast<u64>(v) | (static_cast<u64>(cv) << 32);
        } else {
          atomicOr(&p.ctl[b].error_bits, static_cast<u32>(BFX_DEVICE_ERROR_QUEUE_OVERFLOW));
        }
      }
    }
  }
}

// Frontier push (see frontier.cuh).
#include "frontier.cuh"

// ---------------------------------------------------------------------------
// Jacobi pull: lane = query lane, 32/W destination vertices per warp.
// d_next[v,l] = min(d[v,l], min over admitted in-edges of d[u,l] + w).
// ---------------------------------------------------------------------------

template <bool kCount>
__device__ __forceinline__ void jacobi_item(const LaunchParams& p, const DBatch& B, DCtl& C, u32 item, u32 r,
                                            u32 widx, Work& wk) {
  const u32 lane = lane_id();
  const u32 sub = lane >> B.shift;
  const u32 ql = lane & (B.W - 1u);
  const u32 vpw = 32u >> B.shift;
  const u32 cv = item * vpw + sub;
  const u64* const dr = B.dist[r & 1u];
  u64* const dw = B.dist[(r & 1u) ^ 1u];
  u32 changed = 0u;
  if (cv < B.U) {
    const u32 v = B.c2g[cv];
    const uint2 vt = B.tiles[__ldg(p.g.owner + v)];
    const u64 idx = (static_cast<u64>(cv) << B.shift) + ql;
    const u64 old = dev::ld_cg(dr + idx);
    u64 best = old;
    if (kCount) wk.c[7] += 1;  // every vertex-lane item reads its label and writes the other slot
    if ((vt.x >> ql) & 1u) {
      const u32 cb = __ldg(p.g.csc_off + v), ce = __ldg(p.g.csc_off + v + 1);
      if (kCount) wk.c[8] += ce - cb;
      for (u32 e = cb; e < ce; ++e) {
        const uint4 rec = __ldg(p.g.csc + e);
        const uint2 su = B.tiles[rec.w];
        if ((su.x >> ql) & 1u) {
          const u32 sb = dev::hi(dev::ld_cg(dr + ((static_cast<u64>(rec.x - su.y) << B.shift) + ql)));
          if (sb != dev::kInfBits) {
            const u64 cand = dev::candidate(sb, rec.y, rec.z);
            best = cand < best ? cand : best;
            if (kCount) wk.c[9] += 1;
          }
        }
      }
      if (dev::hi(best) != dev::hi(old)) changed = 1u << ql;
      if (kCount) wk.c[10] += changed != 0u;
    }
    dw[idx] = best;
  }
  const u32 any = __reduce_or_sync(0xFFFFFFFFu, changed);
  if (lane == 0 && any != 0u && (dev::ld_cg(&C.changed[widx]) & any) != any) atomicOr(&C.changed[widx], any);
}

// ---------------------------------------------------------------------------
// Dense chaotic push: every admitted (source vertex, lane) pushes all of its
// admitted out-edges in place each round.
// ---------------------------------------------------------------------------

template <bool kCount>
__device__ __forceinline__ void dense_item(const LaunchParams& p, const DBatch& B, DCtl& C, u32 item, u32 exec,
                                           u32 widx, Work& wk) {
  const u32 lane = lane_id();
  const u32 sub = lane >> B.shift;
  const u32 ql = lane & (B.W - 1u);
  const u32 vpw = 32u >> B.shift;
  const u32 cu = item * vpw + sub;
  u32 changed = 0u;
  if (cu < B.U) {
    const u32 u = B.c2g[cu];
    const uint2 ut = B.tiles[__ldg(p.g.owner + u)];
    if (((ut.x & exec) >> ql) & 1u) {
      const u32 sb = dev::hi(dev::ld_cg(B.dist[0] + ((static_cast<u64>(cu) << B.shift) + ql)));
      if (sb != dev::kInfBits) {
        const u32 rb = __ldg(p.g.csr_off + u), re = __ldg(p.g.csr_off + u + 1);
        if (kCount) {
          wk.c[0] += 1;
          wk.c[1] += re - rb;
          wk.c[2] += 1;
        }
        for (u32 e = rb; e < re; ++e) {
          const uint4 rec = __ldg(p.g.csr + e);
          const uint2 dt = B.tiles[rec.w];
          if ((dt.x >> ql) & 1u) {
            const u64 cand = dev::candidate(sb, rec.y, rec.z);
            u64* const target = B.dist[0] + ((static_cast<u64>(rec.x - dt.y) << B.shift) + ql);
            const u64 cur = dev::ld_cg(target);
            if (kCount) wk.c[3] += 1;
            if (cand < cur) {
              dev::red_min(target, cand);
              const bool dec = dev::hi(cand) < dev::hi(cur);
              if (dec) changed = 1u << ql;
              if (kCount) {
                wk.c[6] += 1;
                wk.c[5] += dec;
              }
            }
          }
        }
      }
    }
  }
  const u32 any = __reduce_or_sync(0xFFFFFFFFu, changed);
  if (lane == 0 && any != 0u && (dev::ld_cg(&C.changed[widx]) & any) != any) atomicOr(&C.changed[widx], any);
}

// ---------------------------------------------------------------------------
// One round over every batch.  Returns false when the launch must stop.
// Called by every block of the grid; `prefix` is dynamic shared memory of
// nb+1 words.
// ---------------------------------------------------------------------------

__device__ __forceinline__ u32 batch_exec(const LaunchParams& p, u32 b, u32 ridx) {
  const u32 ch = dev::ld_cg(&p.ctl[b].changed[ridx]);
  if (engine_of(p, b) == BFX_ENGINE_JACOBI_PULL) return ch != 0u ? p.batches[b].valid : 0u;
  return p.per_lane ? ch : (ch != 0u ? p.batches[b].valid : 0u);
}

// Far pile size of the batch's current generation: the three pile counters
// and the generation are read together (one dependent step, not two).
__device__ __forceinline__ u32 current_far_count(const DCtl& C, u32 r) {
  const u32 g = dev::ld_cg(&C.gen[r & 1u]) % 3u;
  const u32 f0 = dev::ld_cg(&C.fcount[0]), f1 = dev::ld_cg(&C.fcount[1]), f2 = dev::ld_cg(&C.fcount[2]);
  return g == 0u ? f0 : (g == 1u ? f1 : f2);
}

__device__ u32 round_work(const LaunchParams& p, u32 r, u32* prefix) {
  const u32 ridx = r % 3u;
  block_prefix(prefix, p.nb, [&](u32 b) {
    const DBatch& B = p.batches[b];
    const DCtl& C = p.ctl[b];
    // every counter the batch's item count can depend on, loaded up front
    const u32 eng = engine_of(p, b);
    const u32 count = dev::ld_cg(&C.count[ridx]);
    const u32 changed = dev::ld_cg(&C.changed[ridx]);
    const u32 far = current_far_count(C, r);
    const u32 U = B.U;
    if (eng == BFX_ENGINE_FRONTIER_PUSH) {
      const u32 n = min(count, U);
      if (n != 0u) {  // warp items: a pack of chunks (chunked), flat_entries_per_item(n) entries (flat), 4 or 1 entries
        if (p.flat >= 2u) return chunk_slots(n, U) | kPackable;
        return p.flat ? (n + flat_entries_per_item(n) - 1u) / flat_entries_per_item(n) : (B.W <= 8u ? (n + 3u) >> 2 : n);
      }
      const u32 f = min(far, U);
      return (f + kSplitPerItem - 1u) / kSplitPerItem;  // split round: kSplitPerItem far entries per warp item
    }
    const u32 exec = eng == BFX_ENGINE_JACOBI_PULL || !p.per_lane ? (changed != 0u ? B.valid : 0u) : changed;
    return exec != 0u ? (((U << B.shift) + 31u) >> 5) : 0u;
  }, p.flat >= 2u ? p.cpack : 1u);
  return prefix[p.nb];
}

// kChunked: compiled for the chunked frontier layout only (a separate
// kernel instantiation, so the other layouts keep their register budget).
// The warp's claim stages and far-pile minimum (flat and chunked layouts)
// serve one (round, batch): flushed when the warp moves to another batch and
// at the end of the round, before the grid barrier.
// Work distribution: block k owns the warp items k, k + G, k + 2G, ... (G
// blocks), and its warps take them one at a time from a shared-memory
// counter, so a warp that drew cheap items takes more of them and the
// block's warps finish together; consecutive items stay on neighbouring
// blocks at the same time (the index order of dense chunked rounds).
template <bool kCount, u32 kItems, bool kChunked, bool kPairs = false>
__device__ void round_body(const LaunchParams& p, u32 r, const u32* prefix, Work& wk) {
  __shared__ u32 s_next_item;
  const u32 ridx = r % 3u, widx = (r + 1u) % 3u;
  const u32 total = prefix[p.nb];
  const u32 pack = s_round_pack;  // chunk slots per warp item of this round (round_work)
  Stages st{{0u, 0u}, 0xFFFFFFFFu};
  u32 staged_batch = 0xFFFFFFFFu;
  if (threadIdx.x == 0u) s_next_item = 0u;
  __syncthreads();
  for (;;) {
    u32 k = 0u;
    if (lane_id() == 0u) k = atomicAdd(&s_next_item, 1u);
    k = __shfl_sync(0xFFFFFFFFu, k, 0);
    const u64 wl = blockIdx.x + static_cast<u64>(k) * gridDim.x;
    if (wl >= total) break;
    const u32 w = static_cast<u32>(wl);
    const u32 b = find_batch(prefix, p.nb, w);
    const DBatch& B = p.batches[b];
    DCtl& C = p.ctl[b];
    const u32 item = w - prefix[b];
    const u32 eng = engine_of(p, b);
    if (eng == BFX_ENGINE_FRONTIER_PUSH) {
      // read once per warp and broadcast: the branch below and the sizes the
      // frontier bodies see are warp-uniform by construction
      u32 n = 0u, g = 0u, tau = 0u, f = 0u, tau_next = 0u;
      if (lane_id() == 0u) {
        n = min(dev::ld_cg(&C.count[ridx]), B.U);
        g = dev::ld_cg(&C.gen[r & 1u]);
        tau = dev::ld_cg(&C.tau[r & 1u]);
        if (n == 0u) {
          f = min(dev::ld_cg(&C.fcount[g % 3u]), B.U);
          tau_next = split_threshold(C, tau, g % 3u);
        }
      }
      n = __shfl_sync(0xFFFFFFFFu, n, 0);
      g = __shfl_sync(0xFFFFFFFFu, g, 0);
      tau = __shfl_sync(0xFFFFFFFFu, tau, 0);
      f = __shfl_sync(0xFFFFFFFFu, f, 0);
      tau_next = __shfl_sync(0xFFFFFFFFu, tau_next, 0);
      const FrontierView V = frontier_view(B, r & 1u, g % 3u, (g + 1u) % 3u);
      if (b != staged_batch) {
        // near round: claims to the next queue, parked lanes to pile g % 3;
        // split round: pile g % 3 is read and re-parked lanes go to g + 1
        stages_flush(st);
        staged_batch = b;
        const u32 po = n != 0u ? g % 3u : (g + 1u) % 3u;
        if (lane_id() == 0u) {
          const u32 wib = threadIdx.x >> 5;
          s_stage_queue[kNear][wib] = StageQueue{V.queue_w, &C.count[widx], &C.error_bits, V.U};
          s_stage_queue[kFar][wib] = StageQueue{n != 0u ? V.pile : V.pile_out, &C.fcount[po], &C.error_bits, V.U};
          s_fmin_target[wib] = &C.fmin[po];
        }
        __syncwarp();
      }
      if (n != 0u) {
        if (kChunked) {
          // a pack of queue words (sparse round) or of chunk slots in index
          // order (dense round)
          frontier_flat<kCount, kItems, true, kPairs>(p, V, C, item, n, 32u, tau, st, wk, chunk_dense(n, V.U, 5u),
                                                      pack);
        } else if (p.flat) {
          frontier_flat<kCount, kItems, false>(p, V, C, item, n, flat_entries_per_item(n), tau, st, wk);
        } else if (B.W <= 8u) {
          frontier_group<kCount, 8>(p, V, C, item, n, r & 1u, widx, tau, g % 3u, wk);
        } else {
          frontier_group<kCount, 32>(p, V, C, item, n, r & 1u, widx, tau, g % 3u, wk);
        }
      } else if (kChunked) {
        split_group<kCount, true>(p, V, C, item, f, tau_next, st, wk);
      } else {
        split_group<kCount, false>(p, V, C, item, f, tau_next, st, wk);
      }
    } else if (eng == BFX_ENGINE_JACOBI_PULL) {
      jacobi_item<kCount>(p, B, C, item, r, widx, wk);
    } else {
      dense_item<kCount>(p, B, C, item, batch_exec(p, b, ridx), widx, wk);
    }
  }
  stages_flush(st);
}

// Bookkeeping at the start of round r, done by block 0 (threads striding
// over the batches): rounds counter per batch, clear the rotating slot that
// round r+1 will write.  A batch's counters are loaded together before any
// of them is used.
__device__ void round_bookkeeping(const LaunchParams& p, u32 r) {
  const u32 ridx = r % 3u, zidx = (r + 2u) % 3u;
#pragma unroll 4
  for (u32 b = threadIdx.x; b < p.nb; b += blockDim.x) {
    DCtl& C = p.ctl[b];
    bool work;
    const u32 eng = engine_of(p, b);
    const u32 g = dev::ld_cg(&C.gen[r & 1u]);
    const u32 tau = dev::ld_cg(&C.tau[r & 1u]);
    const u32 count = dev::ld_cg(&C.count[ridx]);
    const u32 far = current_far_count(C, r);
    if (eng == BFX_ENGINE_FRONTIER_PUSH) {
      // near round, split round (near frontier empty, far pile not), or idle;
      // generation and threshold of round r+1 go to the other parity slot.
      const bool near = count != 0u;
      const bool split = !near && far != 0u;
      work = near || split;
      if (split) {
        C.fcount[(g + 2u) % 3u] = 0u;  // idle since two splits ago; the next split writes it
        C.fmin[(g + 2u) % 3u] = 0xFFFFFFFFu;
        C.gen[(r + 1u) & 1u] = g + 1u;
        C.tau[(r + 1u) & 1u] = split_threshold(C, tau, g % 3u);
      } else {
        C.gen[(r + 1u) & 1u] = g;
        C.tau[(r + 1u) & 1u] = tau;
      }
    } else {
      work = batch_exec(p, b, ridx) != 0u;
    }
    if (work) C.rounds = r + 1u;
    C.count[zidx] = 0u;
    C.changed[zidx] = 0u;
  }
  if (threadIdx.x == 0u) p.run->items[zidx] = 0u;  // tiled layout: the block-item counter of round r + 2
}

// Frontier batches whose round r is a near/far split round (round trace
// only; reads slots that the bookkeeping of round r does not write).
// Executed by one whole warp, lanes striding over the batches.
__device__ u32 split_batches(const LaunchParams& p, u32 r) {
  u32 n = 0u;
  for (u32 b = lane_id(); b < p.nb; b += 32u) {
    if (engine_of(p, b) != BFX_ENGINE_FRONTIER_PUSH) continue;
    const DCtl& C = p.ctl[b];
    const u32 g = dev::ld_cg(&C.gen[r & 1u]);
    n += dev::ld_cg(&C.count[r % 3u]) == 0u && dev::ld_cg(&C.fcount[g % 3u]) != 0u;
  }
  return __reduce_add_sync(0xFFFFFFFFu, n);
}

// Round trace words 2 and 3: the active (vertex, lane) pairs and lane-edge
// relaxations of round r, added per warp from the counters' growth since the
// previous round.
__device__ void trace_round_work(const LaunchParams& p, u32 r, const Work& wk, u64 (&traced)[2]) {
  u64 x[2] = {wk.c[2] - traced[0], wk.c[3] - traced[1]};
  traced[0] = wk.c[2];
  traced[1] = wk.c[3];
  for (int i = 0; i < 2; ++i) {
    for (int o = 16; o > 0; o >>= 1) x[i] += __shfl_down_sync(0xFFFFFFFFu, x[i], o);
    if (lane_id() == 0 && x[i]) {
      atomicAdd(reinterpret_cast<unsigned long long*>(&p.round_trace[4u * r + 2u + i]), x[i]);
    }
  }
}

// Adds each thread's counters into the launch-wide totals.
__device__ void flush_work(const LaunchParams& p, Work& wk) {
  for (int i = 0; i < kWorkCounters; ++i) {
    u64 x = wk.c[i];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xFFFFFFFFu, x, o);
    const int slot = i < 7 ? i : i + 1;  // work[7] holds the round count
    if (lane_id() == 0 && x) atomicAdd(reinterpret_cast<unsigned long long*>(&p.run->work[slot]), x);
  }
}

// kMinBlocks = resident 512-thread blocks per SM the register budget is set
// for, or kBlocks256x3 = three 256-thread blocks per SM (80 registers, 24
// warps per SM; chunked layout only).
// for: 3 -> 40 registers per thread (48 warps per SM), 2 -> 64 registers
// (32 warps per SM; no spills in the group layout, a few in the flat one).
// kItems = flat-layout work items per thread per iteration.
constexpr int kBlocks256x3 = 5;
template <bool kCount, int kMinBlocks, u32 kItems, bool kChunked = false, bool kPairs = false>
__global__ void __launch_bounds__(kMinBlocks == kBlocks256x3 ? 256 : 512, kMinBlocks == kBlocks256x3 ? 3 : kMinBlocks)
    persistent_kernel(LaunchParams p) {
  extern __shared__ u32 prefix[];
  const u32 nblocks = gridDim.x;
  Work wk;
  wk.zero();
  u64 traced[2] = {0u, 0u};
  const u64 t0 = dev::global_ns();
  u32 r = 0;
  for (;; ++r) {
    const u32 total = round_work(p, r, prefix);
    if (total == 0u || r >= p.max_rounds) break;
    if (blockIdx.x == 0) round_bookkeeping(p, r);
    if (p.round_trace != nullptr && blockIdx.x == 0 && threadIdx.x < 32u && r < p.trace_cap) {
      const u64 t = dev::global_ns();
      const u32 splits = split_batches(p, r);
      if (threadIdx.x == 0u) {
        p.round_trace[4u * r] = t;
        p.round_trace[4u * r + 1u] = total | (static_cast<u64>(splits) << 32);
      }
    }
    round_body<kCount, kItems, kChunked, kPairs>(p, r, prefix, wk);
    if (kCount && p.round_trace != nullptr && r < p.trace_cap) trace_round_work(p, r, wk, traced);
    // Past the launch budget block 0 raises the barrier's abort before it
    // arrives, so every block leaves after this round.
    if (blockIdx.x == 0 && threadIdx.x == 0 && dev::global_ns() - t0 > p.budget_ns) {
      atomicExch(&p.run->sync.abort, 1u);
    }
    if (!dev::grid_barrier(&p.run->sync, nblocks, kBarrierTimeoutNs)) {
      if (threadIdx.x == 0) atomicExch(&p.run->abort, 1u);
      break;
    }
  }
  if (kCount) flush_work(p, wk);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    p.run->round = r;
    p.run->done = 1u;
    p.run->work[7] = r;
  }
}

// Host-poll modes: one round per launch over a fixed grid ...
template <bool kCount, bool kChunked = false>
__global__ void __launch_bounds__(512, 3) round_kernel(LaunchParams p) {
  extern __shared__ u32 prefix[];
  if (dev::ld_cg(&p.run->done) != 0u) return;
  const u32 r = dev::ld_cg(&p.run->round);
  const u32 total = round_work(p, r, prefix);
  if (total == 0u) return;
  Work wk;
  wk.zero();
  round_body<kCount, 2, kChunked>(p, r, prefix, wk);
  if (kCount) flush_work(p, wk);
}

// ... followed by a one-block advance: stop test, bookkeeping, next round.
__global__ void advance_kernel(LaunchParams p) {
  extern __shared__ u32 prefix[];
  if (dev::ld_cg(&p.run->done) != 0u) return;
  const u32 r = dev::ld_cg(&p.run->round);
  // Bookkeeping for the round that just ran happens before the next one
  // starts; the stop test looks at the round that would run next.
  round_bookkeeping(p, r);
  __syncthreads();
  const u32 next_total = round_work(p, r + 1u, prefix);
  if (threadIdx.x == 0) {
    p.run->round = r + 1u;
    p.run->work[7] = r + 1u;
    if (next_total == 0u || static_cast<u64>(r + 1u) >= p.max_rounds) p.run->done = 1u;
  }
}

// Before the first host-poll round: stop immediately if nothing to do.
__global__ void start_kernel(LaunchParams p) {
  extern __shared__ u32 prefix[];
  const u32 total = round_work(p, 0u, prefix);
  if (threadIdx.x == 0) {
    p.run->round = 0u;
    p.run->done = (total == 0u || p.max_rounds == 0u) ? 1u : 0u;
  }
}

// Tiled frontier layout (see tiled.cuh).
#include "tiled.cuh"

// ---------------------------------------------------------------------------
// Finalize: one block per batch.  Reached / miss lanes from target
// finiteness (src/hip/batched_frontier_push.hip.cpp:971-1010), pending lanes
// for round-limited stops, and the reference-format controller and status.
// ---------------------------------------------------------------------------

__global__ void finalize_kernel(LaunchParams p, bfx_device_controller* controllers, bfx_device_run_status* statuses) {
  const u32 b = blockIdx.x;
  const u32 eng = engine_of(p, b);
  const DBatch& B = p.batches[b];
  DCtl& C = p.ctl[b];
  __shared__ u32 s_missing, s_active;
  if (threadIdx.x == 0) {
    s_missing = 0u;
    s_active = 0u;
  }
  __syncthreads();
  const u32 r_end = p.run->round;
  const u32 ridx = r_end % 3u;
  const bool aborted = p.run->abort != 0u;
  bool pending;
  if (eng == BFX_ENGINE_FRONTIER_PUSH) {
    pending = C.count[ridx] != 0u || C.fcount[C.gen[r_end & 1u] % 3u] != 0u;
  } else {
    pending = batch_exec(p, b, ridx) != 0u;
  }
  const u32 final_slot = eng == BFX_ENGINE_JACOBI_PULL ? (C.rounds & 1u) : 0u;
  const u64* const d = B.dist[final_slot];
  for (u32 i = threadIdx.x; i < B.tgt_count; i += blockDim.x) {
    const u32 lane = lane_of_position(B.tgt_off, B.W, i);
    const u32 v = B.tgt[i];
    const uint2 t = B.tiles[p.g.owner[v]];
    bool reached = false;
    if ((t.x >> lane) & 1u) reached = dev::hi(d[(static_cast<u64>(v - t.y) << B.shift) + lane]) != dev::kInfBits;
    if (!reached) atomicOr(&s_missing, 1u << lane);
  }
  if (pending && !aborted) {
    if (eng == BFX_ENGINE_FRONTIER_PUSH) {
      const u32* const mk = B.mask[r_end & 1u];
      u32 acc = 0u;
      for (u32 i = threadIdx.x; i < B.U; i += blockDim.x) acc |= mk[i] | B.fmask[i];
      acc = __reduce_or_sync(0xFFFFFFFFu, acc);
      if (lane_id() == 0 && acc) atomicOr(&s_active, acc);
    } else if (threadIdx.x == 0) {
      s_active = C.changed[ridx];
    }
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  u32 error_bits = C.error_bits;
  u32 stop;
  if (aborted) {
    error_bits |= BFX_DEVICE_ERROR_DEVICE_FAILURE;
  }
  if (error_bits & BFX_DEVICE_ERROR_DEVICE_FAILURE) {
    stop = BFX_STOP_DEVICE_FAILURE;
    error_bits = BFX_DEVICE_ERROR_DEVICE_FAILURE;
  } else if (error_bits & BFX_DEVICE_ERROR_QUEUE_OVERFLOW) {
    stop = BFX_STOP_QUEUE_OVERFLOW;
    error_bits = BFX_DEVICE_ERROR_QUEUE_OVERFLOW;
  } else if (error_bits != 0u) {
    stop = BFX_STOP_INVALID_CONTROLLER_STATE;
    error_bits = BFX_DEVICE_ERROR_INVALID_CONTROLLER_STATE;
  } else if (!pending) {
    stop = BFX_STOP_CONVERGED;
  } else {
    stop = BFX_STOP_MAXIMUM_ROUNDS;
  }
  const bool converged = stop == BFX_STOP_CONVERGED;
  const u32 valid = B.valid;
  const u32 active = converged || error_bits ? 0u : (s_active & valid);
  const u32 conv_lanes = converged ? valid : ((p.per_lane && !error_bits) ? (valid & ~active) : 0u);
  bfx_device_run_status st;
  st.final_distance_slot = final_slot;
  st.converged = converged ? 1u : 0u;
  st.rounds_completed = C.rounds;
  st.reached_target_mask = converged ? (valid & ~s_missing) : 0u;
  st.bounding_box_miss_mask = converged ? (valid & s_missing) : 0u;
  st.valid_lane_mask = valid;
  st.active_lane_mask = active;
  st.converged_lane_mask = conv_lanes;
  st.stop_reason = stop;
  st.error_bits = error_bits;
  st.reserved0 = 0u;
  statuses[b] = st;
  bfx_device_controller c;
  memset(&c, 0, sizeof(c));
  c.valid_lane_mask = valid;
  c.active_lane_mask = active;
  c.converged_lane_mask = conv_lanes;
  c.engine_kind = eng;
  c.enable_per_lane_convergence = p.per_lane;
  c.rounds_completed = C.rounds;
  c.maximum_rounds = p.max_rounds;
  c.distance_read_slot = final_slot;
  c.distance_write_slot = eng == BFX_ENGINE_JACOBI_PULL ? (final_slot ^ 1u) : 0u;
  c.frontier_read_slot = r_end & 1u;
  c.frontier_write_slot = (r_end & 1u) ^ 1u;
  c.frontier_size[r_end & 1u] = eng == BFX_ENGINE_FRONTIER_PUSH ? C.count[ridx] : 0u;
  c.done = 1u;
  c.stop_reason = stop;
  c.error_bits = error_bits;
  controllers[b] = c;
}

// Graph-sized label image of one batch: bits / predecessor edge ids.
__global__ void expand_kernel(DGraph g, DBatch B, u32 slot, u32* bits, u32* preds) {
  const u64 n = static_cast<u64>(g.V) << B.shift;
  for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<u64>(gridDim.x) * blockDim.x) {
    const u32 v = static_cast<u32>(i >> B.shift);
    const u32 l = static_cast<u32>(i & (B.W - 1u));
    const uint2 t = B.tiles[g.owner[v]];
    u64 w = dev::kUnreached;
    if ((t.x >> l) & 1u) w = B.dist[slot][(static_cast<u64>(v - t.y) << B.shift) + l];
    if (bits) bits[i] = dev::hi(w);
    if (preds) {
      const u32 lo = static_cast<u32>(w);
      preds[i] = (lo == 0u || lo == 0xFFFFFFFFu) ? 0xFFFFFFFFu : lo - 1u;
    }
  }
}

// One lane of a batch as a graph-sized image.
__global__ void expand_lane_kernel(DGraph g, DBatch B, u32 slot, u32 lane, u32* bits, u32* preds) {
  for (u32 v = blockIdx.x * blockDim.x + threadIdx.x; v < g.V; v += gridDim.x * blockDim.x) {
    const uint2 t = B.tiles[g.owner[v]];
    u64 w = dev::kUnreached;
    if ((t.x >> lane) & 1u) w = B.dist[slot][(static_cast<u64>(v - t.y) << B.shift) + lane];
    if (bits) bits[v] = dev::hi(w);
    if (preds) {
      const u32 lo = static_cast<u32>(w);
      preds[v] = (lo == 0u || lo == 0xFFFFFFFFu) ? 0xFFFFFFFFu : lo - 1u;
    }
  }
}

// Largest finite distance bits per batch over the final labels (grid-stride
// over the union vertices of all batches, as init_kernel); out[b] starts at 0.
__global__ void label_bound_kernel(LaunchParams p, const bfx_device_run_status* statuses, u32* out) {
  const u64 tid = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x;
  const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
  const u32 total_units = p.unit_base[p.nb];
  u32 best = 0u, best_b = 0xFFFFFFFFu;
  for (u64 u = tid; u < total_units; u += stride) {
    const u32 b = find_batch(p.unit_base, p.nb, static_cast<u32>(u));
    if (b != best_b) {
      if (best_b != 0xFFFFFFFFu && best != 0u) atomicMax(out + best_b, best);
      best_b = b;
      best = 0u;
    }
    const DBatch& B = p.batches[b];
    const u32 cv = static_cast<u32>(u) - p.unit_base[b];
    const u64* const d = B.dist[statuses[b].final_distance_slot] + (static_cast<u64>(cv) << B.shift);
    for (u32 l = 0; l < B.W; ++l) {
      const u32 h = dev::hi(d[l]);
      if (h < dev::kInfBits && h > best) best = h;
    }
  }
  if (best_b != 0xFFFFFFFFu && best != 0u) atomicMax(out + best_b, best);
}

// ---------------------------------------------------------------------------
// Device-side batch description preparation (bfx_prepare_batches_from_queries):
// the per-batch image prepare_batch_device_description builds on the host
// (src/batch_layout.cpp:1056-1296) -- dense tile lane masks, one vertex range
// per union tile with its compact offset, lane terminal slices -- built from
// the batches' lane -> query assignment and the queries' selected tiles and
// terminals.
// ---------------------------------------------------------------------------

// The uploaded query and lane image.  Per query q: tiles [tile_off[q],
// tile_off[q+1]), sources and targets likewise; per batch b: lanes
// [lane_base[b], lane_base[b+1]) with their query indices; per lane its
// first entry in the flattened (lane, tile) list.
struct QueryImage {
  const u32* tile_off;
  const u32* tiles;
  const u32* src_off;
  const u32* srcs;
  const u32* tgt_off;
  const u32* tgts;
  const u32* lane_base;      // [nb+1]
  const u32* lane_query;     // [lanes]
  const u32* lane_tile_base; // [lanes+1]
  u32 nb, lanes;
};

// Scatter: every (lane, selected tile) ORs the lane's bit into its batch's
// dense tile mask.
__global__ void desc_mask_kernel(QueryImage q, uint2* tiles, u64 tstride) {
  const u32 total = q.lane_tile_base[q.lanes];
  for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    const u32 lane_g = find_batch(q.lane_tile_base, q.lanes, i);
    const u32 b = find_batch(q.lane_base, q.nb, lane_g);
    const u32 lane = lane_g - q.lane_base[b];
    const u32 qi = q.lane_query[lane_g];
    const u32 t = q.tiles[q.tile_off[qi] + (i - q.lane_tile_base[lane_g])];
    atomicOr(&tiles[b * tstride + t].x, 1u << lane);
  }
}

// One block per batch: union tile count, union vertex count, and the count
// of union tiles whose mask is not every valid lane (0 with R == T: a
// full-graph batch).  out[4b..4b+3] = {R, U, partial tiles, 0}.
__global__ void desc_count_kernel(const u32* tile_off, u32 T, const uint2* tiles, u64 tstride, const u32* valid,
                                  u32* out) {
  __shared__ u32 s_acc[3];
  const u32 b = blockIdx.x;
  if (threadIdx.x == 0u) s_acc[0] = s_acc[1] = s_acc[2] = 0u;
  __syncthreads();
  u32 r = 0u, u = 0u, partial = 0u;
  for (u32 t = threadIdx.x; t < T; t += blockDim.x) {
    const u32 m = tiles[b * tstride + t].x;
    if (m != 0u) {
      ++r;
      u += tile_off[t + 1] - tile_off[t];
      partial += m != valid[b];
    }
  }
  r = __reduce_add_sync(0xFFFFFFFFu, r);
  u = __reduce_add_sync(0xFFFFFFFFu, u);
  partial = __reduce_add_sync(0xFFFFFFFFu, partial);
  if (lane_id() == 0u) {
    atomicAdd(&s_acc[0], r);
    atomicAdd(&s_acc[1], u);
    atomicAdd(&s_acc[2], partial);
  }
  __syncthreads();
  if (threadIdx.x == 0u) {
    out[4u * b] = s_acc[0];
    out[4u * b + 1u] = s_acc[1];
    out[4u * b + 2u] = s_acc[2];
    out[4u * b + 3u] = 0u;
  }
}

// One block per batch: union tiles in increasing order with their vertex
// ranges, compact offsets and the tile table's compact biases (block scans
// over the tile ids), then the lane terminal slices; a terminal whose owner
// tile is not selected for its lane sets *error.
__global__ void desc_fill_kernel(QueryImage q, const u32* owner, const u32* tile_off, u32 T, uint2* tiles,
                                 u64 tstride, const DBatch* batches, u32* error) {
  __shared__ u32 s_f[32], s_v[32], s_tot[2];
  __shared__ u32 s_carry[2];
  const u32 b = blockIdx.x;
  const DBatch& B = batches[b];
  uint4* ranges = const_cast<uint4*>(B.ranges);
  u32* roff = const_cast<u32*>(B.range_off);
  uint2* tb = tiles + b * tstride;
  if (threadIdx.x == 0u) s_carry[0] = s_carry[1] = 0u;
  __syncthreads();
  const u32 nw = blockDim.x >> 5, wib = threadIdx.x >> 5, lane = lane_id();
  for (u32 base = 0; base < T; base += blockDim.x) {
    const u32 t = base + threadIdx.x;
    const u32 m = t < T ? tb[t].x : 0u;
    const u32 size = m != 0u ? tile_off[t + 1] - tile_off[t] : 0u;
    // block exclusive scans of (union flag, union vertices)
    u32 f = m != 0u ? 1u : 0u, v = size;
    for (u32 o = 1; o < 32u; o <<= 1) {
      const u32 yf = __shfl_up_sync(0xFFFFFFFFu, f, o);
      const u32 yv = __shfl_up_sync(0xFFFFFFFFu, v, o);
      if (lane >= o) {
        f += yf;
        v += yv;
      }
    }
    if (lane == 31u) {
      s_f[wib] = f;
      s_v[wib] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0u) {
      u32 af = 0u, av = 0u;
      for (u32 w = 0; w < nw; ++w) {
        const u32 xf = s_f[w], xv = s_v[w];
        s_f[w] = af;
        s_v[w] = av;
        af += xf;
        av += xv;
      }
      s_tot[0] = af;  // this chunk's union tiles and vertices
      s_tot[1] = av;
    }
    __syncthreads();
    const u32 idx = s_carry[0] + s_f[wib] + f - (m != 0u ? 1u : 0u);
    const u32 off = s_carry[1] + s_v[wib] + v - size;
    if (m != 0u) {
      ranges[idx] = make_uint4(t, tile_off[t], tile_off[t + 1], m);
      roff[idx] = off;
      tb[t].y = tile_off[t] - off;
    }
    __syncthreads();
    if (threadIdx.x == 0u) {
      s_carry[0] += s_tot[0];
      s_carry[1] += s_tot[1];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0u) roff[B.range_count] = s_carry[1];
  // terminal slices: lanes in order, invalid lanes empty
  u32* so = const_cast<u32*>(B.src_off);
  u32* src = const_cast<u32*>(B.src);
  u32* to = const_cast<u32*>(B.tgt_off);
  u32* tgt = const_cast<u32*>(B.tgt);
  const u32 lanes = q.lane_base[b + 1] - q.lane_base[b];
  if (threadIdx.x == 0u) {
    u32 ns = 0u, nt = 0u;
    so[0] = to[0] = 0u;
    for (u32 l = 0; l < B.W; ++l) {
      if (l < lanes) {
        const u32 qi = q.lane_query[q.lane_base[b] + l];
        ns += q.src_off[qi + 1] - q.src_off[qi];
        nt += q.tgt_off[qi + 1] - q.tgt_off[qi];
      }
      so[l + 1] = ns;
      to[l + 1] = nt;
    }
  }
  __syncthreads();
  for (u32 l = wib; l < lanes; l += nw) {
    const u32 qi = q.lane_query[q.lane_base[b] + l];
    const u32 s0 = q.src_off[qi], s1 = q.src_off[qi + 1], t0 = q.tgt_off[qi], t1 = q.tgt_off[qi + 1];
    const u32 sb = so[l], tb0 = to[l];
    for (u32 k = lane; k < s1 - s0; k += 32u) {
      const u32 v = q.srcs[s0 + k];
      src[sb + k] = v;
      if (((tb[owner[v]].x >> l) & 1u) == 0u) atomicOr(error, 1u);
    }
    for (u32 k = lane; k < t1 - t0; k += 32u) {
      const u32 v = q.tgts[t0 + k];
      tgt[tb0 + k] = v;
      if (((tb[owner[v]].x >> l) & 1u) == 0u) atomicOr(error, 1u);
    }
  }
}

// ---------------------------------------------------------------------------
}  // namespace bfx

namespace bfx {
namespace {

void upload(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  if (bytes) BFX_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
}

void check_layout(const bfx_device_graph_layout32& L) {
  require(L.owner_tiles && L.csr_row_offsets && L.csr_destinations && L.csr_weights && L.csc_column_offsets &&
              L.csc_sources && L.csc_weights && L.csc_edge_ids,
          "device layout arrays must be non-null");
  const std::uint32_t V = L.vertex_count, E = L.edge_count, T = L.tile_count;
  require(T >= 1, "device layout needs at least one tile");
  require(L.csr_row_offsets[0] == 0 && L.csr_row_offsets[V] == E, "invalid CSR offsets");
  require(L.csc_column_offsets[0] == 0 && L.csc_column_offsets[V] == E, "invalid CSC offsets");
  for (std::uint32_t v = 0; v < V; ++v) {
    require(L.csr_row_offsets[v] <= L.csr_row_offsets[v + 1], "invalid CSR offsets");
    require(L.csc_column_offsets[v] <= L.csc_column_offsets[v + 1], "invalid CSC offsets");
    require(L.owner_tiles[v] < T, "owner tile out of range");
    require(v == 0 || L.owner_tiles[v] >= L.owner_tiles[v - 1], "owner tiles must be contiguous spans");
  }
  for (std::uint32_t e = 0; e < E; ++e) {
    if (L.csr_destinations[e] >= V || L.csc_sources[e] >= V) throw std::out_of_range("edge endpoint out of range");
    if (L.csc_edge_ids[e] >= E) throw std::out_of_range("edge id out of range");
    require(L.csr_weights[e] >= 0.0F && L.csc_weights[e] >= 0.0F, "invalid stored weight");
  }
}

}  // namespace
}  // namespace bfx

extern "C" {

int bfx_abi_version(void) { return BFX_ABI_VERSION; }

const char* bfx_last_error(void) { return bfx::g_last_error.c_str(); }

int bfx_device_count(int* count) {
  return bfx::guarded([&] {
    bfx::require(count != nullptr, "null output");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
      cudaGetLastError();
      n = 0;
    }
    *count = n;
  });
}

int bfx_resident_graph_upload(const bfx_device_graph_layout32* layout, int device, bfx_resident_graph** out) {
  return bfx::guarded([&] {
    bfx::require(layout && out, "null argument");
    *out = nullptr;
    const bfx_device_graph_layout32& L = *layout;
    bfx::check_layout(L);
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
      cudaGetLastError();
      throw bfx::Error(BFX_ERR_NO_DEVICE, "no CUDA device is available");
    }
    if (device < 0 || device >= n) throw std::out_of_range("device index");
    BFX_CUDA(cudaSetDevice(device));
    const std::uint32_t V = L.vertex_count, E = L.edge_count, T = L.tile_count;
    // Stable EdgeId per CSR position: given, or matched from the CSC image
    // (each CSC entry (dst, src, eid) is one CSR entry of row src).
    std::vector<std::uint32_t> csr_eid;
    const std::uint32_t* eids = L.csr_edge_ids;
    if (!eids) {
      csr_eid.assign(E, 0xFFFFFFFFu);
      std::vector<std::uint32_t> cursor(L.csr_row_offsets, L.csr_row_offsets + V);
      // CSR rows are ordered by (dst tile, dst, eid); visiting CSC entries in
      // increasing eid per (src, dst) pair reproduces that order.
      std::vector<std::uint64_t> order(E);
      for (std::uint32_t v = 0; v < V; ++v) {
        for (std::uint32_t q = L.csc_column_offsets[v]; q < L.csc_column_offsets[v + 1]; ++q) order[q] = q;
      }
      std::vector<std::uint32_t> col_of(E);
      for (std::uint32_t v = 0; v < V; ++v) {
        for (std::uint32_t q = L.csc_column_offsets[v]; q < L.csc_column_offsets[v + 1]; ++q) col_of[q] = v;
      }
      std::sort(order.begin(), order.end(), [&](std::uint64_t a, std::uint64_t b) {
        const std::uint32_t sa = L.csc_sources[a], sb = L.csc_sources[b];
        if (sa != sb) return sa < sb;
        const std::uint32_t da = col_of[a], db = col_of[b];
        if (L.owner_tiles[da] != L.owner_tiles[db]) return L.owner_tiles[da] < L.owner_tiles[db];
        if (da != db) return da < db;
        return L.csc_edge_ids[a] < L.csc_edge_ids[b];
      });
      for (std::uint64_t i = 0; i < E; ++i) {
        const std::uint32_t q = static_cast<std::uint32_t>(order[i]);
        const std::uint32_t p = cursor[L.csc_sources[q]]++;
        bfx::require(L.csr_destinations[p] == col_of[q], "CSR and CSC images disagree");
        csr_eid[p] = L.csc_edge_ids[q];
      }
      eids = csr_eid.data();
    }
    auto G = std::make_unique<bfx_resident_graph>();
    G->device = device;
    G->tile_vertex_offsets.assign(T + 1U, 0U);
    for (std::uint32_t v = 0; v < V; ++v) ++G->tile_vertex_offsets[L.owner_tiles[v] + 1U];
    for (std::uint32_t t = 0; t < T; ++t) G->tile_vertex_offsets[t + 1] += G->tile_vertex_offsets[t];

    std::vector<uint4> csr(E), csc(E);
    std::vector<std::uint32_t> eid_src(E, 0U);
    std::vector<uint2> lrun(V);
    bfx::parallel_for(V, 0, [&](std::uint64_t b, std::uint64_t e) {
      for (std::uint64_t v = b; v < e; ++v) {
        // own-tile run: rows are ordered by destination tile, so the edges
        // into v's own tile are contiguous
        std::uint32_t lb = L.csr_row_offsets[v], lc = 0;
        for (std::uint32_t p = L.csr_row_offsets[v]; p < L.csr_row_offsets[v + 1]; ++p) {
          if (L.owner_tiles[L.csr_destinations[p]] == L.owner_tiles[v]) {
            if (lc == 0) lb = p;
            ++lc;
          }
        }
        lrun[v] = make_uint2(lb, lc);
        for (std::uint32_t p = L.csr_row_offsets[v]; p < L.csr_row_offsets[v + 1]; ++p) {
          const std::uint32_t d = L.csr_destinations[p];
          std::uint32_t wb;
          std::memcpy(&wb, &L.csr_weights[p], 4);
          csr[p] = make_uint4(d, wb, eids[p] + 1U, L.owner_tiles[d]);
          if (eids[p] >= E) throw std::out_of_range("csr edge id out of range");
          eid_src[eids[p]] = static_cast<std::uint32_t>(v);
        }
        for (std::uint32_t q = L.csc_column_offsets[v]; q < L.csc_column_offsets[v + 1]; ++q) {
          const std::uint32_t s = L.csc_sources[q];
          std::uint32_t wb;
          std::memcpy(&wb, &L.csc_weights[q], 4);
          csc[q] = make_uint4(s, wb, L.csc_edge_ids[q] + 1U, L.owner_tiles[s]);
        }
      }
    });
    const size_t o_owner = 0;
    const size_t o_csr_off = bfx::align256(o_owner + size_t{V} * 4);
    const size_t o_csc_off = bfx::align256(o_csr_off + (size_t{V} + 1) * 4);
    const size_t o_csr = bfx::align256(o_csc_off + (size_t{V} + 1) * 4);
    const size_t o_csc = bfx::align256(o_csr + size_t{E} * 16);
    const size_t o_eid_src = bfx::align256(o_csc + size_t{E} * 16);
    const size_t o_lrun = bfx::align256(o_eid_src + size_t{E} * 4);
    const size_t o_toff = bfx::align256(o_lrun + size_t{V} * 8);
    const size_t total = bfx::align256(o_toff + (size_t{T} + 1) * 4);
    G->mem.reserve(total, device);
    char* base = static_cast<char*>(G->mem.ptr);
    BFX_CUDA(cudaMemcpy(base + o_owner, L.owner_tiles, size_t{V} * 4, cudaMemcpyHostToDevice));
    BFX_CUDA(cudaMemcpy(base + o_csr_off, L.csr_row_offsets, (size_t{V} + 1) * 4, cudaMemcpyHostToDevice));
    BFX_CUDA(cudaMemcpy(base + o_csc_off, L.csc_column_offsets, (size_t{V} + 1) * 4, cudaMemcpyHostToDevice));
    BFX_CUDA(cudaMemcpy(base + o_csr, csr.data(), size_t{E} * 16, cudaMemcpyHostToDevice));
    BFX_CUDA(cudaMemcpy(base + o_csc, csc.data(), size_t{E} * 16, cudaMemcpyHostToDevice));
    BFX_CUDA(cudaMemcpy(base + o_eid_src, eid_src.data(), size_t{E} * 4, cudaMemcpyHostToDevice));
    BFX_CUDA(cudaMemcpy(base + o_lrun, lrun.data(), size_t{V} * 8, cudaMemcpyHostToDevice));
    BFX_CUDA(cudaMemcpy(base + o_toff, G->tile_vertex_offsets.data(), (size_t{T} + 1) * 4, cudaMemcpyHostToDevice));
    double wsum = 0.0;
    for (std::uint32_t e = 0; e < E; ++e) wsum += L.csr_weights[e];
    G->mean_weight = E ? wsum / E : 0.0;
    G->g.V = V;
    G->g.E = E;
    G->g.T = T;
    G->g.owner = reinterpret_cast<const std::uint32_t*>(base + o_owner);
    G->g.csr_off = reinterpret_cast<const std::uint32_t*>(base + o_csr_off);
    G->g.csc_off = reinterpret_cast<const std::uint32_t*>(base + o_csc_off);
    G->g.csr = reinterpret_cast<const uint4*>(base + o_csr);
    G->g.csc = reinterpret_cast<const uint4*>(base + o_csc);
    G->g.eid_src = reinterpret_cast<const std::uint32_t*>(base + o_eid_src);
    G->g.lrun = reinterpret_cast<const uint2*>(base + o_lrun);
    G->g.tile_off = reinterpret_cast<const std::uint32_t*>(base + o_toff);
    G->bytes = total;
    {
      const std::uint32_t size0 = G->tile_vertex_offsets[1] - G->tile_vertex_offsets[0];
      bool uniform = true;
      for (std::uint32_t t = 0; t < T && uniform; ++t) {
        uniform = G->tile_vertex_offsets[t + 1] - G->tile_vertex_offsets[t] == size0;
      }
      std::uint32_t shift = 8;
      if (uniform && size0 >= 32u && size0 <= 256u && (size0 & (size0 - 1u)) == 0u) {
        shift = static_cast<std::uint32_t>(__builtin_ctz(size0));
      } else if (uniform && size0 < 32u) {
        shift = 5;
      }
      G->tile_shift = shift;
    }
    *out = G.release();
  });
}

int bfx_resident_graph_destroy(bfx_resident_graph* graph) {
  return bfx::guarded([&] { delete graph; });
}

int bfx_workspace_graph_stats(bfx_workspace* ws, double out[2]) {
  return bfx::guarded([&] {
    bfx::require(ws && out, "null argument");
    out[0] = ws->graph->mean_weight;
    out[1] = static_cast<double>(ws->graph->g.E);
  });
}

int bfx_resident_graph_info(const bfx_resident_graph* graph, uint64_t out[4]) {
  return bfx::guarded([&] {
    bfx::require(graph && out, "null argument");
    out[0] = graph->g.V;
    out[1] = graph->g.E;
    out[2] = graph->g.T;
    out[3] = graph->bytes;
  });
}

int bfx_workspace_create(bfx_resident_graph* graph, bfx_workspace** out) {
  return bfx::guarded([&] {
    bfx::require(graph && out, "null argument");
    *out = nullptr;
    BFX_CUDA(cudaSetDevice(graph->device));
    auto ws = std::make_unique<bfx_workspace>();
    ws->graph = graph;
    BFX_CUDA(cudaStreamCreateWithFlags(&ws->stream, cudaStreamNonBlocking));
    for (auto& e : ws->ev) BFX_CUDA(cudaEventCreate(&e));
    BFX_CUDA(cudaDeviceGetAttribute(&ws->sm_count, cudaDevAttrMultiProcessorCount, graph->device));
    *out = ws.release();
  });
}

int bfx_workspace_destroy(bfx_workspace* ws) {
  return bfx::guarded([&] {
    if (!ws) return;
    cudaSetDevice(ws->graph->device);
    if (ws->stream) cudaStreamSynchronize(ws->stream);
    if (ws->chunk_exec) cudaGraphExecDestroy(ws->chunk_exec);
    for (auto& e : ws->ev) {
      if (e) cudaEventDestroy(e);
    }
    if (ws->stream) cudaStreamDestroy(ws->stream);
    delete ws;
  });
}

int bfx_workspace_stream(bfx_workspace* ws, void** stream) {
  return bfx::guarded([&] {
    bfx::require(ws && stream, "null argument");
    *stream = ws->stream;
  });
}

int bfx_workspace_bytes(bfx_workspace* ws, uint64_t* bytes) {
  return bfx::guarded([&] {
    bfx::require(ws && bytes, "null argument");
    *bytes = ws->meta.bytes + ws->arena.bytes + ws->tile_tables.bytes + ws->qimage.bytes;
  });
}

}  // extern "C"

namespace bfx {
namespace {

// Per-batch sizes of a prepared set.
struct BatchSizes {
  u32 U, R, S, Tg, W, shift, valid, full;
};

// Where a batch's description arrays sit in the metadata block.
struct DescArrays {
  size_t src_off, src, tgt_off, tgt, ranges, range_off;
};

// Lays out a prepared set: the metadata block (batch records, controllers,
// launch state, unit and source prefixes, statuses, controllers, then each
// batch's description arrays), the arena (per-batch labels -- two slots, so
// one prepare serves every engine -- pending masks, queues, compact map, far
// pile state, chunk bitmaps, row tables) and the tile tables (one dense
// {lane mask, compact bias} table per batch).  Fills ws->batches with device
// pointers, the staging header (records, prefixes) and the launch
// parameters; the caller writes the description arrays and uploads.
struct Layout {
  size_t o_up, meta_total;
  std::vector<DescArrays> arrays;
};

Layout lay_out_batches(bfx_workspace* ws, std::uint32_t count, const std::vector<BatchSizes>& sz) {
  const DGraph& g = ws->graph->g;
  const size_t o_batch = 0;
  const size_t o_ctl = align256(o_batch + count * sizeof(DBatch));
  const size_t o_run = align256(o_ctl + count * sizeof(DCtl));
  const size_t o_ubase = align256(o_run + sizeof(DRun));
  const size_t o_sbase = align256(o_ubase + (count + 1) * 4);
  const size_t o_status = align256(o_sbase + (count + 1) * 4);
  const size_t o_ctrl = align256(o_status + count * sizeof(bfx_device_run_status));
  Layout L;
  L.o_up = align256(o_ctrl + count * sizeof(bfx_device_controller));
  L.arrays.resize(count);
  size_t up = L.o_up;
  for (std::uint32_t b = 0; b < count; ++b) {
    const BatchSizes& s = sz[b];
    DescArrays& a = L.arrays[b];
    a.src_off = up;
    up += align256((s.W + 1) * 4);
    a.src = up;
    up += align256(size_t{s.S} * 4);
    a.tgt_off = up;
    up += align256((s.W + 1) * 4);
    a.tgt = up;
    up += align256(size_t{s.Tg} * 4);
    a.ranges = up;
    up += align256(size_t{s.R} * 16);
    a.range_off = up;
    up += align256((size_t{s.R} + 1) * 4);
  }
  L.meta_total = up;
  std::vector<size_t> arena_off(count);
  size_t arena_total = 0;
  for (std::uint32_t b = 0; b < count; ++b) {
    arena_off[b] = arena_total;
    const size_t U = sz[b].U;
    arena_total += align256(U * sz[b].W * 8) * 2 + align256(U * 4) * 5 + align256(U * 8) * 7 +
                   align256((U + 1023) / 1024 * 4) * 2;
  }
  const size_t tile_table_bytes = align256(size_t{g.T} * 8);
  const bool grew = L.meta_total > ws->meta.bytes || arena_total > ws->arena.bytes ||
                    tile_table_bytes * count > ws->tile_tables.bytes;
  ws->meta.reserve(L.meta_total, ws->graph->device);
  ws->arena.reserve(arena_total, ws->graph->device);
  ws->tile_tables.reserve(tile_table_bytes * count, ws->graph->device);
  if (grew) ++ws->generation;
  ws->staging.reserve(L.meta_total);
  char* hb = static_cast<char*>(ws->staging.ptr);
  char* db = static_cast<char*>(ws->meta.ptr);
  char* ab = static_cast<char*>(ws->arena.ptr);
  char* tb = static_cast<char*>(ws->tile_tables.ptr);
  std::memset(hb, 0, L.o_up);
  ws->batches.assign(count, DBatch{});
  std::uint32_t* ubase = reinterpret_cast<std::uint32_t*>(hb + o_ubase);
  std::uint32_t* sbase = reinterpret_cast<std::uint32_t*>(hb + o_sbase);
  std::uint64_t usum = 0, ssum = 0;
  for (std::uint32_t b = 0; b < count; ++b) {
    const BatchSizes& s = sz[b];
    const DescArrays& da = L.arrays[b];
    DBatch& B = ws->batches[b];
    B.W = s.W;
    B.shift = s.shift;
    B.valid = s.valid;
    B.U = s.U;
    B.src_count = s.S;
    B.tgt_count = s.Tg;
    B.range_count = s.R;
    B.full = s.full;
    B.src_off = reinterpret_cast<const std::uint32_t*>(db + da.src_off);
    B.src = reinterpret_cast<const std::uint32_t*>(db + da.src);
    B.tgt_off = reinterpret_cast<const std::uint32_t*>(db + da.tgt_off);
    B.tgt = reinterpret_cast<const std::uint32_t*>(db + da.tgt);
    B.ranges = reinterpret_cast<const uint4*>(db + da.ranges);
    B.range_off = reinterpret_cast<const std::uint32_t*>(db + da.range_off);
    char* a = ab + arena_off[b];
    const size_t U = s.U;
    B.dist[0] = reinterpret_cast<u64*>(a);
    a += align256(U * s.W * 8);
    B.dist[1] = reinterpret_cast<u64*>(a);
    a += align256(U * s.W * 8);
    B.mask[0] = reinterpret_cast<std::uint32_t*>(a);
    a += align256(U * 4);
    B.mask[1] = reinterpret_cast<std::uint32_t*>(a);
    a += align256(U * 4);
    B.queue[0] = reinterpret_cast<u64*>(a);
    a += align256(U * 8);
    B.queue[1] = reinterpret_cast<u64*>(a);
    a += align256(U * 8);
    B.c2g = reinterpret_cast<std::uint32_t*>(a);
    a += align256(U * 4);
    B.fmask = reinterpret_cast<std::uint32_t*>(a);
    a += align256(U * 4);
    B.fbound = reinterpret_cast<std::uint32_t*>(a);
    a += align256(U * 4);
    for (int k = 0; k < 3; ++k) {
      B.fpile[k] = reinterpret_cast<u64*>(a);
      a += align256(U * 8);
    }
    for (int k = 0; k < 2; ++k) {
      B.cmask[k] = reinterpret_cast<std::uint32_t*>(a);
      a += align256((U + 1023) / 1024 * 4);
    }
    B.crow = reinterpret_cast<uint2*>(a);
    a += align256(U * 8);
    B.clrun = reinterpret_cast<uint2*>(a);
    a += align256(U * 8);
    B.tiles = reinterpret_cast<uint2*>(tb + tile_table_bytes * b);
    ubase[b] = static_cast<std::uint32_t>(usum);
    sbase[b] = static_cast<std::uint32_t>(ssum);
    usum += U;
    ssum += s.S;
    if (usum > 0xFFFFFFFFull) throw std::overflow_error("total union vertices exceed 32 bits");
  }
  ubase[count] = static_cast<std::uint32_t>(usum);
  sbase[count] = static_cast<std::uint32_t>(ssum);
  std::memcpy(hb + o_batch, ws->batches.data(), count * sizeof(DBatch));
  ws->nb = count;
  ws->src_total = ssum;
  ws->params = LaunchParams{};
  ws->params.g = g;
  ws->params.batches = reinterpret_cast<const DBatch*>(db + o_batch);
  ws->params.ctl = reinterpret_cast<DCtl*>(db + o_ctl);
  ws->params.run = reinterpret_cast<DRun*>(db + o_run);
  ws->params.unit_base = reinterpret_cast<const std::uint32_t*>(db + o_ubase);
  ws->params.nb = count;
  ws->src_base = reinterpret_cast<u32*>(db + o_sbase);
  ws->d_status = reinterpret_cast<bfx_device_run_status*>(db + o_status);
  ws->d_ctrl = reinterpret_cast<bfx_device_controller*>(db + o_ctrl);
  ws->executed = false;
  return L;
}

}  // namespace
}  // namespace bfx

extern "C" {

int bfx_prepare_batches(bfx_workspace* ws, uint32_t count, const bfx_batch_description* batches) {
  return bfx::guarded([&] {
    bfx::require(ws != nullptr, "null workspace");
    bfx::require(count > 0 && batches, "at least one batch is required");
    if (count > bfx::kMaxBatchesPerLaunch) throw std::length_error("too many batches for one launch");
    BFX_CUDA(cudaSetDevice(ws->graph->device));
    const bfx::DGraph& g = ws->graph->g;
    const auto& tvo = ws->graph->tile_vertex_offsets;
    // Validate descriptions (validate_batch_device_description,
    // include/bfnew/batch_layout.hpp:176-199) and size everything.
    std::vector<bfx::BatchSizes> sz(count);
    for (std::uint32_t b = 0; b < count; ++b) {
      const bfx_batch_description& d = batches[b];
      const std::uint32_t W = d.lane_width;
      bfx::require(W == 1 || W == 8 || W == 16 || W == 32, "unsupported lane width");
      const std::uint32_t wmask = W == 32 ? 0xFFFFFFFFu : ((1u << W) - 1u);
      bfx::require(d.valid_lane_mask != 0 && (d.valid_lane_mask & ~wmask) == 0, "invalid valid lane mask");
      bfx::require(d.tile_count == g.T, "description tile count does not match the graph");
      bfx::require(d.source_offsets && d.target_offsets && d.tile_lane_masks && d.union_tiles &&
                       (d.range_count == 0 || d.selected_vertex_ranges),
                   "null description array");
      bfx::require(d.source_offsets[0] == 0 && d.target_offsets[0] == 0, "invalid terminal offsets");
      for (std::uint32_t l = 0; l < W; ++l) {
        bfx::require(d.source_offsets[l + 1] >= d.source_offsets[l] && d.target_offsets[l + 1] >= d.target_offsets[l],
                     "invalid terminal offsets");
        const bool valid = (d.valid_lane_mask >> l) & 1u;
        const bool has_s = d.source_offsets[l + 1] > d.source_offsets[l];
        const bool has_t = d.target_offsets[l + 1] > d.target_offsets[l];
        bfx::require(valid ? (has_s && has_t) : (!has_s && !has_t), "invalid terminal payload");
      }
      const std::uint32_t S = d.source_offsets[W], Tg = d.target_offsets[W];
      bfx::require(S == 0 || d.sources, "null sources");
      bfx::require(Tg == 0 || d.targets, "null targets");
      bfx::require(d.range_count == d.union_tile_count, "one vertex range per union tile is required");
      std::uint64_t U = 0;
      for (std::uint32_t i = 0; i < d.union_tile_count; ++i) {
        const std::uint32_t t = d.union_tiles[i];
        if (t >= g.T) throw std::out_of_range("union tile out of range");
        bfx::require(i == 0 || t > d.union_tiles[i - 1], "union tiles must be strictly increasing");
        const bfx_batch_vertex_range& r = d.selected_vertex_ranges[i];
        bfx::require(r.begin == tvo[t] && r.end == tvo[t + 1], "vertex range does not match its tile");
        bfx::require(r.lane_mask == d.tile_lane_masks[t] && r.lane_mask != 0 && (r.lane_mask & ~d.valid_lane_mask) == 0,
                     "invalid tile lane mask");
        U += r.end - r.begin;
      }
      bfx::require(U > 0, "batch has no selected vertices");
      if (U > 0x7FFFFFFFull) throw std::overflow_error("union vertex count exceeds the device index range");
      for (std::uint32_t l = 0; l < W; ++l) {
        for (std::uint32_t i = d.source_offsets[l]; i < d.source_offsets[l + 1]; ++i) {
          const std::uint32_t v = d.sources[i];
          if (v >= g.V) throw std::out_of_range("source out of range");
        }
        for (std::uint32_t i = d.target_offsets[l]; i < d.target_offsets[l + 1]; ++i) {
          if (d.targets[i] >= g.V) throw std::out_of_range("target out of range");
        }
      }
      // Full-graph batch: every tile in order, each selected by every valid
      // lane -- the frontier then needs no tile-table lookup per edge.
      bool full = d.range_count == g.T;
      for (std::uint32_t i = 0; full && i < d.range_count; ++i) {
        full = d.union_tiles[i] == i && d.selected_vertex_ranges[i].lane_mask == d.valid_lane_mask;
      }
      sz[b] = bfx::BatchSizes{static_cast<std::uint32_t>(U), d.range_count, S, Tg, W,
                              static_cast<std::uint32_t>(__builtin_ctz(W)), d.valid_lane_mask, full ? 1u : 0u};
    }
    // Terminal ownership: a terminal's owner tile must be selected for its
    // lane (terminal_owner_tile_not_selected, src/query.cpp:221-236).
    auto owner_of = [&](std::uint32_t v) {
      return static_cast<std::uint32_t>(std::upper_bound(tvo.begin(), tvo.end(), v) - tvo.begin()) - 1U;
    };
    for (std::uint32_t b = 0; b < count; ++b) {
      const bfx_batch_description& d = batches[b];
      for (std::uint32_t l = 0; l < d.lane_width; ++l) {
        for (std::uint32_t i = d.source_offsets[l]; i < d.source_offsets[l + 1]; ++i) {
          bfx::require((d.tile_lane_masks[owner_of(d.sources[i])] >> l) & 1u, "terminal owner tile not selected");
          bfx::require(i == d.source_offsets[l] || d.sources[i] > d.sources[i - 1], "noncanonical sources");
        }
        for (std::uint32_t i = d.target_offsets[l]; i < d.target_offsets[l + 1]; ++i) {
          bfx::require((d.tile_lane_masks[owner_of(d.targets[i])] >> l) & 1u, "terminal owner tile not selected");
          bfx::require(i == d.target_offsets[l] || d.targets[i] > d.targets[i - 1], "noncanonical targets");
        }
      }
    }
    const bfx::Layout L = bfx::lay_out_batches(ws, count, sz);
    char* hb = static_cast<char*>(ws->staging.ptr);
    for (std::uint32_t b = 0; b < count; ++b) {
      const bfx_batch_description& d = batches[b];
      const bfx::BatchSizes& s = sz[b];
      const bfx::DescArrays& a = L.arrays[b];
      std::memcpy(hb + a.src_off, d.source_offsets, (s.W + 1) * 4);
      if (s.S) std::memcpy(hb + a.src, d.sources, size_t{s.S} * 4);
      std::memcpy(hb + a.tgt_off, d.target_offsets, (s.W + 1) * 4);
      if (s.Tg) std::memcpy(hb + a.tgt, d.targets, size_t{s.Tg} * 4);
      uint4* ranges = reinterpret_cast<uint4*>(hb + a.ranges);
      std::uint32_t* roff = reinterpret_cast<std::uint32_t*>(hb + a.range_off);
      roff[0] = 0;
      for (std::uint32_t i = 0; i < s.R; ++i) {
        const bfx_batch_vertex_range& r = d.selected_vertex_ranges[i];
        ranges[i] = make_uint4(d.union_tiles[i], r.begin, r.end, r.lane_mask);
        roff[i + 1] = roff[i] + (r.end - r.begin);
      }
    }
    bfx::upload(ws->meta.ptr, hb, L.meta_total, ws->stream);
    ws->last_h2d = L.meta_total;
    // Tile tables must read 0 outside the union (init_kernel writes the union).
    BFX_CUDA(cudaMemsetAsync(ws->tile_tables.ptr, 0, bfx::align256(size_t{g.T} * 8) * count, ws->stream));
    // Staging must outlive the async copy: synchronise before the host may
    // reuse it (the next prepare overwrites it).
    BFX_CUDA(cudaStreamSynchronize(ws->stream));
  });
}

int bfx_prepare_batches_from_queries(bfx_workspace* ws, uint32_t batch_count, const bfx_batch_lanes* batches,
                                     uint32_t query_count, const bfx_route_query* queries) {
  return bfx::guarded([&] {
    using bfx::u32;
    bfx::require(ws != nullptr, "null workspace");
    bfx::require(batch_count > 0 && batches && queries, "at least one batch is required");
    if (batch_count > bfx::kMaxBatchesPerLaunch) throw std::length_error("too many batches for one launch");
    BFX_CUDA(cudaSetDevice(ws->graph->device));
    const bfx::DGraph& g = ws->graph->g;
    // Host checks of the image (validate_batch_device_description's terms,
    // include/bfnew/batch_layout.hpp:176-199): lane widths and counts, query
    // indices, strictly increasing tiles and terminals in range.  Terminal
    // ownership is checked on the device.
    std::vector<std::uint8_t> used(query_count, 0);
    std::vector<u32> lane_base(batch_count + 1, 0U), lane_query, lane_tile_base(1, 0U);
    std::vector<bfx::BatchSizes> sz(batch_count);
    for (u32 b = 0; b < batch_count; ++b) {
      const bfx_batch_lanes& d = batches[b];
      const u32 W = d.lane_width;
      bfx::require(W == 1 || W == 8 || W == 16 || W == 32, "unsupported lane width");
      bfx::require(d.lane_count >= 1 && d.lane_count <= W, "lane count must be 1..lane width");
      bfx::require(d.query_index_by_lane != nullptr, "null lane query indices");
      u32 S = 0, Tg = 0;
      for (u32 l = 0; l < d.lane_count; ++l) {
        const u32 qi = d.query_index_by_lane[l];
        if (qi >= query_count) throw std::out_of_range("lane query index out of range");
        const bfx_route_query& r = queries[qi];
        if (!used[qi]) {
          bfx::require(r.source_count > 0 && r.target_count > 0, "route queries require sources and targets");
          bfx::require(r.selected_tile_count > 0 && r.selected_tiles && r.sources && r.targets, "null query array");
          for (u32 i = 0; i < r.selected_tile_count; ++i) {
            if (r.selected_tiles[i] >= g.T) throw std::out_of_range("selected tile out of range");
            bfx::require(i == 0 || r.selected_tiles[i] > r.selected_tiles[i - 1],
                         "selected tiles must be strictly increasing");
          }
          for (u32 i = 0; i < r.source_count; ++i) {
            if (r.sources[i] >= g.V) throw std::out_of_range("source out of range");
            bfx::require(i == 0 || r.sources[i] > r.sources[i - 1], "noncanonical sources");
          }
          for (u32 i = 0; i < r.target_count; ++i) {
            if (r.targets[i] >= g.V) throw std::out_of_range("target out of range");
            bfx::require(i == 0 || r.targets[i] > r.targets[i - 1], "noncanonical targets");
          }
          used[qi] = 1;
        }
        S += r.source_count;
        Tg += r.target_count;
        lane_query.push_back(qi);
        lane_tile_base.push_back(lane_tile_base.back() + r.selected_tile_count);
      }
      lane_base[b + 1] = static_cast<u32>(lane_query.size());
      const u32 valid = d.lane_count == 32 ? 0xFFFFFFFFu : ((1u << d.lane_count) - 1u);
      sz[b] = bfx::BatchSizes{0, 0, S, Tg, W, static_cast<u32>(__builtin_ctz(W)), valid, 0};
    }
    // The query image: per-query tiles and terminals (concatenated), lane
    // tables, batch valid masks; one upload.
    std::vector<u32> qt_off(query_count + 1, 0U), qs_off(query_count + 1, 0U), qg_off(query_count + 1, 0U);
    for (u32 qi = 0; qi < query_count; ++qi) {
      const bfx_route_query& r = queries[qi];
      qt_off[qi + 1] = qt_off[qi] + (used[qi] ? r.selected_tile_count : 0U);
      qs_off[qi + 1] = qs_off[qi] + (used[qi] ? r.source_count : 0U);
      qg_off[qi + 1] = qg_off[qi] + (used[qi] ? r.target_count : 0U);
    }
    const u32 lanes = static_cast<u32>(lane_query.size());
    size_t o = 0;
    auto slot = [&](size_t words) {
      const size_t at = o;
      o = bfx::align256(o + words * 4);
      return at;
    };
    const size_t o_qt_off = slot(query_count + 1), o_qt = slot(qt_off[query_count]);
    const size_t o_qs_off = slot(query_count + 1), o_qs = slot(qs_off[query_count]);
    const size_t o_qg_off = slot(query_count + 1), o_qg = slot(qg_off[query_count]);
    const size_t o_lb = slot(batch_count + 1), o_lq = slot(lanes), o_ltb = slot(lanes + 1);
    const size_t o_valid = slot(batch_count), o_count = slot(4 * size_t{batch_count}), o_err = slot(1);
    const size_t image_bytes = o;
    ws->qimage.reserve(image_bytes, ws->graph->device);
    ws->staging.reserve(image_bytes);
    char* hb = static_cast<char*>(ws->staging.ptr);
    char* qb = static_cast<char*>(ws->qimage.ptr);
    auto put = [&](size_t at, const u32* src, size_t words) {
      if (words) std::memcpy(hb + at, src, words * 4);
    };
    put(o_qt_off, qt_off.data(), query_count + 1);
    put(o_qs_off, qs_off.data(), query_count + 1);
    put(o_qg_off, qg_off.data(), query_count + 1);
    for (u32 qi = 0; qi < query_count; ++qi) {
      if (!used[qi]) continue;
      const bfx_route_query& r = queries[qi];
      put(o_qt + size_t{qt_off[qi]} * 4, r.selected_tiles, r.selected_tile_count);
      put(o_qs + size_t{qs_off[qi]} * 4, r.sources, r.source_count);
      put(o_qg + size_t{qg_off[qi]} * 4, r.targets, r.target_count);
    }
    put(o_lb, lane_base.data(), batch_count + 1);
    put(o_lq, lane_query.data(), lanes);
    put(o_ltb, lane_tile_base.data(), lanes + 1);
    for (u32 b = 0; b < batch_count; ++b) reinterpret_cast<u32*>(hb + o_valid)[b] = sz[b].valid;
    reinterpret_cast<u32*>(hb + o_err)[0] = 0U;
    bfx::upload(qb, hb, image_bytes, ws->stream);
    bfx::QueryImage q{};
    q.tile_off = reinterpret_cast<const u32*>(qb + o_qt_off);
    q.tiles = reinterpret_cast<const u32*>(qb + o_qt);
    q.src_off = reinterpret_cast<const u32*>(qb + o_qs_off);
    q.srcs = reinterpret_cast<const u32*>(qb + o_qs);
    q.tgt_off = reinterpret_cast<const u32*>(qb + o_qg_off);
    q.tgts = reinterpret_cast<const u32*>(qb + o_qg);
    q.lane_base = reinterpret_cast<const u32*>(qb + o_lb);
    q.lane_query = reinterpret_cast<const u32*>(qb + o_lq);
    q.lane_tile_base = reinterpret_cast<const u32*>(qb + o_ltb);
    q.nb = batch_count;
    q.lanes = lanes;
    // Tile masks on the device, then the union sizes (one small readback
    // sizes the arena).
    const size_t tile_table_bytes = bfx::align256(size_t{g.T} * 8);
    const std::uint64_t tstride = tile_table_bytes / 8;
    ws->tile_tables.reserve(tile_table_bytes * batch_count, ws->graph->device);
    uint2* tiles = static_cast<uint2*>(ws->tile_tables.ptr);
    BFX_CUDA(cudaMemsetAsync(tiles, 0, tile_table_bytes * batch_count, ws->stream));
    const int wide = ws->sm_count * 8;
    bfx::desc_mask_kernel<<<wide, 256, 0, ws->stream>>>(q, tiles, tstride);
    BFX_CUDA(cudaGetLastError());
    u32* d_count = reinterpret_cast<u32*>(qb + o_count);
    bfx::desc_count_kernel<<<batch_count, 512, 0, ws->stream>>>(g.tile_off, g.T, tiles, tstride,
                                                                reinterpret_cast<const u32*>(qb + o_valid), d_count);
    BFX_CUDA(cudaGetLastError());
    std::vector<u32> counts(4 * size_t{batch_count});
    BFX_CUDA(cudaMemcpyAsync(counts.data(), d_count, counts.size() * 4, cudaMemcpyDeviceToHost, ws->stream));
    BFX_CUDA(cudaStreamSynchronize(ws->stream));
    for (u32 b = 0; b < batch_count; ++b) {
      sz[b].R = counts[4 * b];
      sz[b].U = counts[4 * b + 1];
      sz[b].full = (sz[b].R == g.T && counts[4 * b + 2] == 0U) ? 1U : 0U;
      bfx::require(sz[b].U > 0, "batch has no selected vertices");
    }
    // Layout, records, then the description arrays written on the device.
    const bfx::Layout L = bfx::lay_out_batches(ws, batch_count, sz);
    bfx::upload(ws->meta.ptr, ws->staging.ptr, L.o_up, ws->stream);
    ws->last_h2d = image_bytes + L.o_up;
    u32* d_err = reinterpret_cast<u32*>(qb + o_err);
    bfx::desc_fill_kernel<<<batch_count, 512, 0, ws->stream>>>(q, g.owner, g.tile_off, g.T, tiles, tstride,
                                                               ws->params.batches, d_err);
    BFX_CUDA(cudaGetLastError());
    u32 err = 0;
    BFX_CUDA(cudaMemcpyAsync(&err, d_err, 4, cudaMemcpyDeviceToHost, ws->stream));
    BFX_CUDA(cudaStreamSynchronize(ws->stream));
    if (err) {
      ws->nb = 0;
      throw std::invalid_argument("terminal owner tile not selected");
    }
  });
}

int bfx_fetch_prepared_description(bfx_workspace* ws, uint32_t batch, uint32_t counts[5], uint32_t* source_offsets,
                                   uint32_t* sources, uint32_t* target_offsets, uint32_t* targets,
                                   uint32_t* union_tiles, uint32_t* tile_lane_masks,
                                   bfx_batch_vertex_range* selected_vertex_ranges) {
  return bfx::guarded([&] {
    bfx::require(ws && counts, "null argument");
    bfx::require(ws->nb > 0, "no prepared batches");
    if (batch >= ws->nb) throw std::out_of_range("batch index");
    BFX_CUDA(cudaSetDevice(ws->graph->device));
    const bfx::DBatch& B = ws->batches[batch];
    counts[0] = B.W;
    counts[1] = B.valid;
    counts[2] = B.src_count;
    counts[3] = B.tgt_count;
    counts[4] = B.range_count;
    if (!(source_offsets && sources && target_offsets && targets && union_tiles && tile_lane_masks &&
          selected_vertex_ranges)) {
      return;  // counts only
    }
    const std::uint32_t T = ws->graph->g.T;
    std::vector<uint4> ranges(B.range_count);
    BFX_CUDA(cudaMemcpyAsync(source_offsets, B.src_off, (B.W + 1) * 4, cudaMemcpyDeviceToHost, ws->stream));
    if (B.src_count)
      BFX_CUDA(cudaMemcpyAsync(sources, B.src, size_t{B.src_count} * 4, cudaMemcpyDeviceToHost, ws->stream));
    BFX_CUDA(cudaMemcpyAsync(target_offsets, B.tgt_off, (B.W + 1) * 4, cudaMemcpyDeviceToHost, ws->stream));
    if (B.tgt_count)
      BFX_CUDA(cudaMemcpyAsync(targets, B.tgt, size_t{B.tgt_count} * 4, cudaMemcpyDeviceToHost, ws->stream));
    if (B.range_count)
      BFX_CUDA(cudaMemcpyAsync(ranges.data(), B.ranges, size_t{B.range_count} * 16, cudaMemcpyDeviceToHost,
                               ws->stream));
    BFX_CUDA(cudaStreamSynchronize(ws->stream));
    // dense masks from the prepared ranges (the tile table itself is
    // completed by the launch's init)
    std::fill(tile_lane_masks, tile_lane_masks + T, 0U);
    for (std::uint32_t i = 0; i < B.range_count; ++i) {
      union_tiles[i] = ranges[i].x;
      selected_vertex_ranges[i] = bfx_batch_vertex_range{ranges[i].y, ranges[i].z, ranges[i].w};
      if (ranges[i].x < T) tile_lane_masks[ranges[i].x] = ranges[i].w;
    }
  });
}

}  // extern "C"

namespace bfx {
namespace {

void validate_options(const bfx_gpu_run_options& o, bool allow_auto = false) {
  if (o.engine > 2u && !(allow_auto && o.engine == BFX_ENGINE_AUTO)) throw std::invalid_argument("invalid engine");
  if (o.control_mode > 2u) throw std::invalid_argument("invalid control mode");
  if (o.rounds_per_chunk == 0u) throw std::invalid_argument("invalid rounds per chunk");
  if (o.block_size == 0u || o.block_size % 32u != 0u || o.block_size > 512u)
    throw std::invalid_argument("invalid block size");
  if (o.grid_policy > 1u) throw std::invalid_argument("invalid grid policy");
  if (o.grid_policy == 1u && o.blocks_per_wgp == 0u) throw std::invalid_argument("invalid blocks per SM");
  if (o.grid_policy == 0u && o.blocks_per_wgp != 0u) throw std::invalid_argument("invalid blocks per SM");
  if (o.instrumentation > 2u) throw std::invalid_argument("invalid instrumentation");
  if (o.maximum_rounds == 0u) throw std::invalid_argument("invalid maximum rounds");
  if (o.enable_per_lane_convergence > 1u) throw std::invalid_argument("invalid per-lane convergence flag");
}

int grid_blocks(bfx_workspace* ws, const void* kernel, int block, size_t smem, const bfx_gpu_run_options& o) {
  int per_sm = 0;
  BFX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, smem));
  if (per_sm <= 0) throw Error(BFX_ERR_CUDA, "kernel cannot be resident with this block size");
  if (o.grid_policy == 1u) {
    if (static_cast<int>(o.blocks_per_wgp) > per_sm)
      throw std::invalid_argument("blocks per SM exceed the cooperative residency limit");
    per_sm = static_cast<int>(o.blocks_per_wgp);
  }
  return per_sm * ws->sm_count;
}

// Persistent kernel instantiation: 64 registers (two 512-thread blocks per
// SM) with 2, 3 or 4 flat work items per thread, or 40 registers with 2;
// the chunked layout has its own: 64 registers with 2 items, or 80 (blocks
// of at most 256 threads) with 2, 3 or 4.
const void* persistent_entry(bool count, std::uint32_t registers, std::uint32_t items, bool chunked, bool pairs) {
  const bool wide = registers != 40u;
  if (chunked && !pairs && registers == 80u) {
    if (items == 3u) {
      return count ? reinterpret_cast<const void*>(persistent_kernel<true, kBlocks256x3, 3, true>)
                   : reinterpret_cast<const void*>(persistent_kernel<false, kBlocks256x3, 3, true>);
    }
    if (items == 4u) {
      return count ? reinterpret_cast<const void*>(persistent_kernel<true, kBlocks256x3, 4, true>)
                   : reinterpret_cast<const void*>(persistent_kernel<false, kBlocks256x3, 4, true>);
    }
    return count ? reinterpret_cast<const void*>(persistent_kernel<true, kBlocks256x3, 2, true>)
                 : reinterpret_cast<const void*>(persistent_kernel<false, kBlocks256x3, 2, true>);
  }
  if (chunked && pairs) {
    return count ? reinterpret_cast<const void*>(persistent_kernel<true, 2, 2, true, true>)
                 : reinterpret_cast<const void*>(persistent_kernel<false, 2, 2, true, true>);
  }
  if (chunked) {
    return count ? reinterpret_cast<const void*>(persistent_kernel<true, 2, 2, true>)
                 : reinterpret_cast<const void*>(persistent_kernel<false, 2, 2, true>);
  }
  if (!wide) {
    return count ? reinterpret_cast<const void*>(persistent_kernel<true, 3, 2>)
                 : reinterpret_cast<const void*>(persistent_kernel<false, 3, 2>);
  }
  if (items == 3u) {
    return count ? reinterpret_cast<const void*>(persistent_kernel<true, 2, 3>)
                 : reinterpret_cast<const void*>(persistent_kernel<false, 2, 3>);
  }
  if (items == 4u) {
    return count ? reinterpret_cast<const void*>(persistent_kernel<true, 2, 4>)
                 : reinterpret_cast<const void*>(persistent_kernel<false, 2, 4>);
  }
  return count ? reinterpret_cast<const void*>(persistent_kernel<true, 2, 2>)
               : reinterpret_cast<const void*>(persistent_kernel<false, 2, 2>);
}

// A per-batch launch parameter array (engines, steps, mappings) on the
// device.  Uploaded only when it differs from the last upload, after the
// workspace stream drained, so a launch still in flight never sees a
// half-written array and no staging buffer is rewritten under an
// asynchronous copy.
const std::uint32_t* upload_batch_words(bfx_workspace* ws, DeviceBuffer& dev, std::vector<std::uint32_t>& uploaded,
                                        const std::vector<std::uint32_t>& words) {
  if (dev.ptr == nullptr || uploaded != words) {
    BFX_CUDA(cudaStreamSynchronize(ws->stream));
    dev.reserve(words.size() * 4, ws->graph->device);
    BFX_CUDA(cudaMemcpy(dev.ptr, words.data(), words.size() * 4, cudaMemcpyHostToDevice));
    uploaded = words;
  }
  return static_cast<const std::uint32_t*>(dev.ptr);
}

void execute(bfx_workspace* ws, const bfx_gpu_run_options& o) {
  require(ws->nb > 0, "no prepared batches");
  validate_options(o, true);
  BFX_CUDA(cudaSetDevice(ws->graph->device));
  LaunchParams p = ws->params;
  p.engine = o.engine;
  p.per_lane = o.enable_per_lane_convergence;
  p.max_rounds = o.maximum_rounds;
  p.budget_ns = kLaunchBudgetNs;
  p.engines = nullptr;
  p.deltas = nullptr;
  p.flat = ws->frontier_layout == BFX_FRONTIER_FLAT ? 1u : (ws->frontier_layout == BFX_FRONTIER_CHUNKED ? 2u : 0u);
  p.cshift = 5u;
  p.cpack = ws->chunk_pack;
  p.tile_stage_min = ws->tile_stage_min;
  p.tile_iters = ws->tile_iters;
  p.tile_wmax = 1u;
  if (ws->frontier_layout == BFX_FRONTIER_TILED) {
    // the tiled layout runs in persistent mode; host-poll modes use the
    // chunked layout's round kernels
    p.flat = o.control_mode == BFX_CONTROL_PERSISTENT_COOPERATIVE ? 3u : 2u;
    if (p.flat == 3u) {
      p.tshift = ws->graph->tile_shift;
      for (const DBatch& b : ws->batches) p.tile_wmax = std::max(p.tile_wmax, b.W);
      if (!ws->batch_mappings.empty()) {
        require(ws->batch_mappings.size() == ws->nb, "per-batch mappings do not match the prepared batches");
        p.mappings = upload_batch_words(ws, ws->mappings_dev, ws->mappings_uploaded, ws->batch_mappings);
      }
    }
  }
  p.round_trace = nullptr;
  p.trace_cap = 0u;
  p.amin = ws->relax_atomic;
  p.edge_major = ws->edge_major;
  if (o.instrumentation == 2u && o.control_mode == BFX_CONTROL_PERSISTENT_COOPERATIVE) {
    ws->round_trace.reserve(size_t{kRoundTraceCap} * 32u, ws->graph->device);
    BFX_CUDA(cudaMemsetAsync(ws->round_trace.ptr, 0, size_t{kRoundTraceCap} * 32u, ws->stream));
    p.round_trace = static_cast<u64*>(ws->round_trace.ptr);
    p.trace_cap = kRoundTraceCap;
  }
  if (!ws->batch_deltas.empty()) {
    require(ws->batch_deltas.size() == ws->nb, "per-batch deltas do not match the prepared batches");
    std::vector<std::uint32_t> bits(ws->nb);
    std::memcpy(bits.data(), ws->batch_deltas.data(), ws->nb * 4);
    p.deltas = upload_batch_words(ws, ws->deltas_dev, ws->deltas_uploaded, bits);
  }
  if (o.engine == BFX_ENGINE_AUTO) {
    // Per-batch engines chosen by bfx_autotune / bfx_set_batch_engines
    // (frontier push where none was chosen).
    std::vector<std::uint32_t> eng(ws->nb, BFX_ENGINE_FRONTIER_PUSH);
    if (ws->batch_engines.size() == ws->nb) eng = ws->batch_engines;
    p.engines = upload_batch_words(ws, ws->engines_dev, ws->engines_uploaded, eng);
    p.engine = BFX_ENGINE_FRONTIER_PUSH;
  }
  const int block = static_cast<int>(o.block_size);
  const size_t smem = (size_t{ws->nb} + 1) * 4;
  std::uint64_t launches = 0;
  ws->last_host_checks = 0;
  BFX_CUDA(cudaEventRecord(ws->ev[0], ws->stream));
  // init + seed with a wide ordinary grid
  const int wide = ws->sm_count * 8;
  init_kernel<<<wide, 256, 0, ws->stream>>>(p);
  ++launches;
  BFX_CUDA(cudaGetLastError());
  const int seed_blocks = static_cast<int>(std::min<std::uint64_t>(
      std::max<std::uint64_t>(1, (ws->src_total + 255) / 256), static_cast<std::uint64_t>(wide)));
  seed_kernel<<<seed_blocks, 256, 0, ws->stream>>>(p, ws->src_base);
  ++launches;
  BFX_CUDA(cudaGetLastError());
  BFX_CUDA(cudaEventRecord(ws->ev[1], ws->stream));
  if (o.control_mode == BFX_CONTROL_PERSISTENT_COOPERATIVE && p.flat == 3u) {
    require(block == 256 || block == 384, "the tiled frontier layout runs blocks of 256 or 384 threads");
    const void* kfn =
        block == 256 ? (o.instrumentation != 0u ? reinterpret_cast<const void*>(persistent_tiled_kernel<true, 256>)
                                                : reinterpret_cast<const void*>(persistent_tiled_kernel<false, 256>))
                     : (o.instrumentation != 0u ? reinterpret_cast<const void*>(persistent_tiled_kernel<true, 384>)
                                                : reinterpret_cast<const void*>(persistent_tiled_kernel<false, 384>));
    const size_t tsmem = tile_smem_bytes(ws->nb, p.tshift, p.tile_wmax);
    BFX_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(tsmem)));
    const int grid = grid_blocks(ws, kfn, block, tsmem, o);
    void* args[] = {&p};
    BFX_CUDA(cudaLaunchCooperativeKernel(kfn, grid, block, args, tsmem, ws->stream));
    ++launches;
  } else if (o.control_mode == BFX_CONTROL_PERSISTENT_COOPERATIVE) {
    // register budget 0 (default): 80 for the chunked layout with blocks of
    // at most 256 threads, 64 otherwise
    const std::uint32_t regs =
        ws->register_budget != 0u ? ws->register_budget : (p.flat == 2u && block <= 256 ? 80u : 64u);
    const void* kfn = persistent_entry(o.instrumentation != 0u, regs, ws->flat_items, p.flat == 2u,
                                       ws->chunk_pairs != 0u);
    require(!(regs == 80u && p.flat == 2u && ws->chunk_pairs == 0u) || block <= 256,
            "the 80-register chunked kernel needs blocks of at most 256 threads");
    const int grid = grid_blocks(ws, kfn, block, smem, o);
    void* args[] = {&p};
    BFX_CUDA(cudaLaunchCooperativeKernel(kfn, grid, block, args, smem, ws->stream));
    ++launches;
  } else {
    const std::uint32_t K = o.control_mode == BFX_CONTROL_PER_ROUND_HOST_POLL ? 1u : o.rounds_per_chunk;
    const bool chunked = p.flat == 2u;
    const void* kfn = o.instrumentation
                          ? (chunked ? reinterpret_cast<const void*>(round_kernel<true, true>)
                                     : reinterpret_cast<const void*>(round_kernel<true, false>))
                          : (chunked ? reinterpret_cast<const void*>(round_kernel<false, true>)
                                     : reinterpret_cast<const void*>(round_kernel<false, false>));
    const int grid = grid_blocks(ws, kfn, block, smem, o);
    start_kernel<<<1, 1024, smem, ws->stream>>>(p);
    ++launches;
    BFX_CUDA(cudaGetLastError());
    // Capture K x (round, advance) once per workspace generation / K / engine.
    const bool reuse = ws->chunk_exec && ws->chunk_rounds == K && ws->chunk_grid == grid &&
                       ws->chunk_instr == o.instrumentation &&
                       ws->chunk_block == block && std::memcmp(&ws->chunk_params, &p, sizeof(p)) == 0;
    if (!reuse) {
      if (ws->chunk_exec) cudaGraphExecDestroy(ws->chunk_exec);
      ws->chunk_exec = nullptr;
      cudaGraph_t graph;
      BFX_CUDA(cudaStreamBeginCapture(ws->stream, cudaStreamCaptureModeThreadLocal));
      for (std::uint32_t k = 0; k < K; ++k) {
        if (o.instrumentation) {
          if (chunked) {
            round_kernel<true, true><<<grid, block, smem, ws->stream>>>(p);
          } else {
            round_kernel<true, false><<<grid, block, smem, ws->stream>>>(p);
          }
        } else {
          if (chunked) {
            round_kernel<false, true><<<grid, block, smem, ws->stream>>>(p);
          } else {
            round_kernel<false, false><<<grid, block, smem, ws->stream>>>(p);
          }
        }
        advance_kernel<<<1, 1024, smem, ws->stream>>>(p);
      }
      BFX_CUDA(cudaStreamEndCapture(ws->stream, &graph));
      const cudaError_t ie = cudaGraphInstantiate(&ws->chunk_exec, graph, 0);
      cudaGraphDestroy(graph);
      BFX_CUDA(ie);
      ws->chunk_rounds = K;
      ws->chunk_grid = grid;
      ws->chunk_block = block;
      ws->chunk_instr = o.instrumentation;
      ws->chunk_params = p;
    }
    // Poll the device controller after every chunk, as the reference's
    // ordinary modes do (src/hip/batched_frontier_push.hip.cpp:1613-1654).
    ws->status_host.reserve(256);
    std::uint32_t* const done_host = static_cast<std::uint32_t*>(ws->status_host.ptr);
    const std::uint64_t max_chunks = (o.maximum_rounds + K - 1) / K + 1;
    ws->last_host_checks = 0;
    const auto t0 = std::chrono::steady_clock::now();
    for (std::uint64_t c = 0; c < max_chunks; ++c) {
      BFX_CUDA(cudaMemcpyAsync(done_host, &p.run->done, 4, cudaMemcpyDeviceToHost, ws->stream));
      BFX_CUDA(cudaStreamSynchronize(ws->stream));
      ++ws->last_host_checks;
      if (*done_host) break;
      if (std::chrono::steady_clock::now() - t0 > std::chrono::nanoseconds(kLaunchBudgetNs)) {
        // same outcome as a persistent launch past its budget: device_failure
        BFX_CUDA(cudaMemsetAsync(&p.run->abort, 1, 1, ws->stream));
        break;
      }
      BFX_CUDA(cudaGraphLaunch(ws->chunk_exec, ws->stream));
      launches += 2ull * K;
    }
  }
  BFX_CUDA(cudaGetLastError());
  BFX_CUDA(cudaEventRecord(ws->ev[2], ws->stream));
  finalize_kernel<<<ws->nb, 256, 0, ws->stream>>>(p, ws->d_ctrl, ws->d_status);
  ++launches;
  BFX_CUDA(cudaGetLastError());
  BFX_CUDA(cudaEventRecord(ws->ev[3], ws->stream));
  ws->last_launches = launches;
  ws->executed = true;
  ws->paths_ready = false;
  ws->params.engine = o.engine;
  ws->params.per_lane = o.enable_per_lane_convergence;
}

}  // namespace
}  // namespace bfx

extern "C" {

int bfx_set_register_budget(bfx_workspace* ws, uint32_t registers) {
  return bfx::guarded([&] {
    bfx::require(ws != nullptr, "null argument");
    bfx::require(registers == 0u || registers == 40u || registers == 64u || registers == 80u,
                 "register budget must be 0 (automatic), 40, 64 or 80");
    ws->register_budget = registers;
  });
}

int bfx_set_chunk_pack(bfx_workspace* ws, uint32_t pack) {
  return bfx::guarded([&] {
    bfx::require(ws != nullptr, "null argument");
    bfx::require(pack == 1u || pack == 2u || pack == 4u || pack == 8u, "chunk pack must be 1, 2, 4 or 8");
    ws->chunk_pack = pack;
  });
}

int bfx_get_chunk_pack(bfx_workspace* ws, uint32_t* pack) {
  return bfx::guarded([&] {
    bfx::require(ws != nullptr && pack != nullptr, "null argument");
    *pack = ws->chunk_pack;
  });
}

int bfx_set_chunk_pairs(bfx_workspace* ws, uint32_t mode) {
  return bfx::guarded([&] {
    bfx::require(ws != nullptr, "null argument");
    bfx::require(mode <= 1u, "chunk pair mode must be 0 or 1");
    ws->chunk_pairs = mode;
  });
}

int bfx_set_flat_order(bfx_workspace* ws, uint32_t edge_major) {
  return bfx::guarded([&] {
    bfx::require(ws != nullptr, "null argument");
    bfx::require(edge_major <= 1u, "flat work order must be 0 or 1");
    ws->edge_major = edge_major;
  });
}

int bfx_set_relax_atomic(bfx_workspace* ws, uint32_t mode) {
  return bfx::guarded([&] {
    bfx::require(ws != nullptr, "null argument");
    bfx::require(mode <= 1u, "relaxation mode must be 0 or 1");
    ws->relax_atomic = mode;
  });
}

int bfx_set_flat_items(bfx_workspace* ws, uint32_t items) {
  return bfx::guarded([&] {
    bfx::require(ws != nullptr, "null argument");
    bfx::require(items >= 2u && items <= 4u, "flat work items per thread must be 2, 3 or 4");
    ws->flat_items = items;
  });
}

int bfx_set_frontier_layout(bfx_workspace* ws, uint32_t layout) {
  return bfx::guarded([&] {
    bfx::require(ws != nullptr, "null argument");
    bfx::require(layout == BFX_FRONTIER_GROUPS || layout == BFX_FRONTIER_FLAT || layout == BFX_FRONTIER_CHUNKED ||
                     layout == BFX_FRONTIER_TILED,
                 "invalid frontier layout");
    ws->frontier_layout = layout;
  });
}

int bfx_set_tile_stage_min(bfx_workspace* ws, uint32_t lane_edges) {
  return bfx::guarded([&] {
    bfx::require(ws != nullptr, "null argument");
    ws->tile_stage_min = lane_edges;
  });
}

int bfx_set_batch_mappings(bfx_workspace* ws, uint32_t count, const uint32_t* mappings) {
  return bfx::guarded([&] {
    bfx::require(ws != nullptr, "null workspace");
    bfx::require(count == 0 || mappings != nullptr, "null mappings");
    for (std::uint32_t i = 0; i < count; ++i) {
      bfx::require(mappings[i] == BFX_MAPPING_CHUNKS || mappings[i] == BFX_MAPPING_TILE_VISITS, "invalid mapping");
    }
    ws->batch_mappings.assign(mappings, mappings + count);
  });
}

int bfx_get_frontier_mapping(bfx_workspace* ws, uint32_t* layout, uint32_t count, uint32_t* mappings) {
  return bfx::guarded([&] {
    bfx::require(ws && layout, "null argument");
    *layout = ws->frontier_layout;
    for (std::uint32_t i = 0; i < count; ++i) {
      bfx::require(mappings != nullptr, "null mappings");
      mappings[i] = i < ws->batch_mappings.size() ? ws->batch_mappings[i] : BFX_MAPPING_TILE_VISITS;
    }
  });
}

int bfx_set_tile_passes(bfx_workspace* ws, uint32_t passes) {
  return bfx::guarded([&] {
    bfx::require(ws != nullptr, "null argument");
    bfx::require(passes >= 1u && passes <= 1024u, "tile passes must be 1..1024");
    ws->tile_iters = passes;
  });
}

int bfx_execute(bfx_workspace* ws, const bfx_gpu_run_options* options) {
  return bfx::guarded([&] {
    bfx::require(ws && options, "null argument");
    bfx::execute(ws, *options);
  });
}

int bfx_fetch_statuses(bfx_workspace* ws, bfx_device_run_status* statuses, bfx_device_controller* controllers) {
  return bfx::guarded([&] {
    bfx::require(ws != nullptr, "null workspace");
    bfx::require(ws->executed, "no executed batches");
    BFX_CUDA(cudaSetDevice(ws->graph->device));
    const size_t sb = ws->nb * sizeof(bfx_device_run_status);
    const size_t cb = ws->nb * sizeof(bfx_device_controller);
    ws->status_host.reserve(sb + cb + 256);
    char* h = static_cast<char*>(ws->status_host.ptr);
    if (statuses) BFX_CUDA(cudaMemcpyAsync(h, ws->d_status, sb, cudaMemcpyDeviceToHost, ws->stream));
    if (controllers) BFX_CUDA(cudaMemcpyAsync(h + sb, ws->d_ctrl, cb, cudaMemcpyDeviceToHost, ws->stream));
    BFX_CUDA(cudaStreamSynchronize(ws->stream));
    if (statuses) std::memcpy(statuses, h, sb);
    if (controllers) std::memcpy(controllers, h + sb, cb);
    ws->last_d2h = (statuses ? sb : 0) + (controllers ? cb : 0);
  });
}

int bfx_run_batches(bfx_workspace* ws, uint32_t count, const bfx_batch_description* batches,
                    const bfx_gpu_run_options* options, bfx_device_run_status* statuses) {
  int rc = bfx_prepare_batches(ws, count, batches);
  if (rc != BFX_OK) return rc;
  rc = bfx_execute(ws, options);
  if (rc != BFX_OK) return rc;
  return bfx_fetch_statuses(ws, statuses, nullptr);
}

int bfx_download_labels(bfx_workspace* ws, uint32_t batch, uint32_t* distance_bits, uint32_t* predecessor_edges) {
  return bfx::guarded([&] {
    bfx::require(ws != nullptr, "null workspace");
    bfx::require(ws->executed, "no executed batches");
    if (batch >= ws->nb) throw std::out_of_range("batch index");
    BFX_CUDA(cudaSetDevice(ws->graph->device));
    const bfx::DBatch& B = ws->batches[batch];
    const size_t n = static_cast<size_t>(ws->graph->g.V) << B.shift;
    bfx_device_run_status st;
    BFX_CUDA(cudaMemcpyAsync(&st, ws->d_status + batch, sizeof(st), cudaMemcpyDeviceToHost, ws->stream));
    BFX_CUDA(cudaStreamSynchronize(ws->stream));
    const std::uint32_t slot = st.final_distance_slot;
    std::uint32_t* d_out = nullptr;
    BFX_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&d_out), n * 8, ws->stream));
    bfx::expand_kernel<<<ws->sm_count * 8, 256, 0, ws->stream>>>(ws->graph->g, B, slot, d_out, d_out + n);
    const cudaError_t le = cudaGetLastError();
    if (le == cudaSuccess) {
      if (distance_bits) cudaMemcpyAsync(distance_bits, d_out, n * 4, cudaMemcpyDeviceToHost, ws->stream);
      if (predecessor_edges) cudaMemcpyAsync(predecessor_edges, d_out + n, n * 4, cudaMemcpyDeviceToHost, ws->stream);
    }
    cudaFreeAsync(d_out, ws->stream);
    BFX_CUDA(le);
    BFX_CUDA(cudaStreamSynchronize(ws->stream));
  });
}

int bfx_download_lane_labels(bfx_workspace* ws, uint32_t batch, uint32_t lane, uint32_t* distance_bits,
                             uint32_t* predecessor_edges) {
  return bfx::guarded([&] {
    bfx::require(ws != nullptr, "null workspace");
    bfx::require(ws->executed, "no executed batches");
    if (batch >= ws->nb) throw std::out_of_range("batch index");
    const bfx::DBatch& B = ws->batches[batch];
    if (lane >= B.W) throw std::out_of_range("lane index");
    BFX_CUDA(cudaSetDevice(ws->graph->device));
    const size_t n = ws->graph->g.V;
    bfx_device_run_status st;
    BFX_CUDA(cudaMemcpyAsync(&st, ws->d_status + batch, sizeof(st), cudaMemcpyDeviceToHost, ws->stream));
    BFX_CUDA(cudaStreamSynchronize(ws->stream));
    std::uint32_t* d_out = nullptr;
    BFX_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&d_out), n * 8, ws->stream));
    bfx::expand_lane_kernel<<<ws->sm_count * 8, 256, 0, ws->stream>>>(ws->graph->g, B, st.final_distance_slot, lane,
                                                                      d_out, d_out + n);
    const cudaError_t le = cudaGetLastError();
    if (le == cudaSuccess) {
      if (distance_bits) cudaMemcpyAsync(distance_bits, d_out, n * 4, cudaMemcpyDeviceToHost, ws->stream);
      if (predecessor_edges) cudaMemcpyAsync(predecessor_edges, d_out + n, n * 4, cudaMemcpyDeviceToHost, ws->stream);
    }
    cudaFreeAsync(d_out, ws->stream);
    BFX_CUDA(le);
    BFX_CUDA(cudaStreamSynchronize(ws->stream));
  });
}

int bfx_fetch_label_bounds(bfx_workspace* ws, uint32_t* max_finite_distance_bits) {
  return bfx::guarded([&] {
    bfx::require(ws && max_finite_distance_bits, "null argument");
    bfx::require(ws->executed, "no executed batches");
    BFX_CUDA(cudaSetDevice(ws->graph->device));
    std::uint32_t* d_out = nullptr;
    BFX_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&d_out), size_t{ws->nb} * 4, ws->stream));
    cudaError_t e = cudaMemsetAsync(d_out, 0, size_t{ws->nb} * 4, ws->stream);
    if (e == cudaSuccess) {
      bfx::label_bound_kernel<<<ws->sm_count * 8, 256, 0, ws->stream>>>(ws->params, ws->d_status, d_out);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
      e = cudaMemcpyAsync(max_finite_distance_bits, d_out, size_t{ws->nb} * 4, cudaMemcpyDeviceToHost, ws->stream);
    }
    cudaFreeAsync(d_out, ws->stream);
    BFX_CUDA(e);
    BFX_CUDA(cudaStreamSynchronize(ws->stream));
  });
}

int bfx_fetch_work_statistics(bfx_workspace* ws, bfx_device_work_statistics* stats, uint64_t counters[8]) {
  return bfx::guarded([&] {
    bfx::require(ws != nullptr, "null workspace");
    bfx::require(ws->executed, "no executed batches");
    BFX_CUDA(cudaSetDevice(ws->graph->device));
    std::uint64_t raw[16];
    BFX_CUDA(cudaMemcpyAsync(raw, ws->params.run->work, sizeof(raw), cudaMemcpyDeviceToHost, ws->stream));
    BFX_CUDA(cudaStreamSynchronize(ws->stream));
    // totals over the engines: Jacobi items count as entries and source reads
    const std::uint64_t w[8] = {raw[0] + raw[8], raw[1] + raw[9], raw[2] + raw[8], raw[3] + raw[10],
                                raw[4],          raw[5] + raw[11], raw[6],         raw[7]};
    if (counters) std::memcpy(counters, w, sizeof(w));
    if (stats) {
      std::memset(stats, 0, sizeof(*stats));
      stats->edges_examined = w[3];
      stats->successful_decreases = w[5];
      stats->active_vertices = w[0];
      stats->active_lane_rounds = w[2];
      stats->kernel_dispatches = ws->last_launches;
      stats->atomic_attempts = w[6];
      stats->successful_atomic_updates = w[5];
      stats->queue_claims = w[4];
      stats->full_edge_rounds = ws->params.engine == BFX_ENGINE_FRONTIER_PUSH ? 0u : w[7];
      stats->host_checks = ws->last_host_checks;
      stats->host_synchronizations = ws->last_host_checks;
      stats->controller_copies = ws->last_host_checks;
    }
  });
}

int bfx_fetch_round_trace(bfx_workspace* ws, uint32_t capacity, uint64_t* trace, uint32_t* rounds) {
  return bfx::guarded([&] {
    bfx::require(ws && rounds, "null argument");
    bfx::require(ws->executed, "no executed batches");
    BFX_CUDA(cudaSetDevice(ws->graph->device));
    std::uint64_t w[8];
    BFX_CUDA(cudaMemcpyAsync(w, ws->params.run->work, sizeof(w), cudaMemcpyDeviceToHost, ws->stream));
    BFX_CUDA(cudaStreamSynchronize(ws->stream));
    bfx::require(ws->round_trace.ptr != nullptr, "no traced run (instrumentation 2, persistent control)");
    const std::uint32_t n = static_cast<std::uint32_t>(std::min<std::uint64_t>(w[7], bfx::kRoundTraceCap));
    *rounds = n;
    if (trace && capacity) {
      const std::uint32_t m = std::min(n, capacity);
      BFX_CUDA(cudaMemcpy(trace, ws->round_trace.ptr, size_t{m} * 32u, cudaMemcpyDeviceToHost));
    }
  });
}

int bfx_fetch_engine_work(bfx_workspace* ws, uint64_t counters[16]) {
  return bfx::guarded([&] {
    bfx::require(ws && counters, "null argument");
    bfx::require(ws->executed, "no executed batches");
    BFX_CUDA(cudaSetDevice(ws->graph->device));
    BFX_CUDA(cudaMemcpyAsync(counters, ws->params.run->work, 16 * sizeof(std::uint64_t), cudaMemcpyDeviceToHost,
                             ws->stream));
    BFX_CUDA(cudaStreamSynchronize(ws->stream));
  });
}

int bfx_last_execute_timing(bfx_workspace* ws, float out[2]) {
  return bfx::guarded([&] {
    bfx::require(ws && out, "null argument");
    bfx::require(ws->executed, "no executed batches");
    BFX_CUDA(cudaSetDevice(ws->graph->device));
    BFX_CUDA(cudaEventSynchronize(ws->ev[3]));
    BFX_CUDA(cudaEventElapsedTime(&out[0], ws->ev[1], ws->ev[2]));
    BFX_CUDA(cudaEventElapsedTime(&out[1], ws->ev[0], ws->ev[3]));
  });
}

int bfx_workspace_transfer_bytes(bfx_workspace* ws, uint64_t out[2]) {
  return bfx::guarded([&] {
    bfx::require(ws && out, "null argument");
    out[0] = ws->last_h2d;
    out[1] = ws->last_d2h;
  });
}

int bfx_set_batch_deltas(bfx_workspace* ws, uint32_t count, const float* deltas) {
  return bfx::guarded([&] {
    bfx::require(ws != nullptr, "null workspace");
    bfx::require(count == 0 || deltas != nullptr, "null deltas");
    for (std::uint32_t i = 0; i < count; ++i) {
      bfx::require(deltas[i] > 0.0f, "near/far steps must be positive (+inf: plain frontier)");
    }
    ws->batch_deltas.assign(deltas, deltas + count);
  });
}

int bfx_set_batch_engines(bfx_workspace* ws, uint32_t count, const uint32_t* engines) {
  return bfx::guarded([&] {
    bfx::require(ws != nullptr, "null workspace");
    bfx::require(count == 0 || engines != nullptr, "null engines");
    for (std::uint32_t i = 0; i < count; ++i) bfx::require(engines[i] <= 2u, "invalid engine");
    ws->batch_engines.assign(engines, engines + count);
  });
}

int bfx_last_launch_count(bfx_workspace* ws, uint64_t* launches) {
  return bfx::guarded([&] {
    bfx::require(ws && launches, "null argument");
    *launches = ws->last_launches;
  });
}

int bfx_run_query(bfx_workspace* ws, uint32_t source_count, const uint32_t* sources, uint32_t target_count,
                  const uint32_t* targets, uint32_t selected_tile_count, const uint32_t* selected_tiles,
                  const bfx_gpu_run_options* options, bfx_device_run_status* status) {
  return bfx::guarded([&] {
    bfx::require(ws && options && status, "null argument");
    bfx::require(source_count > 0 && target_count > 0, "route queries require sources and targets");
    bfx::require(sources && targets && selected_tiles && selected_tile_count > 0, "null query array");
    const auto& tvo = ws->graph->tile_vertex_offsets;
    const std::uint32_t T = ws->graph->g.T;
    std::vector<std::uint32_t> masks(T, 0U);
    std::vector<bfx_batch_vertex_range> ranges(selected_tile_count);
    for (std::uint32_t i = 0; i < selected_tile_count; ++i) {
      const std::uint32_t t = selected_tiles[i];
      if (t >= T) throw std::out_of_range("selected tile out of range");
      bfx::require(i == 0 || t > selected_tiles[i - 1], "selected tiles must be strictly increasing");
      masks[t] = 1U;
      ranges[i] = bfx_batch_vertex_range{tvo[t], tvo[t + 1], 1U};
    }
    const std::uint32_t so[2] = {0U, source_count};
    const std::uint32_t to[2] = {0U, target_count};
    bfx_batch_description d;
    std::memset(&d, 0, sizeof(d));
    d.lane_width = 1;
    d.valid_lane_mask = 1;
    d.source_offsets = so;
    d.sources = sources;
    d.target_offsets = to;
    d.targets = targets;
    d.union_tile_count = selected_tile_count;
    d.tile_count = T;
    d.union_tiles = selected_tiles;
    d.tile_lane_masks = masks.data();
    d.range_count = selected_tile_count;
    d.selected_vertex_ranges = ranges.data();
    // The plain per-query engine runs the options' engine as given: per-batch
    // engines, near/far steps and mappings of the workspace's batch set do
    // not apply (they are kept for that set).
    struct Keep {
      bfx_workspace* ws;
      std::vector<std::uint32_t> engines, mappings;
      std::vector<float> deltas;
      explicit Keep(bfx_workspace* w) : ws(w) {
        engines.swap(w->batch_engines);
        deltas.swap(w->batch_deltas);
        mappings.swap(w->batch_mappings);
      }
      ~Keep() {
        ws->batch_engines.swap(engines);
        ws->batch_deltas.swap(deltas);
        ws->batch_mappings.swap(mappings);
      }
    } keep(ws);
    int rc = bfx_run_batches(ws, 1, &d, options, status);
    if (rc != BFX_OK) throw bfx::Error(rc, bfx_last_error());
  });
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Static-scratch single-query entry point (bfx_run_query_static).
//
// For callers that must not allocate device memory at call time: processes
// whose device memory is carved up and owned by another runtime (a host
// application or framework that hands the GPU's memory to its own pool and
// forbids other allocations), and latency-critical loops that cannot afford
// an allocation's implicit synchronisation.  bfx_run_query allocates its
// workspace on first use and grows it; this variant keeps every scratch
// buffer (labels, pending masks, frontier queues, tile table, batch records,
// launch state) in one file-scope device array of fixed size, so a call
// allocates nothing.  It runs the persistent cooperative control mode only,
// without instrumentation, on the legacy default stream with synchronous
// copies.
// ---------------------------------------------------------------------------

namespace bfx {
namespace {
constexpr size_t kStaticScratchBytes = size_t{32} << 20;  // 32 MiB per device
constexpr int kMaxStaticDevices = 64;
}  // namespace
}  // namespace bfx

// Every device that loads libbfx.so holds this array until the process exits.
// All calls on a device share it, and each call leaves its contents behind:
// the call re-initialises everything it reads (labels, masks, queues, tile
// table, counters) before relaxing.
static __device__ __align__(256) unsigned char bfx_static_scratch[bfx::kStaticScratchBytes];

namespace bfx {
namespace {

std::mutex g_static_mutex;
void* g_static_base[kMaxStaticDevices] = {};

// Device address of bfx_static_scratch on the current device, resolved once
// per device with cudaGetSymbolAddress (the host-side name is only a
// stand-in; kernels must be given this address).  The address is kept for
// the life of the process, so a cudaDeviceReset between calls is not
// supported (the module, and with it the array, may move).
cudaError_t static_scratch_base(int device, void** out) {
  std::lock_guard<std::mutex> lock(g_static_mutex);
  if (g_static_base[device] == nullptr) {
    void* p = nullptr;
    const cudaError_t rc = cudaGetSymbolAddress(&p, bfx_static_scratch);
    if (rc != cudaSuccess) return rc;
    g_static_base[device] = p;
  }
  *out = g_static_base[device];
  return cudaSuccess;
}

// Final label of every target of a width-1 batch: distance bits and the
// predecessor edge id (0xffffffff for sources and unreached targets).
__global__ void gather_targets_kernel(DGraph g, const DBatch* batch, const bfx_device_run_status* status,
                                      u32* out_bits, u32* out_pred) {
  const DBatch& B = *batch;
  const u32 slot = status->final_distance_slot;
  for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < B.tgt_count; i += gridDim.x * blockDim.x) {
    const u32 v = B.tgt[i];
    const uint2 t = B.tiles[g.owner[v]];
    const u64 w = (t.x & 1u) ? B.dist[slot][v - t.y] : dev::kUnreached;
    const u32 lo = static_cast<u32>(w);
    out_bits[i] = dev::hi(w);
    out_pred[i] = (lo == 0u || lo == 0xFFFFFFFFu) ? 0xFFFFFFFFu : lo - 1u;
  }
}

void copy_in(char* base, size_t off, const void* src, size_t bytes) {
  if (bytes) BFX_CUDA(cudaMemcpy(base + off, src, bytes, cudaMemcpyHostToDevice));
}

}  // namespace
}  // namespace bfx

extern "C" int bfx_run_query_static(const bfx_resident_graph* graph, uint32_t source_count, const uint32_t* sources,
                                    uint32_t target_count, const uint32_t* targets, uint32_t selected_tile_count,
                                    const uint32_t* selected_tiles, const bfx_gpu_run_options* options,
                                    bfx_device_run_status* status, uint32_t* target_distance_bits,
                                    uint32_t* target_predecessor_edges) {
  return bfx::guarded([&] {
    using bfx::u32;
    using bfx::u64;
    bfx::require(graph && options && status && target_distance_bits && target_predecessor_edges, "null argument");
    bfx::require(source_count > 0 && target_count > 0, "route queries require sources and targets");
    bfx::require(sources && targets && selected_tiles && selected_tile_count > 0, "null query array");
    bfx::validate_options(*options);
    bfx::require(options->control_mode == BFX_CONTROL_PERSISTENT_COOPERATIVE,
                 "the static-scratch query runs the persistent cooperative control mode only");
    bfx::require(options->instrumentation == 0u, "the static-scratch query has no instrumentation");
    if (graph->device < 0 || graph->device >= bfx::kMaxStaticDevices) throw std::out_of_range("device index");
    const std::vector<std::uint32_t>& tvo = graph->tile_vertex_offsets;
    const u32 T = graph->g.T, V = graph->g.V;
    u64 U = 0;
    for (u32 i = 0; i < selected_tile_count; ++i) {
      const u32 t = selected_tiles[i];
      if (t >= T) throw std::out_of_range("selected tile out of range");
      bfx::require(i == 0 || t > selected_tiles[i - 1], "selected tiles must be strictly increasing");
      U += tvo[t + 1] - tvo[t];
    }
    bfx::require(U > 0, "query selects no vertices");
    auto selected = [&](u32 v) {
      const u32 owner = static_cast<u32>(std::upper_bound(tvo.begin(), tvo.end(), v) - tvo.begin()) - 1U;
      return std::binary_search(selected_tiles, selected_tiles + selected_tile_count, owner);
    };
    for (u32 i = 0; i < source_count; ++i) {
      if (sources[i] >= V) throw std::out_of_range("source out of range");
      bfx::require(i == 0 || sources[i] > sources[i - 1], "noncanonical sources");
      bfx::require(selected(sources[i]), "terminal owner tile not selected");
    }
    for (u32 i = 0; i < target_count; ++i) {
      if (targets[i] >= V) throw std::out_of_range("target out of range");
      bfx::require(i == 0 || targets[i] > targets[i - 1], "noncanonical targets");
      bfx::require(selected(targets[i]), "terminal owner tile not selected");
    }
    // Layout inside the static array.
    const size_t S = source_count, Tg = target_count, R = selected_tile_count;
    const size_t o_batch = 0;
    const size_t o_ctl = bfx::align256(o_batch + sizeof(bfx::DBatch));
    const size_t o_run = bfx::align256(o_ctl + sizeof(bfx::DCtl));
    const size_t o_ubase = bfx::align256(o_run + sizeof(bfx::DRun));
    const size_t o_sbase = bfx::align256(o_ubase + 8);
    const size_t o_status = bfx::align256(o_sbase + 8);
    const size_t o_ctrl = bfx::align256(o_status + sizeof(bfx_device_run_status));
    const size_t o_soff = bfx::align256(o_ctrl + sizeof(bfx_device_controller));
    const size_t o_src = bfx::align256(o_soff + 8);
    const size_t o_toff = bfx::align256(o_src + S * 4);
    const size_t o_tgt = bfx::align256(o_toff + 8);
    const size_t o_ranges = bfx::align256(o_tgt + Tg * 4);
    const size_t o_roff = bfx::align256(o_ranges + R * 16);
    const size_t o_out = bfx::align256(o_roff + (R + 1) * 4);
    const size_t o_dist0 = bfx::align256(o_out + Tg * 8);
    const size_t o_dist1 = bfx::align256(o_dist0 + U * 8);
    const size_t o_mask0 = bfx::align256(o_dist1 + U * 8);
    const size_t o_mask1 = bfx::align256(o_mask0 + U * 4);
    const size_t o_q0 = bfx::align256(o_mask1 + U * 4);
    const size_t o_q1 = bfx::align256(o_q0 + U * 8);
    const size_t o_c2g = bfx::align256(o_q1 + U * 8);
    const size_t o_fmask = bfx::align256(o_c2g + U * 4);
    const size_t o_fbound = bfx::align256(o_fmask + U * 4);
    const size_t o_fp0 = bfx::align256(o_fbound + U * 4);
    const size_t o_fp1 = bfx::align256(o_fp0 + U * 8);
    const size_t o_fp2 = bfx::align256(o_fp1 + U * 8);
    const size_t o_tiles = bfx::align256(o_fp2 + U * 8);
    const size_t total = bfx::align256(o_tiles + size_t{T} * 8);
    if (total > bfx::kStaticScratchBytes) {
      throw std::overflow_error("query needs more than the 32 MiB static scratch (union of " + std::to_string(U) +
                                " vertices); use bfx_run_query");
    }
    BFX_CUDA(cudaSetDevice(graph->device));
    void* vbase = nullptr;
    BFX_CUDA(bfx::static_scratch_base(graph->device, &vbase));
    char* base = static_cast<char*>(vbase);
    // Batch record (width 1) pointing into the array.
    bfx::DBatch B{};
    B.W = 1;
    B.shift = 0;
    B.valid = 1;
    B.U = static_cast<u32>(U);
    B.src_count = static_cast<u32>(S);
    B.tgt_count = static_cast<u32>(Tg);
    B.range_count = static_cast<u32>(R);
    B.dist[0] = reinterpret_cast<u64*>(base + o_dist0);
    B.dist[1] = reinterpret_cast<u64*>(base + o_dist1);
    B.mask[0] = reinterpret_cast<u32*>(base + o_mask0);
    B.mask[1] = reinterpret_cast<u32*>(base + o_mask1);
    B.queue[0] = reinterpret_cast<u64*>(base + o_q0);
    B.queue[1] = reinterpret_cast<u64*>(base + o_q1);
    B.c2g = reinterpret_cast<u32*>(base + o_c2g);
    B.fmask = reinterpret_cast<u32*>(base + o_fmask);
    B.fbound = reinterpret_cast<u32*>(base + o_fbound);
    B.fpile[0] = reinterpret_cast<u64*>(base + o_fp0);
    B.fpile[1] = reinterpret_cast<u64*>(base + o_fp1);
    B.fpile[2] = reinterpret_cast<u64*>(base + o_fp2);
    B.tiles = reinterpret_cast<uint2*>(base + o_tiles);
    B.src_off = reinterpret_cast<const u32*>(base + o_soff);
    B.src = reinterpret_cast<const u32*>(base + o_src);
    B.tgt_off = reinterpret_cast<const u32*>(base + o_toff);
    B.tgt = reinterpret_cast<const u32*>(base + o_tgt);
    B.ranges = reinterpret_cast<const uint4*>(base + o_ranges);
    B.range_off = reinterpret_cast<const u32*>(base + o_roff);
    const u32 ubase[2] = {0U, static_cast<u32>(U)};
    const u32 soff[2] = {0U, source_count};
    const u32 toff[2] = {0U, target_count};
    bfx::copy_in(base, o_batch, &B, sizeof(B));
    bfx::copy_in(base, o_ubase, ubase, 8);
    bfx::copy_in(base, o_sbase, soff, 8);
    bfx::copy_in(base, o_soff, soff, 8);
    bfx::copy_in(base, o_src, sources, S * 4);
    bfx::copy_in(base, o_toff, toff, 8);
    bfx::copy_in(base, o_tgt, targets, Tg * 4);
    // Vertex ranges and their compact offsets, streamed through a stack buffer.
    {
      constexpr u32 kChunk = 256;
      uint4 rbuf[kChunk];
      u32 obuf[kChunk];
      u32 acc = 0;
      for (u32 i0 = 0; i0 < R; i0 += kChunk) {
        const u32 n = std::min<u32>(kChunk, static_cast<u32>(R) - i0);
        for (u32 k = 0; k < n; ++k) {
          const u32 t = selected_tiles[i0 + k];
          rbuf[k] = make_uint4(t, tvo[t], tvo[t + 1], 1U);
          obuf[k] = acc;
          acc += tvo[t + 1] - tvo[t];
        }
        bfx::copy_in(base, o_ranges + size_t{i0} * 16, rbuf, size_t{n} * 16);
        bfx::copy_in(base, o_roff + size_t{i0} * 4, obuf, size_t{n} * 4);
      }
      bfx::copy_in(base, o_roff + R * 4, &acc, 4);
    }
    // The tile table must read 0 outside the selection (the previous call's
    // entries are still there); everything else is reset by init_kernel.
    BFX_CUDA(cudaMemset(base + o_tiles, 0, size_t{T} * 8));
    bfx::LaunchParams p{};
    p.g = graph->g;
    p.batches = reinterpret_cast<const bfx::DBatch*>(base + o_batch);
    p.ctl = reinterpret_cast<bfx::DCtl*>(base + o_ctl);
    p.run = reinterpret_cast<bfx::DRun*>(base + o_run);
    p.unit_base = reinterpret_cast<const u32*>(base + o_ubase);
    p.nb = 1;
    p.engine = options->engine;
    p.per_lane = options->enable_per_lane_convergence;
    p.max_rounds = options->maximum_rounds;
    p.budget_ns = bfx::kLaunchBudgetNs;
    int sms = 0;
    BFX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, graph->device));
    bfx::init_kernel<<<sms * 8, 256>>>(p);
    BFX_CUDA(cudaGetLastError());
    bfx::seed_kernel<<<static_cast<int>((S + 255) / 256), 256>>>(p, reinterpret_cast<const u32*>(base + o_sbase));
    BFX_CUDA(cudaGetLastError());
    const int block = static_cast<int>(options->block_size);
    const size_t smem = 8;
    int per_sm = 0;
    BFX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, reinterpret_cast<const void*>(bfx::persistent_kernel<false, 3, 2>), block, smem));
    if (per_sm <= 0) throw bfx::Error(BFX_ERR_CUDA, "kernel cannot be resident with this block size");
    if (options->grid_policy == 1u) {
      if (static_cast<int>(options->blocks_per_wgp) > per_sm)
        throw std::invalid_argument("blocks per SM exceed the cooperative residency limit");
      per_sm = static_cast<int>(options->blocks_per_wgp);
    }
    void* args[] = {&p};
    BFX_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(bfx::persistent_kernel<false, 3, 2>),
                                         per_sm * sms, block, args, smem, 0));
    auto* d_status = reinterpret_cast<bfx_device_run_status*>(base + o_status);
    bfx::finalize_kernel<<<1, 256>>>(p, reinterpret_cast<bfx_device_controller*>(base + o_ctrl), d_status);
    BFX_CUDA(cudaGetLastError());
    u32* out = reinterpret_cast<u32*>(base + o_out);
    bfx::gather_targets_kernel<<<static_cast<int>((Tg + 255) / 256), 256>>>(graph->g, p.batches, d_status, out,
                                                                          out + Tg);
    BFX_CUDA(cudaGetLastError());
    BFX_CUDA(cudaMemcpy(status, d_status, sizeof(*status), cudaMemcpyDeviceToHost));
    BFX_CUDA(cudaMemcpy(target_distance_bits, out, Tg * 4, cudaMemcpyDeviceToHost));
    BFX_CUDA(cudaMemcpy(target_predecessor_edges, out + Tg, Tg * 4, cudaMemcpyDeviceToHost));
  });
}

// ---------------------------------------------------------------------------
// Barrier self-test (failure detection without a GPU fault).  A cooperative
// grid runs `rounds` grid barriers; when absent_block < gridDim.x that block
// never arrives, so the others' bounded waits run out after timeout_ns, raise
// the abort flag and return -- the same path a stuck engine launch takes.
// out = {aborted, barriers passed by block 0 (all blocks when none is
// absent), blocks that observed the abort, 0}.
// ---------------------------------------------------------------------------

namespace bfx {
namespace {

__global__ void barrier_selftest_kernel(dev::GridSync* gs, u32 rounds, u32 absent_block, u64 timeout_ns, u32* out) {
  if (blockIdx.x == absent_block) return;  // never arrives: nothing else sets the generation
  u32 passed = 0;
  for (u32 r = 0; r < rounds; ++r) {
    if (!dev::grid_barrier(gs, gridDim.x, timeout_ns)) break;
    ++passed;
  }
  if (threadIdx.x == 0) {
    if (passed < rounds) atomicAdd(&out[2], 1u);
    if (blockIdx.x == (absent_block == 0u ? 1u : 0u)) out[1] = passed;
    if (gs->abort) out[0] = 1u;
  }
}

}  // namespace
}  // namespace bfx

extern "C" int bfx_barrier_selftest(int device, uint32_t rounds, uint32_t absent_block, uint64_t timeout_ns,
                                    uint32_t out[4]) {
  return bfx::guarded([&] {
    bfx::require(out != nullptr, "null output");
    bfx::require(timeout_ns > 0 && timeout_ns <= 2000000000ull, "timeout must be in (0, 2 s]");
    BFX_CUDA(cudaSetDevice(device));
    int sms = 0, per_sm = 0;
    BFX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    BFX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, reinterpret_cast<const void*>(bfx::barrier_selftest_kernel), 128, 0));
    const int grid = std::max(2, std::min(per_sm, 2) * sms);
    void* mem = nullptr;
    BFX_CUDA(cudaMalloc(&mem, 256));
    cudaError_t err = cudaMemset(mem, 0, 256);
    auto* gs = static_cast<bfx::dev::GridSync*>(mem);
    auto* dout = reinterpret_cast<std::uint32_t*>(static_cast<char*>(mem) + 64);
    if (err == cudaSuccess) {
      void* args[] = {&gs, &rounds, &absent_block, &timeout_ns, &dout};
      err = cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(bfx::barrier_selftest_kernel), grid, 128, args,
                                        0, 0);
    }
    if (err == cudaSuccess) err = cudaDeviceSynchronize();
    if (err == cudaSuccess) err = cudaMemcpy(out, dout, 16, cudaMemcpyDeviceToHost);
    out[3] = static_cast<std::uint32_t>(grid);
    cudaFree(mem);
    BFX_CUDA(err);
  });
}
