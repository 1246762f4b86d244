// Tiled frontier push (BFX_FRONTIER_TILED; included by engine.cu after the
// Jacobi and dense items).
//
// The claim unit is a block of 2^cshift consecutive compact vertices -- one
// spatial tile when every tile holds 2^cshift vertices, as vertices are
// ordered by tile and a batch's union tiles are concatenated in compact
// order.  A block item of the persistent grid is one such unit of one
// batch ("visit"):
//   1. the block reads the unit's pending lanes (and clears them) and its
//      compact row table, and sums the lane-edge work;
//   2. with enough work it stages the unit's label rows (2^cshift x W packed
//      words, contiguous in the vertex-major layout) in shared memory and
//      relaxes in local iterations: every pending (vertex, lane) pushes all
//      its admitted out-edges; a target inside the unit is relaxed with a
//      64-bit atomicMin in shared memory and, on a decrease below the
//      threshold, marked pending for the next local iteration; a target
//      outside goes through the global path (pre-read, red.min, pending
//      lane OR, unit claim through the chunk bitmap, staged queue append).
//      Iterations repeat until no local lane is pending (or a cap, whose
//      leftovers are handed to the next round);
//   3. changed labels are written back with red.min -- another block may
//      have lowered the same word meanwhile through an inter-tile edge, and
//      that improvement is also queued for the next round, so the min keeps
//      both;
//   4. a unit with little work skips the staging and relaxes every target in
//      global memory, like the chunked layout.
// Near/far thresholds apply unchanged: a decrease at or above tau parks the
// lane on the far pile (global far mask, bound and pile), local or not.
// Within a pass the work list is flat over the block: (vertex, lane, edge)
// items ordered vertex-major, two per thread in flight; a thread finds its
// item's vertex by binary search over the block's inclusive work scan.
#pragma once

// Shared-memory layout of a tiled visit, after the round prefix:
// labels S[n][W] then six u32 arrays of n = 2^cshift entries.
struct TileSmem {
  u64* S;
  u32* P;    // pending lanes for the next local iteration
  u32* M;    // lanes processed in this pass
  u32* CH;   // lanes whose staged label changed (written back)
  u32* WI;   // inclusive lane-edge work scan
  u32* RB;   // CSR row begin
  u32* DG;   // out-degree
};

constexpr u32 kTileLocalIterations = 32;

__device__ __forceinline__ TileSmem tile_smem(u32* prefix, u32 nb, u32 cshift, u32 wmax) {
  const size_t off = ((static_cast<size_t>(nb) + 1u) * 4u + 15u) & ~static_cast<size_t>(15);
  char* base = reinterpret_cast<char*>(prefix) + off;
  const u32 n = 1u << cshift;
  TileSmem t;
  t.S = reinterpret_cast<u64*>(base);
  u32* a = reinterpret_cast<u32*>(base + static_cast<size_t>(n) * wmax * 8u);
  t.P = a;
  t.M = a + n;
  t.CH = a + 2u * n;
  t.WI = a + 3u * n;
  t.RB = a + 4u * n;
  t.DG = a + 5u * n;
  return t;
}

// Dynamic shared memory of the tiled kernel (host and device agree).
__host__ __device__ inline size_t tile_smem_bytes(u32 nb, u32 cshift, u32 wmax) {
  const size_t off = ((static_cast<size_t>(nb) + 1u) * 4u + 15u) & ~static_cast<size_t>(15);
  const size_t n = size_t{1} << cshift;
  return off + n * wmax * 8u + 6u * n * 4u;
}

// Block-wide inclusive scan of one value per thread (blockDim.x <= 1024).
__device__ __forceinline__ u32 block_inclusive_scan(u32 x, u32* warp_sums, u32& total) {
  const u32 lane = lane_id(), wib = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (u32 o = 1; o < 32u; o <<= 1) {
    const u32 y = __shfl_up_sync(0xFFFFFFFFu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31u) warp_sums[wib] = x;
  __syncthreads();
  if (wib == 0u) {
    u32 w = lane < nw ? warp_sums[lane] : 0u;
    for (u32 o = 1; o < 32u; o <<= 1) {
      const u32 y = __shfl_up_sync(0xFFFFFFFFu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < nw) warp_sums[lane] = w;  // inclusive over warps
  }
  __syncthreads();
  const u32 before = wib == 0u ? 0u : warp_sums[wib - 1u];
  total = warp_sums[nw - 1u];
  __syncthreads();  // warp_sums is reused by the next scan
  return x + before;
}

// A decrease at or above the threshold: the lane is parked (far mask, bound,
// pile).  Returns true when this OR parked the vertex on the pile.
__device__ __forceinline__ bool tile_park(const FrontierView& B, Stages& st, u32 cdst, u32 bit, u32 dist_bits) {
  st.fd = min(st.fd, dist_bits);
  dev::red_min_u32(B.fbound + cdst, dist_bits);
  return atomicOr(B.fmask + cdst, bit) == 0u;
}

// One pass over the snapshot M[0..n) of a visit: every (vertex, lane) in M
// pushes its admitted out-edges.  kStaged: source labels and in-unit
// targets live in S (shared memory); otherwise everything is global.
// Executed by the whole block; `total` is the block's lane-edge work.
template <bool kCount, bool kStaged>
__device__ __forceinline__ void tile_pass(const LaunchParams& p, const FrontierView& B, const TileSmem& sm, u32 c0,
                                          u32 n, u32 total, u32 tau_bits, Stages& st, Work& wk) {
  const u32 cs = p.cshift;
  const u32 shift = B.shift;
  u32 known_chunk = 0xFFFFFFFFu;
  for (u32 base = 0; base < total; base += 2u * blockDim.x) {
    // decode two items per thread
    u32 ii[2], ll[2], ee[2];
    bool live[2];
#pragma unroll
    for (u32 u = 0; u < 2u; ++u) {
      const u32 w = base + u * blockDim.x + threadIdx.x;
      live[u] = w < total;
      ii[u] = ll[u] = ee[u] = 0u;
      if (live[u]) {
        u32 lo = 0u, hi = n;  // smallest i with WI[i] > w
        while (lo < hi) {
          const u32 mid = (lo + hi) >> 1;
          if (sm.WI[mid] > w) hi = mid; else lo = mid + 1u;
        }
        const u32 i = lo;
        const u32 excl = i == 0u ? 0u : sm.WI[i - 1u];
        const u32 r = w - excl;
        const u32 deg = sm.DG[i];
        const u32 j = r / deg;
        ii[u] = i;
        ee[u] = sm.RB[i] + (r - j * deg);
        ll[u] = __fns(sm.M[i], 0u, static_cast<int>(j) + 1);
      }
    }
    uint4 rec[2];
    u32 src[2];
#pragma unroll
    for (u32 u = 0; u < 2u; ++u) {
      if (live[u]) {
        rec[u] = __ldg(p.g.csr + ee[u]);
        const u64 si = (static_cast<u64>(ii[u]) << shift) + ll[u];
        src[u] = kStaged ? dev::hi(*reinterpret_cast<volatile u64*>(sm.S + si))
                         : dev::hi(dev::ld_cg(B.dist + (static_cast<u64>(c0) << shift) + si));
      }
    }
    // admission and compact target
    u32 cdst[2], bitv[2];
    bool relax[2], local[2];
    u64 cand[2], cur[2];
#pragma unroll
    for (u32 u = 0; u < 2u; ++u) {
      relax[u] = false;
      local[u] = false;
      cdst[u] = 0u;
      bitv[u] = 1u << ll[u];
      if (live[u] && src[u] != dev::kInfBits) {
        const uint2 dt = B.full ? make_uint2(B.valid, 0u) : B.tiles[rec[u].w];
        cdst[u] = rec[u].x - dt.y;
        relax[u] = (dt.x >> ll[u]) & 1u;
        cand[u] = dev::candidate(src[u], rec[u].y, rec[u].z);
        local[u] = kStaged && (cdst[u] - c0) < n;
      }
    }
#pragma unroll
    for (u32 u = 0; u < 2u; ++u) {
      if (relax[u]) {
        if (local[u]) {
          cur[u] = *reinterpret_cast<volatile u64*>(sm.S + ((static_cast<u64>(cdst[u] - c0) << shift) + ll[u]));
        } else {
          cur[u] = dev::ld_cg(B.dist + ((static_cast<u64>(cdst[u]) << shift) + ll[u]));
        }
      }
    }
    bool near_claim[2], far_claim[2];
#pragma unroll
    for (u32 u = 0; u < 2u; ++u) {
      near_claim[u] = far_claim[u] = false;
      if (!relax[u]) continue;
      if (kCount) {
        wk.c[3] += 1;
        if (local[u]) wk.c[13] += 1;
      }
      if (cand[u] >= cur[u]) continue;
      u64 old = cur[u];
      if (local[u]) {
        const u32 j = cdst[u] - c0;
        old = atomicMin(reinterpret_cast<unsigned long long*>(sm.S + ((static_cast<u64>(j) << shift) + ll[u])),
                        static_cast<unsigned long long>(cand[u]));
        if (cand[u] >= old) continue;
        atomicOr(sm.CH + j, bitv[u]);
      } else {
        dev::red_min(B.dist + ((static_cast<u64>(cdst[u]) << shift) + ll[u]), cand[u]);
      }
      if (kCount) {
        wk.c[6] += 1;
        wk.c[5] += dev::hi(cand[u]) < dev::hi(old);
      }
      if (dev::hi(cand[u]) >= dev::hi(old)) continue;  // same distance, smaller edge id: nothing to propagate
      if (dev::hi(cand[u]) < tau_bits) {
        if (local[u]) {
          atomicOr(sm.P + (cdst[u] - c0), bitv[u]);
        } else {
          dev::red_or(B.mask_w + cdst[u], bitv[u]);
          const u32 chunk = cdst[u] >> cs;
          if (chunk != known_chunk) {
            const u32 cb = 1u << (chunk & 31u);
            near_claim[u] = (atomicOr(B.cmask_w + (chunk >> 5), cb) & cb) == 0u;
            known_chunk = chunk;
          }
        }
      } else {
        far_claim[u] = tile_park(B, st, cdst[u], bitv[u], dev::hi(cand[u]));
      }
    }
#pragma unroll
    for (u32 u = 0; u < 2u; ++u) {
      if (kCount && near_claim[u]) wk.c[4] += 1;
      stage_push(st, kNear, near_claim[u], cdst[u] >> cs);
      stage_push(st, kFar, far_claim[u], queue_word(cdst[u], cdst[u]));
    }
  }
}

// Snapshot of the pending lanes for a pass: M = P, P = 0, inclusive work
// scan into WI; returns the block's lane-edge work (block-uniform).
__device__ __forceinline__ u32 tile_snapshot(const TileSmem& sm, u32 n, u32* warp_sums) {
  u32 work = 0u;
  const u32 i = threadIdx.x;
  if (i < n) {
    const u32 m = sm.P[i];
    sm.M[i] = m;
    sm.P[i] = 0u;
    work = static_cast<u32>(__popc(m)) * sm.DG[i];
  }
  u32 total = 0u;
  const u32 incl = block_inclusive_scan(work, warp_sums, total);
  if (i < n) sm.WI[i] = incl;
  __syncthreads();
  return total;
}

// One visit: block item `item` of a near round of a frontier batch (n_queued
// queued units; dense rounds enumerate every unit).  Executed by the whole
// block; every branch is block-uniform.
template <bool kCount>
__device__ void tile_visit(const LaunchParams& p, const FrontierView& B, DCtl& C, u32 item, u32 n_queued,
                           u32 tau_bits, const TileSmem& sm, Stages& st, Work& wk) {
  __shared__ u32 s_warp[32];
  __shared__ u32 s_unit;
  const u32 cs = p.cshift;
  const u32 units = chunk_count(B.U, cs);
  if (threadIdx.x == 0u) {
    u32 unit;
    if (chunk_dense(n_queued, B.U, cs)) {
      // dense round: the item is unit slot `item`; a clear bit means no work
      const u32 word = dev::ld_cg(B.cmask_r + (item >> 5));
      unit = ((word >> (item & 31u)) & 1u) ? item : 0xFFFFFFFEu;
    } else {
      unit = static_cast<u32>(dev::ld_cg(B.queue_r + item));
      if (unit >= units) {
        atomicOr(&C.error_bits, static_cast<u32>(BFX_DEVICE_ERROR_INVALID_CONTROLLER_STATE));
        unit = 0xFFFFFFFEu;
      }
    }
    if (unit < units) atomicAnd(B.cmask_r + (unit >> 5), ~(1u << (unit & 31u)));
    s_unit = unit;
  }
  __syncthreads();
  const u32 unit = s_unit;
  if (unit >= units) return;
  const u32 c0 = unit << cs;
  const u32 n = min(1u << cs, B.U - c0);
  // 1. pending lanes (cleared) and rows
  const u32 i = threadIdx.x;
  u32 work = 0u;
  if (i < n) {
    const u32 m = dev::ld_cg(B.mask_r + c0 + i) & B.valid;
    const uint2 row = __ldg(B.crow + c0 + i);
    if (m != 0u) B.mask_r[c0 + i] = 0u;
    sm.P[i] = m;
    sm.CH[i] = 0u;
    sm.RB[i] = row.x;
    sm.DG[i] = row.y;
    work = static_cast<u32>(__popc(m)) * row.y;
    if (kCount && m != 0u) {
      wk.c[0] += 1;
      wk.c[1] += row.y;
      wk.c[2] += __popc(m);
    }
  }
  u32 total = 0u;
  (void)block_inclusive_scan(work, s_warp, total);  // block total (the pass rescans)
  if (total == 0u) return;
  if (total < p.tile_stage_min) {
    // 4. little work: relax in place
    const u32 t = tile_snapshot(sm, n, s_warp);
    tile_pass<kCount, false>(p, B, sm, c0, n, t, tau_bits, st, wk);
    __syncthreads();
    return;
  }
  // 2. stage the label rows (n x W words, 256-byte aligned: c0 is a multiple of 32)
  {
    const u32 words = n << B.shift;
    const u64* g = B.dist + (static_cast<u64>(c0) << B.shift);
    const uint4* g4 = reinterpret_cast<const uint4*>(g);
    uint4* s4 = reinterpret_cast<uint4*>(sm.S);
    for (u32 k = threadIdx.x; k < (words >> 1); k += blockDim.x) s4[k] = __ldcg(g4 + k);
    if ((words & 1u) && threadIdx.x == 0u) sm.S[words - 1u] = dev::ld_cg(g + words - 1u);
  }
  if (kCount && threadIdx.x == 0u) wk.c[14] += 1;
  __syncthreads();
  for (u32 it = 0; it < kTileLocalIterations; ++it) {
    const u32 t = tile_snapshot(sm, n, s_warp);
    if (t == 0u) break;
    if (kCount && i < n && sm.M[i] != 0u) {
      if (it > 0u) {
        wk.c[0] += 1;
        wk.c[1] += sm.DG[i];
        wk.c[2] += __popc(sm.M[i]);
      }
    }
    tile_pass<kCount, true>(p, B, sm, c0, n, t, tau_bits, st, wk);
    __syncthreads();
  }
  // leftovers after the cap: the next round picks them up
  bool claim = false;
  if (i < n && sm.P[i] != 0u) {
    dev::red_or(B.mask_w + c0 + i, sm.P[i]);
    const u32 cb = 1u << (unit & 31u);
    claim = (atomicOr(B.cmask_w + (unit >> 5), cb) & cb) == 0u;
  }
  stage_push(st, kNear, claim, unit);
  // 3. write back the changed labels
  {
    const u32 words = n << B.shift;
    u64* g = B.dist + (static_cast<u64>(c0) << B.shift);
    for (u32 k = threadIdx.x; k < words; k += blockDim.x) {
      if ((sm.CH[k >> B.shift] >> (k & ((1u << B.shift) - 1u))) & 1u) dev::red_min(g + k, sm.S[k]);
    }
  }
  __syncthreads();
}

// One round of the tiled layout: block items drawn from a per-round counter.
// Frontier near rounds: one unit visit per item; split rounds: 32 far
// entries per warp of the block; Jacobi / dense batches: one warp item per
// warp of the block.  Every branch is block-uniform (the item, its batch and
// the batch's round values are broadcast through shared memory).
template <bool kCount>
__device__ void round_body_tiled(const LaunchParams& p, u32 r, u32* prefix, Work& wk) {
  __shared__ u32 s_item;
  __shared__ u32 s_vals[5];
  const u32 ridx = r % 3u, widx = (r + 1u) % 3u;
  const u32 total = prefix[p.nb];
  const u32 nw = blockDim.x >> 5, wib = threadIdx.x >> 5;
  const TileSmem sm = tile_smem(prefix, p.nb, p.cshift, p.tile_wmax);
  Stages st{{0u, 0u}, 0xFFFFFFFFu};
  u32 staged_batch = 0xFFFFFFFFu;
  for (;;) {
    if (threadIdx.x == 0u) s_item = atomicAdd(&p.run->items[ridx], 1u);
    __syncthreads();
    const u32 w = s_item;
    __syncthreads();
    if (w >= total) break;
    const u32 b = find_batch(prefix, p.nb, w);
    const DBatch& B = p.batches[b];
    DCtl& C = p.ctl[b];
    const u32 item = w - prefix[b];
    const u32 eng = engine_of(p, b);
    if (eng == BFX_ENGINE_FRONTIER_PUSH) {
      if (threadIdx.x == 0u) {
        const u32 n = min(dev::ld_cg(&C.count[ridx]), B.U);
        const u32 g = dev::ld_cg(&C.gen[r & 1u]);
        const u32 tau = dev::ld_cg(&C.tau[r & 1u]);
        s_vals[0] = n;
        s_vals[1] = g;
        s_vals[2] = tau;
        s_vals[3] = n == 0u ? min(dev::ld_cg(&C.fcount[g % 3u]), B.U) : 0u;
        s_vals[4] = n == 0u ? split_threshold(C, tau, g % 3u) : 0u;
      }
      __syncthreads();
      const u32 n = s_vals[0], g = s_vals[1], tau = s_vals[2], f = s_vals[3], tau_next = s_vals[4];
      __syncthreads();
      const FrontierView V = frontier_view(B, r & 1u, g % 3u, (g + 1u) % 3u);
      if (b != staged_batch) {
        stages_flush(st);
        staged_batch = b;
        const u32 po = n != 0u ? g % 3u : (g + 1u) % 3u;
        if (lane_id() == 0u) {
          s_stage_queue[kNear][wib] = StageQueue{V.queue_w, &C.count[widx], &C.error_bits, V.U};
          s_stage_queue[kFar][wib] = StageQueue{n != 0u ? V.pile : V.pile_out, &C.fcount[po], &C.error_bits, V.U};
          s_fmin_target[wib] = &C.fmin[po];
        }
        __syncwarp();
      }
      if (n != 0u) {
        tile_visit<kCount>(p, V, C, item, n, tau, sm, st, wk);
      } else {
        split_group<kCount, true>(p, V, C, item * nw + wib, f, tau_next, st, wk);
      }
    } else if (eng == BFX_ENGINE_JACOBI_PULL) {
      jacobi_item<kCount>(p, B, C, item * nw + wib, r, widx, wk);
    } else {
      dense_item<kCount>(p, B, C, item * nw + wib, batch_exec(p, b, ridx), widx, wk);
    }
  }
  stages_flush(st);
}

// Persistent cooperative kernel of the tiled layout: 256-thread blocks, two
// per SM by launch bounds (the staged labels take up to 64 KB per block).
template <bool kCount>
__global__ void __launch_bounds__(256, 2) persistent_tiled_kernel(LaunchParams p) {
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
    round_body_tiled<kCount>(p, r, prefix, wk);
    if (kCount && p.round_trace != nullptr && r < p.trace_cap) trace_round_work(p, r, wk, traced);
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
