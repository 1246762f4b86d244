// Tiled frontier push (BFX_FRONTIER_TILED; included by engine.cu after the
// Jacobi and dense items).
//
// Claims and queues are the chunked layout's (32-vertex chunks, chunk
// bitmaps, staged appends).  Sparse rounds run exactly as there, as warp
// items each warp draws on its own (the chunked round body).  Dense rounds --
// at least half of a batch's chunk slots pending -- visit whole tiles
// instead: a block item is one unit of 2^tshift consecutive compact vertices,
// which is one spatial tile when every tile holds 2^tshift vertices
// (vertices are ordered by tile, and a batch's union tiles are concatenated
// in compact order).  A visit:
//   1. reads and clears the unit's chunk bits and its vertices' pending
//      lanes, and their row tables: CSR row, and the own-tile run (a row is
//      sorted by destination tile, so the edges into the vertex's own tile
//      are contiguous; the resident graph keeps them per vertex);
//   2. with enough work, stages the unit's label rows (2^tshift x W packed
//      words, contiguous in the vertex-major layout) in shared memory and
//      runs local passes: every pending (vertex, lane) relaxes its own-tile
//      run against the staged labels with a 64-bit atomicMin in shared
//      memory; a decrease below the threshold makes the target pending for
//      the next pass and marks it for the global push.  Passes repeat until
//      no lane of the unit is pending (or a cap; the rest is handed to the
//      next round);
//   3. pushes the other edges of every marked (vertex, lane) once, with its
//      final label, through the global path (pre-read, red.min, pending lane
//      OR, chunk claim, staged append) -- a loop in which every item is a
//      global relaxation, so no warp waits on one slow item among fast ones;
//   4. writes the changed labels back with red.min (another block may have
//      lowered the same word through an inter-tile edge meanwhile; that
//      improvement is queued for the next round as well, and the min keeps
//      both);
//   5. a unit with little pending work skips the staging and relaxes all its
//      edges in global memory in one pass.
// Near/far thresholds apply unchanged: a decrease at or above tau parks the
// lane on the far pile (global far mask, bound and pile), local or not.
// Within a pass the work list is flat over the block: (vertex, lane, edge)
// items ordered vertex-major, two per thread in flight; a thread finds its
// item's vertex by binary search over the block's inclusive work scan.
#pragma once

// Shared-memory layout of a tiled visit, after the round prefix:
// labels S[n][W] then nine u32 arrays of n = 2^tshift entries.
struct TileSmem {
  u64* S;
  u32* P;    // lanes pending for the next local pass
  u32* G;    // lanes whose other edges are pushed by the global pass
  u32* M;    // lanes of the current pass
  u32* CH;   // lanes whose staged label changed (written back)
  u32* WI;   // inclusive lane-edge work scan of the current pass
  u32* RB;   // CSR row begin
  u32* DG;   // out-degree
  u32* LB;   // own-tile run: first CSR index
  u32* LC;   // own-tile run: edge count
};

constexpr u32 kTileArrays = 9;

// Dynamic shared memory: the round's two prefixes (block items, warp items;
// nb + 1 words each), then the visit arrays.
__device__ __forceinline__ TileSmem tile_smem(u32* prefix, u32 nb, u32 tshift, u32 wmax) {
  const size_t off = ((static_cast<size_t>(nb) + 1u) * 8u + 15u) & ~static_cast<size_t>(15);
  char* base = reinterpret_cast<char*>(prefix) + off;
  const u32 n = 1u << tshift;
  TileSmem t;
  t.S = reinterpret_cast<u64*>(base);
  u32* a = reinterpret_cast<u32*>(base + static_cast<size_t>(n) * wmax * 8u);
  t.P = a;
  t.G = a + n;
  t.M = a + 2u * n;
  t.CH = a + 3u * n;
  t.WI = a + 4u * n;
  t.RB = a + 5u * n;
  t.DG = a + 6u * n;
  t.LB = a + 7u * n;
  t.LC = a + 8u * n;
  return t;
}

// Dynamic shared memory of the tiled kernel (host and device agree).
__host__ __device__ inline size_t tile_smem_bytes(u32 nb, u32 tshift, u32 wmax) {
  const size_t off = ((static_cast<size_t>(nb) + 1u) * 8u + 15u) & ~static_cast<size_t>(15);
  const size_t n = size_t{1} << tshift;
  return off + n * wmax * 8u + kTileArrays * n * 4u;
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

// Pass kinds: kLocal relaxes the own-tile runs against the staged labels;
// kGlobal pushes the other edges of the marked lanes (sources staged);
// kInPlace relaxes every edge in global memory (unstaged visit).
enum TilePass : u32 { kLocal = 0, kGlobal = 1, kInPlace = 2 };

// Snapshot for a pass: M = src (src cleared), per-vertex lane-edge work of
// the pass kind, inclusive scan into WI.  Returns the block's work.
template <u32 kKind>
__device__ __forceinline__ u32 tile_snapshot(const TileSmem& sm, u32* src, u32 n, u32* warp_sums) {
  u32 work = 0u;
  const u32 i = threadIdx.x;
  if (i < n) {
    const u32 m = src[i];
    sm.M[i] = m;
    src[i] = 0u;
    const u32 edges = kKind == kLocal ? sm.LC[i] : (kKind == kGlobal ? sm.DG[i] - sm.LC[i] : sm.DG[i]);
    work = static_cast<u32>(__popc(m)) * edges;
  }
  u32 total = 0u;
  const u32 incl = block_inclusive_scan(work, warp_sums, total);
  if (i < n) sm.WI[i] = incl;
  __syncthreads();
  return total;
}

// One pass over the snapshot M[0..n) (see TilePass).  Executed by the whole
// block; `total` is the pass's lane-edge work.
template <bool kCount, u32 kKind>
__device__ __forceinline__ void tile_pass(const LaunchParams& p, const FrontierView& B, const TileSmem& sm, u32 c0,
                                          u32 n, u32 total, u32 tau_bits, Stages& st, Work& wk) {
  const u32 shift = B.shift;
  u32 known_chunk = 0xFFFFFFFFu;
  for (u32 base = 0; base < total; base += 2u * blockDim.x) {
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
        const u32 r = w - (i == 0u ? 0u : sm.WI[i - 1u]);
        const u32 lc = sm.LC[i];
        const u32 deg = kKind == kLocal ? lc : (kKind == kGlobal ? sm.DG[i] - lc : sm.DG[i]);
        const u32 j = r / deg;
        const u32 k = r - j * deg;
        ii[u] = i;
        if (kKind == kLocal) {
          ee[u] = sm.LB[i] + k;
        } else if (kKind == kGlobal) {
          // the row without its own-tile run [LB, LB + LC)
          const u32 before = sm.LB[i] - sm.RB[i];
          ee[u] = k < before ? sm.RB[i] + k : sm.LB[i] + lc + (k - before);
        } else {
          ee[u] = sm.RB[i] + k;
        }
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
        src[u] = kKind != kInPlace ? dev::hi(*reinterpret_cast<volatile u64*>(sm.S + si))
                                   : dev::hi(dev::ld_cg(B.dist + (static_cast<u64>(c0) << shift) + si));
      }
    }
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
        // own-tile edges whose target lies in the staged unit (all of them
        // when tiles and units coincide)
        local[u] = kKind == kLocal && (cdst[u] - c0) < n;
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
          atomicOr(sm.G + (cdst[u] - c0), bitv[u]);
        } else {
          dev::red_or(B.mask_w + cdst[u], bitv[u]);
          const u32 chunk = cdst[u] >> 5;
          if (chunk != known_chunk) {
            const u32 cb = 1u << (chunk & 31u);
            near_claim[u] = (atomicOr(B.cmask_w + (chunk >> 5), cb) & cb) == 0u;
            known_chunk = chunk;
          }
        }
      } else {
        st.fd = min(st.fd, dev::hi(cand[u]));
        dev::red_min_u32(B.fbound + cdst[u], dev::hi(cand[u]));
        far_claim[u] = atomicOr(B.fmask + cdst[u], bitv[u]) == 0u;
      }
    }
#pragma unroll
    for (u32 u = 0; u < 2u; ++u) {
      if (kCount && near_claim[u]) wk.c[4] += 1;
      stage_push(st, kNear, near_claim[u], cdst[u] >> 5);
      stage_push(st, kFar, far_claim[u], queue_word(cdst[u], cdst[u]));
    }
  }
}

// One visit of a dense round: tile unit `unit` of a frontier batch.
// Executed by the whole block; every branch is block-uniform.
template <bool kCount>
__device__ void tile_visit(const LaunchParams& p, const FrontierView& B, u32 unit, u32 tau_bits, const TileSmem& sm,
                           Stages& st, Work& wk) {
  __shared__ u32 s_warp[32];
  __shared__ u32 s_live;
  const u32 ts = p.tshift;
  const u32 c0 = unit << ts;
  const u32 n = min(1u << ts, B.U - c0);
  // the unit's chunk bits (2^(ts-5) bits of one word): read and clear
  if (threadIdx.x == 0u) {
    const u32 first = c0 >> 5, count = (n + 31u) >> 5;
    const u32 bits = (count >= 32u ? 0xFFFFFFFFu : ((1u << count) - 1u)) << (first & 31u);
    s_live = (atomicAnd(B.cmask_r + (first >> 5), ~bits) & bits) != 0u;
  }
  __syncthreads();
  if (!s_live) return;
  // 1. pending lanes (cleared) and row tables
  const u32 i = threadIdx.x;
  u32 work = 0u;
  if (i < n) {
    const u32 m = dev::ld_cg(B.mask_r + c0 + i) & B.valid;
    const uint2 row = __ldg(B.crow + c0 + i);
    const uint2 lr = __ldg(B.clrun + c0 + i);
    if (m != 0u) B.mask_r[c0 + i] = 0u;
    sm.P[i] = m;
    sm.G[i] = m;
    sm.CH[i] = 0u;
    sm.RB[i] = row.x;
    sm.DG[i] = row.y;
    sm.LB[i] = lr.x;
    sm.LC[i] = lr.y;
    work = static_cast<u32>(__popc(m)) * row.y;
    if (kCount && m != 0u) {
      wk.c[0] += 1;
      wk.c[1] += row.y;
      wk.c[2] += __popc(m);
    }
  }
  u32 total = 0u;
  (void)block_inclusive_scan(work, s_warp, total);
  if (total == 0u) return;
  if (total < p.tile_stage_min) {
    // 5. little work: every edge in global memory, one pass
    const u32 t = tile_snapshot<kInPlace>(sm, sm.P, n, s_warp);
    tile_pass<kCount, kInPlace>(p, B, sm, c0, n, t, tau_bits, st, wk);
    __syncthreads();
    return;
  }
  // 2. stage the label rows (n x W words; 256-byte aligned as c0 is a multiple of 32)
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
  for (u32 it = 0; it < p.tile_iters; ++it) {
    const u32 t = tile_snapshot<kLocal>(sm, sm.P, n, s_warp);
    if (t == 0u) break;
    if (kCount && it > 0u && i < n && sm.M[i] != 0u) {
      wk.c[0] += 1;
      wk.c[1] += sm.LC[i];
      wk.c[2] += __popc(sm.M[i]);
    }
    tile_pass<kCount, kLocal>(p, B, sm, c0, n, t, tau_bits, st, wk);
    __syncthreads();
  }
  // leftovers after the cap: the next round relaxes all their edges
  bool claim = false;
  if (i < n && sm.P[i] != 0u) {
    dev::red_or(B.mask_w + c0 + i, sm.P[i]);
    sm.G[i] &= ~sm.P[i];
    const u32 chunk = (c0 + i) >> 5;
    const u32 cb = 1u << (chunk & 31u);
    claim = (atomicOr(B.cmask_w + (chunk >> 5), cb) & cb) == 0u;
  }
  stage_push(st, kNear, claim, (c0 + i) >> 5);
  __syncthreads();
  // 3. the other edges of every marked lane, once, with its final label
  {
    const u32 t = tile_snapshot<kGlobal>(sm, sm.G, n, s_warp);
    tile_pass<kCount, kGlobal>(p, B, sm, c0, n, t, tau_bits, st, wk);
  }
  // 4. write back the changed labels
  {
    const u32 words = n << B.shift;
    u64* g = B.dist + (static_cast<u64>(c0) << B.shift);
    for (u32 k = threadIdx.x; k < words; k += blockDim.x) {
      if ((sm.CH[k >> B.shift] >> (k & ((1u << B.shift) - 1u))) & 1u) dev::red_min(g + k, sm.S[k]);
    }
  }
  __syncthreads();
}

// Work of round r in two prefixes: block items (one tile visit per unit of a
// frontier batch in a dense near round, for batches mapped to tile visits)
// and warp items (everything else, as the chunked layout counts them: a
// pack of queued chunks per sparse near item, a pack of chunk slots of a
// dense round of a batch mapped to chunks, 256 far entries per split item,
// Jacobi / dense warp items).
__device__ __forceinline__ bool visits_tiles(const LaunchParams& p, u32 b) {
  return p.mappings == nullptr || p.mappings[b] == BFX_MAPPING_TILE_VISITS;
}

__device__ u32 round_work_tiled(const LaunchParams& p, u32 r, u32* prefix_block, u32* prefix_warp) {
  const u32 ridx = r % 3u;
  block_prefix(prefix_block, p.nb, [&](u32 b) -> u32 {
    if (engine_of(p, b) != BFX_ENGINE_FRONTIER_PUSH || !visits_tiles(p, b)) return 0u;
    const DBatch& B = p.batches[b];
    const u32 n = min(dev::ld_cg(&p.ctl[b].count[ridx]), B.U);
    return n != 0u && chunk_dense(n, B.U, 5u) ? chunk_count(B.U, p.tshift) : 0u;
  });
  block_prefix(prefix_warp, p.nb, [&](u32 b) -> u32 {
    const DBatch& B = p.batches[b];
    if (engine_of(p, b) == BFX_ENGINE_FRONTIER_PUSH) {
      const DCtl& C = p.ctl[b];
      const u32 n = min(dev::ld_cg(&C.count[ridx]), B.U);
      // dense rounds of a batch mapped to chunks: every chunk slot, in index
      // order, as the chunked layout runs them
      if (n != 0u) {
        return chunk_dense(n, B.U, 5u) && visits_tiles(p, b) ? 0u : (chunk_slots(n, B.U) | kPackable);
      }
      const u32 f = min(dev::ld_cg(&C.fcount[dev::ld_cg(&C.gen[r & 1u]) % 3u]), B.U);
      return (f + kSplitPerItem - 1u) / kSplitPerItem;
    }
    return batch_exec(p, b, ridx) != 0u ? (((B.U << B.shift) + 31u) >> 5) : 0u;
  }, p.cpack);
  return prefix_block[p.nb] + prefix_warp[p.nb];
}

// One round of the tiled layout.  Phase 1: block items drawn from a
// per-round counter, one tile visit each (block-uniform branches only,
// their values broadcast through shared memory).  Phase 2: the warp items,
// run by the chunked layout's round body (each warp draws its own items).
template <bool kCount>
__device__ void round_body_tiled(const LaunchParams& p, u32 r, u32* prefix_block, u32* prefix_warp, Work& wk) {
  __shared__ u32 s_item;
  __shared__ u32 s_vals[3];
  const u32 ridx = r % 3u, widx = (r + 1u) % 3u;
  const u32 total = prefix_block[p.nb];
  const u32 wib = threadIdx.x >> 5;
  const TileSmem sm = tile_smem(prefix_block, p.nb, p.tshift, p.tile_wmax);
  Stages st{{0u, 0u}, 0xFFFFFFFFu};
  u32 staged_batch = 0xFFFFFFFFu;
  while (total != 0u) {
    if (threadIdx.x == 0u) s_item = atomicAdd(&p.run->items[ridx], 1u);
    __syncthreads();
    const u32 w = s_item;
    __syncthreads();
    if (w >= total) break;
    const u32 b = find_batch(prefix_block, p.nb, w);
    const DBatch& B = p.batches[b];
    DCtl& C = p.ctl[b];
    if (threadIdx.x == 0u) {
      s_vals[0] = dev::ld_cg(&C.gen[r & 1u]);
      s_vals[1] = dev::ld_cg(&C.tau[r & 1u]);
    }
    __syncthreads();
    const u32 g = s_vals[0], tau = s_vals[1];
    __syncthreads();
    const FrontierView V = frontier_view(B, r & 1u, g % 3u, (g + 1u) % 3u);
    if (b != staged_batch) {
      stages_flush(st);
      staged_batch = b;
      if (lane_id() == 0u) {
        s_stage_queue[kNear][wib] = StageQueue{V.queue_w, &C.count[widx], &C.error_bits, V.U};
        s_stage_queue[kFar][wib] = StageQueue{V.pile, &C.fcount[g % 3u], &C.error_bits, V.U};
        s_fmin_target[wib] = &C.fmin[g % 3u];
      }
      __syncwarp();
    }
    tile_visit<kCount>(p, V, w - prefix_block[b], tau, sm, st, wk);
  }
  stages_flush(st);
  __syncthreads();
  round_body<kCount, 2, true>(p, r, prefix_warp, wk);
}

// Persistent cooperative kernel of the tiled layout: blocks of kThreads
// (256: up to 128 registers; 384: 80), two per SM by launch bounds (the
// staged labels take up to 64 KB per block).
template <bool kCount, int kThreads>
__global__ void __launch_bounds__(kThreads, 2) persistent_tiled_kernel(LaunchParams p) {
  extern __shared__ u32 prefix[];
  const u32 nblocks = gridDim.x;
  Work wk;
  wk.zero();
  u64 traced[2] = {0u, 0u};
  const u64 t0 = dev::global_ns();
  u32 r = 0;
  u32* const prefix_warp = prefix + (p.nb + 1u);
  for (;; ++r) {
    const u32 total = round_work_tiled(p, r, prefix, prefix_warp);
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
    round_body_tiled<kCount>(p, r, prefix, prefix_warp, wk);
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
