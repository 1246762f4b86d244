// Frontier push round bodies (included by engine.cu after the device records):
// frontier_group (sub-warp groups per queued vertex), frontier_flat (flat
// (lane, edge) work list over queued vertices or, with kChunked, over queued
// 32-vertex chunks -- the default), split_group (near/far split rounds).
//
// frontier_group: one warp item covers EPW = 32 / S queue entries of one batch: a group of S
// threads per entry (S = 8 for batches of <= 8 lanes, 32 otherwise).  Within
// a group the entry's k active lanes are spread over aligned sub-groups of
// kp = 2^ceil(log2 k) threads, so a group relaxes S / kp edges per step and
// all groups of the warp step together (the step count is the warp's
// maximum, so every shuffle has the full warp).
//
// Per entry the dependent chain is short: the group leader loads the queue
// word {vertex, compact index}, the pending lanes and the row bounds in one
// go and clears the pending lanes with a plain store -- the read slot is
// only written in the previous round, and every vertex is queued at most
// once per round, so no atomic is needed.  Each thread pre-reads its
// destination label and issues a non-returning 64-bit min only for a smaller
// candidate; success bits are OR-combined per edge; the first lane of the
// edge ORs them into the next round's pending lanes and the warp claims
// queue slots with one atomicAdd.
#pragma once

// Registers-only view of one batch for one round of the frontier engine:
// the per-round slots (read / write pending masks and queues, the far pile
// of this generation) are selected once per warp item, so the round body
// never re-reads the batch record from global memory after its atomics.
struct FrontierView {
  u64* dist;
  u32* mask_r;
  u32* mask_w;
  u64* queue_r;
  u64* queue_w;
  const uint2* tiles;
  u32* fmask;
  u32* fbound;    // lower bound of each vertex's parked labels
  u64* pile;      // near round: far pile being filled; split round: pile read
  u64* pile_out;  // split round: pile written
  const uint2* crow;  // compact index -> {CSR row begin, out-degree} (chunked layout)
  const uint2* clrun; // compact index -> own-tile run {first CSR index, count} (tiled layout)
  u32* cmask_r;       // chunk bitmaps (chunked layout): read and write slots
  u32* cmask_w;
  u32 shift, valid, U, full;
};

__device__ __forceinline__ FrontierView frontier_view(const DBatch& b, u32 rd, u32 pile, u32 pile_out) {
  FrontierView v;
  v.dist = b.dist[0];
  v.mask_r = b.mask[rd];
  v.mask_w = b.mask[rd ^ 1u];
  v.queue_r = b.queue[rd];
  v.queue_w = b.queue[rd ^ 1u];
  v.tiles = b.tiles;
  v.fmask = b.fmask;
  v.fbound = b.fbound;
  v.pile = b.fpile[pile];
  v.pile_out = b.fpile[pile_out];
  v.crow = b.crow;
  v.clrun = b.clrun;
  v.cmask_r = b.cmask[rd];
  v.cmask_w = b.cmask[rd ^ 1u];
  v.shift = b.shift;
  v.valid = b.valid;
  v.U = b.U;
  v.full = b.full;
  return v;
}

// Claims staged per warp in shared memory and appended to their queue with
// one atomicAdd per 32 or more entries.  A stage lives for the warp's items
// of one (round, batch) -- round_body flushes it when the warp moves on to
// another batch and at the end of the round -- so the queue counters, one
// address per batch that every warp appends to, see one atomic per 32
// claims instead of one per warp step.  Two stages per warp: kNear (the next
// round's queue) and kFar (the far pile).  The buffers and the queue
// descriptors live in shared memory; a thread keeps only the warp-uniform
// entry counts in registers.
constexpr u32 kStage = 64;  // entries per warp stage: < 32 before a push adds <= 32
constexpr u32 kNear = 0u, kFar = 1u;

struct StageQueue {
  u64* queue;
  u32* counter;  // queue size
  u32* err;      // the batch's error bits (queue overflow)
  u32 cap;       // queue capacity (the batch's union vertex count)
};

__shared__ u64 s_stage_buf[2][16][kStage];  // blocks of up to 512 threads
__shared__ StageQueue s_stage_queue[2][16];
__shared__ u32* s_fmin_target[16];           // fmin of the far pile the warp parks on

struct Stages {
  u32 n[2];  // staged entries per stage (warp-uniform)
  u32 fd;    // smallest parked distance seen by this thread (folded by farmin_flush)
};

// Executed by all 32 threads.
__device__ __forceinline__ void stage_flush(Stages& st, u32 k) {
  if (st.n[k] == 0u) return;  // warp-uniform
  const u32 wib = threadIdx.x >> 5;
  const StageQueue q = s_stage_queue[k][wib];
  __syncwarp();
  const u32 lane = lane_id();
  u32 pos = 0u;
  if (lane == 0u) pos = atomicAdd(q.counter, st.n[k]);
  pos = __shfl_sync(0xFFFFFFFFu, pos, 0);
  for (u32 i = lane; i < st.n[k]; i += 32u) {
    if (pos + i < q.cap) {
      q.queue[pos + i] = s_stage_buf[k][wib][i];
    } else {
      atomicOr(q.err, static_cast<u32>(BFX_DEVICE_ERROR_QUEUE_OVERFLOW));
    }
  }
  __syncwarp();
  st.n[k] = 0u;
}

// Appends the claiming threads' queue words to stage k; flushes at >= 32
// staged.  Executed by all 32 threads.
__device__ __forceinline__ void stage_push(Stages& st, u32 k, bool claim, u64 word) {
  const u32 lane = lane_id();
  const u32 cm = __ballot_sync(0xFFFFFFFFu, claim);
  if (claim) s_stage_buf[k][threadIdx.x >> 5][st.n[k] + __popc(cm & ((1u << lane) - 1u))] = word;
  st.n[k] += static_cast<u32>(__popc(cm));
  if (st.n[k] >= 32u) stage_flush(st, k);
}

// Folds the threads' smallest parked distances into the pile's fmin (one
// atomicMin per warp and (round, batch)).  Executed by all 32 threads.
__device__ __forceinline__ void farmin_flush(Stages& st) {
  const u32 x = __reduce_min_sync(0xFFFFFFFFu, st.fd);
  if (lane_id() == 0u && x != 0xFFFFFFFFu) atomicMin(s_fmin_target[threadIdx.x >> 5], x);
  st.fd = 0xFFFFFFFFu;
}

__device__ __forceinline__ void stages_flush(Stages& st) {
  stage_flush(st, kNear);
  stage_flush(st, kFar);
  farmin_flush(st);
}

__device__ __forceinline__ u64 queue_word(u32 v, u32 cv) {
  return static_cast<u64>(v) | (static_cast<u64>(cv) << 32);
}

template <bool kCount, u32 S>
__device__ __forceinline__ void frontier_group(const LaunchParams& p, const FrontierView& B, DCtl& C, u32 item, u32 count,
                                               u32 rd, u32 widx, u32 tau_bits, u32 pile, Work& wk) {
  constexpr u32 EPW = 32u / S;
  const u32 lane = lane_id();
  const u32 sl = lane & (S - 1u);
  const u32 leader = lane & ~(S - 1u);
  const u32 entry = item * EPW + (lane / S);
  const bool live = entry < count;
  u32* const mask_r = B.mask_r;
  u32 v = 0u, cv = 0u, m = 0u, rb = 0u, re = 0u;
  if (live && sl == 0u) {
    const u64 q = dev::ld_cg(B.queue_r + entry);
    v = static_cast<u32>(q);
    cv = static_cast<u32>(q >> 32);
    if (v < p.g.V && cv < B.U) {
      m = dev::ld_cg(mask_r + cv) & B.valid;
      rb = __ldg(p.g.csr_off + v);
      re = __ldg(p.g.csr_off + v + 1u);
      mask_r[cv] = 0u;
    } else {
      // a queue word outside the batch: record it and skip the entry
      atomicOr(&C.error_bits, static_cast<u32>(BFX_DEVICE_ERROR_INVALID_CONTROLLER_STATE));
      v = cv = 0u;
    }
  }
  v = __shfl_sync(0xFFFFFFFFu, v, static_cast<int>(leader));
  cv = __shfl_sync(0xFFFFFFFFu, cv, static_cast<int>(leader));
  m = __shfl_sync(0xFFFFFFFFu, m, static_cast<int>(leader));
  rb = __shfl_sync(0xFFFFFFFFu, rb, static_cast<int>(leader));
  re = __shfl_sync(0xFFFFFFFFu, re, static_cast<int>(leader));
  const u32 k = __popc(m);
  const u32 s = k <= 1u ? 0u : 32u - __clz(k - 1u);
  const u32 kp = 1u << s;  // <= S by construction (k <= W <= S)
  const u32 G = S >> s;    // edges per step for this entry
  const u32 slot = sl >> s;
  const u32 j = sl & (kp - 1u);
  const bool has_lane = live && j < k;
  if (kCount && live && sl == 0u) {
    wk.c[0] += 1;
    wk.c[1] += re - rb;
    wk.c[2] += k;
  }
  u32 ql = 0u, src_bits = dev::kInfBits;
  if (has_lane) {
    u32 mm = m;
    for (u32 t = 0; t < j; ++t) mm &= mm - 1u;  // drop the j lowest active lanes
    ql = __ffs(mm) - 1u;
    src_bits = dev::hi(dev::ld_cg(B.dist + ((static_cast<u64>(cv) << B.shift) + ql)));
  }
  const u32 steps_mine = live ? (re - rb + G - 1u) / G : 0u;
  const u32 steps = __reduce_max_sync(0xFFFFFFFFu, steps_mine);
  // Sub-group sizes differ between the entries of one warp, so the OR
  // combine runs the warp's largest trip count (every full-mask shuffle is
  // executed by all 32 threads) and each thread keeps only the partners
  // inside its own sub-group.
  const u32 kp_warp = __reduce_max_sync(0xFFFFFFFFu, kp);
  u32* const mask_w = B.mask_w;
  u64* const queue_w = B.queue_w;
  for (u32 st = 0; st < steps; ++st) {
    const u32 e = rb + st * G + slot;
    u32 bits = 0u, fbits = 0u, cdst = 0u, dstv = 0u, fd = 0xFFFFFFFFu;
    if (has_lane && e < re) {
      const uint4 rec = __ldg(p.g.csr + e);
      const uint2 dt = B.tiles[rec.w];
      cdst = rec.x - dt.y;
      dstv = rec.x;
      if (((dt.x >> ql) & 1u) && src_bits != dev::kInfBits) {
        const u64 cand = dev::candidate(src_bits, rec.y, rec.z);
        u64* const target = B.dist + ((static_cast<u64>(cdst) << B.shift) + ql);
        const u64 cur = dev::ld_cg(target);
        if (kCount) wk.c[3] += 1;
        if (cand < cur) {
          dev::red_min(target, cand);
          if (dev::hi(cand) < dev::hi(cur)) {
            // near: below this round's threshold; far: parked until a split
            if (dev::hi(cand) < tau_bits) {
              bits = 1u << ql;
            } else {
              fbits = 1u << ql;
              fd = dev::hi(cand);
              dev::red_min_u32(B.fbound + cdst, fd);
            }
          }
          if (kCount) {
            wk.c[6] += 1;
            wk.c[5] += (bits | fbits) != 0u;
          }
        }
      }
    }
    for (u32 o = 1; o < kp_warp; o <<= 1) {
      const u32 xb = __shfl_xor_sync(0xFFFFFFFFu, bits, o);
      const u32 xf = __shfl_xor_sync(0xFFFFFFFFu, fbits, o);
      if (o < kp) {
        bits |= xb;
        fbits |= xf;
      }
    }
    if (__any_sync(0xFFFFFFFFu, fbits != 0u)) {
      // smallest parked distance of the pile (one atomic per warp step)
      fd = __reduce_min_sync(0xFFFFFFFFu, fd);
      if (lane == 0u) atomicMin(&C.fmin[pile], fd);
      bool fclaim = false;
      if (j == 0u && fbits != 0u) fclaim = atomicOr(B.fmask + cdst, fbits) == 0u;
      const u32 fm = __ballot_sync(0xFFFFFFFFu, fclaim);
      if (fm != 0u) {
        const u32 first = __ffs(fm) - 1u;
        u32 pos = 0u;
        if (lane == first) pos = atomicAdd(&C.fcount[pile], static_cast<u32>(__popc(fm)));
        pos = __shfl_sync(0xFFFFFFFFu, pos, static_cast<int>(first));
        if (fclaim) {
          const u32 at = pos + __popc(fm & ((1u << lane) - 1u));
          if (at < B.U) {
            B.pile[at] = static_cast<u64>(dstv) | (static_cast<u64>(cdst) << 32);
          } else {
            atomicOr(&C.error_bits, static_cast<u32>(BFX_DEVICE_ERROR_QUEUE_OVERFLOW));
          }
        }
      }
    }
    bool claim = false;
    if (j == 0u && bits != 0u) claim = atomicOr(mask_w + cdst, bits) == 0u;
    const u32 cm = __ballot_sync(0xFFFFFFFFu, claim);
    if (cm != 0u) {
      const u32 first = __ffs(cm) - 1u;
      u32 pos = 0u;
      if (lane == first) pos = atomicAdd(&C.count[widx], static_cast<u32>(__popc(cm)));
      pos = __shfl_sync(0xFFFFFFFFu, pos, static_cast<int>(first));
      if (claim) {
        if (kCount) wk.c[4] += 1;
        const u32 at = pos + __popc(cm & ((1u << lane) - 1u));
        if (at < B.U) {
          queue_w[at] = static_cast<u64>(dstv) | (static_cast<u64>(cdst) << 32);
        } else {
          atomicOr(&C.error_bits, static_cast<u32>(BFX_DEVICE_ERROR_QUEUE_OVERFLOW));
        }
      }
    }
  }
}

// Split round of the near/far frontier: the batch's near frontier is empty,
// so the threshold advances (split_threshold) and every parked (vertex, lane) of the
// current far pile is re-examined: lanes whose label is now below the new
// threshold join the next round's near frontier, the rest move to the next
// pile.  The batch runs no near round in the same round, so the far masks it
// reads are stable and are cleared with plain stores.
//
// A warp item covers kSplitPerItem (256) pile entries, eight per thread: the
// eight entries' pile words, far masks and bounds are loaded together, and
// the entries that stay parked whole (bound not below the new threshold) --
// usually most of the pile -- are appended to the next pile with one counter
// atomic for the item and plain stores, so a pile of millions of entries
// does not serialise on its counter.  The other entries re-read their parked
// labels; their claims are warp-aggregated through the stages.
constexpr u32 kSplitPer = 8u;
constexpr u32 kSplitPerItem = 32u * kSplitPer;

template <bool kCount, bool kChunked>
__device__ __forceinline__ void split_group(const LaunchParams& p, const FrontierView& B, DCtl& C, u32 item, u32 count,
                                            u32 tau_next, Stages& st, Work& wk) {
  const u32 lane = lane_id();
  const u32 below = (1u << lane) - 1u;
  u64 q[kSplitPer];
  u32 bits[kSplitPer], bound[kSplitPer];
#pragma unroll
  for (u32 j = 0; j < kSplitPer; ++j) {
    const u32 entry = item * kSplitPerItem + j * 32u + lane;
    q[j] = entry < count ? dev::ld_cg(B.pile + entry) : ~u64{0};
  }
#pragma unroll
  for (u32 j = 0; j < kSplitPer; ++j) {
    bits[j] = 0u;
    bound[j] = 0xFFFFFFFFu;
    const u32 cv = static_cast<u32>(q[j] >> 32);
    if (q[j] != ~u64{0}) {
      if (cv < B.U) {
        bits[j] = dev::ld_cg(B.fmask + cv) & B.valid;
        bound[j] = dev::ld_cg(B.fbound + cv);
      } else {
        atomicOr(&C.error_bits, static_cast<u32>(BFX_DEVICE_ERROR_INVALID_CONTROLLER_STATE));
        q[j] = ~u64{0};
      }
    }
  }
  // Every parked label of a vertex is at least its bound (each far
  // improvement lowers it; a split stores the exact minimum of the lanes it
  // re-parks).  When the bound is finite and not below the new threshold,
  // all lanes stay parked: the entry moves to the next pile unread and its
  // far mask stays set.
  u32 stay_mask = 0u, nstay = 0u, stay_rank[kSplitPer];
#pragma unroll
  for (u32 j = 0; j < kSplitPer; ++j) {
    const bool stays = q[j] != ~u64{0} && bits[j] != 0u && bound[j] < dev::kInfBits && bound[j] >= tau_next;
    const u32 bal = __ballot_sync(0xFFFFFFFFu, stays);
    stay_rank[j] = nstay + static_cast<u32>(__popc(bal & below));
    nstay += static_cast<u32>(__popc(bal));
    if (stays) {
      stay_mask |= 1u << j;
      st.fd = min(st.fd, bound[j]);
    }
  }
  if (nstay != 0u) {  // warp-uniform
    const StageQueue sq = s_stage_queue[kFar][threadIdx.x >> 5];
    u32 pos = 0u;
    if (lane == 0u) pos = atomicAdd(sq.counter, nstay);
    pos = __shfl_sync(0xFFFFFFFFu, pos, 0);
#pragma unroll
    for (u32 j = 0; j < kSplitPer; ++j) {
      if ((stay_mask >> j) & 1u) {
        if (pos + stay_rank[j] < sq.cap) {
          sq.queue[pos + stay_rank[j]] = q[j];
        } else {
          atomicOr(sq.err, static_cast<u32>(BFX_DEVICE_ERROR_QUEUE_OVERFLOW));
        }
      }
    }
  }
  if (kCount) {
#pragma unroll
    for (u32 j = 0; j < kSplitPer; ++j) {
      if (q[j] != ~u64{0}) {
        wk.c[0] += 1;
        wk.c[11] += 1;
        if (!((stay_mask >> j) & 1u)) wk.c[12] += static_cast<u32>(__popc(bits[j]));
      }
    }
  }
  // The other entries: their parked lanes are re-read eight at a time (the
  // eight label loads issued back to back).
#pragma unroll 1
  for (u32 j = 0; j < kSplitPer; ++j) {
    const bool go = q[j] != ~u64{0} && !((stay_mask >> j) & 1u);
    if (!__any_sync(0xFFFFFFFFu, go)) continue;
    const u32 v = static_cast<u32>(q[j]), cv = static_cast<u32>(q[j] >> 32);
    u32 near = 0u, far = 0u, fd = 0xFFFFFFFFu;
    if (go) {
      B.fmask[cv] = 0u;
      u64* const row = B.dist + (static_cast<u64>(cv) << B.shift);
      for (u32 rest = bits[j]; rest != 0u;) {
        u32 ls[8], ds[8];
#pragma unroll
        for (u32 i = 0; i < 8u; ++i) {
          ls[i] = rest != 0u ? static_cast<u32>(__ffs(rest)) - 1u : 32u;
          rest &= rest - 1u;
        }
#pragma unroll
        for (u32 i = 0; i < 8u; ++i) ds[i] = ls[i] < 32u ? dev::hi(dev::ld_cg(row + ls[i])) : 0u;
#pragma unroll
        for (u32 i = 0; i < 8u; ++i) {
          if (ls[i] < 32u) {
            if (ds[i] < tau_next) {
              near |= 1u << ls[i];
            } else {
              far |= 1u << ls[i];
              fd = min(fd, ds[i]);
            }
          }
        }
      }
      // the bound of the lanes that stay parked (none: cleared)
      B.fbound[cv] = far != 0u ? fd : 0xFFFFFFFFu;
    }
    // far lanes stay parked (next pile); near lanes join the next round
    bool fclaim = false, claim = false;
    if (far != 0u) fclaim = atomicOr(B.fmask + cv, far) == 0u;
    u64 qword = queue_word(v, cv);  // queue word: {vertex, compact index}, or the chunk (chunked layout)
    if (near != 0u) {
      if (kChunked) {
        dev::red_or(B.mask_w + cv, near);
        const u32 chunk = cv >> p.cshift;
        const u32 bit = 1u << (chunk & 31u);
        claim = (atomicOr(B.cmask_w + (chunk >> 5), bit) & bit) == 0u;
        qword = chunk;
      } else {
        claim = atomicOr(B.mask_w + cv, near) == 0u;
      }
    }
    st.fd = min(st.fd, fd);
    stage_push(st, kFar, fclaim, queue_word(v, cv));
    if (kCount && claim) wk.c[4] += 1;
    stage_push(st, kNear, claim, qword);
  }
}

// Entries per flat warp item for a batch frontier of n entries: 32 from 2,048
// entries up, otherwise the power of two nearest below n / 64 (at least 1),
// so a small frontier is spread over up to 64 warps instead of a few.
__device__ __forceinline__ u32 flat_entries_per_item(u32 n) {
  const u32 e = n >> 6;
  if (e >= 32u) return 32u;
  return e == 0u ? 1u : 1u << (31u - __clz(e));
}

// Flat frontier round body: one warp item covers `epi` queue entries
// (flat_entries_per_item of the batch's frontier size).  Every thread below epi loads one entry's header (queue word, pending lanes, row
// bounds) -- 32 independent header chains per warp -- and the entries'
// (lane, out-edge) pairs are flattened into one work list, entry-major, then
// lane, then edge.  The warp walks the list 64 items per iteration, two per
// thread, with the memory accesses of the two items interleaved phase by
// phase (record and source label, tile entry, target label, pending-word OR)
// so each thread keeps two dependent chains in flight.  A thread finds the
// entry of a work item by a binary search over the warp's inclusive work scan
// (five shuffles).  Every thread ORs its own success into the next round's
// pending word; the OR that turns the word non-zero claims the vertex.  A
// far success (near/far frontier) ORs its lane into the far mask the same
// way and the OR that turns it non-zero parks the vertex on the far pile;
// the smallest parked distance is kept per thread (Stages::fd).  The ORs'
// results are read one iteration later (after the next items' first loads
// are issued), and claimed vertices are staged in the warp's shared-memory
// stages (Stages) and appended to the next queue or the far pile with one
// counter atomic per 32 or more claims, off the per-step chain.  All loops
// are warp-uniform.

struct FlatItem {
  bool live;
  u32 ql, ed, cv;
};

// edge_major: work items ordered entry, then edge, then lane (consecutive
// threads relax the lanes of one edge, whose labels are adjacent); otherwise
// entry, then lane, then edge.
__device__ __forceinline__ FlatItem flat_decode(u32 w, u32 total, u32 incl, u32 excl, u32 cv, u32 m, u32 rb,
                                                u32 deg, bool edge_major) {
  u32 e = 0u;
  for (u32 s = 16u; s > 0u; s >>= 1) {
    if (__shfl_sync(0xFFFFFFFFu, incl, static_cast<int>(e + s - 1u)) <= w) e += s;
  }
  const u32 ecv = __shfl_sync(0xFFFFFFFFu, cv, static_cast<int>(e));
  const u32 em = __shfl_sync(0xFFFFFFFFu, m, static_cast<int>(e));
  const u32 erb = __shfl_sync(0xFFFFFFFFu, rb, static_cast<int>(e));
  const u32 edeg = __shfl_sync(0xFFFFFFFFu, deg, static_cast<int>(e));
  const u32 eexcl = __shfl_sync(0xFFFFFFFFu, excl, static_cast<int>(e));
  FlatItem it{w < total, 0u, 0u, ecv};
  if (it.live) {
    const u32 r = w - eexcl;
    u32 j;  // lane ordinal within the entry
    if (edge_major) {
      const u32 k = static_cast<u32>(__popc(em));
      const u32 edge = r / k;
      j = r - edge * k;
      it.ed = erb + edge;
    } else {
      j = r / edeg;
      it.ed = erb + (r - j * edeg);
    }
    u32 mm = em;
    for (u32 t = 0; t < j; ++t) mm &= mm - 1u;
    it.ql = __ffs(mm) - 1u;
  }
  return it;
}

// kChunked: the item is a pack of `pack` (the round's pack, at most
// LaunchParams::cpack and kPackMax) chunk slots -- in a sparse round consecutive queue words,
// each naming a queued 32-vertex chunk (compact indices 32 c .. 32 c + 31);
// in a dense round consecutive chunk slots in index order, of which only
// those whose bit is set in the chunk bitmap are read.  The pending lanes
// and the compact row table {row begin, out-degree} of each chunk's 32
// vertices are read together (the next chunk's loads are issued before the
// current one is compacted), and the vertices with pending lanes are
// compacted into a per-warp ring in shared memory, so a work list covers up
// to 32 active vertices of several chunks instead of the few a single chunk
// holds.  Successes set the pending lane with a non-returning OR and claim
// the target's chunk through the chunk bitmap.
// kPairs (chunked only): the warp walks the group's (entry, lane) pairs, one
// per thread, each over its entry's out-edges -- no per-edge decode.
constexpr u32 kNoChunk = 0xFFFFFFFFu;
constexpr u32 kPackMax = 8u;              // chunk slots per warp item, at most
__shared__ uint4 s_pack[16][64];          // per warp: ring of {compact index, pending lanes, row begin, degree}

// Chunked near round of a batch with n queued chunks: sparse rounds walk
// the queue (claim order); once at least half of the batch's chunk slots are
// pending, the items are all chunk slots in index order and a warp skips the
// slots whose bit is clear.  Concurrent warps then relax neighbouring
// chunks, whose target labels (intra-tile edges) are shared in the L2.
// cshift: the claim unit is 2^cshift compact vertices (5: 32-vertex chunks).
// chunk_slots: the round's slots (queue words or chunk slots), of which a
// warp item takes the round's pack.
__device__ __forceinline__ u32 chunk_count(u32 U, u32 cshift) { return (U + (1u << cshift) - 1u) >> cshift; }
__device__ __forceinline__ bool chunk_dense(u32 n, u32 U, u32 cshift) { return 2u * n >= chunk_count(U, cshift); }
__device__ __forceinline__ u32 chunk_slots(u32 n, u32 U) { return chunk_dense(n, U, 5u) ? chunk_count(U, 5u) : n; }

template <bool kCount, u32 kItems, bool kChunked, bool kPairs = false>
__device__ __forceinline__ void frontier_flat(const LaunchParams& p, const FrontierView& B, DCtl& C, u32 item, u32 count,
                                              u32 epi, u32 tau_bits, Stages& st, Work& wk, bool dense = false,
                                              u32 pack = 1u) {
  const u32 lane = lane_id();
  // Claims of the previous step: their pending-word and far-mask ORs stay
  // in flight while the next step decodes its items and issues its first
  // loads.  p_old / f_old == 0: the OR claimed the vertex (or its chunk).
  u32 p_old[kItems], p_v[kItems], p_cv[kItems], f_old[kItems], f_v[kItems], f_cv[kItems];
  u32 known_chunk = 0xFFFFFFFFu;  // chunked layout: last chunk whose bit this thread ORed
#pragma unroll
  for (u32 u = 0; u < kItems; ++u) {
    p_old[u] = f_old[u] = 1u;
    p_v[u] = p_cv[u] = f_v[u] = f_cv[u] = 0u;
  }
  // One step: kItems (lane, edge) items per thread, memory phases interleaved.
  auto step = [&](const FlatItem (&it)[kItems], u32 (&src)[kItems], bool load_src) {
    u32 bits[kItems], fbits[kItems], cdst[kItems], dstv[kItems];
    uint4 rec[kItems];
    uint2 dt[kItems];
#pragma unroll
    for (u32 u = 0; u < kItems; ++u) bits[u] = fbits[u] = cdst[u] = dstv[u] = 0u;
#pragma unroll
    for (u32 u = 0; u < kItems; ++u) {
      if (it[u].live) {
        if (load_src) src[u] = dev::hi(dev::ld_cg(B.dist + ((static_cast<u64>(it[u].cv) << B.shift) + it[u].ql)));
        rec[u] = __ldg(p.g.csr + it[u].ed);
      }
    }
    bool any_claim = false;
#pragma unroll
    for (u32 u = 0; u < kItems; ++u) any_claim |= p_old[u] == 0u || f_old[u] == 0u;
    if (__any_sync(0xFFFFFFFFu, any_claim)) {  // claims are rare: one vote skips the stage pushes
#pragma unroll
      for (u32 u = 0; u < kItems; ++u) {
        if (kCount && p_old[u] == 0u) wk.c[4] += 1;
        stage_push(st, kNear, p_old[u] == 0u, queue_word(p_v[u], p_cv[u]));
        stage_push(st, kFar, f_old[u] == 0u, queue_word(kChunked ? f_cv[u] : f_v[u], f_cv[u]));
      }
    }
#pragma unroll
    for (u32 u = 0; u < kItems; ++u) {
      if (it[u].live) {
        // full-graph batch: compact index = vertex id, every lane admitted
        dt[u] = B.full ? make_uint2(B.valid, 0u) : B.tiles[rec[u].w];
        cdst[u] = rec[u].x - dt[u].y;
        dstv[u] = rec[u].x;
      }
    }
    u64 cur[kItems], cand[kItems];
    bool relax[kItems];
#pragma unroll
    for (u32 u = 0; u < kItems; ++u) {
      relax[u] = it[u].live && ((dt[u].x >> it[u].ql) & 1u) && src[u] != dev::kInfBits;
      if (relax[u]) {
        cand[u] = dev::candidate(src[u], rec[u].y, rec[u].z);
        u64* const target = B.dist + ((static_cast<u64>(cdst[u]) << B.shift) + it[u].ql);
        // returning min (one L2 read-modify-write) or pre-read + min on success
        cur[u] = p.amin ? dev::atom_min(target, cand[u]) : dev::ld_cg(target);
      }
    }
#pragma unroll
    for (u32 u = 0; u < kItems; ++u) {
      if (relax[u]) {
        if (kCount) wk.c[3] += 1;
        if (cand[u] < cur[u]) {
          if (!p.amin) dev::red_min(B.dist + ((static_cast<u64>(cdst[u]) << B.shift) + it[u].ql), cand[u]);
          if (dev::hi(cand[u]) < dev::hi(cur[u])) {
            if (dev::hi(cand[u]) < tau_bits) {
              bits[u] = 1u << it[u].ql;
            } else {
              fbits[u] = 1u << it[u].ql;
              st.fd = min(st.fd, dev::hi(cand[u]));
              dev::red_min_u32(B.fbound + cdst[u], dev::hi(cand[u]));
            }
          }
          if (kCount) {
            wk.c[6] += 1;
            wk.c[5] += (bits[u] | fbits[u]) != 0u;
          }
        }
      }
    }
    // the far-mask and pending-word ORs are issued here; their results are
    // read by the next iteration (or after the loop)
#pragma unroll
    for (u32 u = 0; u < kItems; ++u) {
      f_old[u] = fbits[u] != 0u ? atomicOr(B.fmask + cdst[u], fbits[u]) : 1u;
      if (!kChunked) f_v[u] = dstv[u];  // the chunked layout's split rounds read only the compact index
      f_cv[u] = cdst[u];
    }
#pragma unroll
    for (u32 u = 0; u < kItems; ++u) {
      if (kChunked) {
        // pending lane with a non-returning OR; the chunk bit's OR claims.
        // A chunk this thread already ORed in this item is known to be set
        // for the round, so its bit is not ORed again.
        const u32 chunk = cdst[u] >> 5;
        const u32 bit = 1u << (chunk & 31u);
        p_old[u] = 1u;
        if (bits[u] != 0u) {
          dev::red_or(B.mask_w + cdst[u], bits[u]);
          if (chunk != known_chunk) {
            p_old[u] = atomicOr(B.cmask_w + (chunk >> 5), bit) & bit;
            known_chunk = chunk;
          }
        }
        p_v[u] = chunk;
        p_cv[u] = 0u;
      } else {
        p_old[u] = bits[u] != 0u ? atomicOr(B.mask_w + cdst[u], bits[u]) : 1u;
        p_v[u] = dstv[u];
        p_cv[u] = cdst[u];
      }
    }
  };
  // The work list of one group of up to 32 entries, one per thread
  // (m == 0: no entry).
  auto relax_entries = [&](const u32 cv, const u32 m, const u32 rb, const u32 deg) {
    if (kPairs) {
      // Pair mode: each thread takes one (entry, lane) pair of the item and
      // walks that entry's edges kItems per step; one source read per pair,
      // no per-edge decode.
      const u32 k = static_cast<u32>(__popc(m));
      u32 kincl = k;
      for (u32 o = 1; o < 32u; o <<= 1) {
        const u32 y = __shfl_up_sync(0xFFFFFFFFu, kincl, o);
        if (lane >= o) kincl += y;
      }
      const u32 kexcl = kincl - k;
      const u32 pairs = __shfl_sync(0xFFFFFFFFu, kincl, 31);
      for (u32 pbase = 0; pbase < pairs; pbase += 32u) {
        const u32 pi = pbase + lane;
        u32 e = 0u;
        for (u32 s = 16u; s > 0u; s >>= 1) {
          if (__shfl_sync(0xFFFFFFFFu, kincl, static_cast<int>(e + s - 1u)) <= pi) e += s;
        }
        const u32 ecv = __shfl_sync(0xFFFFFFFFu, cv, static_cast<int>(e));
        const u32 em = __shfl_sync(0xFFFFFFFFu, m, static_cast<int>(e));
        const u32 erb = __shfl_sync(0xFFFFFFFFu, rb, static_cast<int>(e));
        const u32 edeg = __shfl_sync(0xFFFFFFFFu, deg, static_cast<int>(e));
        const u32 eexcl = __shfl_sync(0xFFFFFFFFu, kexcl, static_cast<int>(e));
        const bool plive = pi < pairs;
        u32 pql = 0u, psrc = dev::kInfBits;
        if (plive) {
          u32 mm = em;
          for (u32 t = 0; t < pi - eexcl; ++t) mm &= mm - 1u;
          pql = __ffs(mm) - 1u;
          psrc = dev::hi(dev::ld_cg(B.dist + ((static_cast<u64>(ecv) << B.shift) + pql)));
        }
        const u32 steps = __reduce_max_sync(0xFFFFFFFFu, plive ? edeg : 0u);
        for (u32 s = 0; s < steps; s += kItems) {
          FlatItem it[kItems];
          u32 src[kItems];
  #pragma unroll
          for (u32 u = 0; u < kItems; ++u) {
            it[u] = FlatItem{plive && s + u < edeg, pql, erb + s + u, ecv};
            src[u] = psrc;
          }
          step(it, src, false);
        }
      }
    } else {
      const u32 work = static_cast<u32>(__popc(m)) * deg;
      u32 incl = work;
      for (u32 o = 1; o < 32u; o <<= 1) {
        const u32 y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
      }
      const u32 excl = incl - work;
      const u32 total = __shfl_sync(0xFFFFFFFFu, incl, 31);
      for (u32 base = 0; base < total; base += 32u * kItems) {
        FlatItem it[kItems];
        u32 src[kItems];
  #pragma unroll
        for (u32 u = 0; u < kItems; ++u) {
          it[u] = flat_decode(base + 32u * u + lane, total, incl, excl, cv, m, rb, deg, p.edge_major != 0u);
          src[u] = dev::kInfBits;
        }
        step(it, src, true);
      }
    }
  };
  if (kChunked) {
    // Pack: lane j < pack holds slot j's chunk (kNoChunk: none).
    const u32 K = pack;
    const u32 nchunks = chunk_count(B.U, 5u);
    const u32 s0 = item * K;
    u32 my_chunk = kNoChunk;
    if (lane < K) {
      const u32 s = s0 + lane;
      if (dense) {
        if (s < nchunks && ((dev::ld_cg(B.cmask_r + (s >> 5)) >> (s & 31u)) & 1u) != 0u) my_chunk = s;
      } else if (s < count) {
        my_chunk = static_cast<u32>(dev::ld_cg(B.queue_r + s));
        if (my_chunk >= nchunks) {
          atomicOr(&C.error_bits, static_cast<u32>(BFX_DEVICE_ERROR_INVALID_CONTROLLER_STATE));
          my_chunk = kNoChunk;
        }
      }
    }
    u32 rest = __ballot_sync(0xFFFFFFFFu, my_chunk != kNoChunk);
    if (rest == 0u) return;  // warp-uniform: no slot of the pack is pending
    // the read slot's chunk bits are cleared for the round after next (a
    // dense pack's slots share one bitmap word: K divides 32)
    if (dense) {
      if (lane == 0u) atomicAnd(B.cmask_r + (s0 >> 5), ~(rest << (s0 & 31u)));
    } else if (my_chunk != kNoChunk) {
      atomicAnd(B.cmask_r + (my_chunk >> 5), ~(1u << (my_chunk & 31u)));
    }
    // One chunk's pending lanes and rows per thread (vertex 32 c + lane).
    auto load_chunk = [&](u32 j, u32& ccv, u32& cm, uint2& crow) {
      const u32 chunk = __shfl_sync(0xFFFFFFFFu, my_chunk, static_cast<int>(j));
      ccv = (chunk << 5) + lane;
      cm = 0u;
      crow = make_uint2(0u, 0u);
      if (ccv < B.U) {
        cm = dev::ld_cg(B.mask_r + ccv) & B.valid;
        crow = __ldg(B.crow + ccv);
      }
    };
    uint4* const ring = s_pack[threadIdx.x >> 5];
    const u32 below = (1u << lane) - 1u;
    u32 head = 0u, held = 0u;  // ring: entries [head, head + held) wait for a group (warp-uniform)
    u32 ncv, nm;
    uint2 nrow;
    load_chunk(static_cast<u32>(__ffs(rest)) - 1u, ncv, nm, nrow);
    rest &= rest - 1u;
    bool loaded = true;  // ncv / nm / nrow hold a chunk not yet compacted
    for (;;) {
      while (loaded && held < 32u) {
        const u32 ccv = ncv, cm = nm;
        const uint2 crow = nrow;
        loaded = rest != 0u;
        if (loaded) {  // the next chunk's loads go out before this one is compacted
          load_chunk(static_cast<u32>(__ffs(rest)) - 1u, ncv, nm, nrow);
          rest &= rest - 1u;
        }
        const bool act = cm != 0u;
        if (act) {
          B.mask_r[ccv] = 0u;
          if (kCount) {
            wk.c[0] += 1;
            wk.c[1] += crow.y;
            wk.c[2] += __popc(cm);
          }
        }
        const u32 bal = __ballot_sync(0xFFFFFFFFu, act);
        if (act) ring[(head + held + static_cast<u32>(__popc(bal & below))) & 63u] = make_uint4(ccv, cm, crow.x, crow.y);
        held += static_cast<u32>(__popc(bal));
      }
      if (held == 0u) break;
      __syncwarp();
      const u32 take = min(held, 32u);
      uint4 e = make_uint4(0u, 0u, 0u, 0u);
      if (lane < take) e = ring[(head + lane) & 63u];
      __syncwarp();
      head += take;
      held -= take;
      relax_entries(e.x, e.y, e.z, e.w);
    }
  } else {
    const u32 entry = item * epi + lane;  // epi entries per item (a power of two <= 32)
    u32 cv = 0u, m = 0u, rb = 0u, deg = 0u;
    if (lane < epi && entry < count) {
      const u64 q = dev::ld_cg(B.queue_r + entry);
      const u32 v = static_cast<u32>(q);
      cv = static_cast<u32>(q >> 32);
      if (v < p.g.V && cv < B.U) {
        m = dev::ld_cg(B.mask_r + cv) & B.valid;
        rb = __ldg(p.g.csr_off + v);
        deg = __ldg(p.g.csr_off + v + 1u) - rb;
        B.mask_r[cv] = 0u;
      } else {
        atomicOr(&C.error_bits, static_cast<u32>(BFX_DEVICE_ERROR_INVALID_CONTROLLER_STATE));
        cv = 0u;
      }
      if (kCount) {
        wk.c[0] += 1;
        wk.c[1] += deg;
        wk.c[2] += __popc(m);
      }
    }
    relax_entries(cv, m, rb, deg);
  }
#pragma unroll
  for (u32 u = 0; u < kItems; ++u) {
    if (kCount && p_old[u] == 0u) wk.c[4] += 1;
    stage_push(st, kNear, p_old[u] == 0u, queue_word(p_v[u], p_cv[u]));
    stage_push(st, kFar, f_old[u] == 0u, queue_word(kChunked ? f_cv[u] : f_v[u], f_cv[u]));
  }
}
