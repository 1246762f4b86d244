// Device-side building blocks shared by the relaxation engines: packed
// (distance | predecessor) words, coherent loads, the non-returning 64-bit
// min reduction, and a grid barrier whose waits are bounded in time.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace bfx::dev {

using u32 = std::uint32_t;
using u64 = std::uint64_t;

// A label is one 64-bit word: high half = distance (float bits of a
// non-negative float, whose unsigned order equals float order on
// {+0, finite >= 0, +inf}, src/hip/batched_frontier_push.hip.cpp:377-394);
// low half = 1 + stable EdgeId of the predecessor edge.  A source holds
// (0, 0), which no candidate can undercut; an unreached label holds
// (+inf, 0xffffffff).  One unsigned 64-bit min therefore keeps the smallest
// distance and, among equal distances, the smallest stable edge id -- the
// first tight candidate the reference's reconstruction picks
// (src/path_reconstruct.cpp:56-89, src/compact_paths.cpp:98-129).
constexpr u32 kInfBits = 0x7F800000u;
constexpr u64 kUnreached = (static_cast<u64>(kInfBits) << 32) | 0xFFFFFFFFull;
constexpr u64 kSourceWord = 0ull;

__device__ __forceinline__ u32 hi(u64 w) { return static_cast<u32>(w >> 32); }

__device__ __forceinline__ u64 ld_cg(const u64* p) { return __ldcg(reinterpret_cast<const unsigned long long*>(p)); }
__device__ __forceinline__ u32 ld_cg(const u32* p) { return __ldcg(p); }

__device__ __forceinline__ void red_min_u32(u32* p, u32 v) {
  asm volatile("red.relaxed.gpu.global.min.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ u32 ld_acquire_gpu(const u32* p) {
  u32 v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void red_min(u64* p, u64 v) {
  asm volatile("red.relaxed.gpu.global.min.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ void red_or(u32* p, u32 v) {
  asm volatile("red.relaxed.gpu.global.or.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Returning 64-bit min at L2: the label before the reduction.
__device__ __forceinline__ u64 atom_min(u64* p, u64 v) {
  u64 old;
  asm volatile("atom.relaxed.gpu.global.min.u64 %0, [%1], %2;" : "=l"(old) : "l"(p), "l"(v) : "memory");
  return old;
}

__device__ __forceinline__ u64 global_ns() {
  u64 t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Candidate label for a relaxation: distance d_src + w rounded to nearest
// (explicit __fadd_rn so no contraction can change a bit), predecessor eid.
__device__ __forceinline__ u64 candidate(u32 src_bits, u32 w_bits, u32 eid_plus_one) {
  const float c = __fadd_rn(__uint_as_float(src_bits), __uint_as_float(w_bits));
  return (static_cast<u64>(__float_as_uint(c)) << 32) | eid_plus_one;
}

struct GridSync {
  u32 arrive;
  u32 generation;
  u32 abort;
  u32 reserved;
};

// Sense-by-generation grid barrier for a cooperatively launched grid.  Every
// wait gives up after `timeout_ns` (or as soon as another block has given
// up): the block then raises `abort` and the caller leaves its loop, so no
// launch can spin forever.
__device__ __forceinline__ bool grid_barrier(GridSync* gs, u32 nblocks, u64 timeout_ns) {
  __shared__ u32 s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    u32 ok = 1;
    const u32 gen = ld_acquire_gpu(&gs->generation);
    __threadfence();
    const u32 ticket = atomicAdd(&gs->arrive, 1u);
    if (ticket == nblocks - 1u) {
      atomicExch(&gs->arrive, 0u);
      __threadfence();
      atomicAdd(&gs->generation, 1u);
    } else {
      const u64 t0 = global_ns();
      while (ld_acquire_gpu(&gs->generation) == gen) {
        if (ld_acquire_gpu(&gs->abort) != 0u) {
          ok = 0;
          break;
        }
        if (global_ns() - t0 > timeout_ns) {
          atomicExch(&gs->abort, 1u);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    if (ld_acquire_gpu(&gs->abort) != 0u) ok = 0;
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0u;
}

}  // namespace bfx::dev
