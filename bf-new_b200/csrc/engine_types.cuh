// Shared declarations of the CUDA translation units: device records of the
// resident graph, batches and launch state, and the host-side resident
// graph / workspace objects behind the C ABI handles.
#pragma once

#include "bfx.h"
#include "bfx_internal.hpp"
#include "device_common.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

namespace bfx {

#define BFX_CUDA(call)                                                                          \
  do {                                                                                          \
    cudaError_t err_ = (call);                                                                  \
    if (err_ != cudaSuccess) {                                                                  \
      throw ::bfx::Error(err_ == cudaErrorMemoryAllocation ? BFX_ERR_OUT_OF_MEMORY : BFX_ERR_CUDA, \
                         std::string(#call) + ": " + cudaGetErrorString(err_));                \
    }                                                                                           \
  } while (0)

using dev::u32;
using dev::u64;

// ---------------------------------------------------------------------------
// Device structures
// ---------------------------------------------------------------------------

struct DGraph {
  u32 V, E, T, reserved;
  const u32* owner;    // [V]
  const u32* csr_off;  // [V+1]
  const uint4* csr;    // [E] {dst, weight bits, eid+1, dst tile}
  const u32* csc_off;  // [V+1]
  const uint4* csc;    // [E] {src, weight bits, eid+1, src tile}
  const u32* eid_src;  // [E] source vertex of each stable edge id
  const uint2* lrun;   // [V] own-tile run of each CSR row {first CSR index, count} (rows are sorted by
                       // destination tile, so a vertex's edges into its own tile are contiguous)
  const u32* tile_off; // [T+1] first vertex of each tile
};

struct DBatch {
  u32 W, shift, valid, U;
  u32 src_count, tgt_count, range_count;
  u32 full;            // every tile selected by every valid lane, compact index == vertex id
  u64* dist[2];        // [U*W] labels (slot 1 only for Jacobi)
  u32* mask[2];        // [U] pending lane masks (frontier)
  u64* queue[2];       // [U] frontier entries {vertex, compact index << 32}, or chunk ids (chunked layout)
  u32* c2g;            // [U] compact -> global vertex
  uint2* tiles;        // [T] {lane mask, compact bias}
  const u32* src_off;  // [W+1]
  const u32* src;
  const u32* tgt_off;  // [W+1]
  const u32* tgt;
  const uint4* ranges;    // [R] {tile, begin, end, lane mask}
  const u32* range_off;   // [R+1] compact offsets
  u32* fmask;             // [U] far lanes (near/far frontier)
  u32* fbound;            // [U] lower bound of the vertex's parked labels (float bits; 0xffffffff: none)
  u64* fpile[3];          // [U] far piles {vertex, compact index << 32}, rotating by far generation
                          // (chunked layout: the vertex field holds the compact index)
  u32* cmask[2];          // [ceil(U/1024)] chunk bitmaps (chunked frontier): bit c = chunk c pending
  uint2* crow;            // [U] {CSR row begin, out-degree} per compact vertex (chunked frontier)
  uint2* clrun;           // [U] own-tile run {first CSR index, count} per compact vertex (tiled frontier)
};

struct DCtl {
  u32 count[3];    // frontier sizes, rotating by round
  u32 changed[3];  // Jacobi/dense: lanes whose distance changed, rotating
  u32 rounds;      // rounds executed with work
  u32 missing;     // finalize: lanes with an unreached target
  u32 active;      // finalize: lanes still pending at the stop
  u32 error_bits;
  // Near/far frontier: far pile sizes by generation % 3; generation and
  // threshold (float bits) double-buffered by round parity.
  u32 fcount[3];
  u32 fmin[3];     // smallest parked distance per far pile (float bits)
  u32 gen[2];
  u32 tau[2];
  u32 delta;       // threshold step (float bits); +inf = plain frontier
};

// Threshold of the split that consumes far pile `pile`: tau + delta, raised
// above the pile's smallest parked distance so every split moves at least
// one (vertex, lane) to the near frontier (progress even when tau + delta
// rounds back to tau).
__device__ __forceinline__ u32 split_threshold(const DCtl& C, u32 tau, u32 pile) {
  const u32 stepped = __float_as_uint(__fadd_rn(__uint_as_float(tau), __uint_as_float(C.delta)));
  const u32 fmin = C.fmin[pile];
  const u32 above = fmin >= 0x7F800000u ? fmin : fmin + 1u;  // next float above fmin
  return stepped > above ? stepped : above;
}

struct DRun {
  dev::GridSync sync;
  u32 round;       // next round (host-poll modes)
  u32 done;        // all batches stopped
  u32 stop;        // launch-wide stop reason
  u32 abort;       // device failure seen
  u64 max_rounds;
  u64 launches;
  u64 work[16];    // launch-wide work counters: [0..6] push engines, [7] rounds, [8..11] Jacobi, [12..13] splits,
                   // [14..15] tiled visits (lane-edge relaxations inside shared memory, staged visits)
  u32 items[3];    // tiled layout: block items drawn in round r from items[r % 3] (cleared two rounds ahead)
  u32 reserved[5];
};

// Work counters of an instrumented run (instrumentation >= 1):
// 0 queue entries processed, 1 edge records read, 2 active (vertex, lane)
// source reads, 3 lane-edge relaxations, 4 queue claims, 5 distance
// decreases, 6 min-reductions issued, 7 rounds executed.
// Per-thread work counters of an instrumented run: c[0..6] frontier and
// dense push (entries / vertex items, edge records, source reads, lane-edge
// relaxations, queue claims, decreases, min-reductions), c[7..10] Jacobi
// pull (vertex-lane items, in-edge records, relaxations, changes), c[11..12]
// near/far split rounds (far pile entries scanned, parked lanes re-read),
// c[13..14] tiled visits (lane-edge relaxations in shared memory, visits
// that staged their labels).
constexpr int kWorkCounters = 15;
struct Work {
  u64 c[kWorkCounters];
  __device__ void zero() {
    for (int i = 0; i < kWorkCounters; ++i) c[i] = 0;
  }
};

constexpr u32 kMaxBatchesPerLaunch = 4096;
constexpr u64 kBarrierTimeoutNs = 2000000000ull;  // 2 s per barrier wait
constexpr u64 kLaunchBudgetNs = 30000000000ull;   // 30 s per relaxation launch

struct LaunchParams {
  DGraph g;
  const DBatch* batches;
  DCtl* ctl;
  DRun* run;
  const u32* unit_base;  // [nb+1] prefix of U (init / finalize)
  u32 nb;
  u32 engine;            // engine of every batch when `engines` is null
  u32 per_lane;
  u32 flat;              // frontier layout: 0 sub-warp groups, 1 flat work list, 2 chunked flat work list,
                         // 3 tiled (a block visits 2^cshift compact vertices with their labels in shared memory)
  u64 max_rounds;
  u64 budget_ns;         // wall-clock budget of one relaxation launch; past it the launch stops (device_failure)
  const u32* engines;    // [nb] per-batch engine (autotuned launches) or null
  const u32* deltas;     // [nb] near/far threshold steps (float bits) or null (plain frontier)
  u64* round_trace;      // instrumentation 2: per round {start %globaltimer, warp items | split batches << 32,
                         // active pairs, lane-edge relaxations}; null otherwise
  u32 trace_cap;         // rounds the trace holds
  u32 amin;              // flat frontier: 1 = returning min per relaxation, 0 = pre-read + min on success
  u32 edge_major;        // flat frontier work order: 1 = entry, edge, lane; 0 = entry, lane, edge
  u32 cshift;            // chunked / tiled layouts: a claim unit is 2^cshift consecutive compact vertices
                         // (5: 32-vertex chunks)
  u32 cpack;             // chunked / tiled layouts: chunk slots per warp item (1, 2, 4 or 8)
  u32 tile_stage_min;    // tiled layout: lane-edge work below which a block visit relaxes in place (no staging)
  u32 tile_wmax;         // tiled layout: widest batch of the launch (sizes the staged label rows)
  u32 tile_iters;        // tiled layout: local relaxation passes per visit before the rest waits a round
  u32 tshift;            // tiled layout: a dense round visits units of 2^tshift compact vertices (the tile size)
  const u32* mappings;   // tiled layout, [nb] or null (every batch visits tiles): BFX_MAPPING_* per batch
};

constexpr u32 kRoundTraceCap = 65536;

__device__ __forceinline__ u32 engine_of(const LaunchParams& p, u32 b) {
  return p.engines ? p.engines[b] : p.engine;
}

// Host side
// ---------------------------------------------------------------------------

inline size_t align256(size_t x) { return (x + 255) & ~size_t{255}; }

struct DeviceBuffer {
  void* ptr{nullptr};
  size_t bytes{0};
  int device{0};
  DeviceBuffer() = default;
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  ~DeviceBuffer() { release(); }
  void release() {
    if (ptr) {
      cudaSetDevice(device);
      cudaFree(ptr);
    }
    ptr = nullptr;
    bytes = 0;
  }
  // Grows geometrically; contents are not preserved.
  void reserve(size_t need, int dev) {
    if (need <= bytes && ptr) return;
    release();
    device = dev;
    size_t cap = std::max(need, bytes + bytes / 2);
    cap = (cap + 255) & ~size_t{255};
    BFX_CUDA(cudaMalloc(&ptr, cap));
    bytes = cap;
  }
};

struct PinnedBuffer {
  void* ptr{nullptr};
  size_t bytes{0};
  PinnedBuffer() = default;
  PinnedBuffer(const PinnedBuffer&) = delete;
  PinnedBuffer& operator=(const PinnedBuffer&) = delete;
  ~PinnedBuffer() {
    if (ptr) cudaFreeHost(ptr);
  }
  void reserve(size_t need) {
    if (need <= bytes && ptr) return;
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    size_t cap = std::max(need, bytes + bytes / 2);
    cap = (cap + 255) & ~size_t{255};
    BFX_CUDA(cudaHostAlloc(&ptr, cap, cudaHostAllocDefault));
    bytes = cap;
  }
};

}  // namespace bfx

struct bfx_resident_graph {
  int device{0};
  bfx::DGraph g{};
  bfx::DeviceBuffer mem;
  std::vector<std::uint32_t> tile_vertex_offsets;  // host copy, [T+1]
  std::uint64_t bytes{0};
  double mean_weight{0.0};
  // Tiled frontier claim unit: log2 of the tile size when every tile holds
  // the same power-of-two count of vertices in [32, 256], else 8 (units then
  // straddle tiles, which costs locality but not correctness); at least 5.
  std::uint32_t tile_shift{8};
};

struct bfx_workspace {
  bfx_resident_graph* graph{nullptr};
  cudaStream_t stream{nullptr};
  int sm_count{0};
  // Prepared batch set.
  std::uint32_t nb{0};
  std::uint64_t src_total{0};
  std::vector<bfx::DBatch> batches;
  bfx::DeviceBuffer meta;   // DBatch[], DCtl[], DRun, unit_base, src_base, uploaded descriptions
  bfx::DeviceBuffer arena;  // labels, masks, queues, c2g, row tables
  bfx::DeviceBuffer tile_tables;  // per batch dense {lane mask, compact bias} over all tiles
  bfx::DeviceBuffer qimage;       // device-side preparation: the uploaded query and lane image
  bfx::PinnedBuffer staging;
  bfx::PinnedBuffer status_host;
  size_t meta_bytes{0};
  size_t arena_bytes{0};
  bool needs_slot2{false};
  bfx::LaunchParams params{};
  bfx::u32* src_base{nullptr};
  bfx_device_run_status* d_status{nullptr};
  bfx_device_controller* d_ctrl{nullptr};
  std::uint64_t last_launches{0};
  std::uint64_t last_host_checks{0};
  std::uint64_t last_h2d{0}, last_d2h{0};
  cudaEvent_t ev[4]{};  // execute start, relaxation start, relaxation end, execute end
  bool executed{false};
  // Host-poll graph cache, keyed by the exact launch parameters.
  cudaGraphExec_t chunk_exec{nullptr};
  std::uint32_t chunk_rounds{0};
  int chunk_grid{0};
  int chunk_block{0};
  std::uint32_t chunk_instr{0};
  bfx::LaunchParams chunk_params{};
  std::uint64_t generation{0};
  // Compact path reconstruction state (summaries pass -> payload pass).
  bfx::DeviceBuffer paths;       // summaries, offsets, flags, search scratch
  bfx::PinnedBuffer paths_host;
  std::uint32_t path_first_batch{0};
  std::uint32_t path_batch_count{0};
  std::uint64_t path_targets{0};
  std::uint64_t path_vertices{0};  // payload sizes after the summaries pass
  std::uint64_t path_edges{0};
  bool paths_ready{false};
  bfx::DeviceBuffer adjoint;     // per-edge exact accumulators, upstream values, result
  std::vector<std::uint32_t> batch_engines;  // per-batch engine for BFX_ENGINE_AUTO launches
  std::vector<float> batch_deltas;           // per-batch near/far steps (empty: plain frontier)
  std::vector<std::uint32_t> batch_mappings; // tiled layout: per-batch dense-round mapping (empty: tile visits)
  bfx::DeviceBuffer mappings_dev;
  std::uint32_t frontier_layout = 2;         // BFX_FRONTIER_CHUNKED (default) / _FLAT / _GROUPS
  std::uint32_t relax_atomic = 0;            // flat frontier relaxation: 0 pre-read + min, 1 returning min
  std::uint32_t edge_major = 0;              // flat frontier work order (see bfx_set_flat_order)
  std::uint32_t chunk_pairs = 0;             // chunked frontier pair mode (see bfx_set_chunk_pairs)
  std::uint32_t chunk_pack = 4;              // chunk slots per warp item (see bfx_set_chunk_pack)
  std::uint32_t flat_items = 2;              // flat layout: work items per thread per iteration (2..4)
  std::uint32_t register_budget = 0;         // persistent kernel registers per thread: 0 automatic, 40, 64, 80
  std::uint32_t tile_stage_min = 1024;       // tiled layout: lane-edge work from which a visit stages its labels
  std::uint32_t tile_iters = 32;             // tiled layout: local passes per visit
  bfx::DeviceBuffer deltas_dev;
  bfx::DeviceBuffer engines_dev;
  std::vector<std::uint32_t> deltas_uploaded, engines_uploaded, mappings_uploaded;  // contents of the *_dev arrays
  bfx::DeviceBuffer round_trace;  // instrumentation 2 only
};

