/*
 * bfx — batched regional shortest paths on NVIDIA B200 (sm_100a).
 *
 * C ABI of the product library libbfx.so.  Every entry point returns an int
 * status (BFX_OK == 0) and never throws; bfx_last_error() gives the calling
 * thread's last message.  All structs are plain data with fixed layouts; no
 * C++ or torch types cross this boundary.
 *
 * The functions replace the batched relaxation path of the reference engine
 * (amber-bajaj-1/bf-new).  Each declaration names the reference interface it
 * stands in for (file:line in the reference repository).
 */
#ifndef BFX_H
#define BFX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BFX_ABI_VERSION 1

/* Status codes (host errors).  Device-side failures are reported through
 * bfx_device_run_status.error_bits / stop_reason as in the reference. */
enum {
  BFX_OK = 0,
  BFX_ERR_INVALID_ARGUMENT = 1, /* reference: std::invalid_argument */
  BFX_ERR_OUT_OF_RANGE = 2,     /* reference: std::out_of_range */
  BFX_ERR_OVERFLOW = 3,         /* reference: std::overflow_error / length_error */
  BFX_ERR_CUDA = 4,             /* reference: HipRuntimeError (hip/runtime.hpp:22-35) */
  BFX_ERR_NO_DEVICE = 5,
  BFX_ERR_STATE = 6,            /* reference: std::logic_error */
  BFX_ERR_OUT_OF_MEMORY = 7
};

/* Engine, control and stop enums: same values as include/bfnew/gpu_api.hpp:14-55. */
enum { BFX_ENGINE_JACOBI_PULL = 0, BFX_ENGINE_DENSE_CHAOTIC_PUSH = 1, BFX_ENGINE_FRONTIER_PUSH = 2,
       BFX_ENGINE_AUTO = 0xFFFFFFFFu /* bfx extension: the autotuner picks per batch */ };
enum { BFX_CONTROL_PERSISTENT_COOPERATIVE = 0, BFX_CONTROL_CHUNKED_HOST_POLL = 1,
       BFX_CONTROL_PER_ROUND_HOST_POLL = 2 };
enum { BFX_STOP_NONE = 0, BFX_STOP_CONVERGED = 1, BFX_STOP_MAXIMUM_ROUNDS = 2,
       BFX_STOP_QUEUE_OVERFLOW = 3, BFX_STOP_INVALID_CONTROLLER_STATE = 4,
       BFX_STOP_DEVICE_FAILURE = 5 };
enum { BFX_DEVICE_ERROR_QUEUE_OVERFLOW = 1u, BFX_DEVICE_ERROR_INVALID_CONTROLLER_STATE = 2u,
       BFX_DEVICE_ERROR_DEVICE_FAILURE = 4u };

/* Mirrors bfnew::GpuRunOptions (include/bfnew/gpu_api.hpp:57-67), 48 bytes,
 * validated like validate_gpu_run_options (src/gpu_api.cpp:71-105). */
typedef struct bfx_gpu_run_options {
  uint32_t engine;
  uint32_t control_mode;
  uint32_t rounds_per_chunk;
  uint32_t block_size;
  uint32_t grid_policy;      /* 0 occupancy-derived, 1 fixed blocks per SM */
  uint32_t blocks_per_wgp;   /* blocks per SM when grid_policy == 1 */
  uint32_t instrumentation;  /* 0 none, 1 light, 2 debug */
  uint32_t reserved0;
  uint64_t maximum_rounds;
  uint32_t enable_per_lane_convergence;
  uint32_t reserved1;
} bfx_gpu_run_options;

/* Mirrors bfnew::DeviceController (gpu_api.hpp:100-120), 96 bytes. */
typedef struct bfx_device_controller {
  uint32_t valid_lane_mask, active_lane_mask, changed_lane_mask, converged_lane_mask;
  uint32_t execute_lane_mask, engine_kind, enable_per_lane_convergence, reserved0;
  uint64_t rounds_completed, maximum_rounds;
  uint32_t distance_read_slot, distance_write_slot, frontier_read_slot, frontier_write_slot;
  uint64_t frontier_size[2];
  uint32_t next_frontier_lane_mask, done, stop_reason, error_bits;
} bfx_device_controller;

/* Mirrors bfnew::DeviceRunStatus (gpu_api.hpp:176-187), 48 bytes. */
typedef struct bfx_device_run_status {
  uint32_t final_distance_slot;
  uint32_t converged;
  uint64_t rounds_completed;
  uint32_t reached_target_mask;
  uint32_t bounding_box_miss_mask;
  uint32_t valid_lane_mask;
  uint32_t active_lane_mask;
  uint32_t converged_lane_mask;
  uint32_t stop_reason;
  uint32_t error_bits;
  uint32_t reserved0;
} bfx_device_run_status;

/* Mirrors bfnew::DeviceWorkStatistics (gpu_api.hpp:122-150), 168 bytes. */
typedef struct bfx_device_work_statistics {
  uint64_t edges_examined, successful_decreases, active_vertices, active_lane_rounds;
  uint64_t maximum_queue_size, host_checks, host_synchronizations, controller_copies;
  uint64_t kernel_dispatches, expansion_count, atomic_attempts, successful_atomic_updates;
  uint64_t queue_claims, duplicate_suppressions, mask_operations, overflow_events;
  uint64_t high_contention_destinations, changed_flag_updates, full_edge_rounds;
  uint64_t empty_frontier_rounds, small_frontier_rounds;
} bfx_device_work_statistics;

/* Flattened bfnew::DeviceGraphLayout32 (include/bfnew/device_layout.hpp:72-93)
 * plus csr_edge_ids, the stable EdgeId of every CSR position
 * (WeightedGraph::outgoing().edge_ids); NULL derives it from the CSC image.
 * Host pointers. */
typedef struct bfx_device_graph_layout32 {
  uint32_t vertex_count, edge_count, tile_count, csr_run_count, csc_run_count, reserved0;
  const uint32_t *owner_tiles;                /* [V] */
  const uint32_t *csr_row_offsets;            /* [V+1] */
  const uint32_t *csr_destinations;           /* [E] */
  const float *csr_weights;                   /* [E] */
  const uint32_t *csr_row_run_offsets;        /* [V+1] */
  const uint32_t *csr_run_edge_offsets;       /* [csr_run_count+1] */
  const uint32_t *csr_run_destination_tiles;  /* [csr_run_count] */
  const uint32_t *csc_column_offsets;         /* [V+1] */
  const uint32_t *csc_sources;                /* [E] */
  const float *csc_weights;                   /* [E] */
  const uint32_t *csc_edge_ids;               /* [E] */
  const uint32_t *csc_column_run_offsets;     /* [V+1] */
  const uint32_t *csc_run_edge_offsets;       /* [csc_run_count+1] */
  const uint32_t *csc_run_source_tiles;       /* [csc_run_count] */
  const uint32_t *csr_edge_ids;               /* [E] or NULL */
} bfx_device_graph_layout32;

/* bfnew::BatchVertexRange (batch_layout.hpp:23-29), 12 bytes. */
typedef struct bfx_batch_vertex_range {
  uint32_t begin, end, lane_mask;
} bfx_batch_vertex_range;

/* Flattened bfnew::BatchDeviceDescription (batch_layout.hpp:73-120), the
 * device-materialized-run-mask representation.  Host pointers. */
typedef struct bfx_batch_description {
  uint32_t lane_width;       /* 1, 8, 16 or 32 */
  uint32_t valid_lane_mask;
  const uint32_t *source_offsets;  /* [lane_width+1] */
  const uint32_t *sources;         /* [source_offsets[lane_width]] global vertex ids */
  const uint32_t *target_offsets;  /* [lane_width+1] */
  const uint32_t *targets;
  uint32_t union_tile_count;
  uint32_t tile_count;             /* == graph tile_count */
  const uint32_t *union_tiles;     /* [union_tile_count], strictly increasing */
  const uint32_t *tile_lane_masks; /* [tile_count] dense lane mask per tile */
  uint32_t range_count;
  uint32_t reserved0;
  const bfx_batch_vertex_range *selected_vertex_ranges; /* one per union tile */
} bfx_batch_description;

typedef struct bfx_resident_graph bfx_resident_graph;
typedef struct bfx_workspace bfx_workspace;

/* ---- library ---------------------------------------------------------- */
int bfx_abi_version(void);
const char *bfx_last_error(void);
/* Number of CUDA devices visible; 0 without a GPU (never an error). */
int bfx_device_count(int *count);

/* ---- resident graph ----------------------------------------------------
 * Replaces bfnew::hip::ResidentDeviceGraph::upload_once_async
 * (include/bfnew/hip/runtime.hpp:238-270) and its content fingerprint guard.
 * Uploads the checked 32-bit image once; the graph is immutable afterwards. */
int bfx_resident_graph_upload(const bfx_device_graph_layout32 *layout, int device,
                              bfx_resident_graph **out);
int bfx_resident_graph_destroy(bfx_resident_graph *graph);
/* Counts {V, E, T, device bytes}. */
int bfx_resident_graph_info(const bfx_resident_graph *graph, uint64_t out[4]);

/* ---- workspace -----------------------------------------------------------
 * Replaces bfnew::hip::ReusableBatched{Frontier,Jacobi,Dense}Workspace
 * (include/bfnew/hip/batched_frontier_workspace.hpp:28-80): device buffers for
 * terminals, tile tables, labels, activity masks, queues, controllers and
 * statuses, grown geometrically and reused across calls.  A workspace binds
 * one graph and one CUDA stream; calls on it must be sequential. */
int bfx_workspace_create(bfx_resident_graph *graph, bfx_workspace **out);
int bfx_workspace_destroy(bfx_workspace *ws);
/* The workspace's cudaStream_t (as void*), for event timing by callers. */
int bfx_workspace_stream(bfx_workspace *ws, void **stream);
/* Device bytes currently reserved by the workspace. */
int bfx_workspace_bytes(bfx_workspace *ws, uint64_t *bytes);

/* ---- batched execution ---------------------------------------------------
 * bfx_prepare_batches + bfx_execute + bfx_fetch_statuses together replace
 * BatchedFrontierPushEngine::run_compact_status (hip/batched_frontier_push.hpp:
 * 105-116) and its Jacobi / dense twins (hip/batched_jacobi.hpp:137-200,
 * hip/batched_dense_chaotic_push.hpp:105-165), generalised to several batches
 * in one launch.  options->engine selects the relaxation engine for every
 * batch (BFX_ENGINE_AUTO: the autotuner picks per batch). */

/* Validates and uploads `count` batch descriptions (host memory) into the
 * workspace (one H2D transfer).  Replaces workspace.prepare_async
 * (src/hip/batched_frontier_workspace.hip.cpp:178). */
int bfx_prepare_batches(bfx_workspace *ws, uint32_t count, const bfx_batch_description *batches);
/* Runs the prepared batches to convergence (or the round limit) on the
 * workspace stream.  Asynchronous in persistent mode: returns after enqueue.
 * Host-poll modes poll the device controller as the reference does. */
int bfx_execute(bfx_workspace *ws, const bfx_gpu_run_options *options);
/* Synchronises the stream and copies one status (and optionally the final
 * controller image) per prepared batch to host memory. */
int bfx_fetch_statuses(bfx_workspace *ws, bfx_device_run_status *statuses,
                       bfx_device_controller *controllers);
/* All three in sequence: the one call a user makes. */
int bfx_run_batches(bfx_workspace *ws, uint32_t count, const bfx_batch_description *batches,
                    const bfx_gpu_run_options *options, bfx_device_run_status *statuses);

/* Downloads batch `batch`'s final labels as a graph-sized V*W image (vertex-
 * major, contiguous lanes; +inf bits / 0xffffffff outside the lane's selected
 * tiles).  distance_bits: float bit patterns; predecessor_edges: stable EdgeId
 * of the chosen tight in-edge, 0xffffffff for sources and unreached vertices.
 * Either output may be NULL.  Replaces run_with_distances
 * (hip/batched_frontier_push.hpp:122-124). */
int bfx_download_labels(bfx_workspace *ws, uint32_t batch, uint32_t *distance_bits,
                        uint32_t *predecessor_edges);

/* One lane of batch `batch` as a graph-sized V image, same encoding as
 * bfx_download_labels (bfx extension: a width-32 batch over a 16.8M-vertex
 * graph is 4.3 GB whole, so checkers fetch the lanes they compare).  Lanes
 * at or above the batch's width fail with BFX_ERR_OUT_OF_RANGE. */
int bfx_download_lane_labels(bfx_workspace *ws, uint32_t batch, uint32_t lane, uint32_t *distance_bits,
                             uint32_t *predecessor_edges);

/* Largest finite distance (float bits) among the final labels of every
 * prepared batch, one word per batch; 0 when a batch reached nothing but
 * its sources (bfx extension).  Integer costs stay exact in float sums only
 * while every distance is below 2^24 (bits 0x4B800000): checkers of integer-
 * cost workloads assert that bound with this. */
int bfx_fetch_label_bounds(bfx_workspace *ws, uint32_t *max_finite_distance_bits);

/* Device time of the most recent bfx_execute, measured by CUDA events the
 * library records on the workspace stream: out[0] = relaxation kernels
 * (the persistent launch, or all round/advance launches of a host-poll run),
 * out[1] = the whole execute (init, seed, relaxation, finalize), in ms. */
int bfx_last_execute_timing(bfx_workspace *ws, float out[2]);
/* Bytes moved by the most recent bfx_prepare_batches (H2D) and
 * bfx_fetch_statuses (D2H). */
int bfx_workspace_transfer_bytes(bfx_workspace *ws, uint64_t out[2]);

/* ---- compact paths ---------------------------------------------------------
 * Replace ReusableCompactPathWorkspace::reconstruct / run_compact_paths
 * (include/bfnew/hip/compact_path_results.hpp:99-127,
 * hip/batched_frontier_push.hpp:118-121).  Per target of batches
 * [first_batch, first_batch + batch_count) of the last execute, in
 * description order: a summary mirroring bfnew::CompactTargetSummary
 * (include/bfnew/compact_path_types.hpp:31-47, 28 bytes; reached 0/1;
 * reconstruction 0 complete, 1 unreachable, 2 query terminal failure (the
 * lane's run did not converge cleanly), 3 no tight path).  Paths follow the
 * reference's deterministic tight-edge search (src/compact_paths.cpp:131-211).
 * sizes (may be NULL) = {targets, payload vertices, payload edges}. */
typedef struct bfx_compact_target_summary {
  uint32_t target;
  uint32_t selected_source;
  float distance;
  uint32_t path_length;
  uint32_t reached;
  uint32_t reconstruction;
  uint32_t has_selected_source;
} bfx_compact_target_summary;

int bfx_compact_path_summaries(bfx_workspace *ws, uint32_t first_batch, uint32_t batch_count,
                               bfx_compact_target_summary *summaries, uint64_t sizes[3]);
/* Second pass: complete targets' paths concatenated in summary order; per
 * target path_length + 1 vertices (source first) with their final labels and
 * path_length stable edge ids. */
int bfx_compact_path_payload(bfx_workspace *ws, uint32_t *vertices, float *distance_labels, uint32_t *edge_ids);

/* ---- edge-usage adjoint ------------------------------------------------------
 * No counterpart in the reference (a new differentiable interface).  For
 * L = sum_t g_t * dist_t over the targets of the last
 * bfx_compact_path_summaries call (g in its summary order), writes
 * edge_grads[e] = dL/dw_e = sum of g_t over the targets whose path uses the
 * edge with stable id e (E entries).  Paths are recomputed from the final
 * labels (no per-round state is kept); contributions are summed exactly and
 * rounded once to float, so the result is independent of thread order.
 * Accepted g: 0 or magnitude in [2^-40, 2^40); targets that are not
 * complete (unreachable, failed lanes) contribute nothing. */
int bfx_edge_usage_adjoint(bfx_workspace *ws, const float *target_grads, float *edge_grads);
/* Replaces every edge weight of the resident graph; weights_by_edge_id[E] is
 * indexed by stable edge id, finite and non-negative (-0 becomes +0). */
int bfx_resident_graph_set_weights(bfx_resident_graph *graph, const float *weights_by_edge_id);

/* ---- engine autotuner ----------------------------------------------------------
 * No counterpart in the reference (its engine shootout, src/engine_shootout.cpp,
 * only catalogues configurations).  Picks the near/far step of frontier push
 * (plain, or 1/2, 1, 2, 4, 8, 32 or 128 mean edge weights) by timing the whole set
 * in one launch, then per batch shape Jacobi pull or dense chaotic push where
 * it is at least 1.5x faster on the batch alone (cached per lane width, valid
 * lanes, magnitude of union vertices and tiles), and keeps those engines only
 * if the whole set runs faster with them (best of `trials` device timings
 * each).  Then the work mapping, when the workspace is in the chunked or the
 * tiled frontier layout with persistent control and blocks of 256 or 384
 * threads: the other of the two layouts is timed on the whole set and kept
 * if faster (the workspace's layout may change), and under the tiled layout
 * each batch shape's dense rounds are mapped to tile visits or chunk-slot
 * warp items (timed alone, visits where 1.1x faster, cached per shape), the
 * per-batch mix kept only if the whole set runs faster (bfx_get_frontier_mapping
 * reports the outcome); last, 2, 4 and 8 chunk slots per warp item are timed
 * on the whole set and the fastest kept (bfx_get_chunk_pack reports it).  The
 * step, layout and pack are cached per set class (graph, magnitudes of the
 * batch counts per lane width and of the union size) and reused for a later
 * set of the class.  Leaves the workspace prepared with all `count`
 * batches and their engines, steps and mappings, so bfx_execute with
 * options->engine == BFX_ENGINE_AUTO relaxes each batch with its own engine
 * in one launch.  engines_out[count]; deltas_out[count] (may be NULL) =
 * chosen steps (+inf = plain); *measured (may be NULL) = batches that were
 * timed rather than found in the cache. */
int bfx_autotune(bfx_workspace *ws, uint32_t count, const bfx_batch_description *batches,
                 const bfx_gpu_run_options *base, uint32_t trials, uint32_t *engines_out, float *deltas_out,
                 uint32_t *measured);
/* Forgets all cached autotuner choices. */
int bfx_autotune_reset(void);
/* Sets the per-batch engines used by BFX_ENGINE_AUTO launches of the prepared
 * batches (count must equal the prepared batch count at execute time). */
int bfx_set_batch_engines(bfx_workspace *ws, uint32_t count, const uint32_t *engines);
/* Near/far frontier (a bfx scheduling option, results unchanged): per-batch
 * threshold steps for frontier-push batches.  A frontier round relaxes only
 * improvements below the batch's current threshold and parks the others;
 * when nothing below it is left the threshold advances by the step and the
 * parked (vertex, lane) pairs now below it rejoin -- fewer redundant
 * relaxations than a plain frontier.  A split raises the threshold at least
 * above the smallest parked distance, so every split makes progress.  +inf
 * (or an empty set) = plain
 * frontier; steps must be positive.  count must equal the prepared batch
 * count at execute time. */
int bfx_set_batch_deltas(bfx_workspace *ws, uint32_t count, const float *deltas);
/* Frontier-push work layout (a bfx scheduling option, results unchanged):
 * BFX_FRONTIER_FLAT gives a warp 32 entries and walks their
 * (lane, out-edge) pairs as one flat work list, two items per thread per
 * step; BFX_FRONTIER_GROUPS gives each queue entry a sub-warp group of 8
 * threads (batches of <= 8 lanes) or a whole warp; BFX_FRONTIER_CHUNKED
 * (default) queues 32-vertex chunks instead of vertices (a chunk bitmap per round
 * slot, pending lanes set with non-returning ORs) and runs the flat work list
 * over each chunk's vertices in index (spatial) order; BFX_FRONTIER_TILED
 * queues whole tiles (blocks of the graph's tile size, 32..256 vertices) and
 * lets a thread block visit one at a time: it stages the tile's label rows in
 * shared memory, relaxes intra-tile edges there until no lane of the tile is
 * pending, pushes inter-tile edges through global memory and writes the
 * changed labels back (persistent control mode, blocks of 256 threads; the
 * host-poll modes run the chunked layout instead). */
enum { BFX_FRONTIER_GROUPS = 0, BFX_FRONTIER_FLAT = 1, BFX_FRONTIER_CHUNKED = 2, BFX_FRONTIER_TILED = 3 };
int bfx_set_frontier_layout(bfx_workspace *ws, uint32_t layout);
/* Tiled layout: a tile visit whose pending lane-edge work is below
 * `lane_edges` relaxes in global memory without staging its labels (bfx
 * extension; results unchanged; default 1024). */
int bfx_set_tile_stage_min(bfx_workspace *ws, uint32_t lane_edges);
/* Tiled layout: local relaxation passes per staged tile visit (1..1024,
 * default 32); lanes still pending after them are relaxed in the next round
 * (bfx extension; results unchanged). */
int bfx_set_tile_passes(bfx_workspace *ws, uint32_t passes);
/* Tiled layout, per batch (bfx extension; results unchanged): dense rounds
 * as tile visits (BFX_MAPPING_TILE_VISITS, the default) or as chunk-slot
 * warp items like the chunked layout (BFX_MAPPING_CHUNKS).  count 0 clears
 * the setting; otherwise count must equal the prepared batch count at
 * execute time.  bfx_autotune sets these when it keeps the tiled layout. */
enum { BFX_MAPPING_CHUNKS = 0, BFX_MAPPING_TILE_VISITS = 1 };
int bfx_set_batch_mappings(bfx_workspace *ws, uint32_t count, const uint32_t *mappings);
/* The workspace's frontier layout and, for the first `count` batches, their
 * mappings (BFX_MAPPING_TILE_VISITS where none was set). */
int bfx_get_frontier_mapping(bfx_workspace *ws, uint32_t *layout, uint32_t count, uint32_t *mappings);
/* Register budget of the persistent relaxation kernel (a bfx tuning option,
 * results unchanged): 40 registers per thread (three 512-thread blocks per
 * SM), 64 (two 512-thread blocks per SM: no spills in the group layout, few
 * in the flat one) or 80 (three 256-thread blocks per SM, blocks of at most
 * 256 threads; the chunked layout only -- the other layouts keep 64).  0, the
 * default, picks 80 for the chunked layout with blocks of at most 256
 * threads and 64 otherwise. */
int bfx_set_register_budget(bfx_workspace *ws, uint32_t registers);
/* Work items each thread keeps in flight per iteration, 2 (default), 3 or 4
 * -- more independent memory chains against more register spills: the flat
 * layout with the 64-register budget and the chunked layout with the
 * 80-register budget (persistent control).  Other configurations use 2. */
int bfx_set_flat_items(bfx_workspace *ws, uint32_t items);
/* Flat layout: how a relaxation updates the target label -- 0 (default)
 * pre-reads it and issues a non-returning 64-bit min only for a smaller
 * candidate; 1 issues one returning 64-bit min per relaxation and takes the
 * returned label as the comparison. */
int bfx_set_relax_atomic(bfx_workspace *ws, uint32_t mode);
/* Flat and chunked layouts: order of an item's work list -- 0 (default)
 * entry, lane, edge; 1 entry, edge, lane (neighbouring threads relax the
 * lanes of one edge, whose target labels are adjacent). */
int bfx_set_flat_order(bfx_workspace *ws, uint32_t edge_major);
/* Chunked layout, persistent control: how a chunk's work is spread over the
 * warp -- 0 (default) the flat work list of (lane, edge) items; 1 one
 * (vertex, lane) pair per thread walking the vertex's out-edges (no per-edge
 * decode; idle threads where degrees differ).  Host-poll modes use 0. */
int bfx_set_chunk_pairs(bfx_workspace *ws, uint32_t mode);
/* Chunked layout (and the tiled layout's warp items): chunk slots per warp
 * item -- 1, 2, 4 (default) or 8 queue words of a sparse round, or as many
 * consecutive chunk slots of a dense round.  The vertices with pending lanes
 * of the item's chunks are compacted into work lists of up to 32 vertices,
 * so a warp step carries more lane-edge relaxations when few vertices of
 * each chunk are pending. */
int bfx_set_chunk_pack(bfx_workspace *ws, uint32_t pack);
int bfx_get_chunk_pack(bfx_workspace *ws, uint32_t *pack);
/* {mean edge weight, edge count} of the workspace's resident graph. */
int bfx_workspace_graph_stats(bfx_workspace *ws, double out[2]);

/* Failure-detection self-test of the engines' grid barrier (no counterpart
 * in the reference, whose cooperative barrier cannot time out).  Runs
 * `rounds` barriers over a cooperative grid; if absent_block < grid size,
 * that block never arrives and the others' bounded waits give up after
 * timeout_ns (<= 2 s) and raise the abort flag -- the path a stuck engine
 * launch takes to report BFX_STOP_DEVICE_FAILURE.  out = {aborted, barriers
 * passed by a present block, blocks that gave up, grid size}. */
int bfx_barrier_selftest(int device, uint32_t rounds, uint32_t absent_block, uint64_t timeout_ns, uint32_t out[4]);

/* Kernels launched by the most recent bfx_execute (its own kernels only). */
int bfx_last_launch_count(bfx_workspace *ws, uint64_t *launches);

/* Work counters of the most recent bfx_execute run with instrumentation >= 1
 * (the reference's Light level, gpu_api.hpp:40-44): stats in the reference's
 * DeviceWorkStatistics layout; counters (may be NULL) = {queue entries
 * processed, edge records read, active (vertex, lane) source reads, lane-edge
 * relaxations, queue claims, distance decreases, min-reductions issued,
 * rounds}.  Without instrumentation the counters read zero. */
int bfx_fetch_work_statistics(bfx_workspace *ws, bfx_device_work_statistics *stats, uint64_t counters[8]);
/* The same counters split by engine (bfx extension, for per-engine
 * algorithmic byte counts): [0..6] frontier and dense push in the order
 * above, [7] rounds, [8..11] Jacobi pull {vertex-lane items, in-edge records,
 * relaxations, changes}, [12..13] near/far split rounds {far pile entries
 * scanned (also counted in [0]), parked lanes re-read}, [14..15] zero. */
int bfx_fetch_engine_work(bfx_workspace *ws, uint64_t counters[16]);
/* Round trace of the most recent persistent run with instrumentation 2 (bfx
 * extension): per round four words {%globaltimer ns at the round's start,
 * warp items of the round in the low 32 bits | frontier batches in a near/far
 * split round in the high 32 bits, active (vertex, lane) source reads of the
 * round, lane-edge relaxations of the round}, up to 65,536 rounds; capacity
 * counts rounds (4 words each); *rounds = rounds executed.  trace may be NULL
 * to query the count. */
int bfx_fetch_round_trace(bfx_workspace *ws, uint32_t capacity, uint64_t *trace, uint32_t *rounds);

/* ---- plain per-query engine ----------------------------------------------
 * Replaces GpuSsspEngine::run(RouteQuery, GpuRunOptions) (gpu_api.hpp:203-211)
 * as implemented by hip::FrontierPushEngine (hip/frontier_push.hpp:47): one
 * query per launch sequence.  selected_tiles must be strictly increasing. */
int bfx_run_query(bfx_workspace *ws, uint32_t source_count, const uint32_t *sources,
                  uint32_t target_count, const uint32_t *targets,
                  uint32_t selected_tile_count, const uint32_t *selected_tiles,
                  const bfx_gpu_run_options *options, bfx_device_run_status *status);

/* ---- single query without device allocation --------------------------------
 * No counterpart in the reference: a libbfx addition for callers that cannot
 * allocate device memory when they run a query -- processes whose device
 * memory is owned and carved up by another runtime (a host application or
 * framework that hands the whole GPU to its own pool and forbids further
 * allocations), and latency-critical loops that cannot afford an
 * allocation's implicit synchronisation.
 *
 * Same query semantics and status as bfx_run_query under the persistent
 * cooperative control mode, but every scratch buffer (labels, pending masks,
 * frontier queues, tile table, batch records, launch state) lives in one
 * fixed 32 MiB array in the library's device memory, so the call allocates
 * nothing.  Limits and rules:
 *  - the whole query image must fit in 32 MiB (about 76 bytes per selected
 *    vertex plus 8 bytes per graph tile); larger queries fail with
 *    BFX_ERR_OVERFLOW and a message -- use bfx_run_query for them;
 *  - options->control_mode must be BFX_CONTROL_PERSISTENT_COOPERATIVE and
 *    options->instrumentation 0 (otherwise BFX_ERR_INVALID_ARGUMENT); the
 *    engine, block size, grid policy, round limit and per-lane convergence
 *    are honoured;
 *  - every GPU that loads libbfx.so holds the 32 MiB array until exit;
 *  - the first call on a device resolves the array's device address once
 *    (cudaGetSymbolAddress) and keeps it for the process, so resetting the
 *    device (cudaDeviceReset) between calls is not supported, and that first
 *    call should be made before any stream capture begins;
 *  - all calls on a device share the array and leave their data in it (each
 *    call re-initialises what it reads); calls that overlap on the GPU --
 *    from several host threads at once -- race and must be serialised by the
 *    caller;
 *  - work runs on the legacy default stream with synchronous copies, and the
 *    call returns after the results are on the host.
 * Outputs: the status, and per target (canonical order) its distance bits and
 * predecessor stable edge id (0xffffffff for sources and unreached targets). */
int bfx_run_query_static(const bfx_resident_graph *graph, uint32_t source_count, const uint32_t *sources,
                         uint32_t target_count, const uint32_t *targets, uint32_t selected_tile_count,
                         const uint32_t *selected_tiles, const bfx_gpu_run_options *options,
                         bfx_device_run_status *status, uint32_t *target_distance_bits,
                         uint32_t *target_predecessor_edges);

#ifdef __cplusplus
}
#endif
#endif /* BFX_H */
