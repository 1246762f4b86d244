/* bfx expansion loop: regional queries whose targets are not reached inside
 * their selected tiles are retried on geometrically larger regions, then
 * (optionally) on the full graph.
 *
 * Replaces bfnew::run_batched_expansion / run_host_batched_expansion
 * (include/bfnew/batched_expansion.hpp:347-372, src/batched_expansion.cpp:888)
 * and keeps their per-query outcomes: the same schedule kinds, terminal
 * policies, dispositions, attempt and expansion counts and final regions.
 * Each planning pass plans the active queries with the batch planner
 * (bfx_plan_build) and relaxes all batches of the pass together: on the GPU
 * that is one launch per pass (bfx_expansion_run); a caller-supplied runner
 * takes the place of the reference's ExpansionBatchRunner
 * (include/bfnew/batched_expansion.hpp:177-181) in
 * bfx_expansion_run_with_runner.  Every attempt restarts from the query's
 * sources: no labels are carried from a failed attempt.
 *
 * Single host thread; all functions return a bfx status (bfx.h). */
#ifndef BFX_EXPANSION_H
#define BFX_EXPANSION_H

#include "bfx.h"
#include "bfx_host.h"

#ifdef __cplusplus
extern "C" {
#endif

/* bfnew::ExpansionScheduleKind (include/bfnew/batched_expansion.hpp:19-25). */
enum { BFX_EXPANSION_UNSPECIFIED = 0, BFX_EXPANSION_ONE_RING = 1, BFX_EXPANSION_FIXED_RING = 2,
       BFX_EXPANSION_DOUBLING = 3, BFX_EXPANSION_HYBRID = 4 };
/* bfnew::ExpansionTerminalPolicy (:27-30). */
enum { BFX_EXPANSION_FULL_REGION_FALLBACK = 0, BFX_EXPANSION_EXPLICIT_FAILURE = 1 };
/* bfnew::ExpansionQueryDisposition (:186-193). */
enum { BFX_EXPANSION_REACHED = 0, BFX_EXPANSION_UNREACHABLE_IN_FULL_REGION = 1,
       BFX_EXPANSION_LIMIT = 2, BFX_EXPANSION_REGION_STALLED = 3,
       BFX_EXPANSION_IDENTITY_OR_COUNT_OVERFLOW = 4, BFX_EXPANSION_ENGINE_FAILURE = 5 };

/* bfnew::BatchedExpansionOptions (:68-110) without the fields that only feed
 * the reference's schedule-comparison evidence (execution fingerprint) or its
 * compact-path production mode (paths come from bfx_compact_path_* on the
 * workspace instead).  Validated like validate_batched_expansion_options
 * (src/batched_expansion.cpp:831-886). */
typedef struct bfx_expansion_options {
  bfx_gpu_run_options run_options;
  bfx_planner_policy planner_policy;
  uint32_t schedule_kind;                 /* BFX_EXPANSION_ONE_RING .. HYBRID */
  uint32_t fixed_ring_size;               /* FIXED_RING only, >= 2 */
  uint32_t hybrid_small_expansion_count;  /* HYBRID only, >= 1 */
  uint32_t maximum_expansions;            /* scheduled expansions per query */
  uint32_t terminal_policy;               /* BFX_EXPANSION_FULL_REGION_FALLBACK / EXPLICIT_FAILURE */
  uint32_t reserved0;
} bfx_expansion_options;

/* bfnew::ExpansionQueryOutcome (:195-214) without the optional distance
 * image and compact payload; final tiles via bfx_expansion_final_tiles. */
typedef struct bfx_expansion_outcome {
  uint32_t query_id;
  uint32_t disposition;
  uint32_t attempts;
  uint32_t scheduled_expansions;
  uint32_t total_expansions;
  uint32_t used_full_region_fallback;
  uint32_t expansion_generation; /* of the final query */
  uint32_t final_tile_count;
  uint64_t selected_vertex_count;
  uint64_t selected_edge_count;
  uint32_t terminal_stop_reason;
  uint32_t terminal_error_bits;
} bfx_expansion_outcome;

/* The deterministic counters of bfnew::BatchedExpansionMetrics (:238-330);
 * relaxation_launches is bfx's: GPU launches that relaxed a pass. */
typedef struct bfx_expansion_metrics {
  uint64_t input_queries;
  uint64_t initial_reached_queries;
  uint64_t reached_queries;
  uint64_t unreachable_full_region_queries;
  uint64_t expansion_limit_queries;
  uint64_t stalled_region_queries;
  uint64_t identity_or_count_overflow_queries;
  uint64_t engine_failure_queries;
  uint64_t planning_passes;
  uint64_t batches_executed;
  uint64_t initial_batches_executed;
  uint64_t retry_batches_executed;
  uint64_t failed_lane_observations;
  uint64_t failed_origin_valid_lane_observations;
  uint64_t retry_valid_lane_observations;
  uint64_t retry_lane_capacity;
  uint64_t scheduled_expansions;
  uint64_t full_region_fallbacks;
  uint64_t repeated_selected_edge_estimate;
  uint64_t attempted_selected_vertex_count;
  uint64_t attempted_selected_edge_estimate;
  uint64_t final_selected_tile_count;
  uint64_t final_selected_vertex_count;
  uint64_t final_selected_edge_count;
  uint64_t relaxation_launches;
} bfx_expansion_metrics;

/* Tile geometry of the spatially ordered graph (bfx_layout_tiles): tile_xy
 * [2*T] (x, y), has_location[T]; the last tile is the spill tile. */
typedef struct bfx_tile_geometry {
  uint32_t tile_count;
  uint32_t reserved0;
  const int64_t *tile_xy;
  const uint8_t *has_location;
  const uint32_t *tile_vertex_offsets; /* [T+1] */
} bfx_tile_geometry;

/* Runs every batch of one planning pass and writes one status per batch
 * (clean convergence: reached | miss == valid lanes).  Returns 0 on success;
 * any other value aborts the expansion run with BFX_ERR_STATE. */
typedef int (*bfx_expansion_batch_runner)(void *user, uint32_t batch_count, const bfx_batch_description *batches,
                                          bfx_device_run_status *statuses);

typedef struct bfx_expansion_result bfx_expansion_result;

/* GPU runner: each pass is prepared into `ws` and relaxed in one launch with
 * options->run_options (BFX_ENGINE_AUTO is not accepted). */
int bfx_expansion_run(bfx_workspace *ws, const bfx_device_graph_layout32 *layout, const bfx_tile_geometry *tiles,
                      uint32_t query_count, const bfx_route_query *queries, const bfx_expansion_options *options,
                      bfx_expansion_result **out);
/* Caller-supplied runner (the reference's ExpansionBatchRunner boundary). */
int bfx_expansion_run_with_runner(const bfx_device_graph_layout32 *layout, const bfx_tile_geometry *tiles,
                                  uint32_t query_count, const bfx_route_query *queries,
                                  const bfx_expansion_options *options, bfx_expansion_batch_runner runner,
                                  void *user, bfx_expansion_result **out);
int bfx_expansion_destroy(bfx_expansion_result *result);
/* outcomes[query_count], in query-id order. */
int bfx_expansion_outcomes(const bfx_expansion_result *result, bfx_expansion_outcome *outcomes);
/* Final selected tiles of outcome `index` (outcomes[index].final_tile_count entries). */
int bfx_expansion_final_tiles(const bfx_expansion_result *result, uint32_t index, uint32_t *tiles);
int bfx_expansion_metrics_get(const bfx_expansion_result *result, bfx_expansion_metrics *metrics);
/* expansion_count_histogram: *count entries; histogram may be NULL to query the count. */
int bfx_expansion_histogram(const bfx_expansion_result *result, uint32_t *count, uint64_t *histogram);

#ifdef __cplusplus
}
#endif

#endif /* BFX_EXPANSION_H */
