/*
 * bfx host builders — C ABI of the host-side pipeline in libbfx.so that feeds
 * the device engines: spatially ordered device graph image, route queries,
 * the overlap batch planner, batch descriptions, and seeded synthetic
 * workloads.  All functions return BFX_OK (0) or a BFX_ERR_* code from bfx.h
 * and never throw.
 */
#ifndef BFX_HOST_H
#define BFX_HOST_H

#include "bfx.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Flattened bfnew::InputGraph (include/bfnew/graph.hpp:139-165): vertex
 * metadata (graph.hpp:18-37) and edge records (graph.hpp:39-46) with their
 * 16-byte PhysicalProvenance (types.hpp:69-75).  Host pointers. */
typedef struct bfx_input_graph {
  uint32_t vertex_count;
  uint32_t reserved0;
  uint64_t edge_count;
  const int32_t *x;
  const int32_t *y;
  const uint8_t *has_location;
  const uint16_t *resource_class;
  const uint32_t *edge_source;
  const uint32_t *edge_destination;
  const float *edge_weight;
  const uint32_t *provenance_domain;
  const uint32_t *provenance_kind;
  const uint64_t *provenance_record;
} bfx_input_graph;

/* bfnew::SpatialOrderConfig (include/bfnew/spatial.hpp:19-26). */
typedef struct bfx_spatial_order_config {
  int32_t origin_x, origin_y;
  uint32_t tile_width, tile_height;
} bfx_spatial_order_config;

typedef struct bfx_layout bfx_layout;

/* Builds the spatially ordered graph and its checked 32-bit device image.
 * Replaces, in one call, UniformGridPartitioner::partition
 * (src/tiled_graph.cpp:539) -> build_spatially_ordered_graph (src/reorder.cpp:151,
 * canonical edge ids from build_weighted_graph, src/graph_builder.cpp:182) ->
 * build_tile_run_layout (src/device_layout.cpp:186) ->
 * build_device_graph_layout32 (src/device_layout.cpp:395).  The result is
 * identical, array for array, to the reference image on the same input.
 * threads: host threads to use (0 = all hardware threads). */
int bfx_layout_build(const bfx_input_graph *input, const bfx_spatial_order_config *config,
                     uint32_t threads, bfx_layout **out);
int bfx_layout_destroy(bfx_layout *layout);
/* Borrowed view (valid while the layout lives), csr_edge_ids included. */
int bfx_layout_view(const bfx_layout *layout, bfx_device_graph_layout32 *view);
/* Tile table: tile_xy[2*T] (tile_x, tile_y), has_location[T],
 * tile_vertex_offsets[T+1]; any output may be NULL. */
int bfx_layout_tiles(const bfx_layout *layout, int64_t *tile_xy, uint8_t *has_location,
                     uint32_t *tile_vertex_offsets);
/* new_to_old[V]: original input vertex id of every reordered vertex. */
int bfx_layout_new_to_old(const bfx_layout *layout, uint32_t *new_to_old);

/* Canonical bfnew::RouteQuery subset used by the batch path
 * (include/bfnew/query.hpp:13-29): sorted unique sources, targets and
 * selected tiles, global reordered ids. */
typedef struct bfx_route_query {
  uint32_t query_id;
  uint32_t expansion_generation;
  uint32_t source_count;
  uint32_t target_count;
  const uint32_t *sources;
  const uint32_t *targets;
  uint32_t selected_tile_count;
  uint32_t reserved0;
  const uint32_t *selected_tiles;
} bfx_route_query;

/* bfnew::BatchPlannerPolicy (include/bfnew/batch_plan.hpp:27-35). */
typedef struct bfx_planner_policy {
  uint32_t lane_width;
  uint32_t minimum_jaccard_numerator, minimum_jaccard_denominator;
  uint32_t maximum_union_inflation_numerator, maximum_union_inflation_denominator;
  uint32_t narrow_lanes; /* bfx extension: 1 = shrink each batch to the
                            smallest supported width holding its lanes */
} bfx_planner_policy;

typedef struct bfx_plan bfx_plan;

/* Features + greedy overlap plan + one batch description per batch.
 * Replaces make_batch_query_features (src/batch_plan.cpp:578),
 * make_overlapping_batch_plan (src/batch_plan.cpp:680) and
 * prepare_batch_device_description (src/batch_layout.cpp:1056, device-
 * materialized run masks).  Queries must have unique ids.  The plan equals
 * the reference's (same batches, lanes and union tiles) when narrow_lanes==0.
 * layout: any graph image (e.g. a bfx_layout_view); tile_vertex_offsets[T+1]. */
int bfx_plan_build(const bfx_device_graph_layout32 *layout, const uint32_t *tile_vertex_offsets,
                   uint32_t query_count, const bfx_route_query *queries, const bfx_planner_policy *policy,
                   bfx_plan **out);
int bfx_plan_destroy(bfx_plan *plan);
int bfx_plan_batch_count(const bfx_plan *plan, uint32_t *count);
/* Borrowed description of batch b (valid while the plan lives). */
int bfx_plan_description(const bfx_plan *plan, uint32_t batch, bfx_batch_description *out);
/* query_index_by_lane[lane_width] (0xffffffff for padding lanes) and
 * estimates {union_vertex_count, union_edge_estimate,
 * selected_lane_vertex_count, selected_lane_edge_estimate}. */
int bfx_plan_batch_info(const bfx_plan *plan, uint32_t batch, uint32_t *query_index_by_lane,
                        uint64_t estimates[4]);
/* All descriptions as one contiguous array (borrowed). */
int bfx_plan_descriptions(const bfx_plan *plan, const bfx_batch_description **out);

/* ---- device-side batch description preparation ----------------------------
 * Replaces prepare_batch_device_description (src/batch_layout.cpp:1056-1296)
 * run on the host per batch: the caller gives only each batch's lane ->
 * query assignment (lanes 0..lane_count-1 valid, the rest padding) and the
 * queries' canonical terminals and strictly increasing selected tiles; the
 * dense tile lane masks, one vertex range per union tile with its compact
 * offset, and the lane terminal slices are built on the device, into the
 * workspace, with one small readback of the union sizes.  The result is the
 * same prepared set bfx_prepare_batches makes from the host descriptions of
 * the same assignment (ready for bfx_execute).  Errors as
 * bfx_prepare_batches (a terminal whose owner tile its lane does not select
 * is rejected with BFX_ERR_INVALID_ARGUMENT). */
typedef struct bfx_batch_lanes {
  uint32_t lane_width;                 /* 1, 8, 16 or 32 */
  uint32_t lane_count;                 /* 1..lane_width */
  const uint32_t *query_index_by_lane; /* [lane_count] indices into the query array */
} bfx_batch_lanes;

int bfx_prepare_batches_from_queries(bfx_workspace *ws, uint32_t batch_count, const bfx_batch_lanes *batches,
                                     uint32_t query_count, const bfx_route_query *queries);

/* The prepared description of batch `batch` as the device holds it (either
 * prepare path), in bfx_batch_description's arrays: counts = {lane_width,
 * valid_lane_mask, source count, target count, union tile count}; with every
 * array non-NULL also source_offsets[W+1], sources, target_offsets[W+1],
 * targets, union_tiles[R], tile_lane_masks[tile_count] and
 * selected_vertex_ranges[R]. */
int bfx_fetch_prepared_description(bfx_workspace *ws, uint32_t batch, uint32_t counts[5],
                                   uint32_t *source_offsets, uint32_t *sources, uint32_t *target_offsets,
                                   uint32_t *targets, uint32_t *union_tiles, uint32_t *tile_lane_masks,
                                   bfx_batch_vertex_range *selected_vertex_ranges);

/* Seeded synthetic spatial workloads (bfx's own generator; the reference's
 * FPGA artifacts are not available).  PRNG: xoshiro256** seeded by
 * splitmix64.  Vertex i of tile (tx, ty) sits at
 * (tx*sx + i % sx, ty*sy + i / sx) with sx*sy = nodes_per_tile. */
typedef struct bfx_synth_config {
  uint32_t tiles_x, tiles_y;
  uint32_t nodes_per_tile;         /* 64 (8x8), 128 (16x8) or 256 (16x16); any s*s too */
  uint32_t intra_degree;           /* edges to uniform nodes of the own tile */
  uint32_t inter_degree;           /* edges to a uniform 4-neighbour tile at a span */
  uint32_t span_count;
  uint32_t spans[8];
  uint32_t cost_kind;              /* 0: uint costs U[cost_lo, cost_hi] stored as f32;
                                      1: f32 base(span) * lognormal(0, sigma) */
  uint32_t cost_lo, cost_hi;
  float intra_base;                /* cost_kind 1: base of intra-tile edges */
  float span_base[8];              /* cost_kind 1: base per span index */
  float sigma;
  uint32_t reserved0;
  uint64_t seed;
} bfx_synth_config;

/* Sizes {V, E} of the generated graph. */
int bfx_synth_sizes(const bfx_synth_config *config, uint64_t out[2]);
/* Fills caller arrays of the sizes above (x, y: V; edges: E) and the
 * SpatialOrderConfig that tiles them.  stats (may be NULL) receives
 * {inter edges, inter edges redrawn at the border}. */
int bfx_synth_fill(const bfx_synth_config *config, int32_t *x, int32_t *y, uint8_t *has_location,
                   uint16_t *resource_class, uint32_t *edge_source, uint32_t *edge_destination,
                   float *edge_weight, uint32_t *provenance_domain, uint32_t *provenance_kind,
                   uint64_t *provenance_record, bfx_spatial_order_config *order,
                   uint64_t stats[2]);

/* Planner / autotuner co-design (no counterpart in the reference, whose
 * planner takes one fixed policy, src/batch_plan.cpp:680): plans the queries
 * with each candidate policy (bfx_plan_build), tunes and times the whole set
 * as it would run (bfx_autotune, then the fastest of `trials` launches with
 * BFX_ENGINE_AUTO), and reports the fastest.  times_ms[policy_count] receives
 * each candidate's relaxation time, *best its index.  The workspace is left
 * prepared and tuned with the best candidate's plan, which the caller can
 * rebuild with bfx_plan_build and the same policy. */
int bfx_autotune_policy(bfx_workspace *ws, const bfx_device_graph_layout32 *layout,
                        const uint32_t *tile_vertex_offsets, uint32_t query_count, const bfx_route_query *queries,
                        uint32_t policy_count, const bfx_planner_policy *policies, const bfx_gpu_run_options *base,
                        uint32_t trials, uint32_t *best, float *times_ms);

#ifdef __cplusplus
}
#endif
#endif /* BFX_HOST_H */
