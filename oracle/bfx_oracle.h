/*
 * bfx oracle — TEST INFRASTRUCTURE ONLY.  A plain-C restatement of the
 * reference's CPU algorithm for the batched relaxation path, used by tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg as the checker.  It
 * is never linked into, called by, or shipped with the product (libbfx.so).
 *
 * Pinned against the reference: tests/test_oracle_golden.py checks it
 * against golden vectors produced by the reference's own CPU code
 * (oracle/gen_golden.py over oracle/_ref).
 */
#ifndef BFX_ORACLE_H
#define BFX_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Graph image the oracle reads: CSR with stable edge ids, CSC, owner tiles. */
typedef struct oracle_graph {
  uint32_t vertex_count, edge_count, tile_count, reserved0;
  const uint32_t *owner_tiles;
  const uint32_t *csr_row_offsets, *csr_destinations, *csr_edge_ids;
  const float *csr_weights;
  const uint32_t *csc_column_offsets, *csc_sources, *csc_edge_ids;
  const float *csc_weights;
} oracle_graph;

/* One query: canonical sources/targets, selected tile flags (tile_count bytes). */
typedef struct oracle_query {
  uint32_t source_count, target_count;
  const uint32_t *sources, *targets;
  const uint8_t *selected;
} oracle_query;

/* Bounded single-query SSSP on the query's induced subgraph (edges whose two
 * endpoints lie in selected tiles), the reference's dijkstra_oracle on
 * build_induced_query_graph (src/cpu/reference_dijkstra.cpp:32-63,
 * src/query.cpp:286-363).  dist_bits[V]: float bits, +inf outside or
 * unreached.  pred[V]: the smallest stable edge id among tight admitted
 * in-edges (src/compact_paths.cpp:98-129), 0xffffffff for sources,
 * unreached and unselected vertices.  Returns 0. */
int oracle_region_sssp(const oracle_graph *g, const oracle_query *q, uint32_t *dist_bits, uint32_t *pred);

/* Many queries over `threads` pthreads; outputs are q-major [nq][V]. */
int oracle_region_sssp_many(const oracle_graph *g, uint32_t nq, const oracle_query *qs, uint32_t threads,
                            uint32_t *dist_bits, uint32_t *pred);

/* Reference compact-path reconstruction for one target
 * (reconstruct_target, src/compact_paths.cpp:131-230): depth-first search
 * over tight admitted in-edges in stable-edge-id order with backtracking
 * out of zero-weight cycles.  Returns the status (0 complete, 1 unreachable,
 * 3 no tight path, 4 length overflow) and writes up to `cap` edge ids
 * (source first) and cap+1 vertices; *length = edge count. */
int oracle_compact_path(const oracle_graph *g, const oracle_query *q, const uint32_t *dist_bits, uint32_t target,
                        uint32_t cap, uint32_t *vertices, uint32_t *edge_ids, uint32_t *length);

/* Edge-usage adjoint over explicit target paths: grad[e] = sum of g_t over
 * the paths using edge e, summed exactly and rounded once to float (the
 * device adjoint's contract; order independent).  paths: concatenated edge
 * ids, path_offsets[n+1], gvals[n] (0 or |g| in [2^-40, 2^40)).  grad[E] is
 * overwritten.  Returns 0, -1 on a bad edge id, -2 on an out-of-range g. */
int oracle_edge_usage_adjoint(uint32_t edge_count, uint32_t path_count, const uint32_t *path_offsets,
                              const uint32_t *paths, const float *gvals, float *grad);

#ifdef __cplusplus
}
#endif
#endif
