/*
 * bfx oracle — TEST INFRASTRUCTURE ONLY (see bfx_oracle.h).  Plain C, no
 * dependencies.  Restates the reference's CPU algorithm; each function cites
 * the reference lines it follows.  Float additions are plain IEEE binary32
 * adds (compiled without fast-math or contraction), as in the reference.
 */
#define _POSIX_C_SOURCE 200809L
#include "bfx_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define INF_BITS 0x7F800000u
#define NO_EDGE 0xFFFFFFFFu

static float bits_to_f(uint32_t b) {
  float f;
  memcpy(&f, &b, 4);
  return f;
}

static uint32_t f_to_bits(float f) {
  uint32_t b;
  memcpy(&b, &f, 4);
  return b;
}

/* Binary min-heap of (distance, vertex), ordered like QueueEntryGreater
 * (src/cpu/reference_dijkstra.cpp:20-28): distance, then vertex. */
typedef struct {
  float d;
  uint32_t v;
} entry;

typedef struct {
  entry *a;
  size_t n, cap;
} heap;

static int less(entry x, entry y) { return x.d < y.d || (x.d == y.d && x.v < y.v); }

static int heap_push(heap *h, entry e) {
  if (h->n == h->cap) {
    size_t nc = h->cap ? 2 * h->cap : 1024;
    entry *na = (entry *)realloc(h->a, nc * sizeof(entry));
    if (!na) return -1;
    h->a = na;
    h->cap = nc;
  }
  size_t i = h->n++;
  while (i > 0) {
    size_t p = (i - 1) / 2;
    if (!less(e, h->a[p])) break;
    h->a[i] = h->a[p];
    i = p;
  }
  h->a[i] = e;
  return 0;
}

static entry heap_pop(heap *h) {
  entry top = h->a[0];
  entry last = h->a[--h->n];
  size_t i = 0;
  for (;;) {
    size_t l = 2 * i + 1, r = l + 1, m = i;
    entry best = last;
    if (l < h->n && less(h->a[l], best)) {
      m = l;
      best = h->a[l];
    }
    if (r < h->n && less(h->a[r], best)) m = r;
    if (m == i) break;
    h->a[i] = h->a[m];
    i = m;
  }
  if (h->n) h->a[i] = last;
  return top;
}

static int selected_vertex(const oracle_graph *g, const oracle_query *q, uint32_t v) {
  return q->selected[g->owner_tiles[v]] != 0;
}

/* dijkstra_oracle (src/cpu/reference_dijkstra.cpp:32-63) run on the induced
 * query graph (src/query.cpp:286-363): relaxation of an edge requires both
 * endpoints in selected tiles; strict `<` decreases; stale heap entries are
 * skipped when their distance differs from the label. */
int oracle_region_sssp(const oracle_graph *g, const oracle_query *q, uint32_t *dist_bits, uint32_t *pred) {
  const uint32_t V = g->vertex_count;
  float *d = (float *)malloc((size_t)V * sizeof(float));
  if (!d) return -1;
  for (uint32_t v = 0; v < V; ++v) d[v] = INFINITY;
  heap h = {0, 0, 0};
  for (uint32_t i = 0; i < q->source_count; ++i) {
    const uint32_t s = q->sources[i];
    if (!selected_vertex(g, q, s)) continue;
    d[s] = 0.0f;
  }
  for (uint32_t i = 0; i < q->source_count; ++i) {
    const uint32_t s = q->sources[i];
    if (selected_vertex(g, q, s)) heap_push(&h, (entry){0.0f, s});
  }
  while (h.n) {
    const entry e = heap_pop(&h);
    if (e.d != d[e.v]) continue;
    for (uint32_t p = g->csr_row_offsets[e.v]; p < g->csr_row_offsets[e.v + 1]; ++p) {
      const uint32_t t = g->csr_destinations[p];
      if (!selected_vertex(g, q, t)) continue;
      const float cand = e.d + g->csr_weights[p];
      if (cand < d[t]) {
        d[t] = cand;
        heap_push(&h, (entry){cand, t});
      }
    }
  }
  free(h.a);
  /* Predecessor: the smallest stable edge id among tight in-edges whose
   * source is selected and finite (tight_choices, src/compact_paths.cpp:98-129,
   * first entry after the sort by edge id); sources have none. */
  for (uint32_t v = 0; v < V; ++v) {
    dist_bits[v] = f_to_bits(d[v]);
    if (pred) pred[v] = NO_EDGE;
  }
  if (pred) {
    for (uint32_t v = 0; v < V; ++v) {
      if (!isfinite(d[v]) || !selected_vertex(g, q, v)) continue;
      int is_source = 0;
      /* sources are few; a linear scan keeps this free of extra storage */
      for (uint32_t i = 0; i < q->source_count; ++i) {
        if (q->sources[i] == v) {
          is_source = 1;
          break;
        }
      }
      if (is_source) continue;
      uint32_t best = NO_EDGE;
      for (uint32_t c = g->csc_column_offsets[v]; c < g->csc_column_offsets[v + 1]; ++c) {
        const uint32_t u = g->csc_sources[c];
        if (!selected_vertex(g, q, u) || !isfinite(d[u])) continue;
        if (d[u] + g->csc_weights[c] == d[v] && g->csc_edge_ids[c] < best) best = g->csc_edge_ids[c];
      }
      pred[v] = best;
    }
  }
  free(d);
  return 0;
}

typedef struct {
  const oracle_graph *g;
  const oracle_query *qs;
  uint32_t nq;
  uint32_t *dist, *pred;
  uint32_t next;
  pthread_mutex_t mu;
} many_ctx;

static void *many_worker(void *arg) {
  many_ctx *c = (many_ctx *)arg;
  for (;;) {
    pthread_mutex_lock(&c->mu);
    const uint32_t i = c->next++;
    pthread_mutex_unlock(&c->mu);
    if (i >= c->nq) break;
    const size_t off = (size_t)i * c->g->vertex_count;
    oracle_region_sssp(c->g, &c->qs[i], c->dist + off, c->pred ? c->pred + off : NULL);
  }
  return NULL;
}

int oracle_region_sssp_many(const oracle_graph *g, uint32_t nq, const oracle_query *qs, uint32_t threads,
                            uint32_t *dist_bits, uint32_t *pred) {
  if (threads == 0) threads = 1;
  if (threads > 256) threads = 256;
  many_ctx c = {g, qs, nq, dist_bits, pred, 0, PTHREAD_MUTEX_INITIALIZER};
  pthread_t th[256];
  for (uint32_t t = 0; t < threads; ++t) pthread_create(&th[t], NULL, many_worker, &c);
  for (uint32_t t = 0; t < threads; ++t) pthread_join(th[t], NULL);
  return 0;
}

/* Tight admitted in-edges of v sorted by stable edge id
 * (tight_choices, src/compact_paths.cpp:98-129). */
typedef struct {
  uint32_t eid, pred;
} choice;

static int cmp_choice(const void *a, const void *b) {
  const uint32_t x = ((const choice *)a)->eid, y = ((const choice *)b)->eid;
  return x < y ? -1 : (x > y ? 1 : 0);
}

static uint32_t tight_choices(const oracle_graph *g, const oracle_query *q, const uint32_t *dist_bits, uint32_t v,
                              choice *out) {
  uint32_t n = 0;
  const float dv = bits_to_f(dist_bits[v]);
  for (uint32_t c = g->csc_column_offsets[v]; c < g->csc_column_offsets[v + 1]; ++c) {
    const uint32_t u = g->csc_sources[c];
    const float du = bits_to_f(dist_bits[u]);
    if (!selected_vertex(g, q, u) || !isfinite(du)) continue;
    if (du + g->csc_weights[c] == dv) out[n++] = (choice){g->csc_edge_ids[c], u};
  }
  qsort(out, n, sizeof(choice), cmp_choice);
  return n;
}

/* reconstruct_target (src/compact_paths.cpp:131-211). */
int oracle_compact_path(const oracle_graph *g, const oracle_query *q, const uint32_t *dist_bits, uint32_t target,
                        uint32_t cap, uint32_t *vertices, uint32_t *edge_ids, uint32_t *length) {
  const uint32_t V = g->vertex_count;
  *length = 0;
  if (!isfinite(bits_to_f(dist_bits[target]))) return 1;
  uint8_t *on_path = (uint8_t *)calloc(V, 1);
  uint8_t *is_source = (uint8_t *)calloc(V, 1);
  uint32_t *stack_v = (uint32_t *)malloc((size_t)V * 4);
  uint32_t *stack_cursor = (uint32_t *)malloc((size_t)V * 4);
  uint32_t *stack_edge = (uint32_t *)malloc((size_t)V * 4);
  uint32_t maxdeg = 0;
  for (uint32_t v = 0; v < V; ++v) {
    const uint32_t d = g->csc_column_offsets[v + 1] - g->csc_column_offsets[v];
    if (d > maxdeg) maxdeg = d;
  }
  choice *buf = (choice *)malloc(((size_t)maxdeg + 1) * sizeof(choice));
  int status = 3;
  for (uint32_t i = 0; i < q->source_count; ++i) is_source[q->sources[i]] = 1;
  size_t depth = 0;
  stack_v[0] = target;
  stack_cursor[0] = 0;
  on_path[target] = 1;
  depth = 1;
  while (depth) {
    const uint32_t v = stack_v[depth - 1];
    if (is_source[v]) {
      const uint32_t len = (uint32_t)(depth - 1);
      if (len > cap) {
        status = 4;
        break;
      }
      /* stack_edge[k] is the edge from stack_v[k+1] to stack_v[k]. */
      for (uint32_t k = 0; k < depth; ++k) vertices[k] = stack_v[depth - 1 - k];
      for (uint32_t k = 0; k < len; ++k) edge_ids[k] = stack_edge[len - 1 - k];
      *length = len;
      status = 0;
      break;
    }
    const uint32_t n = tight_choices(g, q, dist_bits, v, buf);
    int advanced = 0;
    while (stack_cursor[depth - 1] < n) {
      const choice c = buf[stack_cursor[depth - 1]++];
      if (on_path[c.pred]) continue;
      stack_edge[depth - 1] = c.eid;
      stack_v[depth] = c.pred;
      stack_cursor[depth] = 0;
      on_path[c.pred] = 1;
      ++depth;
      advanced = 1;
      break;
    }
    if (advanced) continue;
    on_path[v] = 0;
    --depth;
  }
  free(on_path);
  free(is_source);
  free(stack_v);
  free(stack_cursor);
  free(stack_edge);
  free(buf);
  return status;
}

/* Correctly rounded (nearest, ties to even) float of the exact value
 * n * 2^-63, n a signed 128-bit integer. */
static float round_fixed63(__int128 n) {
  if (n == 0) return 0.0f;
  const int neg = n < 0;
  unsigned __int128 m = neg ? (unsigned __int128)(-n) : (unsigned __int128)n;
  int p = 127;
  while (((m >> p) & 1) == 0) --p;
  int shift = 0;
  uint64_t mant;
  if (p <= 23) {
    mant = (uint64_t)m;
  } else {
    shift = p - 23;
    mant = (uint64_t)((m >> shift) & 0xFFFFFF);
    const int guard = (int)((m >> (shift - 1)) & 1);
    const int sticky = shift > 1 && (m & (((unsigned __int128)1 << (shift - 1)) - 1)) != 0;
    if (guard && (sticky || (mant & 1))) {
      ++mant;
      if (mant == (1u << 24)) {
        mant >>= 1;
        ++shift;
      }
    }
  }
  const float r = ldexpf((float)mant, shift - 63);
  return neg ? -r : r;
}

/* Edge usage over explicit paths: grad[e] = sum over paths p using e of g_p,
 * summed exactly (fixed point with lsb 2^-63) and rounded once to float --
 * the contract of the device adjoint, independent of summation order.
 * g values must be 0 or have magnitude in [2^-40, 2^40).  grad[E] is
 * overwritten. */
int oracle_edge_usage_adjoint(uint32_t edge_count, uint32_t path_count, const uint32_t *path_offsets,
                              const uint32_t *paths, const float *gvals, float *grad) {
  __int128 *acc = (__int128 *)calloc(edge_count ? edge_count : 1, sizeof(__int128));
  if (!acc) return -1;
  int rc = 0;
  for (uint32_t p = 0; p < path_count && rc == 0; ++p) {
    const float g = gvals[p];
    if (g == 0.0f) continue;
    const float a = fabsf(g);
    if (!(a >= 0x1p-40f && a < 0x1p40f)) {
      rc = -2;
      break;
    }
    const uint32_t bits = f_to_bits(g);
    const int ex = (int)((bits >> 23) & 0xFF);
    const __int128 m = (__int128)((bits & 0x7FFFFF) | 0x800000);
    __int128 v = m << (ex - 87); /* g * 2^63 exactly */
    if (bits >> 31) v = -v;
    for (uint32_t k = path_offsets[p]; k < path_offsets[p + 1]; ++k) {
      const uint32_t e = paths[k];
      if (e >= edge_count) {
        rc = -1;
        break;
      }
      acc[e] += v;
    }
  }
  if (rc == 0) {
    for (uint32_t e = 0; e < edge_count; ++e) grad[e] = round_fixed63(acc[e]);
  }
  free(acc);
  return rc;
}
