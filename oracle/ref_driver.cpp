// Test infrastructure only (never linked into the product): a C ABI over the
// reference's own CPU library so that pytest can (1) generate golden fixtures,
// (2) check the product's host layout/batch builders against the reference's
// builders on the same inputs, and (3) time the reference CPU engine as the
// cpu_baseline.  Compiled by oracle/Makefile directly from the reference
// sources; outputs land in oracle/_ref/ only.
//
// Reference entry points wrapped here (paths relative to the reference repo):
//   UniformGridPartitioner::partition          src/tiled_graph.cpp:539
//   build_tile_run_layout                      src/device_layout.cpp:186
//   build_device_graph_layout32                src/device_layout.cpp:395
//   make_route_query / build_induced_query_graph  src/query.cpp:128 / :286
//   dijkstra_oracle / synchronous_bellman_ford src/cpu/reference_dijkstra.cpp:32,
//                                              src/cpu/reference_bellman_ford.cpp:14
//   reconstruct_compact_path_payload           src/compact_paths.cpp:540
//   make_batch_query_features / make_overlapping_batch_plan  src/batch_plan.cpp:578 / :680
//   prepare_batch_device_description           src/batch_layout.cpp:1056
//   run_host_batched_expansion                 src/batched_expansion.cpp:1681
//   run_host_batched_{frontier_push,jacobi_pull,dense_chaotic_push}
//       src/batched_frontier_push.cpp:648, src/batched_jacobi_pull.cpp:572,
//       src/batched_dense_chaotic_push.cpp:569
// Fixture suites are included from the reference's tests/ directory.

#include "bfnew/batch_layout.hpp"
#include "bfnew/batched_expansion.hpp"
#include "bfnew/batch_plan.hpp"
#include "bfnew/batched_dense_chaotic_push.hpp"
#include "bfnew/batched_frontier_push.hpp"
#include "bfnew/batched_jacobi_pull.hpp"
#include "bfnew/compact_paths.hpp"
#include "bfnew/device_layout.hpp"
#include "bfnew/graph.hpp"
#include "bfnew/query.hpp"
#include "bfnew/selected_region_index.hpp"
#include "bfnew/spatial.hpp"
#include "bfnew/sssp.hpp"

#include "batched_frontier_fixture_suite.hpp"
#include "compact_paths_fixture_suite.hpp"
#include "dense_fixture_suite.hpp"
#include "frontier_fixture_suite.hpp"
#include "graph_fixtures.hpp"
#include "jacobi_fixture_suite.hpp"

#include <atomic>
#include <algorithm>
#include <bit>
#include <cmath>
#include <limits>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <mutex>
#include <optional>
#include <string>
#include <thread>
#include <vector>

using namespace bfnew;

namespace {

struct RefCase {
  std::string name;
  std::optional<PartitionedGraph> partitioned;
  TileRunLayout64 runs;
  DeviceGraphLayout32 layout;
  std::vector<std::uint32_t> csr_edge_ids;
  std::vector<RouteQuery> queries;
  // Optional expectations carried by a reference fixture.
  std::uint32_t expected_reached{1U};
  std::uint32_t expected_miss{0U};
  std::uint32_t four_ulps{0U};
  // Planning state.
  std::optional<SelectedRegionIndex> regions;
  std::vector<BatchQueryFeatures> features;
  BatchPlan plan;
};

std::mutex g_mutex;
std::vector<std::unique_ptr<RefCase>> g_cases;
thread_local std::string g_error;

RefCase* get(int handle) {
  std::lock_guard<std::mutex> lock(g_mutex);
  if (handle < 0 || static_cast<std::size_t>(handle) >= g_cases.size()) {
    return nullptr;
  }
  return g_cases[static_cast<std::size_t>(handle)].get();
}

int store(std::unique_ptr<RefCase> c) {
  std::lock_guard<std::mutex> lock(g_mutex);
  g_cases.push_back(std::move(c));
  return static_cast<int>(g_cases.size() - 1U);
}

void finish_layout(RefCase& c) {
  const WeightedGraph& g = c.partitioned->graph;
  c.runs = build_tile_run_layout(g);
  c.layout = build_device_graph_layout32(g, c.runs);
  c.csr_edge_ids.clear();
  for (const EdgeId e : g.outgoing().edge_ids) {
    c.csr_edge_ids.push_back(static_cast<std::uint32_t>(e.value()));
  }
}

std::unique_ptr<RefCase> from_partitioned(std::string name, PartitionedGraph p) {
  auto c = std::make_unique<RefCase>();
  c->name = std::move(name);
  c->partitioned.emplace(std::move(p));
  finish_layout(*c);
  return c;
}

std::vector<test::JacobiFixtureCase> single_query_suite(const std::string& suite) {
  if (suite == "jacobi") return test::make_jacobi_fixture_suite();
  if (suite == "dense") return test::make_dense_fixture_suite();
  if (suite == "frontier") return test::make_frontier_fixture_suite();
  return {};
}

template <typename T>
void copy_out(T* dst, const std::vector<T>& v) {
  if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(T));
}

template <typename F>
int guarded(F&& f) {
  try {
    return f();
  } catch (const std::exception& e) {
    g_error = e.what();
    return -1;
  }
}

}  // namespace

extern "C" {

const char* ref_last_error() { return g_error.c_str(); }

int ref_case_from_input(
    std::uint32_t nv, const std::int32_t* xs, const std::int32_t* ys,
    const std::uint8_t* has_loc, const std::uint16_t* classes,
    std::uint64_t ne, const std::uint32_t* src, const std::uint32_t* dst,
    const float* w, const std::uint32_t* pdom, const std::uint32_t* pkind,
    const std::uint64_t* prec, std::int32_t ox, std::int32_t oy,
    std::uint32_t tw, std::uint32_t th) {
  return guarded([&] {
    std::vector<VertexMetadata> vertices;
    vertices.reserve(nv);
    for (std::uint32_t v = 0; v < nv; ++v) {
      const ResourceClassId cls{classes[v]};
      vertices.push_back(has_loc[v] ? VertexMetadata::located(xs[v], ys[v], cls)
                                    : VertexMetadata::unlocated(cls));
    }
    std::vector<EdgeInputRecord> edges;
    edges.reserve(ne);
    for (std::uint64_t e = 0; e < ne; ++e) {
      edges.push_back(EdgeInputRecord{
          VertexId{src[e]}, VertexId{dst[e]}, w[e],
          PhysicalProvenance{pdom[e], pkind[e], prec[e]}});
    }
    InputGraph input{std::move(vertices), std::move(edges)};
    const UniformGridPartitioner part{SpatialOrderConfig{ox, oy, tw, th}};
    return store(from_partitioned("input", part.partition(input)));
  });
}

// Synthetic spatial graph straight into the reference's partitioner, so the
// reference arm of the benchmark needs nothing from the product library.
// The generator restates the product's seeded synthetic workload
// (xoshiro256** seeded through splitmix64, multiply-shift uniform integers
// from the top 32 bits, Box-Muller normals in double rounded once to float;
// tiles of tile_width x tile_height local coordinates, row-major tile ids,
// intra-tile edges to another uniform node of the tile, inter-tile edges to a
// uniform 4-neighbour at a uniform span, redrawn up to 16 times off the grid
// and then clamped to the border); tests/test_ref_synth.py checks that both
// produce the same graph.
namespace {

struct SynthRng {
  std::uint64_t s[4];
  explicit SynthRng(std::uint64_t seed) {
    std::uint64_t x = seed;
    for (int i = 0; i < 4; ++i) {
      x += 0x9E3779B97F4A7C15ULL;
      std::uint64_t z = x;
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
      s[i] = z ^ (z >> 31);
    }
  }
  std::uint64_t next() {
    auto rotl = [](std::uint64_t v, int k) { return (v << k) | (v >> (64 - k)); };
    const std::uint64_t out = rotl(s[1] * 5U, 7) * 9U;
    const std::uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return out;
  }
  std::uint32_t uniform(std::uint32_t n) { return static_cast<std::uint32_t>(((next() >> 32) * n) >> 32); }
  double unit() { return static_cast<double>(next() >> 11) / 9007199254740992.0; }
  double gauss() {
    const double a = 1.0 - unit();
    const double b = unit();
    return std::sqrt(-2.0 * std::log(a)) * std::cos(6.283185307179586476925 * b);
  }
};

}  // namespace

int ref_case_synth(std::uint32_t tiles_x, std::uint32_t tiles_y, std::uint32_t nodes, std::uint32_t intra,
                   std::uint32_t inter, std::uint32_t span_count, const std::uint32_t* spans,
                   std::uint32_t cost_kind, std::uint32_t cost_lo, std::uint32_t cost_hi, float intra_base,
                   const float* span_base, float sigma, std::uint64_t seed) {
  return guarded([&] {
    if (tiles_x == 0 || tiles_y == 0 || nodes < 2 || span_count == 0 || span_count > 8) {
      throw std::invalid_argument{"bad synthetic graph parameters"};
    }
    std::uint32_t w = nodes, h = 1;
    if (nodes == 128U) {
      w = 16;
      h = 8;
    } else {
      const auto r = static_cast<std::uint32_t>(std::lround(std::sqrt(static_cast<double>(nodes))));
      if (r * r == nodes) w = h = r;
    }
    const std::uint64_t V = std::uint64_t{tiles_x} * tiles_y * nodes;
    std::vector<VertexMetadata> vertices;
    vertices.reserve(V);
    std::vector<EdgeInputRecord> edges;
    edges.reserve(V * (intra + inter));
    SynthRng rng(seed);
    auto draw_cost = [&](int span) -> float {
      if (cost_kind == 0U) return static_cast<float>(cost_lo + rng.uniform(cost_hi - cost_lo + 1U));
      const double base = span < 0 ? intra_base : span_base[span];
      return static_cast<float>(base * std::exp(static_cast<double>(sigma) * rng.gauss()));
    };
    const int step_x[4] = {1, -1, 0, 0};
    const int step_y[4] = {0, 0, 1, -1};
    std::uint64_t record = 0;
    for (std::uint32_t ty = 0; ty < tiles_y; ++ty) {
      for (std::uint32_t tx = 0; tx < tiles_x; ++tx) {
        const std::uint64_t tile = std::uint64_t{ty} * tiles_x + tx;
        for (std::uint32_t i = 0; i < nodes; ++i) {
          const std::uint64_t v = tile * nodes + i;
          vertices.push_back(VertexMetadata::located(static_cast<std::int32_t>(tx * w + i % w),
                                                     static_cast<std::int32_t>(ty * h + i / w), ResourceClassId{1U}));
          for (std::uint32_t j = 0; j < intra; ++j) {
            std::uint32_t other = rng.uniform(nodes - 1U);
            other += other >= i ? 1U : 0U;
            const float c = draw_cost(-1);
            edges.push_back(EdgeInputRecord{VertexId{static_cast<std::uint32_t>(v)},
                                            VertexId{static_cast<std::uint32_t>(tile * nodes + other)}, c,
                                            PhysicalProvenance{1U, 1U, record++}});
          }
          for (std::uint32_t j = 0; j < inter; ++j) {
            std::int64_t nx = 0, ny = 0;
            std::uint32_t si = 0;
            bool inside = false;
            for (int attempt = 0; attempt < 16 && !inside; ++attempt) {
              const std::uint32_t dir = rng.uniform(4U);
              si = rng.uniform(span_count);
              nx = static_cast<std::int64_t>(tx) + step_x[dir] * static_cast<std::int64_t>(spans[si]);
              ny = static_cast<std::int64_t>(ty) + step_y[dir] * static_cast<std::int64_t>(spans[si]);
              inside = nx >= 0 && ny >= 0 && nx < tiles_x && ny < tiles_y;
            }
            nx = std::clamp<std::int64_t>(nx, 0, tiles_x - 1);
            ny = std::clamp<std::int64_t>(ny, 0, tiles_y - 1);
            const std::uint64_t other_tile = static_cast<std::uint64_t>(ny) * tiles_x + static_cast<std::uint64_t>(nx);
            const std::uint32_t node = rng.uniform(nodes);
            const float c = draw_cost(static_cast<int>(si));
            edges.push_back(EdgeInputRecord{VertexId{static_cast<std::uint32_t>(v)},
                                            VertexId{static_cast<std::uint32_t>(other_tile * nodes + node)}, c,
                                            PhysicalProvenance{1U, 1U, record++}});
          }
        }
      }
    }
    InputGraph input{std::move(vertices), std::move(edges)};
    const UniformGridPartitioner part{SpatialOrderConfig{0, 0, w, h}};
    return store(from_partitioned("synthetic", part.partition(input)));
  });
}

// CPU baseline over several timed steps: the induced graphs of the listed
// queries are built once (in parallel; their wall time goes to
// *induced_wall_seconds), then `warmup` untimed and `steps` timed passes run
// dijkstra_oracle over all of them, one query at a time per host thread.
// step_seconds[i] receives the wall time of timed pass i; *edges_out the
// summed induced edge counts.  dist_out (optional, nq x V floats) receives
// each query's distances of the last pass, mapped back to global ids (+inf
// outside the selected tiles).
int ref_time_dijkstra_steps(int h, std::uint32_t nq, const std::uint32_t* qidx, std::uint32_t threads,
                            std::uint32_t warmup, std::uint32_t steps, double* step_seconds,
                            double* induced_wall_seconds, std::uint64_t* edges_out, float* dist_out) {
  return guarded([&]() -> int {
    RefCase* c = get(h);
    if (!c) throw std::invalid_argument{"bad handle"};
    if (threads == 0) threads = 1;
    const WeightedGraph& g = c->partitioned->graph;
    std::vector<std::optional<InducedQueryGraph>> induced(nq);
    auto run_pool = [&](auto&& body) {
      std::atomic<std::uint32_t> next{0U};
      std::vector<std::thread> pool;
      for (std::uint32_t t = 0; t < threads; ++t) {
        pool.emplace_back([&] {
          for (std::uint32_t i; (i = next.fetch_add(1U)) < nq;) body(i);
        });
      }
      for (auto& th : pool) th.join();
    };
    const auto t0 = std::chrono::steady_clock::now();
    run_pool([&](std::uint32_t i) { induced[i].emplace(build_induced_query_graph(g, c->queries.at(qidx[i]))); });
    if (induced_wall_seconds) {
      *induced_wall_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    std::uint64_t edges = 0;
    for (const auto& ig : induced) edges += ig->graph.edge_count();
    if (edges_out) *edges_out = edges;
    for (std::uint32_t pass = 0; pass < warmup + steps; ++pass) {
      const bool last = pass + 1U == warmup + steps;
      const auto a = std::chrono::steady_clock::now();
      run_pool([&](std::uint32_t i) {
        const SsspResult res = dijkstra_oracle(induced[i]->graph, induced[i]->sources);
        if (last && dist_out) {
          float* d = dist_out + std::uint64_t{i} * g.vertex_count();
          std::fill(d, d + g.vertex_count(), std::numeric_limits<float>::infinity());
          for (std::size_t l = 0; l < induced[i]->local_to_global.size(); ++l) {
            d[induced[i]->local_to_global[l].value()] = res.distances[l];
          }
        }
      });
      const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - a).count();
      if (pass >= warmup && step_seconds) step_seconds[pass - warmup] = wall;
    }
    return 0;
  });
}

int ref_fixture_count(const char* suite_c) {
  const std::string suite{suite_c};
  if (suite == "jacobi" || suite == "dense" || suite == "frontier") {
    return static_cast<int>(single_query_suite(suite).size());
  }
  if (suite == "batched_mixed" || suite == "compact_paths" || suite == "core" ||
      suite == "spatial") {
    return 1;
  }
  return 0;
}

// Builds reference fixture `index` of `suite` as a case.  Single-query suites
// carry one query; "batched_mixed" carries the five-lane overlap fixture
// (tests/batched_jacobi_fixture_suite.hpp:57); "compact_paths" the five
// compact-path queries (tests/compact_paths_fixture_suite.hpp:45).
int ref_case_fixture(const char* suite_c, int index) {
  return guarded([&]() -> int {
    const std::string suite{suite_c};
    if (suite == "jacobi" || suite == "dense" || suite == "frontier") {
      auto cases = single_query_suite(suite);
      if (index < 0 || static_cast<std::size_t>(index) >= cases.size()) {
        throw std::out_of_range{"fixture index"};
      }
      test::JacobiFixtureCase& fc = cases[static_cast<std::size_t>(index)];
      auto c = from_partitioned(fc.name, std::move(fc.partitioned));
      c->queries.push_back(std::move(fc.query));
      c->expected_reached = fc.expected_reached_mask;
      c->expected_miss = fc.expected_miss_mask;
      c->four_ulps = fc.comparison == test::JacobiComparisonPolicy::four_ulps;
      return store(std::move(c));
    }
    if (suite == "batched_mixed") {
      test::BatchedJacobiFixture f = test::make_mixed_duration_batched_jacobi_fixture();
      auto c = from_partitioned("batched_mixed", std::move(f.partitioned));
      c->queries = std::move(f.queries);
      return store(std::move(c));
    }
    if (suite == "compact_paths") {
      test::CompactPathFixture f = test::make_compact_path_fixture();
      auto c = from_partitioned("compact_paths", std::move(f.partitioned));
      c->queries.push_back(std::move(f.cycle_query));
      c->queries.push_back(std::move(f.tie_query));
      c->queries.push_back(std::move(f.bounded_query));
      c->queries.push_back(std::move(f.multisource_query));
      c->queries.push_back(std::move(f.unreachable_query));
      return store(std::move(c));
    }
    throw std::invalid_argument{"unknown fixture suite"};
  });
}

const char* ref_case_name(int h) {
  RefCase* c = get(h);
  return c ? c->name.c_str() : "";
}

void ref_case_free(int h) {
  std::lock_guard<std::mutex> lock(g_mutex);
  if (h >= 0 && static_cast<std::size_t>(h) < g_cases.size()) {
    g_cases[static_cast<std::size_t>(h)].reset();
  }
}

// out: V, E, T, csr_runs, csc_runs, queries, expected_reached, expected_miss, four_ulps
int ref_case_counts(int h, std::uint64_t* out) {
  RefCase* c = get(h);
  if (!c) return -1;
  out[0] = c->layout.vertex_count;
  out[1] = c->layout.edge_count;
  out[2] = c->layout.tile_count;
  out[3] = c->layout.csr_run_destination_tiles.size();
  out[4] = c->layout.csc_run_source_tiles.size();
  out[5] = c->queries.size();
  out[6] = c->expected_reached;
  out[7] = c->expected_miss;
  out[8] = c->four_ulps;
  return 0;
}

// Exports the reference's DeviceGraphLayout32 plus host-only extras:
// csr_edge_ids (WeightedGraph::outgoing().edge_ids), new_to_old, the tile
// coordinate table and tile_vertex_offsets.
int ref_case_layout(
    int h, std::uint32_t* owner_tiles,
    std::uint32_t* csr_row_offsets, std::uint32_t* csr_destinations,
    float* csr_weights, std::uint32_t* csr_row_run_offsets,
    std::uint32_t* csr_run_edge_offsets, std::uint32_t* csr_run_destination_tiles,
    std::uint32_t* csc_column_offsets, std::uint32_t* csc_sources,
    float* csc_weights, std::uint32_t* csc_edge_ids,
    std::uint32_t* csc_column_run_offsets, std::uint32_t* csc_run_edge_offsets,
    std::uint32_t* csc_run_source_tiles, std::uint32_t* csr_edge_ids,
    std::uint32_t* new_to_old, std::int64_t* tile_xy, std::uint8_t* tile_has_loc,
    std::uint32_t* tile_vertex_offsets) {
  RefCase* c = get(h);
  if (!c) return -1;
  const DeviceGraphLayout32& L = c->layout;
  copy_out(owner_tiles, L.owner_tiles);
  copy_out(csr_row_offsets, L.csr_row_offsets);
  copy_out(csr_destinations, L.csr_destinations);
  copy_out(csr_weights, L.csr_weights);
  copy_out(csr_row_run_offsets, L.csr_row_run_offsets);
  copy_out(csr_run_edge_offsets, L.csr_run_edge_offsets);
  copy_out(csr_run_destination_tiles, L.csr_run_destination_tiles);
  copy_out(csc_column_offsets, L.csc_column_offsets);
  copy_out(csc_sources, L.csc_sources);
  copy_out(csc_weights, L.csc_weights);
  copy_out(csc_edge_ids, L.csc_edge_ids);
  copy_out(csc_column_run_offsets, L.csc_column_run_offsets);
  copy_out(csc_run_edge_offsets, L.csc_run_edge_offsets);
  copy_out(csc_run_source_tiles, L.csc_run_source_tiles);
  copy_out(csr_edge_ids, c->csr_edge_ids);
  const WeightedGraph& g = c->partitioned->graph;
  if (new_to_old) {
    for (std::size_t i = 0; i < g.new_to_old().size(); ++i) new_to_old[i] = g.new_to_old()[i].value();
  }
  const auto tiles = g.tile_coordinates();
  for (std::size_t t = 0; t < tiles.size(); ++t) {
    if (tile_xy) {
      tile_xy[2 * t] = tiles[t].tile_x;
      tile_xy[2 * t + 1] = tiles[t].tile_y;
    }
    if (tile_has_loc) tile_has_loc[t] = tiles[t].has_location ? 1U : 0U;
  }
  if (tile_vertex_offsets) {
    const auto off = g.tile_vertex_offsets();
    for (std::size_t t = 0; t < off.size(); ++t) tile_vertex_offsets[t] = static_cast<std::uint32_t>(off[t]);
  }
  return 0;
}

// Adds a query with explicitly selected tiles (sorted/deduplicated here), as
// the reference fixture helper with_exact_selected_tiles does
// (tests/batched_jacobi_fixture_suite.hpp:34).  n_tiles == 0 selects every
// tile of the graph (make_full_region_query, tests/jacobi_fixture_suite.hpp:64).
int ref_query_add(int h, std::uint32_t qid, std::uint32_t ns, const std::uint32_t* srcs,
                  std::uint32_t nt, const std::uint32_t* tgts, std::uint32_t ntiles,
                  const std::uint32_t* tiles) {
  return guarded([&]() -> int {
    RefCase* c = get(h);
    if (!c) throw std::invalid_argument{"bad handle"};
    const WeightedGraph& g = c->partitioned->graph;
    std::vector<VertexId> s, t;
    for (std::uint32_t i = 0; i < ns; ++i) s.push_back(VertexId{srcs[i]});
    for (std::uint32_t i = 0; i < nt; ++i) t.push_back(VertexId{tgts[i]});
    RouteQuery q = make_route_query(QueryId{qid}, g, s, t, 0U);
    std::vector<TileId> sel;
    if (ntiles == 0) {
      for (std::size_t i = 0; i < g.tile_coordinates().size(); ++i) sel.push_back(TileId{static_cast<std::uint32_t>(i)});
    } else {
      for (std::uint32_t i = 0; i < ntiles; ++i) sel.push_back(TileId{tiles[i]});
    }
    c->queries.push_back(test::with_exact_selected_tiles(std::move(q), std::move(sel), g));
    return static_cast<int>(c->queries.size() - 1U);
  });
}

// Adds a query whose selected tiles come from make_route_query with padding
// (src/query.cpp:64-118).
int ref_query_add_padded(int h, std::uint32_t qid, std::uint32_t ns, const std::uint32_t* srcs,
                         std::uint32_t nt, const std::uint32_t* tgts, std::uint32_t padding) {
  return guarded([&]() -> int {
    RefCase* c = get(h);
    if (!c) throw std::invalid_argument{"bad handle"};
    std::vector<VertexId> s, t;
    for (std::uint32_t i = 0; i < ns; ++i) s.push_back(VertexId{srcs[i]});
    for (std::uint32_t i = 0; i < nt; ++i) t.push_back(VertexId{tgts[i]});
    c->queries.push_back(make_route_query(QueryId{qid}, c->partitioned->graph, s, t, padding));
    return static_cast<int>(c->queries.size() - 1U);
  });
}

// out: query_id, n_sources, n_targets, n_selected_tiles
int ref_query_counts(int h, int q, std::uint32_t* out) {
  RefCase* c = get(h);
  if (!c || q < 0 || static_cast<std::size_t>(q) >= c->queries.size()) return -1;
  const RouteQuery& r = c->queries[static_cast<std::size_t>(q)];
  out[0] = r.query_id.value();
  out[1] = static_cast<std::uint32_t>(r.sources.size());
  out[2] = static_cast<std::uint32_t>(r.targets.size());
  out[3] = static_cast<std::uint32_t>(r.selected_tiles.size());
  return 0;
}

int ref_query_export(int h, int q, std::uint32_t* srcs, std::uint32_t* tgts, std::uint32_t* tiles) {
  RefCase* c = get(h);
  if (!c || q < 0 || static_cast<std::size_t>(q) >= c->queries.size()) return -1;
  const RouteQuery& r = c->queries[static_cast<std::size_t>(q)];
  for (std::size_t i = 0; i < r.sources.size(); ++i) srcs[i] = r.sources[i].value();
  for (std::size_t i = 0; i < r.targets.size(); ++i) tgts[i] = r.targets[i].value();
  for (std::size_t i = 0; i < r.selected_tiles.size(); ++i) tiles[i] = r.selected_tiles[i].value();
  return 0;
}

// Bounded Dijkstra on the query's induced graph, mapped back to global ids;
// vertices outside the selected tiles are +inf.  This is exactly the
// reference tests' oracle (tests/batched_frontier_push_test.cpp:55).
int ref_dijkstra(int h, int q, float* dist) {
  return guarded([&]() -> int {
    RefCase* c = get(h);
    if (!c) throw std::invalid_argument{"bad handle"};
    const WeightedGraph& g = c->partitioned->graph;
    const RouteQuery& r = c->queries.at(static_cast<std::size_t>(q));
    const InducedQueryGraph induced = build_induced_query_graph(g, r);
    const SsspResult res = dijkstra_oracle(induced.graph, induced.sources);
    for (std::uint32_t v = 0; v < g.vertex_count(); ++v) dist[v] = std::numeric_limits<float>::infinity();
    for (std::size_t l = 0; l < induced.local_to_global.size(); ++l) {
      dist[induced.local_to_global[l].value()] = res.distances[l];
    }
    return 0;
  });
}

// Synchronous Bellman-Ford on the induced graph (same mapping as above).
int ref_bellman_ford(int h, int q, float* dist) {
  return guarded([&]() -> int {
    RefCase* c = get(h);
    if (!c) throw std::invalid_argument{"bad handle"};
    const WeightedGraph& g = c->partitioned->graph;
    const RouteQuery& r = c->queries.at(static_cast<std::size_t>(q));
    const InducedQueryGraph induced = build_induced_query_graph(g, r);
    const SsspResult res = synchronous_bellman_ford(induced.graph, induced.sources);
    for (std::uint32_t v = 0; v < g.vertex_count(); ++v) dist[v] = std::numeric_limits<float>::infinity();
    for (std::size_t l = 0; l < induced.local_to_global.size(); ++l) {
      dist[induced.local_to_global[l].value()] = res.distances[l];
    }
    return 0;
  });
}

// Compact path reconstruction for query q from a graph-sized distance image.
// Per canonical target i: status[i] (CompactPathStatus), reached[i],
// path_len[i] (edge count); the concatenated paths go to vertices/edge_ids
// (vertices: sum(len+1), edge ids: sum(len)) when capacity allows.
// Returns total edge count, or -1.
long long ref_compact_paths(int h, int q, const float* dist, std::uint32_t* status,
                            std::uint32_t* reached, std::uint32_t* path_len,
                            std::uint32_t* vertices, std::uint64_t vcap,
                            std::uint32_t* edge_ids, std::uint64_t ecap) {
  try {
    RefCase* c = get(h);
    if (!c) throw std::invalid_argument{"bad handle"};
    const WeightedGraph& g = c->partitioned->graph;
    const RouteQuery& r = c->queries.at(static_cast<std::size_t>(q));
    std::span<const float> d{dist, g.vertex_count()};
    const CompactPathPayload p = reconstruct_compact_path_payload(g, r, d);
    std::uint64_t vo = 0, eo = 0;
    for (std::size_t i = 0; i < p.targets.size(); ++i) {
      const CompactTargetPath& t = p.targets[i];
      status[i] = static_cast<std::uint32_t>(t.summary.reconstruction);
      reached[i] = static_cast<std::uint32_t>(t.summary.reached);
      path_len[i] = t.summary.path_length;
      for (const VertexId v : t.vertices) {
        if (vertices && vo < vcap) vertices[vo] = v.value();
        ++vo;
      }
      for (const EdgeId e : t.edge_ids) {
        if (edge_ids && eo < ecap) edge_ids[eo] = static_cast<std::uint32_t>(e.value());
        ++eo;
      }
    }
    return static_cast<long long>(eo);
  } catch (const std::exception& e) {
    g_error = e.what();
    return -1;
  }
}

// Reference planner over all queries of the case.  Returns batch count.
int ref_plan(int h, std::uint32_t lane_width, std::uint32_t jn, std::uint32_t jd,
             std::uint32_t in, std::uint32_t id) {
  return guarded([&]() -> int {
    RefCase* c = get(h);
    if (!c) throw std::invalid_argument{"bad handle"};
    const WeightedGraph& g = c->partitioned->graph;
    c->regions.emplace(g, c->runs);
    c->features = make_batch_query_features(g, *c->regions, c->queries);
    BatchPlannerPolicy policy;
    policy.lane_width = lane_width;
    policy.minimum_jaccard_numerator = jn;
    policy.minimum_jaccard_denominator = jd;
    policy.maximum_union_inflation_numerator = in;
    policy.maximum_union_inflation_denominator = id;
    c->plan = make_overlapping_batch_plan(*c->regions, c->features, policy);
    return static_cast<int>(c->plan.batches.size());
  });
}

// Plan entry b: out_counts = {lane_width, valid_mask, union_tile_count};
// query index per lane (0xffffffff = padding); union tiles and lane masks;
// out_estimates = {union_vertex_count, union_edge_estimate,
// selected_lane_vertex_count, selected_lane_edge_estimate}.
int ref_plan_batch(int h, int b, std::uint32_t* out_counts, std::uint32_t* lane_query,
                   std::uint32_t* union_tiles, std::uint32_t* union_masks,
                   std::uint64_t* out_estimates) {
  RefCase* c = get(h);
  if (!c || b < 0 || static_cast<std::size_t>(b) >= c->plan.batches.size()) return -1;
  const BatchPlanEntry& e = c->plan.batches[static_cast<std::size_t>(b)];
  out_counts[0] = e.lane_width;
  out_counts[1] = e.valid_lane_mask;
  out_counts[2] = static_cast<std::uint32_t>(e.union_tiles.size());
  if (lane_query) {
    for (std::size_t l = 0; l < e.lane_width; ++l) lane_query[l] = e.query_indices_by_lane[l];
  }
  if (union_tiles) {
    for (std::size_t i = 0; i < e.union_tiles.size(); ++i) {
      union_tiles[i] = e.union_tiles[i].value();
      union_masks[i] = e.union_tile_lane_masks[i];
    }
  }
  if (out_estimates) {
    out_estimates[0] = e.union_vertex_count;
    out_estimates[1] = e.union_edge_estimate;
    out_estimates[2] = e.selected_lane_vertex_count;
    out_estimates[3] = e.selected_lane_edge_estimate;
  }
  return 0;
}

std::uint64_t ref_plan_fingerprint(int h) {
  RefCase* c = get(h);
  return c ? fingerprint_batch_plan(c->plan) : 0U;
}

// Prepares the description of plan batch b (device-materialized run masks)
// and exports: counts {lane_width, valid_mask, n_sources, n_targets,
// n_union_tiles, n_ranges}; source/target offsets (W+1 each), sources,
// targets, union tiles, dense tile lane masks (T), ranges (3 per range).
int ref_describe_batch(int h, int b, std::uint32_t* counts, std::uint32_t* source_offsets,
                       std::uint32_t* sources, std::uint32_t* target_offsets,
                       std::uint32_t* targets, std::uint32_t* union_tiles,
                       std::uint32_t* tile_lane_masks, std::uint32_t* ranges) {
  return guarded([&]() -> int {
    RefCase* c = get(h);
    if (!c) throw std::invalid_argument{"bad handle"};
    const BatchPlanEntry& e = c->plan.batches.at(static_cast<std::size_t>(b));
    BatchDeviceDescription d;
    prepare_batch_device_description(c->partitioned->graph, c->runs, c->queries, c->features, e,
                                     BatchRunRepresentation::device_materialized_run_masks, d);
    counts[0] = d.lane_width;
    counts[1] = d.valid_lane_mask;
    counts[2] = static_cast<std::uint32_t>(d.sources.size());
    counts[3] = static_cast<std::uint32_t>(d.targets.size());
    counts[4] = static_cast<std::uint32_t>(d.union_tiles.size());
    counts[5] = static_cast<std::uint32_t>(d.selected_vertex_ranges.size());
    copy_out(source_offsets, d.source_offsets);
    copy_out(sources, d.sources);
    copy_out(target_offsets, d.target_offsets);
    copy_out(targets, d.targets);
    copy_out(union_tiles, d.union_tiles);
    copy_out(tile_lane_masks, d.tile_lane_masks);
    if (ranges) {
      for (std::size_t i = 0; i < d.selected_vertex_ranges.size(); ++i) {
        ranges[3 * i] = d.selected_vertex_ranges[i].begin;
        ranges[3 * i + 1] = d.selected_vertex_ranges[i].end;
        ranges[3 * i + 2] = d.selected_vertex_ranges[i].lane_mask;
      }
    }
    return 0;
  });
}

// Runs a reference portable batched engine (engine 0 Jacobi, 1 dense,
// 2 frontier) on plan batch b, persistent control, unlimited rounds.
// distance_bits: V*W words (vertex-major, contiguous lanes); status: the 48-byte
// DeviceRunStatus image.
int ref_run_batched(int h, int b, int engine, std::uint64_t max_rounds,
                    std::uint32_t* distance_bits, void* status48) {
  return guarded([&]() -> int {
    RefCase* c = get(h);
    if (!c) throw std::invalid_argument{"bad handle"};
    const BatchPlanEntry& e = c->plan.batches.at(static_cast<std::size_t>(b));
    BatchDeviceDescription d;
    prepare_batch_device_description(c->partitioned->graph, c->runs, c->queries, c->features, e,
                                     BatchRunRepresentation::retained_per_run_masks, d);
    GpuRunOptions o;
    o.engine = static_cast<EngineKind>(engine);
    o.control_mode = ControlMode::persistent_cooperative;
    o.maximum_rounds = max_rounds;
    DeviceRunStatus st{};
    std::vector<std::uint32_t> bits;
    if (engine == 2) {
      const auto r = run_host_batched_frontier_push(c->layout, c->queries, e, d, o);
      st = r.result.status;
      bits = r.distance_bits;
    } else if (engine == 1) {
      const auto r = run_host_batched_dense_chaotic_push(c->layout, c->queries, e, d, o);
      st = r.result.status;
      bits = r.distance_bits;
    } else {
      const auto r = run_host_batched_jacobi_pull(c->layout, c->queries, e, d, o);
      st = r.result.status;
      for (const float f : r.final_distances) bits.push_back(std::bit_cast<std::uint32_t>(f));
    }
    copy_out(distance_bits, bits);
    std::memcpy(status48, &st, sizeof(st));
    return 0;
  });
}

// CPU baseline: bounded Dijkstra for the listed queries.  The induced graphs
// are built first (in parallel, not in the returned time); then
// dijkstra_oracle runs one query at a time per host thread over `threads`
// threads.  Returns the wall seconds of the Dijkstra phase; induced_seconds
// receives the summed induced-graph build time, sssp_seconds the summed
// per-query Dijkstra time, edges_out the summed induced edge counts.
double ref_time_dijkstra(int h, std::uint32_t nq, const std::uint32_t* qidx,
                         std::uint32_t threads, double* induced_seconds,
                         double* sssp_seconds, std::uint64_t* edges_out) {
  RefCase* c = get(h);
  if (!c) return -1.0;
  const WeightedGraph& g = c->partitioned->graph;
  std::vector<double> ind(threads, 0.0), ss(threads, 0.0);
  std::vector<std::uint64_t> edges(threads, 0U);
  // Phase 1 (untimed by the caller's figure): induced graphs, in parallel.
  std::vector<std::optional<InducedQueryGraph>> induced(nq);
  {
    std::atomic<std::uint32_t> next{0U};
    std::vector<std::thread> pool;
    for (std::uint32_t t = 0; t < threads; ++t) {
      pool.emplace_back([&, t] {
        for (;;) {
          const std::uint32_t i = next.fetch_add(1U);
          if (i >= nq) break;
          const auto a = std::chrono::steady_clock::now();
          induced[i].emplace(build_induced_query_graph(g, c->queries[qidx[i]]));
          ind[t] += std::chrono::duration<double>(std::chrono::steady_clock::now() - a).count();
          edges[t] += induced[i]->graph.edge_count();
        }
      });
    }
    for (auto& th : pool) th.join();
  }
  // Phase 2 (the returned wall time): dijkstra_oracle, one query per thread.
  std::atomic<std::uint32_t> next{0U};
  const auto t0 = std::chrono::steady_clock::now();
  std::vector<std::thread> pool;
  for (std::uint32_t t = 0; t < threads; ++t) {
    pool.emplace_back([&, t] {
      for (;;) {
        const std::uint32_t i = next.fetch_add(1U);
        if (i >= nq) break;
        const auto b = std::chrono::steady_clock::now();
        const SsspResult res = dijkstra_oracle(induced[i]->graph, induced[i]->sources);
        ss[t] += std::chrono::duration<double>(std::chrono::steady_clock::now() - b).count();
        (void)res;
      }
    });
  }
  for (auto& th : pool) th.join();
  const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  double si = 0, sd = 0;
  std::uint64_t se = 0;
  for (std::uint32_t t = 0; t < threads; ++t) {
    si += ind[t];
    sd += ss[t];
    se += edges[t];
  }
  if (induced_seconds) *induced_seconds = si;
  if (sssp_seconds) *sssp_seconds = sd;
  if (edges_out) *edges_out = se;
  return wall;
}

// Reference expansion loop (run_host_batched_expansion) over all queries of
// the case.  params = {engine, lane_width, jn, jd, in, id, schedule_kind,
// fixed_ring_size, hybrid_count, maximum_expansions, terminal_policy}.
// Per outcome (query-id order) out_outcomes receives 12 u64 fields:
// {query_id, disposition, attempts, scheduled, total, fallback, generation,
// tile_count, vertex_count, edge_count, stop_reason, error_bits};
// out_tiles the concatenated final tiles (capacity tile_cap); out_metrics
// 24 u64 counters in bfx_expansion_metrics order; out_hist up to 64 entries
// (count in out_counts[1]).  out_counts[0] = total tiles written.
int ref_expansion_run(int h, const std::uint64_t* params, std::uint64_t max_rounds, std::uint64_t* out_outcomes,
                      std::uint32_t* out_tiles, std::uint64_t tile_cap, std::uint64_t* out_metrics,
                      std::uint64_t* out_hist, std::uint64_t* out_counts) {
  return guarded([&]() -> int {
    RefCase* c = get(h);
    if (!c) throw std::invalid_argument{"bad handle"};
    const WeightedGraph& g = c->partitioned->graph;
    BatchedExpansionOptions o;
    o.run_options.engine = static_cast<EngineKind>(params[0]);
    o.run_options.maximum_rounds = max_rounds;
    o.planner_policy.lane_width = static_cast<std::uint32_t>(params[1]);
    o.planner_policy.minimum_jaccard_numerator = static_cast<std::uint32_t>(params[2]);
    o.planner_policy.minimum_jaccard_denominator = static_cast<std::uint32_t>(params[3]);
    o.planner_policy.maximum_union_inflation_numerator = static_cast<std::uint32_t>(params[4]);
    o.planner_policy.maximum_union_inflation_denominator = static_cast<std::uint32_t>(params[5]);
    o.execution_configuration_fingerprint = 1U;
    o.schedule.kind = static_cast<ExpansionScheduleKind>(params[6]);
    o.schedule.fixed_ring_size = static_cast<std::uint32_t>(params[7]);
    o.schedule.hybrid_small_expansion_count = static_cast<std::uint32_t>(params[8]);
    o.maximum_expansions = static_cast<std::uint32_t>(params[9]);
    o.terminal_policy = static_cast<ExpansionTerminalPolicy>(params[10]);
    const BatchedExpansionRunResult r =
        run_host_batched_expansion(g, c->partitioned->tiles, c->runs, c->layout, c->queries, o);
    std::uint64_t tiles_written = 0;
    for (std::size_t i = 0; i < r.queries.size(); ++i) {
      const ExpansionQueryOutcome& q = r.queries[i];
      std::uint64_t* f = out_outcomes + 12 * i;
      f[0] = q.final_query.query_id.value();
      f[1] = static_cast<std::uint64_t>(q.disposition);
      f[2] = q.attempts;
      f[3] = q.scheduled_expansions;
      f[4] = q.total_expansions;
      f[5] = q.used_full_region_fallback ? 1U : 0U;
      f[6] = q.final_query.expansion_generation;
      f[7] = q.final_query.selected_tiles.size();
      f[8] = q.selected_vertex_count;
      f[9] = q.selected_edge_count;
      f[10] = q.terminal_stop_reason;
      f[11] = q.terminal_error_bits;
      for (const TileId t : q.final_query.selected_tiles) {
        if (tiles_written >= tile_cap) throw std::length_error{"tile buffer too small"};
        out_tiles[tiles_written++] = t.value();
      }
    }
    const BatchedExpansionMetrics& m = r.metrics;
    const std::uint64_t mv[24] = {m.input_queries, m.initial_reached_queries, m.reached_queries,
                                  m.unreachable_full_region_queries, m.expansion_limit_queries,
                                  m.stalled_region_queries, m.identity_or_count_overflow_queries,
                                  m.engine_failure_queries, m.planning_passes, m.batches_executed,
                                  m.initial_batches_executed, m.retry_batches_executed, m.failed_lane_observations,
                                  m.failed_origin_valid_lane_observations, m.retry_valid_lane_observations,
                                  m.retry_lane_capacity, m.scheduled_expansions, m.full_region_fallbacks,
                                  m.repeated_selected_edge_estimate, m.attempted_selected_vertex_count,
                                  m.attempted_selected_edge_estimate, m.final_selected_tile_count,
                                  m.final_selected_vertex_count, m.final_selected_edge_count};
    std::memcpy(out_metrics, mv, sizeof(mv));
    const std::size_t nh = std::min<std::size_t>(m.expansion_count_histogram.size(), 64U);
    for (std::size_t i = 0; i < nh; ++i) out_hist[i] = m.expansion_count_histogram[i];
    out_counts[0] = tiles_written;
    out_counts[1] = m.expansion_count_histogram.size();
    return static_cast<int>(r.queries.size());
  });
}

}  // extern "C"
