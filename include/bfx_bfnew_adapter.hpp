// bf-new's batched-engine classes over libbfx: the adapter a bf-new build
// compiles (with its own include/ on the include path) and links against
// libbfx.so to run the batched relaxation on a B200 instead of the HIP
// engines.  Header-only.
//
// Replaces, with the same class shape and call pattern:
//   bfnew::hip::BatchedFrontierPushEngine   include/bfnew/hip/batched_frontier_push.hpp:91-144
//   bfnew::hip::BatchedJacobiPullEngine     include/bfnew/hip/batched_jacobi.hpp:137-200
//   bfnew::hip::BatchedDenseChaoticPushEngine include/bfnew/hip/batched_dense_chaotic_push.hpp:105-165
//   bfnew::hip::ResidentDeviceGraph::upload_once  include/bfnew/hip/runtime.hpp:238-270
// The engines take a bf-new BatchDeviceDescription (either run
// representation: libbfx derives run admission from tile_lane_masks) and
// GpuRunOptions, and return bf-new's DeviceRunStatus / CompactTargetSummary
// records, whose layouts equal libbfx's byte for byte (asserted below).
// Errors come back as the exceptions bf-new's HIP layer throws for the same
// conditions (std::invalid_argument, std::out_of_range,
// std::overflow_error, std::runtime_error for device failures).
#pragma once

#include "bfnew/batch_layout.hpp"
#include "bfnew/compact_path_types.hpp"
#include "bfnew/device_layout.hpp"
#include "bfnew/gpu_api.hpp"
#include "bfx.h"

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <span>
#include <stdexcept>
#include <string>
#include <vector>

namespace bfnew::cuda {

// ---- record layouts: bf-new's ABI records and libbfx's are the same bytes
#define BFX_SAME_FIELD(A, B, f) static_assert(offsetof(A, f) == offsetof(B, f) && sizeof(A::f) == sizeof(B::f))
static_assert(sizeof(GpuRunOptions) == sizeof(bfx_gpu_run_options) &&
              alignof(GpuRunOptions) == alignof(bfx_gpu_run_options));
BFX_SAME_FIELD(GpuRunOptions, bfx_gpu_run_options, engine);
BFX_SAME_FIELD(GpuRunOptions, bfx_gpu_run_options, control_mode);
BFX_SAME_FIELD(GpuRunOptions, bfx_gpu_run_options, rounds_per_chunk);
BFX_SAME_FIELD(GpuRunOptions, bfx_gpu_run_options, block_size);
BFX_SAME_FIELD(GpuRunOptions, bfx_gpu_run_options, grid_policy);
BFX_SAME_FIELD(GpuRunOptions, bfx_gpu_run_options, blocks_per_wgp);
BFX_SAME_FIELD(GpuRunOptions, bfx_gpu_run_options, instrumentation);
BFX_SAME_FIELD(GpuRunOptions, bfx_gpu_run_options, maximum_rounds);
BFX_SAME_FIELD(GpuRunOptions, bfx_gpu_run_options, enable_per_lane_convergence);

static_assert(sizeof(DeviceController) == sizeof(bfx_device_controller) &&
              alignof(DeviceController) == alignof(bfx_device_controller));
BFX_SAME_FIELD(DeviceController, bfx_device_controller, valid_lane_mask);
BFX_SAME_FIELD(DeviceController, bfx_device_controller, active_lane_mask);
BFX_SAME_FIELD(DeviceController, bfx_device_controller, changed_lane_mask);
BFX_SAME_FIELD(DeviceController, bfx_device_controller, converged_lane_mask);
BFX_SAME_FIELD(DeviceController, bfx_device_controller, execute_lane_mask);
BFX_SAME_FIELD(DeviceController, bfx_device_controller, engine_kind);
BFX_SAME_FIELD(DeviceController, bfx_device_controller, enable_per_lane_convergence);
BFX_SAME_FIELD(DeviceController, bfx_device_controller, rounds_completed);
BFX_SAME_FIELD(DeviceController, bfx_device_controller, maximum_rounds);
BFX_SAME_FIELD(DeviceController, bfx_device_controller, distance_read_slot);
BFX_SAME_FIELD(DeviceController, bfx_device_controller, distance_write_slot);
BFX_SAME_FIELD(DeviceController, bfx_device_controller, frontier_read_slot);
BFX_SAME_FIELD(DeviceController, bfx_device_controller, frontier_write_slot);
BFX_SAME_FIELD(DeviceController, bfx_device_controller, frontier_size);
BFX_SAME_FIELD(DeviceController, bfx_device_controller, next_frontier_lane_mask);
BFX_SAME_FIELD(DeviceController, bfx_device_controller, done);
BFX_SAME_FIELD(DeviceController, bfx_device_controller, stop_reason);
BFX_SAME_FIELD(DeviceController, bfx_device_controller, error_bits);

static_assert(sizeof(DeviceRunStatus) == sizeof(bfx_device_run_status) &&
              alignof(DeviceRunStatus) == alignof(bfx_device_run_status));
BFX_SAME_FIELD(DeviceRunStatus, bfx_device_run_status, final_distance_slot);
BFX_SAME_FIELD(DeviceRunStatus, bfx_device_run_status, converged);
BFX_SAME_FIELD(DeviceRunStatus, bfx_device_run_status, rounds_completed);
BFX_SAME_FIELD(DeviceRunStatus, bfx_device_run_status, reached_target_mask);
BFX_SAME_FIELD(DeviceRunStatus, bfx_device_run_status, bounding_box_miss_mask);
BFX_SAME_FIELD(DeviceRunStatus, bfx_device_run_status, valid_lane_mask);
BFX_SAME_FIELD(DeviceRunStatus, bfx_device_run_status, active_lane_mask);
BFX_SAME_FIELD(DeviceRunStatus, bfx_device_run_status, converged_lane_mask);
BFX_SAME_FIELD(DeviceRunStatus, bfx_device_run_status, stop_reason);
BFX_SAME_FIELD(DeviceRunStatus, bfx_device_run_status, error_bits);

static_assert(sizeof(DeviceWorkStatistics) == sizeof(bfx_device_work_statistics));
BFX_SAME_FIELD(DeviceWorkStatistics, bfx_device_work_statistics, edges_examined);
BFX_SAME_FIELD(DeviceWorkStatistics, bfx_device_work_statistics, kernel_dispatches);
BFX_SAME_FIELD(DeviceWorkStatistics, bfx_device_work_statistics, small_frontier_rounds);

static_assert(sizeof(BatchVertexRange) == sizeof(bfx_batch_vertex_range));
BFX_SAME_FIELD(BatchVertexRange, bfx_batch_vertex_range, begin);
BFX_SAME_FIELD(BatchVertexRange, bfx_batch_vertex_range, end);
BFX_SAME_FIELD(BatchVertexRange, bfx_batch_vertex_range, lane_mask);

static_assert(sizeof(CompactTargetSummary) == sizeof(bfx_compact_target_summary));
static_assert(offsetof(CompactTargetSummary, target) == offsetof(bfx_compact_target_summary, target));
static_assert(offsetof(CompactTargetSummary, selected_source) ==
              offsetof(bfx_compact_target_summary, selected_source));
static_assert(offsetof(CompactTargetSummary, distance) == offsetof(bfx_compact_target_summary, distance));
static_assert(offsetof(CompactTargetSummary, path_length) == offsetof(bfx_compact_target_summary, path_length));
static_assert(offsetof(CompactTargetSummary, reached) == offsetof(bfx_compact_target_summary, reached));
static_assert(offsetof(CompactTargetSummary, reconstruction) ==
              offsetof(bfx_compact_target_summary, reconstruction));
static_assert(offsetof(CompactTargetSummary, has_selected_source) ==
              offsetof(bfx_compact_target_summary, has_selected_source));
#undef BFX_SAME_FIELD

// ---- enumerations: the same values
static_assert(static_cast<std::uint32_t>(EngineKind::jacobi_pull) == BFX_ENGINE_JACOBI_PULL);
static_assert(static_cast<std::uint32_t>(EngineKind::dense_chaotic_push) == BFX_ENGINE_DENSE_CHAOTIC_PUSH);
static_assert(static_cast<std::uint32_t>(EngineKind::frontier_push) == BFX_ENGINE_FRONTIER_PUSH);
static_assert(static_cast<std::uint32_t>(ControlMode::persistent_cooperative) == BFX_CONTROL_PERSISTENT_COOPERATIVE);
static_assert(static_cast<std::uint32_t>(ControlMode::chunked_host_poll) == BFX_CONTROL_CHUNKED_HOST_POLL);
static_assert(static_cast<std::uint32_t>(ControlMode::per_round_host_poll) == BFX_CONTROL_PER_ROUND_HOST_POLL);

// libbfx status -> the exception bf-new raises for the same condition.
inline void check(int rc) {
  if (rc == BFX_OK) return;
  const std::string m = bfx_last_error();
  switch (rc) {
    case BFX_ERR_INVALID_ARGUMENT: throw std::invalid_argument(m);
    case BFX_ERR_OUT_OF_RANGE: throw std::out_of_range(m);
    case BFX_ERR_OVERFLOW: throw std::overflow_error(m);
    case BFX_ERR_STATE: throw std::logic_error(m);
    default: throw std::runtime_error(m);  // CUDA, no device, out of memory: HipRuntimeError's role
  }
}

// The flattened view libbfx reads: pointers into the description's vectors,
// which must outlive the call.
inline bfx_batch_description flatten(const BatchDeviceDescription& d) {
  if (d.selected_vertex_ranges.size() != d.union_tiles.size()) {
    throw std::invalid_argument("batch description needs one vertex range per union tile");
  }
  bfx_batch_description c{};
  c.lane_width = d.lane_width;
  c.valid_lane_mask = d.valid_lane_mask;
  c.source_offsets = d.source_offsets.data();
  c.sources = d.sources.data();
  c.target_offsets = d.target_offsets.data();
  c.targets = d.targets.data();
  c.union_tile_count = static_cast<std::uint32_t>(d.union_tiles.size());
  c.tile_count = static_cast<std::uint32_t>(d.tile_lane_masks.size());
  c.union_tiles = d.union_tiles.data();
  c.tile_lane_masks = d.tile_lane_masks.data();
  c.range_count = static_cast<std::uint32_t>(d.selected_vertex_ranges.size());
  c.selected_vertex_ranges = reinterpret_cast<const bfx_batch_vertex_range*>(d.selected_vertex_ranges.data());
  return c;
}

// The graph resident on one device (upload_once; immutable afterwards).
class ResidentDeviceGraph {
 public:
  // csr_edge_ids: WeightedGraph::outgoing().edge_ids narrowed to 32 bits, or
  // empty to let libbfx derive them from the CSC image.
  explicit ResidentDeviceGraph(const DeviceGraphLayout32& L, std::span<const std::uint32_t> csr_edge_ids = {},
                               int device = 0) {
    bfx_device_graph_layout32 v{};
    v.vertex_count = L.vertex_count;
    v.edge_count = L.edge_count;
    v.tile_count = L.tile_count;
    v.csr_run_count = static_cast<std::uint32_t>(L.csr_run_destination_tiles.size());
    v.csc_run_count = static_cast<std::uint32_t>(L.csc_run_source_tiles.size());
    v.owner_tiles = L.owner_tiles.data();
    v.csr_row_offsets = L.csr_row_offsets.data();
    v.csr_destinations = L.csr_destinations.data();
    v.csr_weights = L.csr_weights.data();
    v.csr_row_run_offsets = L.csr_row_run_offsets.data();
    v.csr_run_edge_offsets = L.csr_run_edge_offsets.data();
    v.csr_run_destination_tiles = L.csr_run_destination_tiles.data();
    v.csc_column_offsets = L.csc_column_offsets.data();
    v.csc_sources = L.csc_sources.data();
    v.csc_weights = L.csc_weights.data();
    v.csc_edge_ids = L.csc_edge_ids.data();
    v.csc_column_run_offsets = L.csc_column_run_offsets.data();
    v.csc_run_edge_offsets = L.csc_run_edge_offsets.data();
    v.csc_run_source_tiles = L.csc_run_source_tiles.data();
    v.csr_edge_ids = csr_edge_ids.empty() ? nullptr : csr_edge_ids.data();
    check(bfx_resident_graph_upload(&v, device, &graph_));
    vertex_count_ = L.vertex_count;
  }
  ~ResidentDeviceGraph() { bfx_resident_graph_destroy(graph_); }
  ResidentDeviceGraph(const ResidentDeviceGraph&) = delete;
  ResidentDeviceGraph& operator=(const ResidentDeviceGraph&) = delete;
  [[nodiscard]] bfx_resident_graph* get() const noexcept { return graph_; }
  [[nodiscard]] std::uint32_t vertex_count() const noexcept { return vertex_count_; }

 private:
  bfx_resident_graph* graph_{};
  std::uint32_t vertex_count_{};
};

// run_with_distances: the status and the V x W final label image
// (vertex-major, lanes contiguous; +inf outside a lane's selected tiles),
// plus the predecessor stable EdgeId per (vertex, lane) (0xffffffff for
// sources and unreached vertices).
struct BatchedDistanceOutput {
  DeviceRunStatus status{};
  std::vector<std::uint32_t> distance_bits;
  std::vector<std::uint32_t> predecessor_edges;
};

// run_compact_paths: one summary per target of the batch (description
// order) and the complete targets' paths concatenated in summary order.
struct BatchedCompactPathOutput {
  DeviceRunStatus status{};
  std::vector<CompactTargetSummary> summaries;
  std::vector<std::uint32_t> vertices;
  std::vector<float> distance_labels;
  std::vector<std::uint32_t> edge_ids;
};

// One engine kind behind bf-new's batched-engine calls.  Every call relaxes
// its batch set in one persistent launch on the engine's own stream; calls
// must be sequential (as for the HIP engines).  Non-owning: the resident
// graph must outlive the engine.
template <EngineKind kKind>
class BatchedEngine {
 public:
  explicit BatchedEngine(const ResidentDeviceGraph& graph) : graph_(&graph) {
    check(bfx_workspace_create(graph.get(), &ws_));
  }
  ~BatchedEngine() { bfx_workspace_destroy(ws_); }
  BatchedEngine(const BatchedEngine&) = delete;
  BatchedEngine& operator=(const BatchedEngine&) = delete;

  [[nodiscard]] static constexpr EngineKind kind() noexcept { return kKind; }

  [[nodiscard]] DeviceRunStatus run_compact_status(const BatchDeviceDescription& batch, const GpuRunOptions& options) {
    return run_compact_status(std::span<const BatchDeviceDescription>(&batch, 1), options).front();
  }

  // Several batches in one launch (bfx extension of the same call).
  [[nodiscard]] std::vector<DeviceRunStatus> run_compact_status(std::span<const BatchDeviceDescription> batches,
                                                                const GpuRunOptions& options) {
    run(batches, options);
    std::vector<DeviceRunStatus> st(batches.size());
    check(bfx_fetch_statuses(ws_, reinterpret_cast<bfx_device_run_status*>(st.data()), nullptr));
    return st;
  }

  // The reference's status-only call: the status and the final controller.
  [[nodiscard]] std::pair<DeviceRunStatus, DeviceController> run_status_only(const BatchDeviceDescription& batch,
                                                                             const GpuRunOptions& options) {
    run(std::span<const BatchDeviceDescription>(&batch, 1), options);
    DeviceRunStatus st{};
    DeviceController ctrl{};
    check(bfx_fetch_statuses(ws_, reinterpret_cast<bfx_device_run_status*>(&st),
                             reinterpret_cast<bfx_device_controller*>(&ctrl)));
    return {st, ctrl};
  }

  [[nodiscard]] BatchedDistanceOutput run_with_distances(const BatchDeviceDescription& batch,
                                                         const GpuRunOptions& options) {
    BatchedDistanceOutput out;
    out.status = run_compact_status(batch, options);
    const std::size_t n = static_cast<std::size_t>(graph_->vertex_count()) * batch.lane_width;
    out.distance_bits.resize(n);
    out.predecessor_edges.resize(n);
    check(bfx_download_labels(ws_, 0, out.distance_bits.data(), out.predecessor_edges.data()));
    return out;
  }

  [[nodiscard]] BatchedCompactPathOutput run_compact_paths(const BatchDeviceDescription& batch,
                                                           const GpuRunOptions& options) {
    BatchedCompactPathOutput out;
    out.status = run_compact_status(batch, options);
    out.summaries.resize(batch.targets.size());
    std::uint64_t sizes[3] = {0, 0, 0};
    check(bfx_compact_path_summaries(ws_, 0, 1, reinterpret_cast<bfx_compact_target_summary*>(out.summaries.data()),
                                     sizes));
    out.summaries.resize(sizes[0]);
    out.vertices.resize(sizes[1]);
    out.distance_labels.resize(sizes[1]);
    out.edge_ids.resize(sizes[2]);
    check(bfx_compact_path_payload(ws_, out.vertices.data(), out.distance_labels.data(), out.edge_ids.data()));
    return out;
  }

  [[nodiscard]] bfx_workspace* workspace() const noexcept { return ws_; }

 private:
  void run(std::span<const BatchDeviceDescription> batches, const GpuRunOptions& options) {
    std::vector<bfx_batch_description> flat;
    flat.reserve(batches.size());
    for (const BatchDeviceDescription& d : batches) flat.push_back(flatten(d));
    GpuRunOptions o = options;
    o.engine = kKind;
    check(bfx_prepare_batches(ws_, static_cast<std::uint32_t>(flat.size()), flat.data()));
    check(bfx_execute(ws_, reinterpret_cast<const bfx_gpu_run_options*>(&o)));
  }

  const ResidentDeviceGraph* graph_;
  bfx_workspace* ws_{};
};

using BatchedFrontierPushEngine = BatchedEngine<EngineKind::frontier_push>;
using BatchedJacobiPullEngine = BatchedEngine<EngineKind::jacobi_pull>;
using BatchedDenseChaoticPushEngine = BatchedEngine<EngineKind::dense_chaotic_push>;

}  // namespace bfnew::cuda
