// Test infrastructure only: runs bf-new's own batch descriptions through
// include/bfx_bfnew_adapter.hpp -- libbfx behind bf-new's batched-engine
// classes -- and compares every status and label with the reference's
// portable batched engines on the same descriptions
// (run_host_batched_{frontier_push,jacobi_pull,dense_chaotic_push},
// src/batched_frontier_push.cpp:648, src/batched_jacobi_pull.cpp:572,
// src/batched_dense_chaotic_push.cpp:569).  Built by oracle/Makefile into
// oracle/_ref/ (it needs the reference headers and library and libbfx).
// It reuses the reference driver's case registry and fixtures.
#include "ref_driver.cpp"

#include "bfx_bfnew_adapter.hpp"

#include <bit>

extern "C" {

// Without a device: the adapter turns libbfx's "no device" status into the
// std::runtime_error bf-new's HIP layer raises.  Returns 1 when it did.
int adapter_no_device_raises(int h) {
  RefCase* c = get(h);
  if (!c) return -1;
  try {
    bfnew::cuda::ResidentDeviceGraph g(c->layout, c->csr_edge_ids, 0);
    return 0;  // a device exists
  } catch (const std::runtime_error& e) {
    return std::string(e.what()).find("no CUDA device") != std::string::npos ? 1 : 2;
  } catch (...) {
    return 3;
  }
}

// The flattened view of each planned batch's reference description points
// at the description's own vectors, with the counts libbfx reads.  Returns
// the number of batches checked, or -1 on a mismatch.
int adapter_flatten_check(int h) {
  return guarded([&]() -> int {
    RefCase* c = get(h);
    if (!c) throw std::invalid_argument{"bad handle"};
    int checked = 0;
    for (const BatchPlanEntry& e : c->plan.batches) {
      BatchDeviceDescription d;
      prepare_batch_device_description(c->partitioned->graph, c->runs, c->queries, c->features, e,
                                       BatchRunRepresentation::device_materialized_run_masks, d);
      const bfx_batch_description f = bfnew::cuda::flatten(d);
      const bool ok = f.lane_width == d.lane_width && f.valid_lane_mask == d.valid_lane_mask &&
                      f.sources == d.sources.data() && f.targets == d.targets.data() &&
                      f.source_offsets == d.source_offsets.data() && f.target_offsets == d.target_offsets.data() &&
                      f.union_tile_count == d.union_tiles.size() && f.tile_count == d.tile_lane_masks.size() &&
                      f.tile_count == c->layout.tile_count && f.range_count == d.selected_vertex_ranges.size() &&
                      static_cast<const void*>(f.selected_vertex_ranges) == d.selected_vertex_ranges.data();
      if (!ok) return -1;
      ++checked;
    }
    return checked;
  });
}

// Every planned batch of case h (planned by ref_plan) through the adapter's
// `engine` on the GPU and through the reference's portable engine of the
// same kind.  out[6] = {batches, valid lanes, distance-bit mismatches,
// status-field mismatches, predecessor checks (frontier/dense: tight edge
// re-derived from the reference distances), predecessor mismatches}.
int adapter_check_plan(int h, int engine, int representation, std::uint64_t* out) {
  return guarded([&]() -> int {
    RefCase* c = get(h);
    if (!c) throw std::invalid_argument{"bad handle"};
    const WeightedGraph& g = c->partitioned->graph;
    bfnew::cuda::ResidentDeviceGraph resident(c->layout, c->csr_edge_ids, 0);
    bfnew::cuda::BatchedFrontierPushEngine frontier(resident);
    bfnew::cuda::BatchedJacobiPullEngine jacobi(resident);
    bfnew::cuda::BatchedDenseChaoticPushEngine dense(resident);
    std::uint64_t batches = 0, lanes = 0, dist_bad = 0, status_bad = 0, pred_checks = 0, pred_bad = 0;
    for (const BatchPlanEntry& e : c->plan.batches) {
      BatchDeviceDescription d;
      prepare_batch_device_description(
          g, c->runs, c->queries, c->features, e,
          representation == 0 ? BatchRunRepresentation::retained_per_run_masks
                              : BatchRunRepresentation::device_materialized_run_masks,
          d);
      GpuRunOptions o;
      o.engine = static_cast<EngineKind>(engine);
      o.control_mode = ControlMode::persistent_cooperative;
      o.maximum_rounds = std::uint64_t{1} << 40;
      bfnew::cuda::BatchedDistanceOutput gpu;
      if (engine == 2) {
        gpu = frontier.run_with_distances(d, o);
      } else if (engine == 1) {
        gpu = dense.run_with_distances(d, o);
      } else {
        gpu = jacobi.run_with_distances(d, o);
      }
      // the reference's portable engine on the retained-mask description
      BatchDeviceDescription dr;
      prepare_batch_device_description(g, c->runs, c->queries, c->features, e,
                                       BatchRunRepresentation::retained_per_run_masks, dr);
      DeviceRunStatus st{};
      std::vector<std::uint32_t> bits;
      if (engine == 2) {
        const auto r = run_host_batched_frontier_push(c->layout, c->queries, e, dr, o);
        st = r.result.status;
        bits = r.distance_bits;
      } else if (engine == 1) {
        const auto r = run_host_batched_dense_chaotic_push(c->layout, c->queries, e, dr, o);
        st = r.result.status;
        bits = r.distance_bits;
      } else {
        const auto r = run_host_batched_jacobi_pull(c->layout, c->queries, e, dr, o);
        st = r.result.status;
        for (const float f : r.final_distances) bits.push_back(std::bit_cast<std::uint32_t>(f));
      }
      const std::uint32_t W = d.lane_width, V = c->layout.vertex_count;
      if (bits.size() != std::size_t{V} * W || gpu.distance_bits.size() != bits.size()) {
        throw std::logic_error{"label image sizes differ"};
      }
      for (std::uint32_t v = 0; v < V; ++v) {
        for (std::uint32_t l = 0; l < W; ++l) {
          if (!((d.valid_lane_mask >> l) & 1U)) continue;
          const std::size_t i = std::size_t{v} * W + l;
          dist_bad += gpu.distance_bits[i] != bits[i];
        }
      }
      status_bad += gpu.status.converged != st.converged;
      status_bad += gpu.status.reached_target_mask != st.reached_target_mask;
      status_bad += gpu.status.bounding_box_miss_mask != st.bounding_box_miss_mask;
      status_bad += gpu.status.valid_lane_mask != st.valid_lane_mask;
      status_bad += gpu.status.active_lane_mask != st.active_lane_mask;
      status_bad += gpu.status.converged_lane_mask != st.converged_lane_mask;
      status_bad += gpu.status.stop_reason != st.stop_reason;
      status_bad += gpu.status.error_bits != st.error_bits;
      // predecessors: the minimum stable id among tight in-edges from a
      // selected, finite source (src/path_reconstruct.cpp:56-89), derived
      // here from the reference's distances
      const auto& in = g.incoming();
      for (std::uint32_t v = 0; v < V; ++v) {
        for (std::uint32_t l = 0; l < W; ++l) {
          if (!((d.valid_lane_mask >> l) & 1U)) continue;
          const std::size_t i = std::size_t{v} * W + l;
          const float dv = std::bit_cast<float>(bits[i]);
          if (!(dv < std::numeric_limits<float>::infinity())) continue;
          std::uint32_t best = 0xFFFFFFFFU;
          bool is_source = false;
          for (std::uint32_t k = d.source_offsets[l]; k < d.source_offsets[l + 1]; ++k) is_source |= d.sources[k] == v;
          if (!is_source) {
            for (std::size_t q = in.column_offsets[v]; q < in.column_offsets[v + 1]; ++q) {
              const std::uint32_t u = in.sources[q].value();
              const std::uint32_t tu = c->layout.owner_tiles[u];
              if (!((d.tile_lane_masks[tu] >> l) & 1U)) continue;
              const float du = std::bit_cast<float>(bits[std::size_t{u} * W + l]);
              if (!(du < std::numeric_limits<float>::infinity())) continue;
              if (du + in.weights[q] == dv) best = std::min<std::uint32_t>(best, static_cast<std::uint32_t>(in.edge_ids[q].value()));
            }
          }
          ++pred_checks;
          pred_bad += gpu.predecessor_edges[i] != best;
        }
      }
      ++batches;
      lanes += static_cast<std::uint64_t>(std::popcount(d.valid_lane_mask));
    }
    out[0] = batches;
    out[1] = lanes;
    out[2] = dist_bad;
    out[3] = status_bad;
    out[4] = pred_checks;
    out[5] = pred_bad;
    return 0;
  });
}

}  // extern "C"
