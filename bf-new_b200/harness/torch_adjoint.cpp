// Gradient harness only: a libtorch autograd Function over the libbfx C ABI.
//
// forward(w)  -- w: float32 CPU tensor of edge weights by stable edge id.
//                Writes w into the resident graph, relaxes the workspace's
//                prepared batches and returns every target's shortest-path
//                distance (description order) as a float32 tensor.
// backward(g) -- the edge-usage adjoint: dL/dw_e = sum of g_t over targets
//                whose path uses e (bfx_edge_usage_adjoint).  Paths are
//                recomputed from the final labels on the device; nothing per
//                relaxation round is stored.
//
// The graph and workspace are libbfx handles created from Python; the
// workspace must already hold the prepared batches, and a forward's state is
// consumed by its own backward (one forward in flight per workspace).
#include <torch/extension.h>

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "bfx.h"

namespace {

void check(int rc) {
  if (rc != BFX_OK) throw std::runtime_error(std::string("libbfx: ") + bfx_last_error());
}

class ShortestPathDistances : public torch::autograd::Function<ShortestPathDistances> {
 public:
  static torch::Tensor forward(torch::autograd::AutogradContext* ctx, torch::Tensor weights, int64_t graph_handle,
                               int64_t workspace_handle, int64_t batch_count, int64_t engine) {
    auto* graph = reinterpret_cast<bfx_resident_graph*>(graph_handle);
    auto* ws = reinterpret_cast<bfx_workspace*>(workspace_handle);
    TORCH_CHECK(weights.dtype() == torch::kFloat32 && weights.device().is_cpu() && weights.dim() == 1,
                "weights must be a 1-D float32 CPU tensor indexed by stable edge id");
    uint64_t info[4];
    check(bfx_resident_graph_info(graph, info));
    TORCH_CHECK(static_cast<uint64_t>(weights.size(0)) == info[1], "one weight per edge is required");
    auto w = weights.contiguous();
    check(bfx_resident_graph_set_weights(graph, w.data_ptr<float>()));
    bfx_gpu_run_options opts{};
    opts.engine = static_cast<uint32_t>(engine);
    opts.control_mode = BFX_CONTROL_PERSISTENT_COOPERATIVE;
    opts.rounds_per_chunk = 8;
    opts.block_size = 256;
    opts.maximum_rounds = uint64_t{1} << 40;
    opts.enable_per_lane_convergence = 1;
    check(bfx_execute(ws, &opts));
    uint64_t sizes[3] = {0, 0, 0};
    // First call sizes the summary array.
    std::vector<bfx_compact_target_summary> summ(1 << 16);
    int rc = bfx_compact_path_summaries(ws, 0, static_cast<uint32_t>(batch_count), summ.data(), sizes);
    check(rc);
    TORCH_CHECK(sizes[0] <= summ.size(), "too many targets for the harness buffer");
    auto out = torch::empty({static_cast<int64_t>(sizes[0])}, torch::kFloat32);
    float* o = out.data_ptr<float>();
    for (uint64_t i = 0; i < sizes[0]; ++i) o[i] = summ[i].distance;
    ctx->saved_data["ws"] = workspace_handle;
    ctx->saved_data["edges"] = static_cast<int64_t>(info[1]);
    return out;
  }

  static torch::autograd::tensor_list backward(torch::autograd::AutogradContext* ctx,
                                               torch::autograd::tensor_list grads) {
    auto* ws = reinterpret_cast<bfx_workspace*>(ctx->saved_data["ws"].toInt());
    const int64_t edges = ctx->saved_data["edges"].toInt();
    auto g = grads[0].to(torch::kFloat32).contiguous().cpu();
    auto gw = torch::zeros({edges}, torch::kFloat32);
    check(bfx_edge_usage_adjoint(ws, g.data_ptr<float>(), gw.data_ptr<float>()));
    return {gw, torch::Tensor(), torch::Tensor(), torch::Tensor(), torch::Tensor()};
  }
};

torch::Tensor shortest_path_distances(torch::Tensor weights, int64_t graph_handle, int64_t workspace_handle,
                                      int64_t batch_count, int64_t engine) {
  return ShortestPathDistances::apply(weights, graph_handle, workspace_handle, batch_count, engine);
}

}  // namespace

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m) {
  m.def("shortest_path_distances", &shortest_path_distances,
        "Target shortest-path distances as a differentiable function of edge weights (libbfx).");
}
