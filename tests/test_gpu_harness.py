"""Gradient harness: the libtorch torch::autograd::Function over the libbfx C
ABI (bf-new_b200/harness/torch_adjoint.cpp).  Autograd through the target
distances must give exactly bfx_edge_usage_adjoint's gradient."""
import numpy as np
import pytest
import torch

import bfx
from bfx import workloads

pytestmark = pytest.mark.gpu


def test_autograd_function_matches_adjoint(gpu):
    import importlib.util, sys
    from pathlib import Path
    spec = importlib.util.spec_from_file_location(
        "build_harness", Path(bfx.__file__).resolve().parent.parent / "harness" / "build_harness.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    harness = mod.load()

    layout, grid = workloads.build_graph("c1f")
    qs = workloads.box_queries(layout, grid, 24, 8, 32, seed=61, targets=(1, 8), clip=32)
    plan = bfx.make_overlapping_batch_plan(layout, qs, bfx.BatchPlannerPolicy(32, 0, 1, 16, 1, narrow_lanes=True))
    descs = plan.descriptions()
    res = bfx.ResidentDeviceGraph.upload_once(layout)
    ws = bfx.Workspace(res)
    ws.prepare(descs)
    w0 = np.zeros(layout.edge_count, np.float32)
    w0[layout.arrays["csr_edge_ids"]] = layout.arrays["csr_weights"]
    w = torch.tensor(w0, requires_grad=True)
    d = harness.shortest_path_distances(w, res._h.value, ws._h.value, len(descs), bfx.ENGINE_FRONTIER_PUSH)
    finite = torch.isfinite(d)
    g = torch.rand(d.shape[0], generator=torch.Generator().manual_seed(3)) * finite
    loss = (torch.where(finite, d, torch.zeros_like(d)) * g).sum()
    loss.backward()
    direct = ws.edge_usage_adjoint(g.numpy().astype(np.float32))
    np.testing.assert_array_equal(w.grad.numpy().view(np.uint32), direct.view(np.uint32))
    assert float(w.grad.sum()) > 0
    ws.close()
    res.close()
