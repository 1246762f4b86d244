"""bfx_run_query_static: the single-query entry point that allocates no device
memory (all scratch in a fixed 32 MiB array inside libbfx.so).  It serves
callers that cannot allocate while they run a query -- a process whose GPU
memory is owned by another runtime's pool, or a loop that cannot take an
allocation's synchronisation.  Its target labels must equal the oracle's and
bfx_run_query's (the workspace-backed entry point) bit for bit, on two calls
in a row, since the shared array keeps the previous call's contents; and the
device's free memory must not change across calls once the library's
kernels are loaded.

This file is collected last on purpose, so a failure here comes after every
other test has run.
"""
import ctypes as C

import numpy as np
import pytest

import bfx
from bfx import workloads
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def static_query(res, q, opts):
    lib = bfx.load()
    s = np.ascontiguousarray(q.sources, np.uint32)
    t = np.ascontiguousarray(q.targets, np.uint32)
    tl = np.ascontiguousarray(q.selected_tiles, np.uint32)
    st = bfx.DeviceRunStatus()
    bits = np.zeros(len(t), np.uint32)
    pred = np.zeros(len(t), np.uint32)
    P = C.POINTER(C.c_uint32)
    rc = lib.bfx_run_query_static(res._h, C.c_uint32(len(s)), s.ctypes.data_as(P), C.c_uint32(len(t)),
                                  t.ctypes.data_as(P), C.c_uint32(len(tl)), tl.ctypes.data_as(P), C.byref(opts),
                                  C.byref(st), bits.ctypes.data_as(P), pred.ctypes.data_as(P))
    return rc, st, bits, pred


def workspace_query(ws, q, opts):
    st = ws.run_query(q.sources, q.targets, q.selected_tiles, opts)
    labels, preds = ws.download_labels(0, 1)
    return st, labels[q.targets, 0], preds[q.targets, 0]


def free_device_bytes() -> int:
    """cudaMemGetInfo's free bytes of the current device (through the CUDA runtime)."""
    rt = C.CDLL("libcudart.so.12")
    free, total = C.c_size_t(), C.c_size_t()
    assert rt.cudaDeviceSynchronize() == 0
    assert rt.cudaMemGetInfo(C.byref(free), C.byref(total)) == 0
    return free.value


@pytest.mark.parametrize("engine", [bfx.ENGINE_FRONTIER_PUSH, bfx.ENGINE_JACOBI_PULL, bfx.ENGINE_DENSE_CHAOTIC_PUSH],
                         ids=["frontier", "jacobi", "dense"])
def test_static_scratch_query_matches_oracle_and_workspace_twice(gpu, engine):
    layout, grid = workloads.build_graph("c2", scale_tiles=(32, 32))
    qs = workloads.box_queries(layout, grid, 3, 4, 24, seed=77, targets=(2, 6))
    orc = Oracle.from_layout(layout)
    res = bfx.ResidentDeviceGraph.upload_once(layout)
    ws = bfx.Workspace(res)
    opts = bfx.GpuRunOptions(engine=engine)
    for q in qs:
        od, op = orc.region_sssp(q.sources, q.targets, q.selected_tiles)
        tg = np.asarray(q.targets, np.int64)
        ref_st, ref_bits, ref_pred = workspace_query(ws, q, opts)
        np.testing.assert_array_equal(ref_bits, od[tg])
        for _ in range(2):  # two calls in a row share the static array
            rc, st, bits, pred = static_query(res, q, opts)
            assert rc == 0, bfx.load().bfx_last_error()
            for f in ("converged", "reached_target_mask", "bounding_box_miss_mask", "valid_lane_mask",
                      "active_lane_mask", "converged_lane_mask", "stop_reason", "error_bits",
                      "final_distance_slot"):
                assert getattr(st, f) == getattr(ref_st, f), f
            assert st.stop_reason == bfx.STOP_CONVERGED
            np.testing.assert_array_equal(bits, od[tg])  # the oracle's distance bits
            np.testing.assert_array_equal(pred, op[tg])  # the oracle's min-eid tight predecessors
            np.testing.assert_array_equal(bits, ref_bits)
            np.testing.assert_array_equal(pred, ref_pred)
    ws.close()
    res.close()


def test_static_scratch_query_allocates_no_device_memory(gpu):
    layout, grid = workloads.build_graph("c2", scale_tiles=(32, 32))
    qs = workloads.box_queries(layout, grid, 4, 4, 24, seed=91, targets=(1, 4))
    res = bfx.ResidentDeviceGraph.upload_once(layout)
    opts = bfx.GpuRunOptions()
    rc, *_ = static_query(res, qs[0], opts)  # loads the kernels it uses (lazy module loading)
    assert rc == 0, bfx.load().bfx_last_error()
    before = free_device_bytes()
    for q in qs + qs:
        rc, st, _, _ = static_query(res, q, opts)
        assert rc == 0, bfx.load().bfx_last_error()
        assert st.stop_reason == bfx.STOP_CONVERGED
    assert free_device_bytes() == before
    res.close()


def test_static_scratch_rejects_host_poll_modes_and_instrumentation(gpu):
    layout, grid = workloads.build_graph("c2", scale_tiles=(16, 16))
    q = workloads.box_queries(layout, grid, 1, 4, 8, seed=3)[0]
    res = bfx.ResidentDeviceGraph.upload_once(layout)
    for opts in (bfx.GpuRunOptions(control_mode=bfx.CONTROL_CHUNKED),
                 bfx.GpuRunOptions(control_mode=bfx.CONTROL_PER_ROUND), bfx.GpuRunOptions(instrumentation=1)):
        rc, *_ = static_query(res, q, opts)
        assert rc == 1  # BFX_ERR_INVALID_ARGUMENT
    res.close()


def test_static_scratch_rejects_oversized_query(gpu):
    layout, grid = workloads.build_graph("c2", scale_tiles=(96, 96))  # 1.18M vertices > the 32 MiB limit
    q = workloads.full_graph_queries(layout, grid, 1, seed=5)[0]
    res = bfx.ResidentDeviceGraph.upload_once(layout)
    rc, st, _, _ = static_query(res, q, bfx.GpuRunOptions())
    assert rc == 3  # BFX_ERR_OVERFLOW
    assert b"32 MiB" in bfx.load().bfx_last_error()
    res.close()
