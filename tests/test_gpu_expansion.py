"""Expansion loop on the GPU (bfx_expansion_run): every planning pass is
relaxed in one launch by the batched engines and must give the same outcomes,
final regions, metrics and histogram as the loop driven by the oracle (which
tests/test_expansion.py pins to the reference's run_host_batched_expansion)."""
import pytest

import bfx
from bfx import expansion as ex
from bfx import workloads
from oracle.oracle import Oracle
from test_expansion import SCHEDULES, oracle_runner, rich_queries

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    spec = dict(workloads.GRAPHS["c1"])
    g, order, _ = bfx.synth_graph(**spec)
    layout = bfx.build_device_graph_layout(g, order)
    qs = rich_queries(layout, (spec["tiles_x"], spec["tiles_y"]), 1717)
    return layout, qs


@pytest.mark.parametrize("engine", [bfx.ENGINE_FRONTIER_PUSH, bfx.ENGINE_JACOBI_PULL, bfx.ENGINE_DENSE_CHAOTIC_PUSH])
@pytest.mark.parametrize("sched", SCHEDULES[:4], ids=lambda s: f"k{s[0]}r{s[1]}h{s[2]}m{s[3]}t{s[4]}")
def test_gpu_expansion_equals_oracle_loop(gpu, case, sched, engine):
    layout, qs = case
    kind, ring, hyb, mx, term = sched
    opts = ex.ExpansionOptions(schedule_kind=kind, fixed_ring_size=ring, hybrid_small_expansion_count=hyb,
                               maximum_expansions=mx, terminal_policy=term, engine=engine,
                               planner_policy=bfx.BatchPlannerPolicy(32, 1, 8, 2, 1, narrow_lanes=True))
    expect = ex.run_expansion_with_runner(oracle_runner(layout, Oracle.from_layout(layout)), layout, qs, opts)
    res = bfx.ResidentDeviceGraph.upload_once(layout)
    ws = bfx.Workspace(res)
    try:
        got = ex.run_expansion(ws, layout, qs, opts)
    finally:
        ws.close()
        res.close()
    assert got["outcomes"] == expect["outcomes"]
    for a, b in zip(got["final_tiles"], expect["final_tiles"]):
        assert list(a) == list(b)
    m = dict(got["metrics"])
    assert m.pop("relaxation_launches") == m["planning_passes"]  # one launch per pass
    e = dict(expect["metrics"])
    e.pop("relaxation_launches")
    assert m == e
    assert got["histogram"] == expect["histogram"]
