"""The autotuner's set-class cache: a second query set of the same workload
class (same graph, same magnitudes of batch counts per lane width and of the
union size) reuses the first set's near/far step, layout and chunk pack
instead of searching again, and its launch stays bit-exact."""
import pytest

import bfx
from bfx import workloads
from oracle.oracle import Oracle
from test_gpu_engines import check_batches

pytestmark = pytest.mark.gpu


def plan(layout, qs):
    return bfx.make_overlapping_batch_plan(layout, qs, bfx.BatchPlannerPolicy(32, 0, 1, 64, 1, narrow_lanes=True)
                                           ).descriptions()


def test_second_set_of_a_class_reuses_the_step_and_stays_exact(gpu):
    # two sets of 8 full-graph sources on the c1 graph: one width-8 batch
    # over every tile each, so one set class
    layout, grid = workloads.build_graph("c1")
    first = workloads.full_graph_queries(layout, grid, 8, seed=41)
    second = workloads.full_graph_queries(layout, grid, 8, seed=42)
    d1, d2 = plan(layout, first), plan(layout, second)
    assert len(d1) == len(d2) == 1 and d1[0].lane_width == d2[0].lane_width == 8
    res = bfx.ResidentDeviceGraph.upload_once(layout)
    ws = bfx.Workspace(res)
    bfx.load().bfx_autotune_reset()
    e1, _ = ws.autotune(d1)
    steps1 = {x for e, x in zip(e1, ws.tuned_deltas) if e == bfx.ENGINE_FRONTIER_PUSH}
    pack1 = ws.chunk_pack()
    assert pack1 in (2, 4, 8)
    ws.set_chunk_pack(1)  # the cached class pack replaces it
    e2, _ = ws.autotune(d2)
    steps2 = {x for e, x in zip(e2, ws.tuned_deltas) if e == bfx.ENGINE_FRONTIER_PUSH}
    assert len(steps1) == 1 and steps2 <= steps1  # the cached class step
    assert ws.chunk_pack() == pack1
    ws.execute(bfx.GpuRunOptions(engine=bfx.ENGINE_AUTO))
    st = ws.fetch_statuses()
    labels = [ws.download_labels(b, d.lane_width) for b, d in enumerate(d2)]
    lanes = [[second[i] if i != bfx.NO_EDGE else None for i in d.query_index_by_lane] for d in d2]
    check_batches(layout, d2, lanes, st, labels, Oracle.from_layout(layout))
    ws.close()
    res.close()
