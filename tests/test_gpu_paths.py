"""GPU compact paths (the reference's ReusableCompactPathWorkspace::reconstruct):
summaries and payloads equal the reference's reconstruct_compact_path_payload
on every golden fixture -- including the zero-weight cycle that needs the
backtracking search -- and the oracle's search on regional c1 queries."""
import numpy as np
import pytest

import bfx
from bfx import workloads
from golden_cases import GOLDEN, fixture_paths, load_case
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def run_paths(layout, descs, engine=bfx.ENGINE_FRONTIER_PUSH):
    res = bfx.ResidentDeviceGraph.upload_once(layout)
    ws = bfx.Workspace(res)
    ws.prepare(descs)
    ws.execute(bfx.GpuRunOptions(engine=engine))
    st = ws.fetch_statuses()
    paths = ws.compact_paths()
    ws.close()
    res.close()
    return st, paths


@pytest.mark.parametrize("path", fixture_paths(), ids=lambda p: p.stem)
@pytest.mark.parametrize("engine", [bfx.ENGINE_FRONTIER_PUSH, bfx.ENGINE_JACOBI_PULL], ids=["frontier", "jacobi"])
def test_compact_paths_match_reference_fixtures(gpu, path, engine):
    case = load_case(path)
    descs = [bfx.make_description(case.layout, [gq.query], 1) for gq in case.queries]
    _, paths = run_paths(case.layout, descs, engine)
    k = 0
    for gq in case.queries:
        for ti, (st, verts, edges) in enumerate(gq.paths()):
            p = paths[k]
            k += 1
            assert p["target"] == gq.query.targets[ti]
            assert p["reconstruction"] == st, (case.name, ti, p)
            if st == 0:
                assert p["reached"] == 1
                np.testing.assert_array_equal(p["vertices"], verts)
                np.testing.assert_array_equal(p["edges"], edges)
                np.testing.assert_array_equal(p["labels"].view(np.uint32), gq.dist[verts])
                assert p["selected_source"] == verts[0] and p["path_length"] == len(edges)
            elif st == 1:
                assert p["reached"] == 0 and np.isinf(p["distance"])
    assert k == len(paths)


def test_zero_weight_cycle_target_uses_backtracking(gpu):
    """tests/compact_paths_fixture_suite.hpp:45: min-id predecessors cycle
    for the first query's target; the device search backtracks like the
    reference and returns the reference path."""
    case = load_case(GOLDEN / "compact_paths.npz")
    gq = case.queries[0]
    _, paths = run_paths(case.layout, [bfx.make_description(case.layout, [gq.query], 1)])
    st, verts, edges = gq.paths()[0]
    assert paths[0]["reconstruction"] == 0
    np.testing.assert_array_equal(paths[0]["vertices"], verts)
    np.testing.assert_array_equal(paths[0]["edges"], edges)


def test_compact_paths_regional_multi_batch(gpu):
    layout, grid = workloads.build_graph("c1f")
    qs = workloads.box_queries(layout, grid, 40, 4, 20, seed=12, targets=(1, 12))
    plan = bfx.make_overlapping_batch_plan(layout, qs, bfx.BatchPlannerPolicy(32, 0, 1, 8, 1, narrow_lanes=True))
    descs = plan.descriptions()
    st, paths = run_paths(layout, descs)
    orc = Oracle.from_layout(layout)
    k = 0
    for d in descs:
        for lane in range(d.lane_width):
            qi = int(d.query_index_by_lane[lane])
            if qi == bfx.NO_EDGE:
                continue
            q = qs[qi]
            dist, _ = orc.region_sssp(q.sources, q.targets, q.selected_tiles)
            for t in q.targets:
                p = paths[k]
                k += 1
                assert p["target"] == t
                ost, overts, oedges = orc.compact_path(q.sources, q.targets, q.selected_tiles, dist, int(t))
                assert p["reconstruction"] == ost
                if ost == 0:
                    np.testing.assert_array_equal(p["vertices"], overts)
                    np.testing.assert_array_equal(p["edges"], oedges)
    assert k == len(paths)


def test_round_limited_lanes_report_terminal_failure(gpu):
    layout, grid = workloads.build_graph("c1")
    qs = workloads.full_graph_queries(layout, grid, 8, seed=3)
    d = bfx.make_description(layout, qs, 8)
    res = bfx.ResidentDeviceGraph.upload_once(layout)
    ws = bfx.Workspace(res)
    ws.prepare([d])
    ws.execute(bfx.GpuRunOptions(maximum_rounds=2))
    paths = ws.compact_paths()
    assert all(p["reconstruction"] == 2 and p["reached"] == 0 for p in paths)
    ws.close()
    res.close()


def test_many_backtracking_targets_searched_in_parallel(gpu):
    """Forty copies of the zero-weight-cycle query (lanes of five width-8
    batches) hand forty targets to the backtracking search at once; the
    searches run one per thread over the search slots, each with its own
    stacks and marks, and every path equals the reference's."""
    case = load_case(GOLDEN / "compact_paths.npz")
    gq = case.queries[0]
    descs = [bfx.make_description(case.layout, [gq.query] * 8, 8) for _ in range(5)]
    _, paths = run_paths(case.layout, descs)
    st, verts, edges = gq.paths()[0]
    per_query = len(gq.query.targets)
    assert len(paths) == 40 * per_query
    for k in range(40):
        p = paths[k * per_query]
        assert p["reconstruction"] == st == 0
        np.testing.assert_array_equal(p["vertices"], verts)
        np.testing.assert_array_equal(p["edges"], edges)
