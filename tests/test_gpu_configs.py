"""Parity on the configurations the benchmark times, at their stated sizes.

The benchmark's own workloads (bfx.workloads.bench_workload: the same graph,
query set, planner policy and autotuned engines / near/far steps, one
persistent launch) are compared with the oracle's bounded Dijkstra on each
query's induced region -- the reference tests' differential check
(tests/batched_frontier_push_test.cpp:55 in the reference) -- distances and
min-eid tight predecessors, bit for bit:

  c2  every lane of every batch (256 regional queries, 2.1M V / 16.8M E);
  c3  four seeded lanes of each of the two full-graph W=32 batches
      (16.8M V / 168M E);
  c5  64 seeded regional lanes and two full-graph lanes of the 4,096 + 16
      query set in one launch.

Each runs with the chunked and the tiled frontier layouts.  The
integer-cost configurations (c3, c5) also assert that every finite distance
is below 2^24, the range in which float sums of integer costs are exact.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

import bfx
from bfx import workloads
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

TWO_POW_24_BITS = 0x4B800000  # float bits of 2^24
THREADS = max(1, min(32, os.cpu_count() or 1))


LAYOUTS = {"chunked": bfx.FRONTIER_CHUNKED, "tiled": bfx.FRONTIER_TILED}


def tuned_launch(resident, wl, layout="chunked", pack=None):
    """Plan, autotune (engines and near/far steps per batch) and run the set
    in one launch, as the benchmark does."""
    plan = bfx.make_overlapping_batch_plan(wl.layout, wl.queries, wl.policy)
    descs = plan.descriptions()
    ws = bfx.Workspace(resident)
    ws.set_frontier_layout(LAYOUTS[layout])
    if pack is not None:
        ws.set_chunk_pack(pack)
    engines, _ = ws.autotune(descs)
    ws.execute(bfx.GpuRunOptions(engine=bfx.ENGINE_AUTO))
    statuses = ws.fetch_statuses()
    return ws, descs, engines, statuses


def valid_lanes(d):
    return [l for l in range(d.lane_width) if (d.valid_lane_mask >> l) & 1]


def compare_lanes(ws, orc, wl, descs, picks, chunk=16):
    """Bit-exact comparison of the picked (batch, lane) labels with the
    oracle; returns (lanes checked, distance mismatches, predecessor
    mismatches, reached targets)."""
    checked = dist_bad = pred_bad = reached = 0
    for i in range(0, len(picks), chunk):
        part = picks[i:i + chunk]
        qs = [wl.queries[int(descs[b].query_index_by_lane[l])] for b, l in part]
        od, op = orc.region_sssp_many(qs, THREADS)
        for k, (b, l) in enumerate(part):
            bits, pred = ws.download_lane(b, l)
            dist_bad += int(np.count_nonzero(bits != od[k]))
            pred_bad += int(np.count_nonzero(pred != op[k]))
            reached += int(np.count_nonzero(od[k][np.asarray(qs[k].targets, np.int64)] != 0x7F800000))
            checked += 1
    return checked, dist_bad, pred_bad, reached


def assert_statuses(statuses):
    for s in statuses:
        assert s.stop_reason == bfx.STOP_CONVERGED, s.as_dict()
        assert s.error_bits == 0


@pytest.fixture(scope="module")
def c3_graph(gpu):
    wl = workloads.bench_workload("c3")
    resident = bfx.ResidentDeviceGraph.upload_once(wl.layout)
    orc = Oracle.from_layout(wl.layout)
    yield wl, resident, orc
    resident.close()


@pytest.fixture(scope="module")
def c2_graph(gpu):
    wl = workloads.bench_workload("c2")
    resident = bfx.ResidentDeviceGraph.upload_once(wl.layout)
    yield wl, resident, Oracle.from_layout(wl.layout)
    resident.close()


@pytest.mark.parametrize("layout,pack", [("chunked", None), ("tiled", None), ("chunked", 1), ("chunked", 8)])
def test_c2_every_lane_bit_exact(c2_graph, layout, pack):
    wl, resident, orc = c2_graph
    ws, descs, engines, statuses = tuned_launch(resident, wl, layout, pack)
    assert_statuses(statuses)
    picks = [(b, l) for b, d in enumerate(descs) for l in valid_lanes(d)]
    assert len(picks) == len(wl.queries) == 256
    checked, dist_bad, pred_bad, reached = compare_lanes(ws, orc, wl, descs, picks)
    assert (checked, dist_bad, pred_bad) == (256, 0, 0)
    # every query's target is inside its own box, so every lane reaches it
    assert sum(bin(s.reached_target_mask).count("1") for s in statuses) == reached
    ws.close()


@pytest.mark.parametrize("layout", ["chunked", "tiled"])
def test_c3_sampled_full_graph_lanes_bit_exact(c3_graph, layout):
    wl, resident, orc = c3_graph
    ws, descs, engines, statuses = tuned_launch(resident, wl, layout)
    assert_statuses(statuses)
    assert len(descs) == 2 and all(d.lane_width == 32 for d in descs)
    rng = np.random.default_rng(3030)
    picks = [(b, int(l)) for b in range(len(descs)) for l in rng.choice(valid_lanes(descs[b]), 4, replace=False)]
    checked, dist_bad, pred_bad, _ = compare_lanes(ws, orc, wl, descs, picks, chunk=8)
    assert (checked, dist_bad, pred_bad) == (8, 0, 0)
    bounds = ws.label_bounds()
    assert bounds.max() < TWO_POW_24_BITS, f"distance {np.uint32(bounds.max()).view(np.float32)} >= 2^24"
    ws.close()


@pytest.mark.parametrize("layout", ["chunked", "tiled"])
def test_c5_sampled_regional_and_full_lanes_bit_exact(c3_graph, layout):
    wl3, resident, orc = c3_graph
    queries, _ = workloads.bench_queries("c5", wl3.layout, wl3.grid)
    wl = workloads.BenchWorkload("c5", None, None, wl3.layout, wl3.grid, queries, [],
                                 bfx.BatchPlannerPolicy(32, 1, 8, 2, 1, narrow_lanes=True), "", True)
    ws, descs, engines, statuses = tuned_launch(resident, wl, layout)
    assert_statuses(statuses)
    n_regional = 4096
    lanes = [(b, l) for b, d in enumerate(descs) for l in valid_lanes(d)]
    assert len(lanes) == len(queries) == 4096 + 16
    regional = [x for x in lanes if int(descs[x[0]].query_index_by_lane[x[1]]) < n_regional]
    full = [x for x in lanes if int(descs[x[0]].query_index_by_lane[x[1]]) >= n_regional]
    rng = np.random.default_rng(5050)
    picks = [regional[int(i)] for i in rng.choice(len(regional), 64, replace=False)]
    picks += [full[int(i)] for i in rng.choice(len(full), 2, replace=False)]
    checked, dist_bad, pred_bad, _ = compare_lanes(ws, orc, wl, descs, picks)
    assert (checked, dist_bad, pred_bad) == (66, 0, 0)
    bounds = ws.label_bounds()
    assert bounds.max() < TWO_POW_24_BITS, f"distance {np.uint32(bounds.max()).view(np.float32)} >= 2^24"
    ws.close()


def test_lane_download_and_label_bounds_match_full_image(gpu):
    """The one-lane download equals the lane's column of the full image, and
    the label bound equals the largest finite distance in it (c1 graph)."""
    layout, grid = workloads.build_graph("c1")
    qs = workloads.full_graph_queries(layout, grid, 8, seed=101)
    resident = bfx.ResidentDeviceGraph.upload_once(layout)
    ws = bfx.Workspace(resident)
    ws.prepare([bfx.make_description(layout, qs, 8)])
    ws.execute(bfx.GpuRunOptions())
    assert_statuses(ws.fetch_statuses())
    full_bits, full_pred = ws.download_labels(0, 8)
    for lane in range(8):
        bits, pred = ws.download_lane(0, lane)
        np.testing.assert_array_equal(bits, full_bits[:, lane])
        np.testing.assert_array_equal(pred, full_pred[:, lane])
    finite = full_bits[full_bits < 0x7F800000]
    assert int(ws.label_bounds()[0]) == int(finite.max())
    with pytest.raises(IndexError):
        ws.download_lane(0, 8)
    ws.close()
    resident.close()
