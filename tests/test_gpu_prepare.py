"""Device-side batch description preparation (bfx_prepare_batches_from_queries):
from each batch's lane -> query assignment and the queries' tiles and
terminals alone, the device builds the same prepared description the host
planner's prepare_batch_device_description image gives (byte for byte: lane
terminal slices, dense tile lane masks, union tiles, vertex ranges), and the
launch on it gives the oracle's labels."""
import numpy as np
import pytest

import bfx
from bfx import workloads
from oracle.oracle import Oracle
from test_gpu_engines import check_batches

pytestmark = pytest.mark.gpu

FIELDS = ("source_offsets", "sources", "target_offsets", "targets", "union_tiles", "tile_lane_masks", "ranges")


def assert_same_description(got, want):
    assert got.lane_width == want.lane_width and got.valid_lane_mask == want.valid_lane_mask
    for f in FIELDS:
        np.testing.assert_array_equal(getattr(got, f), getattr(want, f), err_msg=f)


def lane_lists(descs):
    return [(d.lane_width, [int(q) for q in d.query_index_by_lane[:bin(d.valid_lane_mask).count("1")]])
            for d in descs]


@pytest.fixture(scope="module")
def regional():
    layout, grid = workloads.build_graph("c2", scale_tiles=(32, 32))
    qs = workloads.box_queries(layout, grid, 60, 2, 16, seed=31, targets=(1, 4))
    plan = bfx.make_overlapping_batch_plan(layout, qs, bfx.BatchPlannerPolicy(32, 0, 1, 8, 1, narrow_lanes=True))
    return layout, qs, plan.descriptions()


def test_device_prepared_descriptions_equal_host_planner(gpu, regional):
    layout, qs, descs = regional
    res = bfx.ResidentDeviceGraph.upload_once(layout)
    ws = bfx.Workspace(res)
    ws.prepare(descs)  # host path, read back
    for b, d in enumerate(descs):
        assert_same_description(ws.prepared_description(b), d)
    ws.prepare_from_queries(lane_lists(descs), qs)  # device path
    for b, d in enumerate(descs):
        assert_same_description(ws.prepared_description(b), d)
    ws.execute(bfx.GpuRunOptions())
    st = ws.fetch_statuses()
    labels = [ws.download_labels(b, d.lane_width) for b, d in enumerate(descs)]
    lanes = [[qs[i] if i != bfx.NO_EDGE else None for i in d.query_index_by_lane] for d in descs]
    check_batches(layout, descs, lanes, st, labels, Oracle.from_layout(layout))
    ws.close()
    res.close()


@pytest.mark.parametrize("layout_kind", [bfx.FRONTIER_CHUNKED, bfx.FRONTIER_TILED], ids=["chunked", "tiled"])
def test_device_prepared_full_graph_batch(gpu, layout_kind):
    """A full-graph batch (every tile, every lane): the device path marks it
    full like the host path, and labels equal the oracle's."""
    c1 = workloads.make_workload("c1")
    d = bfx.make_description(c1.layout, c1.queries, 8)
    res = bfx.ResidentDeviceGraph.upload_once(c1.layout)
    ws = bfx.Workspace(res)
    ws.set_frontier_layout(layout_kind)
    ws.prepare_from_queries([(8, list(range(8)))], c1.queries)
    assert_same_description(ws.prepared_description(0), d)
    ws.execute(bfx.GpuRunOptions())
    st = ws.fetch_statuses()
    check_batches(c1.layout, [d], [c1.queries], st, [ws.download_labels(0, 8)], Oracle.from_layout(c1.layout))
    ws.close()
    res.close()


def test_device_prepare_rejects_bad_images(gpu, regional):
    layout, qs, descs = regional
    res = bfx.ResidentDeviceGraph.upload_once(layout)
    ws = bfx.Workspace(res)
    with pytest.raises(ValueError):
        ws.prepare_from_queries([(8, [])], qs)  # no valid lane
    with pytest.raises(ValueError):
        ws.prepare_from_queries([(8, list(range(9)))], qs)  # more lanes than the width
    with pytest.raises(IndexError):
        ws.prepare_from_queries([(1, [len(qs)])], qs)  # query index out of range
    bad = bfx.RouteQuery(0, [int(qs[0].sources[0])], [int(qs[1].targets[0])], qs[0].selected_tiles)
    if not np.isin(layout.arrays["owner_tiles"][bad.targets[0]], qs[0].selected_tiles):
        with pytest.raises(ValueError, match="owner tile"):
            ws.prepare_from_queries([(1, [0])], [bad])
    ws.close()
    res.close()


def test_device_prepared_c2_set_equals_host_planner(gpu):
    """The benchmark's 256-query c2 set (90 batches over 16,384 tiles)."""
    wl = workloads.bench_workload("c2")
    descs = bfx.make_overlapping_batch_plan(wl.layout, wl.queries, wl.policy).descriptions()
    res = bfx.ResidentDeviceGraph.upload_once(wl.layout)
    ws = bfx.Workspace(res)
    ws.prepare_from_queries(lane_lists(descs), wl.queries)
    for b, d in enumerate(descs):
        assert_same_description(ws.prepared_description(b), d)
    ws.execute(bfx.GpuRunOptions())
    assert all(s.stop_reason == bfx.STOP_CONVERGED for s in ws.fetch_statuses())
    ws.close()
    res.close()
