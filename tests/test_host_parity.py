"""CPU parity of the host builders against the reference's own code:
the device graph image (canonical edge ids, spatial order, runs) and the
batch planner + descriptions.  Uses the reference library built by
oracle/Makefile when present; the hashed c1 layout is always checked."""
import hashlib

import numpy as np
import pytest

import bfx
from bfx import workloads
from golden_cases import GOLDEN
from oracle.oracle import Ref

needs_ref = pytest.mark.skipif(not Ref.available(), reason="reference library not built here (oracle/_ref)")


def layout_hash(a):
    h = hashlib.sha256()
    for k in sorted(a):
        h.update(k.encode())
        h.update(np.ascontiguousarray(a[k]).tobytes())
    return h.hexdigest()


def test_c1_layout_equals_reference_hash():
    z = np.load(GOLDEN / "synthetic_c1.npz")
    layout, _ = workloads.build_graph("c1")
    assert layout_hash(layout.arrays) == str(z["layout_sha256"])


def random_input(seed, V=300, E=1500):
    """Irregular input: negative coordinates, unlocated vertices, parallel and
    self edges, zero and duplicate weights, repeated provenance records."""
    rng = np.random.default_rng(seed)
    x = rng.integers(-40, 40, V).astype(np.int32)
    y = rng.integers(-25, 30, V).astype(np.int32)
    has = (rng.random(V) > 0.1).astype(np.uint8)
    cls = rng.integers(0, 3, V).astype(np.uint16)
    src = rng.integers(0, V, E).astype(np.uint32)
    dst = rng.integers(0, V, E).astype(np.uint32)
    dst[:40] = src[:40]
    src[40:80] = src[80:120]
    dst[40:80] = dst[80:120]
    w = rng.choice(np.array([0.0, -0.0, 0.5, 1.0, 2.25, 3.0], np.float32), E)
    w[200:] = rng.random(E - 200).astype(np.float32) * 4
    pd = rng.integers(1, 3, E).astype(np.uint32)
    pk = rng.integers(1, 4, E).astype(np.uint32)
    pr = rng.integers(0, 50, E).astype(np.uint64)
    g = bfx.InputGraph(x, y, has, cls, src, dst, w, pd, pk, pr)
    order = bfx.SpatialOrderConfig(-3, 2, int(rng.integers(3, 9)), int(rng.integers(2, 7)))
    return g, order


@needs_ref
@pytest.mark.parametrize("seed", range(6))
def test_layout_equals_reference_on_irregular_inputs(seed):
    g, order = random_input(seed)
    ours = bfx.build_device_graph_layout(g, order)
    ref = Ref()
    h = ref.case_from_input(g, order)
    a, t = ref.layout(h)
    for k in a:
        np.testing.assert_array_equal(ours.arrays[k].view(np.uint32), a[k].view(np.uint32), err_msg=k)
    for k in ("new_to_old", "tile_xy", "has_location", "tile_vertex_offsets"):
        np.testing.assert_array_equal(ours.tiles[k], t[k], err_msg=k)
    ref.free(h)


@needs_ref
@pytest.mark.parametrize("width,policy", [(32, (1, 8, 2, 1)), (16, (1, 8, 2, 1)), (8, (0, 1, 4, 1)),
                                          (32, (0, 1, 64, 1)), (1, (1, 8, 2, 1))])
def test_planner_and_descriptions_equal_reference(width, policy):
    layout, grid = workloads.build_graph("c1")
    qs = workloads.box_queries(layout, grid, 40, 2, 12, seed=31, targets=(1, 3))
    qs += workloads.full_graph_queries(layout, grid, 3, seed=32, first_id=40)
    ours = bfx.make_overlapping_batch_plan(layout, qs, bfx.BatchPlannerPolicy(width, *policy))
    ref = Ref()
    g, order, _ = bfx.synth_graph(**workloads.GRAPHS["c1"])
    h = ref.case_from_input(g, order)
    for q in qs:
        ref.query_add(h, q.query_id, q.sources, q.targets, q.selected_tiles)
    nb = ref.plan(h, width, *policy)
    assert nb == ours.batch_count
    T = layout.tile_count
    for b in range(nb):
        rb = ref.plan_batch(h, b, width)
        d = ours.descriptions()[b]
        np.testing.assert_array_equal(d.query_index_by_lane, rb["lane_query"])
        assert d.valid_lane_mask == rb["valid"] and d.lane_width == rb["lane_width"]
        np.testing.assert_array_equal(d.union_tiles, rb["union_tiles"])
        assert tuple(ours.estimates[b]) == tuple(int(x) for x in rb["estimates"])
        rd = ref.describe_batch(h, b, T)
        for k in ("source_offsets", "sources", "target_offsets", "targets", "union_tiles", "tile_lane_masks"):
            np.testing.assert_array_equal(getattr(d, k), rd[k], err_msg=k)
        np.testing.assert_array_equal(d.ranges, rd["ranges"])
    ref.free(h)


def test_planner_narrow_lanes_shrinks_width():
    layout, grid = workloads.build_graph("c1")
    qs = workloads.box_queries(layout, grid, 20, 2, 6, seed=3)
    plan = bfx.make_overlapping_batch_plan(layout, qs, bfx.BatchPlannerPolicy(32, narrow_lanes=True))
    for d in plan.descriptions():
        k = bin(d.valid_lane_mask).count("1")
        assert d.lane_width == (1 if k == 1 else 8 if k <= 8 else 16 if k <= 16 else 32)
    covered = sorted(int(i) for d in plan.descriptions() for i in d.query_index_by_lane if i != bfx.NO_EDGE)
    assert covered == list(range(len(qs)))


def test_planner_rejects_bad_queries():
    layout, grid = workloads.build_graph("c1")
    q = workloads.box_queries(layout, grid, 1, 2, 4, seed=1)[0]
    bad = bfx.RouteQuery(1, q.sources, q.targets, q.selected_tiles[1:])  # drops the source tile sometimes
    ok = [q, bfx.RouteQuery(1, q.sources, q.targets, q.selected_tiles)]
    with pytest.raises(ValueError, match="unique"):
        bfx.make_overlapping_batch_plan(layout, [q, bfx.RouteQuery(q.query_id, q.sources, q.targets,
                                                                  q.selected_tiles)])
    with pytest.raises(ValueError):
        bfx.make_overlapping_batch_plan(layout, [q], bfx.BatchPlannerPolicy(lane_width=12))
    del bad, ok
