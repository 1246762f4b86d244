"""The reference arm of the benchmark builds its graphs with the generator
restated in oracle/ref_driver.cpp, so that it loads nothing from libbfx.  Its
graph, partitioned by the reference, must equal the product generator's graph
laid out by libbfx, array for array, and the query samplers must draw the
same query sets from either tile table."""
import numpy as np
import pytest

import bfx
from bfx import workloads
from oracle.oracle import Ref

pytestmark = pytest.mark.skipif(not Ref.available(), reason="reference library (oracle/_ref) not built")

ARRAYS = ["owner_tiles", "csr_row_offsets", "csr_destinations", "csr_weights", "csc_column_offsets", "csc_sources",
          "csc_weights", "csc_edge_ids", "csr_edge_ids"]


@pytest.mark.parametrize("name,tiles", [("c1", None), ("c1f", None), ("c2", (12, 10)), ("c3", (6, 7))])
def test_reference_generator_gives_the_same_graph(name, tiles):
    spec = dict(workloads.GRAPHS[name])
    if tiles:
        spec["tiles_x"], spec["tiles_y"] = tiles
    g, order, _ = bfx.synth_graph(**spec)
    layout = bfx.build_device_graph_layout(g, order)
    ref = Ref()
    h = ref.case_synth(spec)
    a, t = ref.layout(h)
    for k in ARRAYS:
        np.testing.assert_array_equal(a[k].view(np.uint32), layout.arrays[k].view(np.uint32), err_msg=k)
    np.testing.assert_array_equal(t["tile_vertex_offsets"], layout.tiles["tile_vertex_offsets"])
    rt = ref.tiles(h)
    np.testing.assert_array_equal(rt.tiles["tile_xy"], layout.tiles["tile_xy"])
    np.testing.assert_array_equal(rt.tiles["has_location"], layout.tiles["has_location"])
    grid = (spec["tiles_x"], spec["tiles_y"])
    a1 = workloads.box_queries(layout, grid, 20, 2, 6, 11)
    a2 = workloads.box_queries(rt, grid, 20, 2, 6, 11)
    for q1, q2 in zip(a1, a2):
        for f in ("sources", "targets", "selected_tiles"):
            np.testing.assert_array_equal(getattr(q1, f), getattr(q2, f))
    ref.free(h)


def test_stepped_timing_returns_reference_distances():
    spec = dict(workloads.GRAPHS["c2"], tiles_x=8, tiles_y=8)
    ref = Ref()
    h = ref.case_synth(spec)
    rt = ref.tiles(h)
    qs = workloads.box_queries(rt, (8, 8), 6, 2, 5, 4)
    idx = [ref.query_add(h, q.query_id, q.sources, q.targets, q.selected_tiles) for q in qs]
    r = ref.time_dijkstra_steps(h, idx, 2, 1, 3, want_dist=True)
    assert len(r["step_s"]) == 3 and all(x >= 0 for x in r["step_s"])
    for i, q in enumerate(qs):
        np.testing.assert_array_equal(r["dist"][i], ref.dijkstra(h, idx[i], rt.vertex_count))
    ref.free(h)
