"""Edge-usage adjoint (no reference counterpart): dL/dw_e for
L = sum_t g_t * dist_t.  The device result must equal the CPU tree walk over
the oracle's paths bit for bit (integer g = 1 and float g in (0, 1)), and
agree with central finite differences on tie-free edges."""
import numpy as np
import pytest

import bfx
from bfx import workloads
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def weights_by_eid(layout):
    w = np.zeros(layout.edge_count, np.float32)
    w[layout.arrays["csr_edge_ids"]] = layout.arrays["csr_weights"]
    return w


def with_weights(layout, w):
    a = dict(layout.arrays)
    a["csr_weights"] = w[a["csr_edge_ids"]].astype(np.float32)
    a["csc_weights"] = w[a["csc_edge_ids"]].astype(np.float32)
    a["tile_count"] = np.uint32(layout.tile_count)
    return bfx.DeviceGraphLayout(a, layout.tiles)


@pytest.fixture(scope="module")
def nets():
    layout, grid = workloads.build_graph("c1f")
    qs = workloads.box_queries(layout, grid, 64, 8, 48, seed=44, targets=(1, 32), clip=32)
    return layout, qs


def run_adjoint(layout, qs, gvals, weights=None):
    plan = bfx.make_overlapping_batch_plan(layout, qs, bfx.BatchPlannerPolicy(32, 0, 1, 16, 1, narrow_lanes=True))
    descs = plan.descriptions()
    res = bfx.ResidentDeviceGraph.upload_once(layout)
    if weights is not None:
        res.set_weights(weights)
    ws = bfx.Workspace(res)
    ws.prepare(descs)
    ws.execute(bfx.GpuRunOptions())
    paths = ws.compact_paths()
    order = [(qs[int(i)], t) for d in descs for i in d.query_index_by_lane if i != bfx.NO_EDGE
             for t in qs[int(i)].targets]
    g = np.array([gvals[(q.query_id, int(t))] for q, t in order], np.float32)
    grad = ws.edge_usage_adjoint(g)
    ws.close()
    res.close()
    return grad, paths, order, g


def oracle_grad(layout, order, g):
    orc = Oracle.from_layout(layout)
    cache, plist = {}, []
    for q, t in order:
        if q.query_id not in cache:
            cache[q.query_id] = orc.region_sssp(q.sources, q.targets, q.selected_tiles)[0]
        st, _, edges = orc.compact_path(q.sources, q.targets, q.selected_tiles, cache[q.query_id], int(t))
        plist.append(edges if st == 0 else np.zeros(0, np.uint32))
    return orc.edge_usage_adjoint(layout.edge_count, plist, g), cache


@pytest.mark.parametrize("kind", ["ones", "uniform"])
def test_adjoint_equals_cpu_tree_walk_bitwise(gpu, nets, kind):
    layout, qs = nets
    rng = np.random.default_rng(8)
    gvals = {(q.query_id, int(t)): (np.float32(1) if kind == "ones" else rng.random(dtype=np.float32))
             for q in qs for t in q.targets}
    grad, paths, order, g = run_adjoint(layout, qs, gvals)
    og, _ = oracle_grad(layout, order, g)
    np.testing.assert_array_equal(grad.view(np.uint32), og.view(np.uint32))
    if kind == "ones":
        # integer usage counts: every complete path contributes 1 per edge
        counts = np.zeros(layout.edge_count, np.int64)
        for p in paths:
            if p["reconstruction"] == 0:
                counts[p["edges"]] += 1
        np.testing.assert_array_equal(grad, counts.astype(np.float32))


def test_adjoint_matches_finite_differences_on_tie_free_edges(gpu, nets):
    layout, qs = nets
    qs = qs[:16]
    rng = np.random.default_rng(9)
    gvals = {(q.query_id, int(t)): rng.random(dtype=np.float32) for q in qs for t in q.targets}
    grad, paths, order, g = run_adjoint(layout, qs, gvals)
    used = np.nonzero(grad)[0]
    edges = rng.choice(used, size=min(40, len(used)), replace=False)
    w0 = weights_by_eid(layout)
    delta = np.float32(1e-3)
    base_paths = {}
    orc0 = Oracle.from_layout(layout)
    for q, t in order:
        d0 = orc0.region_sssp(q.sources, q.targets, q.selected_tiles)[0]
        base_paths[(q.query_id, int(t))] = orc0.compact_path(q.sources, q.targets, q.selected_tiles, d0, int(t))[2]
    checked = 0
    for e in edges:
        L = {}
        tie_free = True
        for sgn in (1, -1):
            w = w0.copy()
            w[e] = w[e] + sgn * delta
            lay = with_weights(layout, w)
            orc = Oracle.from_layout(lay)
            total = 0.0
            for q, t in order:
                d = orc.region_sssp(q.sources, q.targets, q.selected_tiles)[0]
                _, _, pe = orc.compact_path(q.sources, q.targets, q.selected_tiles, d, int(t))
                if not np.array_equal(pe, base_paths[(q.query_id, int(t))]):
                    tie_free = False
                dt = float(d[int(t)].view(np.float32))
                if np.isfinite(dt):  # unreachable targets do not enter L
                    total += float(gvals[(q.query_id, int(t))]) * dt
            L[sgn] = total
        if not tie_free:
            continue
        fd = (L[1] - L[-1]) / (2 * float(delta))
        assert abs(fd - float(grad[e])) <= 0.05 * max(1.0, abs(float(grad[e]))), (e, fd, grad[e])
        checked += 1
    assert checked >= 10


def test_adjoint_uses_device_weights(gpu, nets):
    """Device weights replaced through bfx_resident_graph_set_weights give the
    labels and gradient of the re-weighted graph."""
    layout, qs = nets
    qs = qs[:8]
    w = weights_by_eid(layout) * np.float32(1.5)
    gvals = {(q.query_id, int(t)): np.float32(1) for q in qs for t in q.targets}
    grad, paths, order, g = run_adjoint(layout, qs, gvals, weights=w)
    og, dists = oracle_grad(with_weights(layout, w), order, g)
    np.testing.assert_array_equal(grad, og)
    for p, (q, t) in zip(paths, order):
        assert np.float32(p["distance"]).view(np.uint32) == dists[q.query_id][int(t)]


# ---- the 512-net configuration: c1 graph with lognormal float costs, 512 nets
# of one source and U[1,32] targets in a box of side U[8,48] tiles clipped to
# 32; target gradients U(0,1) f32 and all ones.

@pytest.fixture(scope="module")
def nets512():
    layout, grid = workloads.build_graph("c1f")
    qs = workloads.box_queries(layout, grid, 512, 8, 48, seed=0xC4, targets=(1, 32), clip=32)
    return layout, qs


@pytest.mark.parametrize("kind", ["uniform", "ones"])
def test_512_nets_adjoint_equals_cpu_tree_walk_bitwise(gpu, nets512, kind):
    layout, qs = nets512
    rng = np.random.default_rng(0xC4)
    gvals = {(q.query_id, int(t)): (np.float32(1) if kind == "ones" else rng.random(dtype=np.float32))
             for q in qs for t in q.targets}
    grad, paths, order, g = run_adjoint(layout, qs, gvals)
    og, dists = oracle_grad(layout, order, g)
    np.testing.assert_array_equal(grad.view(np.uint32), og.view(np.uint32))
    for p, (q, t) in zip(paths, order):
        assert np.float32(p["distance"]).view(np.uint32) == dists[q.query_id][int(t)]


def test_512_nets_adjoint_finite_differences_1000_tie_free_edges(gpu, nets512):
    """Central differences (delta = 1e-3) of L over 1,000 edges whose
    perturbation changes no path, against the adjoint.  L(w +- delta e_k) is
    evaluated by the engine itself with the perturbed weights uploaded through
    bfx_resident_graph_set_weights; the unperturbed labels are pinned to the
    oracle by the test above."""
    layout, qs = nets512
    rng = np.random.default_rng(0xC4F)
    plan = bfx.make_overlapping_batch_plan(layout, qs, bfx.BatchPlannerPolicy(32, 0, 1, 16, 1, narrow_lanes=True))
    descs = plan.descriptions()
    order = [(qs[int(i)], t) for d in descs for i in d.query_index_by_lane if i != bfx.NO_EDGE
             for t in qs[int(i)].targets]
    g = rng.random(len(order), dtype=np.float32)
    res = bfx.ResidentDeviceGraph.upload_once(layout)
    ws = bfx.Workspace(res)
    opts = bfx.GpuRunOptions()
    try:
        ws.prepare(descs)
        ws.execute(opts)
        base = ws.compact_paths(raw=True)
        grad = ws.edge_usage_adjoint(g)
        w0 = weights_by_eid(layout)
        delta = np.float32(1e-3)
        used = rng.permutation(np.nonzero(grad)[0])
        checked = skipped = 0
        for e in used:
            L = {}
            for sgn in (1, -1):
                w = w0.copy()
                w[e] = w[e] + sgn * delta
                res.set_weights(w)
                ws.execute(opts)
                cur = ws.compact_paths(raw=True)
                if not (np.array_equal(cur["edges"], base["edges"]) and
                        np.array_equal(cur["summaries"]["reconstruction"], base["summaries"]["reconstruction"])):
                    break
                d = cur["summaries"]["distance"].astype(np.float64)
                fin = np.isfinite(d)  # unreachable targets do not enter L
                L[sgn] = float(np.sum(g[fin].astype(np.float64) * d[fin]))
            if len(L) != 2:
                skipped += 1
                continue
            fd = (L[1] - L[-1]) / (2 * float(delta))
            assert abs(fd - float(grad[e])) <= 0.05 * max(1.0, abs(float(grad[e]))), (int(e), fd, float(grad[e]))
            checked += 1
            if checked == 1000:
                break
        assert checked == 1000, (checked, skipped)
    finally:
        ws.close()
        res.close()
