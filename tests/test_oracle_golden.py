"""Pins the C oracle (oracle/bfx_oracle.c) against golden vectors produced by
the reference's own CPU code: every fixture suite of the reference's tests for
this path, plus hashed distances of the synthetic c1 configuration."""
import hashlib

import numpy as np
import pytest

import bfx
from bfx import workloads
from golden_cases import GOLDEN, fixture_paths, load_case
from oracle.oracle import Oracle


def walk_preds(pred, target, sources, csr_eid_src):
    """Vertices/edges from a source to `target` following min-eid predecessors."""
    verts, edges, seen = [int(target)], [], {int(target)}
    v = int(target)
    while v not in sources:
        e = int(pred[v])
        if e == bfx.NO_EDGE:
            return None
        v = int(csr_eid_src[e])
        if v in seen:
            return None  # cycle: zero-weight tie, needs the backtracking search
        seen.add(v)
        verts.append(v)
        edges.append(e)
    return np.array(verts[::-1], np.uint32), np.array(edges[::-1], np.uint32)


def edge_sources(layout):
    a = layout.arrays
    E = a["csr_destinations"].shape[0]
    src = np.repeat(np.arange(layout.vertex_count, dtype=np.uint32), np.diff(a["csr_row_offsets"]))
    out = np.zeros(E, np.uint32)
    out[a["csr_edge_ids"]] = src
    return out


@pytest.mark.parametrize("path", fixture_paths(), ids=lambda p: p.stem)
def test_oracle_matches_reference_fixture(path):
    case = load_case(path)
    orc = Oracle.from_layout(case.layout)
    esrc = edge_sources(case.layout)
    for gq in case.queries:
        q = gq.query
        dist, pred = orc.region_sssp(q.sources, q.targets, q.selected_tiles)
        # Both are Dijkstra on the induced graph: bit-identical labels.
        np.testing.assert_array_equal(dist, gq.dist)
        for ti, (st, verts, edges) in enumerate(gq.paths()):
            ost, overts, oedges = orc.compact_path(q.sources, q.targets, q.selected_tiles, gq.dist,
                                                   int(q.targets[ti]))
            assert ost == st
            if st == 0:
                np.testing.assert_array_equal(overts, verts)
                np.testing.assert_array_equal(oedges, edges)
                walked = walk_preds(pred, q.targets[ti], set(int(s) for s in q.sources), esrc)
                if walked is not None:
                    # Acyclic predecessor chains are exactly the reference's path.
                    np.testing.assert_array_equal(walked[0], verts)
                    np.testing.assert_array_equal(walked[1], edges)


def test_golden_covers_reference_suites():
    names = {p.stem.split("_")[0] for p in fixture_paths()}
    assert {"jacobi", "dense", "frontier", "batched", "compact"} <= names
    assert len(fixture_paths()) >= 13 + 2 + 2 + 2


def test_zero_cycle_fixture_needs_backtracking():
    """The reference's zero-weight-cycle fixture (tests/sssp_test.cpp:202) is the
    case where min-eid predecessors form a cycle and the compact-path search
    must backtrack; the oracle reproduces the reference path there."""
    case = load_case(GOLDEN / "compact_paths.npz")
    orc = Oracle.from_layout(case.layout)
    esrc = edge_sources(case.layout)
    gq = case.queries[0]  # cycle query
    q = gq.query
    _, pred = orc.region_sssp(q.sources, q.targets, q.selected_tiles)
    st, verts, edges = gq.paths()[0]
    assert st == 0
    assert walk_preds(pred, q.targets[0], set(int(s) for s in q.sources), esrc) is None
    ost, overts, oedges = orc.compact_path(q.sources, q.targets, q.selected_tiles, gq.dist, int(q.targets[0]))
    assert ost == 0
    np.testing.assert_array_equal(overts, verts)


def test_oracle_matches_reference_on_synthetic_c1():
    z = np.load(GOLDEN / "synthetic_c1.npz")
    layout, _ = workloads.build_graph("c1")
    orc = Oracle.from_layout(layout)
    sample = z["sample_vertices"]
    for i in range(int(z["query_count"])):
        src, tgt, tiles = z[f"Q{i}_sources"], z[f"Q{i}_targets"], z[f"Q{i}_selected_tiles"]
        dist, _ = orc.region_sssp(src, tgt, tiles)
        np.testing.assert_array_equal(dist[sample], z[f"Q{i}_dist_sample"])
        assert hashlib.sha256(dist.tobytes()).hexdigest() == str(z[f"Q{i}_dist_sha256"])
        vo = eo = 0
        for ti, (st, ln) in enumerate(zip(z[f"Q{i}_path_status"], z[f"Q{i}_path_len"])):
            ost, overts, oedges = orc.compact_path(src, tgt, tiles, dist, int(tgt[ti]))
            assert ost == st
            if st == 0:
                np.testing.assert_array_equal(overts, z[f"Q{i}_path_vertices"][vo:vo + ln + 1])
                np.testing.assert_array_equal(oedges, z[f"Q{i}_path_edges"][eo:eo + ln])
                vo += int(ln) + 1
                eo += int(ln)


def exact_round_f32(n: int) -> np.float32:
    """Nearest-even float32 of n * 2^-63 (independent restatement for the test)."""
    from fractions import Fraction
    x = Fraction(n, 1 << 63)
    f = np.float32(float(x))
    # correct the double rounding step, if any, by checking neighbours
    cands = [f, np.nextafter(f, np.float32(np.inf)), np.nextafter(f, np.float32(-np.inf))]
    best = min(cands, key=lambda c: (abs(Fraction(float(c)) - x), int(np.float32(c).view(np.uint32)) & 1))
    return np.float32(best)


def test_oracle_adjoint_is_exact_and_order_free():
    orc = Oracle.from_layout(load_case(fixture_paths()[0]).layout)
    grad = orc.edge_usage_adjoint(5, [np.array([0, 2], np.uint32), np.array([2, 4], np.uint32)],
                                  np.array([0.25, 0.5], np.float32))
    np.testing.assert_array_equal(grad, np.array([0.25, 0, 0.75, 0, 0.5], np.float32))
    rng = np.random.default_rng(3)
    g = (rng.random(400, dtype=np.float32) * np.float32(3)).astype(np.float32) + np.float32(1e-6)
    g[::7] *= np.float32(-1)
    paths = [rng.integers(0, 9, size=rng.integers(1, 6)).astype(np.uint32) for _ in range(400)]
    paths = [np.unique(p) for p in paths]
    grad = orc.edge_usage_adjoint(9, paths, g)
    order = rng.permutation(400)
    grad2 = orc.edge_usage_adjoint(9, [paths[i] for i in order], g[order])
    np.testing.assert_array_equal(grad, grad2)
    for e in range(9):
        n = sum(int(np.float32(gv).astype(np.float64) * 2 ** 63) for gv, p in zip(g, paths) if e in p)
        assert grad[e] == exact_round_f32(n)
