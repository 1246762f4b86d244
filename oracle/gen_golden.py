"""Generates tests/golden/*.npz from the reference's own CPU code.

TEST INFRASTRUCTURE.  Run in a container where the reference sources exist:

    make -C oracle ref && python oracle/gen_golden.py

Every fixture suite the reference's tests hold for this path is exported
(built by the reference's own fixture headers through oracle/ref_driver.cpp):
the device graph image the reference builds, the queries, bounded Dijkstra
distances on each query's induced graph (dijkstra_oracle), compact paths
(reconstruct_compact_path_payload) and, for the five-lane batched fixture,
the reference's portable batched engines' label bits and statuses.  For the
synthetic c1 configuration it records hashes of the reference layout and of
the reference distances so large cases are pinned without large files.
"""
from __future__ import annotations

import hashlib
import sys
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(REPO / "bf-new_b200"))

from oracle.oracle import Ref  # noqa: E402

GOLDEN = REPO / "tests" / "golden"


def layout_hash(a: dict) -> str:
    h = hashlib.sha256()
    for k in sorted(a):
        h.update(k.encode())
        h.update(np.ascontiguousarray(a[k]).tobytes())
    return h.hexdigest()


def export_case(ref: Ref, h: int, out: dict, batched_policy=None) -> None:
    c = ref.counts(h)
    a, t = ref.layout(h)
    for k, v in a.items():
        out["L_" + k] = v
    for k, v in t.items():
        out["T_" + k] = v
    out["tile_count"] = np.uint32(c["T"])
    out["expected_reached"] = np.uint32(c["expected_reached"])
    out["expected_miss"] = np.uint32(c["expected_miss"])
    out["four_ulps"] = np.uint32(c["four_ulps"])
    out["query_count"] = np.uint32(c["queries"])
    V = c["V"]
    for q in range(c["queries"]):
        qd = ref.query(h, q)
        for k, v in qd.items():
            out[f"Q{q}_{k}"] = np.asarray(v)
        d = ref.dijkstra(h, q, V)
        out[f"Q{q}_dist"] = d.view(np.uint32)
        st, rc, ln, verts, edges = ref.compact_paths(h, q, d, len(qd["targets"]))
        out[f"Q{q}_path_status"] = st
        out[f"Q{q}_path_reached"] = rc
        out[f"Q{q}_path_len"] = ln
        out[f"Q{q}_path_vertices"] = verts
        out[f"Q{q}_path_edges"] = edges
    if batched_policy is not None:
        nb = ref.plan(h, *batched_policy)
        out["batch_count"] = np.uint32(nb)
        for b in range(nb):
            pb = ref.plan_batch(h, b, batched_policy[0])
            out[f"B{b}_lane_query"] = pb["lane_query"]
            out[f"B{b}_union_tiles"] = pb["union_tiles"]
            out[f"B{b}_union_masks"] = pb["union_masks"]
            out[f"B{b}_valid"] = np.uint32(pb["valid"])
            out[f"B{b}_lane_width"] = np.uint32(pb["lane_width"])
            for eng in (0, 1, 2):
                bits, st = ref.run_batched(h, b, eng, V, pb["lane_width"])
                out[f"B{b}_E{eng}_bits"] = bits
                out[f"B{b}_E{eng}_status"] = np.array(
                    [st["converged"], st["reached_target_mask"], st["bounding_box_miss_mask"],
                     st["valid_lane_mask"], st["active_lane_mask"], st["converged_lane_mask"], st["stop_reason"],
                     st["error_bits"]], np.uint32)


def main() -> None:
    GOLDEN.mkdir(parents=True, exist_ok=True)
    ref = Ref()
    written = []
    for suite in ("jacobi", "dense", "frontier"):
        for i in range(ref.fixture_count(suite)):
            h = ref.case_fixture(suite, i)
            out = {"suite": np.array(suite), "name": np.array(ref.name(h))}
            export_case(ref, h, out)
            path = GOLDEN / f"{suite}_{i:02d}.npz"
            np.savez_compressed(path, **out)
            written.append(path.name)
            ref.free(h)
    h = ref.case_fixture("batched_mixed", 0)
    out = {"suite": np.array("batched_mixed"), "name": np.array("batched_mixed")}
    # The fixture's own planner policy (tests/batched_jacobi_fixture_suite.hpp:159-165).
    export_case(ref, h, out, batched_policy=(8, 0, 1, 4, 1))
    np.savez_compressed(GOLDEN / "batched_mixed.npz", **out)
    written.append("batched_mixed.npz")
    ref.free(h)
    h = ref.case_fixture("compact_paths", 0)
    out = {"suite": np.array("compact_paths"), "name": np.array("compact_paths")}
    export_case(ref, h, out)
    np.savez_compressed(GOLDEN / "compact_paths.npz", **out)
    written.append("compact_paths.npz")
    ref.free(h)

    # Synthetic c1: the reference's layout and distances as hashes + samples.
    import bfx
    from bfx import workloads
    g, order, _ = bfx.synth_graph(**workloads.GRAPHS["c1"])
    h = ref.case_from_input(g, order)
    a, t = ref.layout(h)
    out = {"layout_sha256": np.array(layout_hash(a)), "V": np.uint32(a["owner_tiles"].shape[0])}
    from bfx import DeviceGraphLayout
    lay = DeviceGraphLayout(a, t)
    grid = (workloads.GRAPHS["c1"]["tiles_x"], workloads.GRAPHS["c1"]["tiles_y"])
    qs = workloads.full_graph_queries(lay, grid, 8, 101)
    qs += workloads.box_queries(lay, grid, 16, 4, 16, 777, first_id=100, targets=(1, 8))
    rng = np.random.default_rng(5)
    sample = rng.integers(0, a["owner_tiles"].shape[0], size=512).astype(np.uint32)
    out["sample_vertices"] = sample
    for i, q in enumerate(qs):
        qi = ref.query_add(h, q.query_id, q.sources, q.targets, q.selected_tiles)
        d = ref.dijkstra(h, qi, a["owner_tiles"].shape[0])
        out[f"Q{i}_sources"] = q.sources
        out[f"Q{i}_targets"] = q.targets
        out[f"Q{i}_selected_tiles"] = q.selected_tiles
        out[f"Q{i}_dist_sha256"] = np.array(hashlib.sha256(d.view(np.uint32).tobytes()).hexdigest())
        out[f"Q{i}_dist_sample"] = d.view(np.uint32)[sample]
        st, rc, ln, verts, edges = ref.compact_paths(h, qi, d, len(q.targets))
        out[f"Q{i}_path_status"] = st
        out[f"Q{i}_path_len"] = ln
        out[f"Q{i}_path_vertices"] = verts
        out[f"Q{i}_path_edges"] = edges
    out["query_count"] = np.uint32(len(qs))
    np.savez_compressed(GOLDEN / "synthetic_c1.npz", **out)
    written.append("synthetic_c1.npz")
    print("wrote", len(written), "fixtures:", " ".join(written))


if __name__ == "__main__":
    main()
