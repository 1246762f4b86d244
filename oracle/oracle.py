"""TEST INFRASTRUCTURE ONLY: Python bindings of the CPU checkers.

* Oracle — the plain-C restatement in oracle/bfx_oracle.c
  (oracle/_build/libbfx_oracle.so), pinned against the reference's golden
  vectors by tests/test_oracle_golden.py.
* Ref — the reference's own CPU library compiled from its sources by
  oracle/Makefile (oracle/_ref/libbfnew_ref_driver.so), optional: present
  where it was built.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
leg may use this module, and only as the checker or the CPU baseline.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "libbfx_oracle.so"
REF_SO = HERE / "_ref" / "libbfnew_ref_driver.so"

u32, u64, f32, P = C.c_uint32, C.c_uint64, C.c_float, C.POINTER


def build(ref: bool = False) -> None:
    subprocess.run(["make", "-s", "-C", str(HERE), "oracle"], check=True)
    if ref:  # where the reference sources are present (BFX_REFERENCE_DIR)
        subprocess.run(["make", "-s", "-C", str(HERE), "ref-if-present"], check=True)


def _p(a, t=u32):
    return None if a is None else a.ctypes.data_as(P(t))


class OracleGraph(C.Structure):
    _fields_ = [("vertex_count", u32), ("edge_count", u32), ("tile_count", u32), ("reserved0", u32),
                ("owner_tiles", P(u32)), ("csr_row_offsets", P(u32)), ("csr_destinations", P(u32)),
                ("csr_edge_ids", P(u32)), ("csr_weights", P(f32)), ("csc_column_offsets", P(u32)),
                ("csc_sources", P(u32)), ("csc_edge_ids", P(u32)), ("csc_weights", P(f32))]


class OracleQuery(C.Structure):
    _fields_ = [("source_count", u32), ("target_count", u32), ("sources", P(u32)), ("targets", P(u32)),
                ("selected", P(C.c_uint8))]


class Oracle:
    """CPU restatement of the reference algorithm (bounded Dijkstra + min-eid tight predecessor)."""

    def __init__(self, arrays: dict, tile_count: int):
        if not ORACLE_SO.exists():
            build()
        self.lib = C.CDLL(str(ORACLE_SO))
        self.a = {k: np.ascontiguousarray(v) for k, v in arrays.items()}
        a = self.a
        self.V = int(a["owner_tiles"].shape[0])
        self.T = int(tile_count)
        self.g = OracleGraph(self.V, int(a["csr_destinations"].shape[0]), self.T, 0, _p(a["owner_tiles"]),
                             _p(a["csr_row_offsets"]), _p(a["csr_destinations"]), _p(a["csr_edge_ids"]),
                             _p(a["csr_weights"], f32), _p(a["csc_column_offsets"]), _p(a["csc_sources"]),
                             _p(a["csc_edge_ids"]), _p(a["csc_weights"], f32))

    @classmethod
    def from_layout(cls, layout) -> "Oracle":
        return cls(layout.arrays, layout.tile_count)

    def _query(self, sources, targets, selected_tiles, keep: list):
        s = np.ascontiguousarray(np.asarray(sources, np.uint32))
        t = np.ascontiguousarray(np.asarray(targets, np.uint32))
        sel = np.zeros(self.T, np.uint8)
        sel[np.asarray(selected_tiles, np.int64)] = 1
        keep += [s, t, sel]
        return OracleQuery(len(s), len(t), _p(s), _p(t), _p(sel, C.c_uint8))

    def region_sssp(self, sources, targets, selected_tiles):
        keep = []
        q = self._query(sources, targets, selected_tiles, keep)
        d = np.empty(self.V, np.uint32)
        pr = np.empty(self.V, np.uint32)
        self.lib.oracle_region_sssp(C.byref(self.g), C.byref(q), _p(d), _p(pr))
        return d, pr

    def region_sssp_many(self, queries, threads: int = 8):
        """queries: objects with .sources/.targets/.selected_tiles; returns (dist[nq,V], pred[nq,V])."""
        keep = []
        qs = (OracleQuery * len(queries))(*[self._query(q.sources, q.targets, q.selected_tiles, keep)
                                           for q in queries])
        d = np.empty((len(queries), self.V), np.uint32)
        pr = np.empty((len(queries), self.V), np.uint32)
        self.lib.oracle_region_sssp_many(C.byref(self.g), u32(len(queries)), qs, u32(threads), _p(d), _p(pr))
        return d, pr

    def compact_path(self, sources, targets, selected_tiles, dist_bits, target, cap: int | None = None):
        keep = []
        q = self._query(sources, targets, selected_tiles, keep)
        cap = cap if cap is not None else self.V
        verts = np.zeros(cap + 1, np.uint32)
        edges = np.zeros(max(cap, 1), np.uint32)
        n = u32()
        db = np.ascontiguousarray(dist_bits, np.uint32)
        st = self.lib.oracle_compact_path(C.byref(self.g), C.byref(q), _p(db), u32(target), u32(cap), _p(verts),
                                          _p(edges), C.byref(n))
        L = n.value
        return st, (verts[:L + 1].copy() if st == 0 else verts[:0]), (edges[:L].copy() if st == 0 else edges[:0])

    def edge_usage_adjoint(self, edge_count: int, paths: list, gvals) -> np.ndarray:
        off = np.zeros(len(paths) + 1, np.uint32)
        off[1:] = np.cumsum([len(p) for p in paths])
        flat = np.ascontiguousarray(np.concatenate(paths) if paths else np.zeros(0), np.uint32)
        g = np.ascontiguousarray(gvals, np.float32)
        grad = np.zeros(edge_count, np.float32)
        rc = self.lib.oracle_edge_usage_adjoint(u32(edge_count), u32(len(paths)), _p(off), _p(flat), _p(g, f32),
                                                _p(grad, f32))
        assert rc == 0
        return grad


class RefTiles:
    """Tile table of a reference case, shaped like a layout's `.tiles` for the
    query samplers (bfx.workloads.box_queries / full_graph_queries)."""

    def __init__(self, tiles: dict, vertex_count: int, tile_count: int):
        self.tiles = tiles
        self.vertex_count = vertex_count
        self.tile_count = tile_count


class Ref:
    """The reference's own CPU library (oracle/_ref), when built."""

    @staticmethod
    def available() -> bool:
        return REF_SO.exists()

    def __init__(self):
        self.lib = C.CDLL(str(REF_SO))
        self.lib.ref_last_error.restype = C.c_char_p
        self.lib.ref_case_name.restype = C.c_char_p
        self.lib.ref_plan_fingerprint.restype = u64
        self.lib.ref_time_dijkstra.restype = C.c_double
        self.lib.ref_compact_paths.restype = C.c_longlong

    def _chk(self, rc):
        if rc < 0:
            raise RuntimeError(self.lib.ref_last_error().decode())
        return rc

    def case_from_input(self, g, order) -> int:
        return self._chk(self.lib.ref_case_from_input(
            u32(g.vertex_count), _p(g.x, C.c_int32), _p(g.y, C.c_int32), _p(g.has_location, C.c_uint8),
            _p(g.resource_class, C.c_uint16), u64(g.edge_count), _p(g.edge_source), _p(g.edge_destination),
            _p(g.edge_weight, f32), _p(g.provenance_domain), _p(g.provenance_kind), _p(g.provenance_record, u64),
            C.c_int32(order.origin_x), C.c_int32(order.origin_y), u32(order.tile_width), u32(order.tile_height)))

    def case_synth(self, spec: dict) -> int:
        """A case from the synthetic graph generator restated in ref_driver.cpp
        (same parameters as bfx.workloads.GRAPHS), partitioned by the reference."""
        spans = np.zeros(8, np.uint32)
        spans[:len(spec["spans"])] = spec["spans"]
        base = np.zeros(8, np.float32)
        base[:len(spec.get("span_base", ()))] = spec.get("span_base", ())
        return self._chk(self.lib.ref_case_synth(
            u32(spec["tiles_x"]), u32(spec["tiles_y"]), u32(spec["nodes_per_tile"]), u32(spec["intra"]),
            u32(spec["inter"]), u32(len(spec["spans"])), _p(spans), u32(spec.get("cost_kind", 0)),
            u32(spec.get("cost_lo", 1)), u32(spec.get("cost_hi", 64)), f32(spec.get("intra_base", 1.0)),
            _p(base, f32), f32(spec.get("sigma", 0.5)), u64(spec["seed"])))

    def tiles(self, h) -> "RefTiles":
        """The case's tile table (coordinates, located flags, vertex offsets)."""
        c = self.counts(h)
        T = c["T"]
        xy = np.zeros(2 * T, np.int64)
        has = np.zeros(T, np.uint8)
        tvo = np.zeros(T + 1, np.uint32)
        nul = [None] * 16
        self._chk(self.lib.ref_case_layout(C.c_int(h), *nul, _p(xy, C.c_int64), _p(has, C.c_uint8), _p(tvo)))
        return RefTiles({"tile_xy": xy.reshape(T, 2), "has_location": has, "tile_vertex_offsets": tvo}, c["V"], T)

    def time_dijkstra_steps(self, h, qidx, threads: int, warmup: int, steps: int, want_dist: bool = False):
        """Induced graphs built once, then `warmup` + `steps` passes of
        dijkstra_oracle over all listed queries (one query per thread)."""
        q = np.ascontiguousarray(qidx, np.uint32)
        walls = np.zeros(max(steps, 1), np.float64)
        ind = C.c_double()
        edges = u64()
        dist = np.zeros((len(q), self.counts(h)["V"]), np.float32) if want_dist else None
        self._chk(self.lib.ref_time_dijkstra_steps(C.c_int(h), u32(len(q)), _p(q), u32(threads), u32(warmup),
                                                   u32(steps), _p(walls, C.c_double), C.byref(ind),
                                                   C.byref(edges), _p(dist, f32)))
        return {"step_s": walls[:steps].tolist(), "induced_wall_s": ind.value, "edges": int(edges.value),
                "dist": dist}

    def fixture_count(self, suite: str) -> int:
        return self.lib.ref_fixture_count(suite.encode())

    def case_fixture(self, suite: str, index: int) -> int:
        return self._chk(self.lib.ref_case_fixture(suite.encode(), C.c_int(index)))

    def name(self, h) -> str:
        return self.lib.ref_case_name(C.c_int(h)).decode()

    def free(self, h):
        self.lib.ref_case_free(C.c_int(h))

    def counts(self, h) -> dict:
        out = (u64 * 9)()
        self._chk(self.lib.ref_case_counts(C.c_int(h), out))
        keys = ("V", "E", "T", "csr_runs", "csc_runs", "queries", "expected_reached", "expected_miss", "four_ulps")
        return dict(zip(keys, (int(x) for x in out)))

    def layout(self, h) -> tuple[dict, dict]:
        c = self.counts(h)
        V, E, T, R1, R2 = c["V"], c["E"], c["T"], c["csr_runs"], c["csc_runs"]
        a = {"owner_tiles": np.zeros(V, np.uint32), "csr_row_offsets": np.zeros(V + 1, np.uint32),
             "csr_destinations": np.zeros(E, np.uint32), "csr_weights": np.zeros(E, np.float32),
             "csr_row_run_offsets": np.zeros(V + 1, np.uint32), "csr_run_edge_offsets": np.zeros(R1 + 1, np.uint32),
             "csr_run_destination_tiles": np.zeros(R1, np.uint32), "csc_column_offsets": np.zeros(V + 1, np.uint32),
             "csc_sources": np.zeros(E, np.uint32), "csc_weights": np.zeros(E, np.float32),
             "csc_edge_ids": np.zeros(E, np.uint32), "csc_column_run_offsets": np.zeros(V + 1, np.uint32),
             "csc_run_edge_offsets": np.zeros(R2 + 1, np.uint32), "csc_run_source_tiles": np.zeros(R2, np.uint32),
             "csr_edge_ids": np.zeros(E, np.uint32)}
        t = {"new_to_old": np.zeros(V, np.uint32), "tile_xy": np.zeros(2 * T, np.int64),
             "has_location": np.zeros(T, np.uint8), "tile_vertex_offsets": np.zeros(T + 1, np.uint32)}
        order = ["owner_tiles", "csr_row_offsets", "csr_destinations", "csr_weights", "csr_row_run_offsets",
                 "csr_run_edge_offsets", "csr_run_destination_tiles", "csc_column_offsets", "csc_sources",
                 "csc_weights", "csc_edge_ids", "csc_column_run_offsets", "csc_run_edge_offsets",
                 "csc_run_source_tiles", "csr_edge_ids"]
        args = [_p(a[k], f32 if a[k].dtype == np.float32 else u32) for k in order]
        self._chk(self.lib.ref_case_layout(C.c_int(h), *args, _p(t["new_to_old"]), _p(t["tile_xy"], C.c_int64),
                                           _p(t["has_location"], C.c_uint8), _p(t["tile_vertex_offsets"])))
        t["tile_xy"] = t["tile_xy"].reshape(T, 2)
        return a, t

    def query_add(self, h, qid, sources, targets, tiles=None) -> int:
        s = np.ascontiguousarray(sources, np.uint32)
        t = np.ascontiguousarray(targets, np.uint32)
        tl = np.ascontiguousarray(tiles if tiles is not None else np.zeros(0), np.uint32)
        return self._chk(self.lib.ref_query_add(C.c_int(h), u32(qid), u32(len(s)), _p(s), u32(len(t)), _p(t),
                                                u32(len(tl)), _p(tl)))

    def query(self, h, q) -> dict:
        c = (u32 * 4)()
        self._chk(self.lib.ref_query_counts(C.c_int(h), C.c_int(q), c))
        s = np.zeros(c[1], np.uint32)
        t = np.zeros(c[2], np.uint32)
        tl = np.zeros(c[3], np.uint32)
        self._chk(self.lib.ref_query_export(C.c_int(h), C.c_int(q), _p(s), _p(t), _p(tl)))
        return {"query_id": int(c[0]), "sources": s, "targets": t, "selected_tiles": tl}

    def dijkstra(self, h, q, V) -> np.ndarray:
        d = np.zeros(V, np.float32)
        self._chk(self.lib.ref_dijkstra(C.c_int(h), C.c_int(q), _p(d, f32)))
        return d

    def bellman_ford(self, h, q, V) -> np.ndarray:
        d = np.zeros(V, np.float32)
        self._chk(self.lib.ref_bellman_ford(C.c_int(h), C.c_int(q), _p(d, f32)))
        return d

    def compact_paths(self, h, q, dist: np.ndarray, ntargets: int):
        d = np.ascontiguousarray(dist, np.float32)
        st = np.zeros(ntargets, np.uint32)
        rc = np.zeros(ntargets, np.uint32)
        ln = np.zeros(ntargets, np.uint32)
        total = self._chk(self.lib.ref_compact_paths(C.c_int(h), C.c_int(q), _p(d, f32), _p(st), _p(rc), _p(ln),
                                                     None, u64(0), None, u64(0)))
        verts = np.zeros(total + ntargets, np.uint32)
        edges = np.zeros(max(total, 1), np.uint32)
        self._chk(self.lib.ref_compact_paths(C.c_int(h), C.c_int(q), _p(d, f32), _p(st), _p(rc), _p(ln),
                                             _p(verts), u64(len(verts)), _p(edges), u64(len(edges))))
        return st, rc, ln, verts, edges[:total]

    def plan(self, h, lane_width=32, jn=1, jd=8, inn=2, ind=1) -> int:
        return self._chk(self.lib.ref_plan(C.c_int(h), u32(lane_width), u32(jn), u32(jd), u32(inn), u32(ind)))

    def plan_batch(self, h, b, lane_width) -> dict:
        cnt = (u32 * 3)()
        self._chk(self.lib.ref_plan_batch(C.c_int(h), C.c_int(b), cnt, None, None, None, None))
        lq = np.zeros(cnt[0], np.uint32)
        ut = np.zeros(cnt[2], np.uint32)
        um = np.zeros(cnt[2], np.uint32)
        est = np.zeros(4, np.uint64)
        self._chk(self.lib.ref_plan_batch(C.c_int(h), C.c_int(b), cnt, _p(lq), _p(ut), _p(um), _p(est, u64)))
        return {"lane_width": int(cnt[0]), "valid": int(cnt[1]), "lane_query": lq, "union_tiles": ut,
                "union_masks": um, "estimates": est}

    def plan_fingerprint(self, h) -> int:
        return int(self.lib.ref_plan_fingerprint(C.c_int(h)))

    def describe_batch(self, h, b, T) -> dict:
        cnt = (u32 * 6)()
        self._chk(self.lib.ref_describe_batch(C.c_int(h), C.c_int(b), cnt, None, None, None, None, None, None,
                                              None))
        W, valid, S, Tg, U, R = (int(x) for x in cnt)
        out = {"lane_width": W, "valid": valid, "source_offsets": np.zeros(W + 1, np.uint32),
               "sources": np.zeros(S, np.uint32), "target_offsets": np.zeros(W + 1, np.uint32),
               "targets": np.zeros(Tg, np.uint32), "union_tiles": np.zeros(U, np.uint32),
               "tile_lane_masks": np.zeros(T, np.uint32), "ranges": np.zeros(3 * R, np.uint32)}
        self._chk(self.lib.ref_describe_batch(C.c_int(h), C.c_int(b), cnt, _p(out["source_offsets"]),
                                              _p(out["sources"]), _p(out["target_offsets"]), _p(out["targets"]),
                                              _p(out["union_tiles"]), _p(out["tile_lane_masks"]), _p(out["ranges"])))
        out["ranges"] = out["ranges"].reshape(R, 3)
        return out

    def run_batched(self, h, b, engine, V, W, max_rounds=1 << 40):
        bits = np.zeros(V * W, np.uint32)
        st = np.zeros(12, np.uint32)
        self._chk(self.lib.ref_run_batched(C.c_int(h), C.c_int(b), C.c_int(engine), u64(max_rounds), _p(bits),
                                           st.ctypes.data_as(C.c_void_p)))
        keys = ("final_distance_slot", "converged", "rounds_lo", "rounds_hi", "reached_target_mask",
                "bounding_box_miss_mask", "valid_lane_mask", "active_lane_mask", "converged_lane_mask",
                "stop_reason", "error_bits", "reserved0")
        return bits.reshape(V, W), dict(zip(keys, (int(x) for x in st)))

    def time_dijkstra(self, h, qidx, threads: int):
        q = np.ascontiguousarray(qidx, np.uint32)
        ind = C.c_double()
        ss = C.c_double()
        edges = u64()
        wall = self.lib.ref_time_dijkstra(C.c_int(h), u32(len(q)), _p(q), u32(threads), C.byref(ind),
                                          C.byref(ss), C.byref(edges))
        return {"wall_s": wall, "induced_s": ind.value, "sssp_s": ss.value, "edges": int(edges.value)}

    def expansion_run(self, h, nq: int, engine: int, policy: tuple, schedule_kind: int, fixed_ring: int,
                      hybrid_count: int, maximum_expansions: int, terminal_policy: int, tile_cap: int,
                      max_rounds: int = 1 << 40) -> dict:
        """Reference run_host_batched_expansion over all queries of case h
        (src/batched_expansion.cpp:1681): outcomes in query-id order."""
        params = np.array([engine, *policy, schedule_kind, fixed_ring, hybrid_count, maximum_expansions,
                           terminal_policy], np.uint64)
        outc = np.zeros(12 * nq, np.uint64)
        tiles = np.zeros(tile_cap, np.uint32)
        metrics = np.zeros(24, np.uint64)
        hist = np.zeros(64, np.uint64)
        counts = np.zeros(2, np.uint64)
        self._chk(self.lib.ref_expansion_run(C.c_int(h), _p(params, u64), u64(max_rounds), _p(outc, u64),
                                             _p(tiles), u64(tile_cap), _p(metrics, u64), _p(hist, u64),
                                             _p(counts, u64)))
        return {"outcomes": outc.reshape(nq, 12), "tiles": tiles[:int(counts[0])], "metrics": metrics,
                "histogram": hist[:int(counts[1])]}
