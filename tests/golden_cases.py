"""Loads the reference-generated golden fixtures (tests/golden/*.npz)."""
from __future__ import annotations

from dataclasses import dataclass
from pathlib import Path

import numpy as np

import bfx

GOLDEN = Path(__file__).resolve().parent / "golden"


@dataclass
class GoldenQuery:
    query: bfx.RouteQuery
    dist: np.ndarray          # reference dijkstra distances (float bits), V
    path_status: np.ndarray   # per canonical target
    path_len: np.ndarray
    path_vertices: np.ndarray  # concatenated, len+1 per complete target
    path_edges: np.ndarray     # concatenated, len per complete target

    def paths(self):
        """[(status, vertices, edges)] per target."""
        out, vo, eo = [], 0, 0
        for st, ln in zip(self.path_status, self.path_len):
            if st == 0:
                out.append((0, self.path_vertices[vo:vo + ln + 1], self.path_edges[eo:eo + ln]))
                vo += int(ln) + 1
                eo += int(ln)
            else:
                out.append((int(st), None, None))
        return out


@dataclass
class GoldenCase:
    name: str
    layout: bfx.DeviceGraphLayout
    queries: list
    expected_reached: int
    expected_miss: int
    four_ulps: bool
    raw: dict


def load_case(path: Path) -> GoldenCase:
    z = dict(np.load(path, allow_pickle=False))
    arrays = {k[2:]: v for k, v in z.items() if k.startswith("L_")}
    arrays["tile_count"] = np.uint32(z["tile_count"])
    tiles = {k[2:]: v for k, v in z.items() if k.startswith("T_")}
    layout = bfx.DeviceGraphLayout(arrays, tiles)
    qs = []
    for q in range(int(z["query_count"])):
        rq = bfx.RouteQuery(int(z[f"Q{q}_query_id"]), z[f"Q{q}_sources"], z[f"Q{q}_targets"],
                            z[f"Q{q}_selected_tiles"])
        qs.append(GoldenQuery(rq, z[f"Q{q}_dist"], z[f"Q{q}_path_status"], z[f"Q{q}_path_len"],
                              z[f"Q{q}_path_vertices"], z[f"Q{q}_path_edges"]))
    return GoldenCase(str(z["name"]), layout, qs, int(z["expected_reached"]), int(z["expected_miss"]),
                      bool(z["four_ulps"]), z)


def fixture_paths() -> list[Path]:
    return sorted(p for p in GOLDEN.glob("*.npz") if p.name != "synthetic_c1.npz")
