"""Seeded synthetic workloads shaped like the benchmark configurations.

The reference's real workload (FPGA routing-contest query artifacts) is not
available, so graphs and query sets with the configured shapes, sizes and
cost distributions are generated here:

  c1  32x32 tiles x 64 nodes, 4 intra + 2 inter (spans 1,2,4), uint costs U[1,64];
      8 full-graph sources, one uniform target each, one batch of width 8.
  c2  128x128 tiles x 128 nodes, 6 intra + 2 inter (spans 1,2,4,8), float costs
      base(span) * lognormal(0, 0.5) with base 1 (intra, span 1), 1.8, 3.2, 6;
      256 regional queries: box side U[4,64] tiles, source and one target uniform
      in the box.
  c3  256x256 tiles x 256 nodes, 7 intra + 3 inter (spans 1,2,4,12), uint costs
      U[1,255]; 64 full-graph sources in batches of 32.
  c4  c1 graph with c2's float costs; 512 nets of one source and U[1,32]
      targets in a box of side U[8,48] clipped to the grid.
  c5  c3 graph; 4096 regional queries (box side U[2,16]) plus 16 full-graph.

Graph generation runs in libbfx (xoshiro256** seeded by splitmix64); query
sampling uses numpy's PCG64 generator seeded per configuration.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import (BatchPlannerPolicy, DeviceGraphLayout, RouteQuery, build_device_graph_layout, make_description,
               make_overlapping_batch_plan, synth_graph)

GRAPHS = {
    "c1": dict(tiles_x=32, tiles_y=32, nodes_per_tile=64, intra=4, inter=2, spans=(1, 2, 4), cost_kind=0,
               cost_lo=1, cost_hi=64, seed=0xC1),
    "c1f": dict(tiles_x=32, tiles_y=32, nodes_per_tile=64, intra=4, inter=2, spans=(1, 2, 4), cost_kind=1,
                intra_base=1.0, span_base=(1.0, 1.8, 3.2), sigma=0.5, seed=0xC4),
    "c2": dict(tiles_x=128, tiles_y=128, nodes_per_tile=128, intra=6, inter=2, spans=(1, 2, 4, 8), cost_kind=1,
               intra_base=1.0, span_base=(1.0, 1.8, 3.2, 6.0), sigma=0.5, seed=0xC2),
    "c3": dict(tiles_x=256, tiles_y=256, nodes_per_tile=256, intra=7, inter=3, spans=(1, 2, 4, 12), cost_kind=0,
               cost_lo=1, cost_hi=255, seed=0xC3),
}


@dataclass
class Workload:
    name: str
    layout: DeviceGraphLayout
    queries: list
    grid: tuple

    def tile_id(self, tx: int, ty: int) -> int:
        return int(self._tile_index[ty, tx])

    def __post_init__(self):
        xy = self.layout.tiles["tile_xy"]
        has = self.layout.tiles["has_location"]
        TX, TY = self.grid
        self._tile_index = np.full((TY, TX), -1, np.int64)
        for t in range(xy.shape[0]):
            if has[t]:
                self._tile_index[xy[t, 1], xy[t, 0]] = t


def build_graph(name: str, threads: int = 0, scale_tiles: tuple | None = None) -> tuple:
    """(layout, grid) for a named graph; scale_tiles overrides the tile grid for small tests."""
    spec = dict(GRAPHS[name])
    if scale_tiles:
        spec["tiles_x"], spec["tiles_y"] = scale_tiles
    g, order, _ = synth_graph(**spec)
    layout = build_device_graph_layout(g, order, threads)
    return layout, (spec["tiles_x"], spec["tiles_y"])


def _vertex_in_tile(layout: DeviceGraphLayout, tile: int, rng) -> int:
    tvo = layout.tiles["tile_vertex_offsets"]
    return int(tvo[tile] + rng.integers(0, int(tvo[tile + 1] - tvo[tile])))


def full_graph_queries(layout, grid, n: int, seed: int, first_id: int = 0, targets_per_query: int = 1):
    rng = np.random.default_rng(seed)
    V = layout.vertex_count
    T = layout.tile_count
    all_tiles = np.arange(T, dtype=np.uint32)
    qs = []
    for i in range(n):
        s = int(rng.integers(0, V))
        t = rng.integers(0, V, size=targets_per_query)
        qs.append(RouteQuery(first_id + i, [s], t, all_tiles))
    return qs


def box_queries(wl_layout, grid, n: int, side_lo: int, side_hi: int, seed: int, first_id: int = 0,
                targets=(1, 1), clip: int | None = None):
    """Regional queries: a box of side U[side_lo, side_hi] tiles (clipped to the
    grid), one source and U[targets] targets uniform in the box."""
    rng = np.random.default_rng(seed)
    TX, TY = grid
    xy = wl_layout.tiles["tile_xy"]
    has = wl_layout.tiles["has_location"]
    index = np.full((TY, TX), -1, np.int64)
    for t in range(xy.shape[0]):
        if has[t]:
            index[xy[t, 1], xy[t, 0]] = t
    qs = []
    for i in range(n):
        sx = min(int(rng.integers(side_lo, side_hi + 1)), clip or TX, TX)
        sy = min(int(rng.integers(side_lo, side_hi + 1)), clip or TY, TY)
        x0 = int(rng.integers(0, TX - sx + 1))
        y0 = int(rng.integers(0, TY - sy + 1))
        tiles = index[y0:y0 + sy, x0:x0 + sx].ravel()
        tiles = np.sort(tiles[tiles >= 0]).astype(np.uint32)

        def pick():
            return _vertex_in_tile(wl_layout, int(tiles[rng.integers(0, len(tiles))]), rng)

        src = pick()
        nt = int(rng.integers(targets[0], targets[1] + 1))
        tg = [pick() for _ in range(nt)]
        qs.append(RouteQuery(first_id + i, [src], tg, tiles))
    return qs


def make_workload(name: str, threads: int = 0, scale_tiles: tuple | None = None, query_count: int | None = None):
    """Graph + query set of a configuration (c1..c5)."""
    graph = {"c1": "c1", "c2": "c2", "c3": "c3", "c4": "c1f", "c5": "c3"}[name]
    layout, grid = build_graph(graph, threads, scale_tiles)
    seed = {"c1": 101, "c2": 202, "c3": 303, "c4": 404, "c5": 505}[name]
    if name == "c1":
        qs = full_graph_queries(layout, grid, query_count or 8, seed)
    elif name == "c2":
        qs = box_queries(layout, grid, query_count or 256, 4, 64, seed)
    elif name == "c3":
        qs = full_graph_queries(layout, grid, query_count or 64, seed)
    elif name == "c4":
        qs = box_queries(layout, grid, query_count or 512, 8, 48, seed, targets=(1, 32), clip=32)
    else:
        qs = box_queries(layout, grid, query_count or 4096, 2, 16, seed)
        qs += full_graph_queries(layout, grid, 16, seed + 1, first_id=len(qs))
    return Workload(name, layout, qs, grid)


def plan_batches(layout, queries, lane_width: int = 32, narrow: bool = True, policy: BatchPlannerPolicy | None = None):
    """Planner + descriptions (the reference's default policy unless given)."""
    policy = policy or BatchPlannerPolicy(lane_width=lane_width, narrow_lanes=narrow)
    return make_overlapping_batch_plan(layout, queries, policy)


def sequential_batches(layout, queries, lane_width: int = 32):
    """Queries packed in order into batches of `lane_width` lanes (no planner)."""
    out = []
    for i in range(0, len(queries), lane_width):
        out.append(make_description(layout, queries[i:i + lane_width], lane_width))
    return out


def shard_batches(lane_edge_estimates, world: int) -> list:
    """Replica sharding: every rank holds the whole graph, batches are split
    so each rank gets a near-equal share of estimated lane-edges (greedy
    longest-first onto the least-loaded rank; ties by rank).  Deterministic,
    so every rank computes the same assignment without communicating."""
    order = sorted(range(len(lane_edge_estimates)), key=lambda b: (-int(lane_edge_estimates[b]), b))
    loads = [0] * world
    shards = [[] for _ in range(world)]
    for b in order:
        r = min(range(world), key=lambda i: (loads[i], i))
        shards[r].append(b)
        loads[r] += int(lane_edge_estimates[b])
    return [sorted(s) for s in shards]


@dataclass
class BenchWorkload:
    """A timed configuration: graph input, layout, query set, the query
    classes the plain per-query baseline samples (queries, sample size) and
    the planner policy."""
    name: str
    graph_input: object
    order: object
    layout: DeviceGraphLayout
    grid: tuple
    queries: list
    classes: list
    policy: BatchPlannerPolicy
    description: str
    uint_costs: bool


def bench_queries(name: str, tiles, grid, rank: int = 0, query_count: int | None = None):
    """(queries, classes) of a timed configuration, from the tile table of its
    layout (`tiles`: any object with the layout's `.tiles` dict and
    `.vertex_count`), so the reference's own layout of the same input gives
    the same queries.  Rank r of a replica run draws its own set (seed
    offset 1000 r)."""
    off = 1000 * rank
    if name == "c2":
        qs = box_queries(tiles, grid, query_count or 256, 4, 64, 202 + off)
        return qs, [(qs, 64)]
    if name in ("c3", "c3small"):
        qs = full_graph_queries(tiles, grid, query_count or (64 if name == "c3" else 32), 303 + off)
        return qs, [(qs, 4 if name == "c3" else 2)]
    if name == "c5":
        regional = box_queries(tiles, grid, query_count or 4096, 2, 16, 505 + off)
        full = full_graph_queries(tiles, grid, 16, 506 + off, first_id=len(regional))
        return regional + full, [(regional, 64), (full, 2)]
    raise ValueError(f"unknown timed workload {name}")


def bench_graph_spec(name: str) -> tuple[dict, tuple]:
    """Synthetic graph parameters and tile grid of a timed configuration."""
    spec = dict(GRAPHS["c3" if name in ("c5", "c3small") else name])
    if name == "c3small":  # c3 generator on 128x128 tiles: a profiling-sized case of the c3 kernel
        spec["tiles_x"] = spec["tiles_y"] = 128
    return spec, (spec["tiles_x"], spec["tiles_y"])


BENCH_DESCRIPTIONS = {
    "c2": ("c2: 256 uneven regional queries (box side U[4,64] tiles) on 128x128 tiles x 128 nodes, "
           "2,097,152 V / 16,777,216 E, f32 lognormal costs"),
    "c3small": ("c3small: 32 full-graph sources in one batch of 32 on 128x128 tiles x 256 nodes, "
                "4,194,304 V / 41,943,040 E, uint costs U[1,255] (profiling-sized c3)"),
    "c3": ("c3: 64 full-graph sources in batches of 32 on 256x256 tiles x 256 nodes, "
           "16,777,216 V / 167,772,160 E, uint costs U[1,255]"),
    "c5": ("c5: 4,096 regional queries (box side U[2,16] tiles) + 16 full-graph sources on 256x256 "
           "tiles x 256 nodes, 16,777,216 V / 167,772,160 E, uint costs U[1,255]"),
}


def bench_workload(name: str, rank: int = 0, query_count: int | None = None, threads: int = 0,
                   keep_input: bool = False) -> BenchWorkload:
    """The exact graph, query set and planner policy that bench.py times.  The
    input graph (edge records, vertex metadata: 4.7 GB on c3) is dropped once
    the layout is built unless `keep_input`."""
    spec, grid = bench_graph_spec(name)
    g, order, _ = synth_graph(**spec)
    layout = build_device_graph_layout(g, order, threads)
    if not keep_input:
        g = None
    queries, classes = bench_queries(name, layout, grid, rank, query_count)
    if name in ("c2", "c5"):
        policy = BatchPlannerPolicy(32, 1, 8, 2, 1, narrow_lanes=True)
    else:
        policy = BatchPlannerPolicy(32, 0, 1, 64, 1)
    return BenchWorkload(name, g, order, layout, grid, queries, classes, policy, BENCH_DESCRIPTIONS[name],
                         spec["cost_kind"] == 0)
