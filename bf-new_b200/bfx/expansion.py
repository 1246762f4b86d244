"""Expansion loop (bfx_expansion.h): regional queries that miss a target are
retried on larger regions -- bfnew::run_batched_expansion
(src/batched_expansion.cpp:888) with the same schedules, terminal policies and
per-query outcomes.  `run_expansion(workspace, ...)` relaxes each planning
pass in one GPU launch; `run_expansion_with_runner(runner, ...)` takes a
caller-supplied pass runner (the reference's ExpansionBatchRunner boundary).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Callable, Sequence

import numpy as np

from . import (BatchDescriptionC, BatchPlannerPolicy, DeviceGraphLayout, DeviceRunStatus, GpuRunOptions,
               PlannerPolicyC, RouteQuery, RouteQueryC, _check, _ptr, load)

u32, u64 = C.c_uint32, C.c_uint64
P = C.POINTER

ONE_RING, FIXED_RING, DOUBLING, HYBRID = 1, 2, 3, 4
FULL_REGION_FALLBACK, EXPLICIT_FAILURE = 0, 1
DISPOSITIONS = ("reached", "unreachable_in_full_region", "expansion_limit", "region_stalled",
                "identity_or_count_overflow", "engine_failure")

OUTCOME_FIELDS = ("query_id", "disposition", "attempts", "scheduled_expansions", "total_expansions",
                  "used_full_region_fallback", "expansion_generation", "final_tile_count", "selected_vertex_count",
                  "selected_edge_count", "terminal_stop_reason", "terminal_error_bits")
METRIC_FIELDS = ("input_queries", "initial_reached_queries", "reached_queries", "unreachable_full_region_queries",
                 "expansion_limit_queries", "stalled_region_queries", "identity_or_count_overflow_queries",
                 "engine_failure_queries", "planning_passes", "batches_executed", "initial_batches_executed",
                 "retry_batches_executed", "failed_lane_observations", "failed_origin_valid_lane_observations",
                 "retry_valid_lane_observations", "retry_lane_capacity", "scheduled_expansions",
                 "full_region_fallbacks", "repeated_selected_edge_estimate", "attempted_selected_vertex_count",
                 "attempted_selected_edge_estimate", "final_selected_tile_count", "final_selected_vertex_count",
                 "final_selected_edge_count")


class ExpansionOptionsC(C.Structure):
    _fields_ = [("run_options", GpuRunOptions), ("planner_policy", PlannerPolicyC), ("schedule_kind", u32),
                ("fixed_ring_size", u32), ("hybrid_small_expansion_count", u32), ("maximum_expansions", u32),
                ("terminal_policy", u32), ("reserved0", u32)]


class ExpansionOutcomeC(C.Structure):
    _fields_ = [(f, u64 if f in ("selected_vertex_count", "selected_edge_count") else u32)
                for f in OUTCOME_FIELDS]


class ExpansionMetricsC(C.Structure):
    _fields_ = [(f, u64) for f in METRIC_FIELDS] + [("relaxation_launches", u64)]


class TileGeometryC(C.Structure):
    _fields_ = [("tile_count", u32), ("reserved0", u32), ("tile_xy", P(C.c_int64)),
                ("has_location", P(C.c_uint8)), ("tile_vertex_offsets", P(u32))]


RunnerFn = C.CFUNCTYPE(C.c_int, C.c_void_p, u32, P(BatchDescriptionC), P(DeviceRunStatus))

assert C.sizeof(ExpansionOutcomeC) == 56 and C.sizeof(ExpansionOptionsC) == 96


@dataclass
class ExpansionOptions:
    """bfnew::BatchedExpansionOptions (include/bfnew/batched_expansion.hpp:68-110)."""
    schedule_kind: int = ONE_RING
    maximum_expansions: int = 4
    terminal_policy: int = FULL_REGION_FALLBACK
    fixed_ring_size: int = 0
    hybrid_small_expansion_count: int = 0
    engine: int = 2
    maximum_rounds: int = 1 << 40
    planner_policy: BatchPlannerPolicy = None

    def c(self) -> ExpansionOptionsC:
        pp = self.planner_policy or BatchPlannerPolicy()
        return ExpansionOptionsC(GpuRunOptions(engine=self.engine, maximum_rounds=self.maximum_rounds), pp.c(),
                                 self.schedule_kind, self.fixed_ring_size, self.hybrid_small_expansion_count,
                                 self.maximum_expansions, self.terminal_policy, 0)


class _Inputs:
    def __init__(self, layout: DeviceGraphLayout, queries: Sequence[RouteQuery]):
        self.view = layout.view()
        self.xy = np.ascontiguousarray(layout.tiles["tile_xy"], np.int64)
        self.loc = np.ascontiguousarray(layout.tiles["has_location"], np.uint8)
        self.tvo = np.ascontiguousarray(layout.tiles["tile_vertex_offsets"], np.uint32)
        self.geo = TileGeometryC(int(layout.tile_count), 0, _ptr(self.xy, C.c_int64), _ptr(self.loc, C.c_uint8),
                                 _ptr(self.tvo))
        self.queries = list(queries)
        self.qc = (RouteQueryC * len(self.queries))(*[q.c() for q in self.queries])


def _collect(h) -> dict:
    lib = load()
    try:
        m = ExpansionMetricsC()
        _check(lib.bfx_expansion_metrics_get(h, C.byref(m)))
        n = int(m.input_queries)
        outs = (ExpansionOutcomeC * n)()
        _check(lib.bfx_expansion_outcomes(h, outs))
        outcomes, tiles = [], []
        for i in range(n):
            o = {f: int(getattr(outs[i], f)) for f in OUTCOME_FIELDS}
            outcomes.append(o)
            t = np.zeros(max(o["final_tile_count"], 1), np.uint32)
            _check(lib.bfx_expansion_final_tiles(h, u32(i), _ptr(t)))
            tiles.append(t[:o["final_tile_count"]])
        cnt = u32()
        _check(lib.bfx_expansion_histogram(h, C.byref(cnt), None))
        hist = (u64 * max(cnt.value, 1))()
        _check(lib.bfx_expansion_histogram(h, C.byref(cnt), hist))
        metrics = {f: int(getattr(m, f)) for f in METRIC_FIELDS}
        metrics["relaxation_launches"] = int(m.relaxation_launches)
        return {"outcomes": outcomes, "final_tiles": tiles, "metrics": metrics,
                "histogram": [int(x) for x in hist[:cnt.value]]}
    finally:
        lib.bfx_expansion_destroy(h)


def run_expansion(workspace, layout: DeviceGraphLayout, queries: Sequence[RouteQuery],
                  options: ExpansionOptions) -> dict:
    """bfx_expansion_run: every planning pass relaxed in one launch on `workspace`."""
    inp = _Inputs(layout, queries)
    h = C.c_void_p()
    _check(load().bfx_expansion_run(workspace._h, C.byref(inp.view), C.byref(inp.geo), u32(len(inp.queries)),
                                    inp.qc, C.byref(options.c()), C.byref(h)))
    return _collect(h)


def run_expansion_with_runner(runner: Callable, layout: DeviceGraphLayout, queries: Sequence[RouteQuery],
                              options: ExpansionOptions) -> dict:
    """bfx_expansion_run_with_runner.  runner(descriptions: list[BatchDescriptionC])
    returns one DeviceRunStatus per batch."""
    inp = _Inputs(layout, queries)
    err = []

    def trampoline(_user, n, descs, statuses):
        try:
            out = runner([descs[i] for i in range(n)])
            for i in range(n):
                statuses[i] = out[i]
            return 0
        except Exception as exc:  # reported through the library's status
            err.append(exc)
            return 1

    fn = RunnerFn(trampoline)
    h = C.c_void_p()
    rc = load().bfx_expansion_run_with_runner(C.byref(inp.view), C.byref(inp.geo), u32(len(inp.queries)), inp.qc,
                                              C.byref(options.c()), fn, None, C.byref(h))
    if err:
        raise err[0]
    _check(rc)
    return _collect(h)
