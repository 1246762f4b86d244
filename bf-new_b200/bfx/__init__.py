"""Python binding of libbfx (ctypes over the C ABI in include/bfx.h, bfx_host.h).

Names mirror the reference's C++ API for the batched relaxation path so the
tests read like the reference's own:

    layout = build_device_graph_layout(input_graph, SpatialOrderConfig(...))
    resident = ResidentDeviceGraph.upload_once(layout)
    plan = make_overlapping_batch_plan(layout, queries, BatchPlannerPolicy())
    engine = BatchedFrontierPushEngine(resident, Workspace(resident))
    statuses = engine.run_compact_status(plan.descriptions(), GpuRunOptions(...))

Errors map like the reference's exceptions: std::invalid_argument ->
ValueError, std::out_of_range -> IndexError, std::overflow_error ->
OverflowError, HipRuntimeError -> BfxCudaError, std::logic_error ->
RuntimeError.  There is no CPU fallback: every engine call runs the CUDA
kernels in libbfx.so and fails loudly without a GPU.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from pathlib import Path
from typing import Sequence

import numpy as np

PKG = Path(__file__).resolve().parent.parent
LIB_PATH = PKG / "lib" / "libbfx.so"

u32, u64, i32, i64, f32 = C.c_uint32, C.c_uint64, C.c_int32, C.c_int64, C.c_float
P = C.POINTER

ENGINE_JACOBI_PULL, ENGINE_DENSE_CHAOTIC_PUSH, ENGINE_FRONTIER_PUSH = 0, 1, 2
ENGINE_AUTO = 0xFFFFFFFF
CONTROL_PERSISTENT, CONTROL_CHUNKED, CONTROL_PER_ROUND = 0, 1, 2
FRONTIER_GROUPS, FRONTIER_FLAT, FRONTIER_CHUNKED, FRONTIER_TILED = 0, 1, 2, 3
MAPPING_CHUNKS, MAPPING_TILE_VISITS = 0, 1
STOP_NONE, STOP_CONVERGED, STOP_MAXIMUM_ROUNDS, STOP_QUEUE_OVERFLOW, STOP_INVALID, STOP_FAILURE = range(6)
INF_BITS = 0x7F800000
NO_EDGE = 0xFFFFFFFF


class BfxCudaError(RuntimeError):
    """A CUDA runtime failure (the reference's HipRuntimeError)."""


class BfxNoDevice(RuntimeError):
    """No CUDA device is visible."""


class GpuRunOptions(C.Structure):
    """bfnew::GpuRunOptions (include/bfnew/gpu_api.hpp:57-67), 48 bytes."""
    _fields_ = [("engine", u32), ("control_mode", u32), ("rounds_per_chunk", u32), ("block_size", u32),
                ("grid_policy", u32), ("blocks_per_wgp", u32), ("instrumentation", u32), ("reserved0", u32),
                ("maximum_rounds", u64), ("enable_per_lane_convergence", u32), ("reserved1", u32)]

    def __init__(self, engine=ENGINE_FRONTIER_PUSH, control_mode=CONTROL_PERSISTENT, rounds_per_chunk=8,
                 block_size=256, grid_policy=0, blocks_per_wgp=0, instrumentation=0,
                 maximum_rounds=1 << 40, enable_per_lane_convergence=1):
        super().__init__(engine, control_mode, rounds_per_chunk, block_size, grid_policy, blocks_per_wgp,
                         instrumentation, 0, maximum_rounds, enable_per_lane_convergence, 0)


class DeviceController(C.Structure):
    """bfnew::DeviceController (gpu_api.hpp:100-120), 96 bytes."""
    _fields_ = [("valid_lane_mask", u32), ("active_lane_mask", u32), ("changed_lane_mask", u32),
                ("converged_lane_mask", u32), ("execute_lane_mask", u32), ("engine_kind", u32),
                ("enable_per_lane_convergence", u32), ("reserved0", u32), ("rounds_completed", u64),
                ("maximum_rounds", u64), ("distance_read_slot", u32), ("distance_write_slot", u32),
                ("frontier_read_slot", u32), ("frontier_write_slot", u32), ("frontier_size", u64 * 2),
                ("next_frontier_lane_mask", u32), ("done", u32), ("stop_reason", u32), ("error_bits", u32)]


class DeviceRunStatus(C.Structure):
    """bfnew::DeviceRunStatus (gpu_api.hpp:176-187), 48 bytes."""
    _fields_ = [("final_distance_slot", u32), ("converged", u32), ("rounds_completed", u64),
                ("reached_target_mask", u32), ("bounding_box_miss_mask", u32), ("valid_lane_mask", u32),
                ("active_lane_mask", u32), ("converged_lane_mask", u32), ("stop_reason", u32),
                ("error_bits", u32), ("reserved0", u32)]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_ if not f.startswith("reserved")}


class CompactTargetSummary(C.Structure):
    """bfnew::CompactTargetSummary (include/bfnew/compact_path_types.hpp:31-47), 28 bytes."""
    _fields_ = [("target", u32), ("selected_source", u32), ("distance", f32), ("path_length", u32),
                ("reached", u32), ("reconstruction", u32), ("has_selected_source", u32)]


class DeviceGraphLayout32View(C.Structure):
    _fields_ = [("vertex_count", u32), ("edge_count", u32), ("tile_count", u32), ("csr_run_count", u32),
                ("csc_run_count", u32), ("reserved0", u32),
                ("owner_tiles", P(u32)), ("csr_row_offsets", P(u32)), ("csr_destinations", P(u32)),
                ("csr_weights", P(f32)), ("csr_row_run_offsets", P(u32)), ("csr_run_edge_offsets", P(u32)),
                ("csr_run_destination_tiles", P(u32)), ("csc_column_offsets", P(u32)), ("csc_sources", P(u32)),
                ("csc_weights", P(f32)), ("csc_edge_ids", P(u32)), ("csc_column_run_offsets", P(u32)),
                ("csc_run_edge_offsets", P(u32)), ("csc_run_source_tiles", P(u32)), ("csr_edge_ids", P(u32))]


class BatchVertexRange(C.Structure):
    _fields_ = [("begin", u32), ("end", u32), ("lane_mask", u32)]


class BatchDescriptionC(C.Structure):
    _fields_ = [("lane_width", u32), ("valid_lane_mask", u32), ("source_offsets", P(u32)), ("sources", P(u32)),
                ("target_offsets", P(u32)), ("targets", P(u32)), ("union_tile_count", u32), ("tile_count", u32),
                ("union_tiles", P(u32)), ("tile_lane_masks", P(u32)), ("range_count", u32), ("reserved0", u32),
                ("selected_vertex_ranges", P(BatchVertexRange))]


class InputGraphC(C.Structure):
    _fields_ = [("vertex_count", u32), ("reserved0", u32), ("edge_count", u64), ("x", P(i32)), ("y", P(i32)),
                ("has_location", P(C.c_uint8)), ("resource_class", P(C.c_uint16)), ("edge_source", P(u32)),
                ("edge_destination", P(u32)), ("edge_weight", P(f32)), ("provenance_domain", P(u32)),
                ("provenance_kind", P(u32)), ("provenance_record", P(u64))]


class SpatialOrderConfig(C.Structure):
    """bfnew::SpatialOrderConfig (include/bfnew/spatial.hpp:19-26)."""
    _fields_ = [("origin_x", i32), ("origin_y", i32), ("tile_width", u32), ("tile_height", u32)]


class RouteQueryC(C.Structure):
    _fields_ = [("query_id", u32), ("expansion_generation", u32), ("source_count", u32), ("target_count", u32),
                ("sources", P(u32)), ("targets", P(u32)), ("selected_tile_count", u32), ("reserved0", u32),
                ("selected_tiles", P(u32))]


class BatchLanesC(C.Structure):
    _fields_ = [("lane_width", u32), ("lane_count", u32), ("query_index_by_lane", P(u32))]


class PlannerPolicyC(C.Structure):
    _fields_ = [("lane_width", u32), ("minimum_jaccard_numerator", u32), ("minimum_jaccard_denominator", u32),
                ("maximum_union_inflation_numerator", u32), ("maximum_union_inflation_denominator", u32),
                ("narrow_lanes", u32)]


class SynthConfig(C.Structure):
    _fields_ = [("tiles_x", u32), ("tiles_y", u32), ("nodes_per_tile", u32), ("intra_degree", u32),
                ("inter_degree", u32), ("span_count", u32), ("spans", u32 * 8), ("cost_kind", u32),
                ("cost_lo", u32), ("cost_hi", u32), ("intra_base", f32), ("span_base", f32 * 8), ("sigma", f32),
                ("reserved0", u32), ("seed", u64)]


assert C.sizeof(GpuRunOptions) == 48 and C.sizeof(DeviceController) == 96 and C.sizeof(DeviceRunStatus) == 48
assert C.sizeof(BatchVertexRange) == 12

_lib = None


def load() -> C.CDLL:
    """Loads libbfx.so (built by bf-new_b200/build.py); raises if absent."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(f"{LIB_PATH} is missing: run python bf-new_b200/build.py")
        lib = C.CDLL(str(LIB_PATH))
        lib.bfx_last_error.restype = C.c_char_p
        _lib = lib
    return _lib


def _check(rc: int) -> None:
    if rc == 0:
        return
    msg = load().bfx_last_error().decode(errors="replace")
    if rc == 1:
        raise ValueError(msg)
    if rc == 2:
        raise IndexError(msg)
    if rc == 3:
        raise OverflowError(msg)
    if rc == 4:
        raise BfxCudaError(msg)
    if rc == 5:
        raise BfxNoDevice(msg)
    if rc == 7:
        raise MemoryError(msg)
    raise RuntimeError(msg)


def _ptr(a: np.ndarray | None, ctype=u32):
    if a is None:
        return None
    return a.ctypes.data_as(P(ctype))


def device_count() -> int:
    n = C.c_int(0)
    _check(load().bfx_device_count(C.byref(n)))
    return n.value


# --------------------------------------------------------------------------
# Host builders
# --------------------------------------------------------------------------

@dataclass
class InputGraph:
    """bfnew::InputGraph as arrays (vertex metadata + edge records)."""
    x: np.ndarray
    y: np.ndarray
    has_location: np.ndarray
    resource_class: np.ndarray
    edge_source: np.ndarray
    edge_destination: np.ndarray
    edge_weight: np.ndarray
    provenance_domain: np.ndarray
    provenance_kind: np.ndarray
    provenance_record: np.ndarray

    def __post_init__(self):
        self.x = np.ascontiguousarray(self.x, np.int32)
        self.y = np.ascontiguousarray(self.y, np.int32)
        self.has_location = np.ascontiguousarray(self.has_location, np.uint8)
        self.resource_class = np.ascontiguousarray(self.resource_class, np.uint16)
        self.edge_source = np.ascontiguousarray(self.edge_source, np.uint32)
        self.edge_destination = np.ascontiguousarray(self.edge_destination, np.uint32)
        self.edge_weight = np.ascontiguousarray(self.edge_weight, np.float32)
        self.provenance_domain = np.ascontiguousarray(self.provenance_domain, np.uint32)
        self.provenance_kind = np.ascontiguousarray(self.provenance_kind, np.uint32)
        self.provenance_record = np.ascontiguousarray(self.provenance_record, np.uint64)

    @property
    def vertex_count(self) -> int:
        return int(self.x.shape[0])

    @property
    def edge_count(self) -> int:
        return int(self.edge_source.shape[0])

    def c(self) -> InputGraphC:
        return InputGraphC(self.vertex_count, 0, self.edge_count, _ptr(self.x, i32), _ptr(self.y, i32),
                           _ptr(self.has_location, C.c_uint8), _ptr(self.resource_class, C.c_uint16),
                           _ptr(self.edge_source), _ptr(self.edge_destination), _ptr(self.edge_weight, f32),
                           _ptr(self.provenance_domain), _ptr(self.provenance_kind), _ptr(self.provenance_record, u64))


LAYOUT_FIELDS = ("owner_tiles", "csr_row_offsets", "csr_destinations", "csr_weights", "csr_row_run_offsets",
                 "csr_run_edge_offsets", "csr_run_destination_tiles", "csc_column_offsets", "csc_sources",
                 "csc_weights", "csc_edge_ids", "csc_column_run_offsets", "csc_run_edge_offsets",
                 "csc_run_source_tiles", "csr_edge_ids")


class DeviceGraphLayout:
    """Owning host image of the checked 32-bit device graph (bfnew::DeviceGraphLayout32
    plus csr_edge_ids), built by libbfx or wrapped from arrays."""

    def __init__(self, arrays: dict, tiles: dict | None = None):
        arrays = dict(arrays)
        tc = arrays.pop("tile_count", None)
        self.arrays = {k: np.ascontiguousarray(v) for k, v in arrays.items()}
        self.tiles = tiles or {}
        self._tile_count = int(np.asarray(tc).reshape(-1)[0]) if tc is not None else None

    @property
    def vertex_count(self) -> int:
        return int(self.arrays["owner_tiles"].shape[0])

    @property
    def edge_count(self) -> int:
        return int(self.arrays["csr_destinations"].shape[0])

    @property
    def tile_count(self) -> int:
        if self._tile_count is not None:
            return self._tile_count
        return int(self.tiles["tile_vertex_offsets"].shape[0] - 1)

    def view(self) -> DeviceGraphLayout32View:
        a = self.arrays
        v = DeviceGraphLayout32View()
        v.vertex_count = self.vertex_count
        v.edge_count = self.edge_count
        v.tile_count = self.tile_count
        v.csr_run_count = a["csr_run_destination_tiles"].shape[0]
        v.csc_run_count = a["csc_run_source_tiles"].shape[0]
        for f in LAYOUT_FIELDS:
            arr = a.get(f)
            setattr(v, f, None if arr is None else _ptr(arr, f32 if arr.dtype == np.float32 else u32))
        return v


def build_device_graph_layout(graph: InputGraph, config: SpatialOrderConfig, threads: int = 0) -> DeviceGraphLayout:
    """UniformGridPartitioner::partition -> build_tile_run_layout ->
    build_device_graph_layout32 (src/tiled_graph.cpp:539, src/device_layout.cpp:186,395) in libbfx."""
    lib = load()
    h = C.c_void_p()
    gc = graph.c()
    _check(lib.bfx_layout_build(C.byref(gc), C.byref(config), u32(threads), C.byref(h)))
    v = DeviceGraphLayout32View()
    _check(lib.bfx_layout_view(h, C.byref(v)))
    V, E, T = v.vertex_count, v.edge_count, v.tile_count
    sizes = {"owner_tiles": V, "csr_row_offsets": V + 1, "csr_destinations": E, "csr_weights": E,
             "csr_row_run_offsets": V + 1, "csr_run_edge_offsets": v.csr_run_count + 1,
             "csr_run_destination_tiles": v.csr_run_count, "csc_column_offsets": V + 1, "csc_sources": E,
             "csc_weights": E, "csc_edge_ids": E, "csc_column_run_offsets": V + 1,
             "csc_run_edge_offsets": v.csc_run_count + 1, "csc_run_source_tiles": v.csc_run_count,
             "csr_edge_ids": E}
    arrays = {}
    for f, n in sizes.items():
        p = getattr(v, f)
        dt = np.float32 if "weights" in f else np.uint32
        arrays[f] = np.ctypeslib.as_array(p, shape=(n,)).view(dt).copy() if n else np.zeros(0, dt)
    tile_xy = np.zeros(2 * T, np.int64)
    has_loc = np.zeros(T, np.uint8)
    tvo = np.zeros(T + 1, np.uint32)
    _check(lib.bfx_layout_tiles(h, _ptr(tile_xy, i64), _ptr(has_loc, C.c_uint8), _ptr(tvo)))
    n2o = np.zeros(V, np.uint32)
    _check(lib.bfx_layout_new_to_old(h, _ptr(n2o)))
    _check(lib.bfx_layout_destroy(h))
    arrays["tile_count"] = np.uint32(T)
    return DeviceGraphLayout(arrays, {"tile_xy": tile_xy.reshape(T, 2), "has_location": has_loc,
                                      "tile_vertex_offsets": tvo, "new_to_old": n2o})


def synth_graph(tiles_x: int, tiles_y: int, nodes_per_tile: int, intra: int, inter: int, spans: Sequence[int],
                cost_kind: int = 0, cost_lo: int = 1, cost_hi: int = 64, intra_base: float = 1.0,
                span_base: Sequence[float] = (), sigma: float = 0.5, seed: int = 1):
    """Seeded synthetic spatial graph; returns (InputGraph, SpatialOrderConfig, stats)."""
    lib = load()
    cfg = SynthConfig()
    cfg.tiles_x, cfg.tiles_y, cfg.nodes_per_tile = tiles_x, tiles_y, nodes_per_tile
    cfg.intra_degree, cfg.inter_degree = intra, inter
    cfg.span_count = len(spans)
    for i, s in enumerate(spans):
        cfg.spans[i] = s
    cfg.cost_kind, cfg.cost_lo, cfg.cost_hi = cost_kind, cost_lo, cost_hi
    cfg.intra_base = intra_base
    for i, b in enumerate(span_base):
        cfg.span_base[i] = b
    cfg.sigma = sigma
    cfg.seed = seed
    sizes = (u64 * 2)()
    _check(lib.bfx_synth_sizes(C.byref(cfg), sizes))
    V, E = int(sizes[0]), int(sizes[1])
    g = InputGraph(np.zeros(V, np.int32), np.zeros(V, np.int32), np.zeros(V, np.uint8), np.zeros(V, np.uint16),
                   np.zeros(E, np.uint32), np.zeros(E, np.uint32), np.zeros(E, np.float32), np.zeros(E, np.uint32),
                   np.zeros(E, np.uint32), np.zeros(E, np.uint64))
    order = SpatialOrderConfig()
    stats = (u64 * 2)()
    _check(lib.bfx_synth_fill(C.byref(cfg), _ptr(g.x, i32), _ptr(g.y, i32), _ptr(g.has_location, C.c_uint8),
                              _ptr(g.resource_class, C.c_uint16), _ptr(g.edge_source), _ptr(g.edge_destination),
                              _ptr(g.edge_weight, f32), _ptr(g.provenance_domain), _ptr(g.provenance_kind),
                              _ptr(g.provenance_record, u64), C.byref(order), stats))
    return g, order, {"inter_edges": int(stats[0]), "inter_redrawn": int(stats[1])}


@dataclass
class RouteQuery:
    """Canonical bfnew::RouteQuery subset (include/bfnew/query.hpp:13-29)."""
    query_id: int
    sources: np.ndarray
    targets: np.ndarray
    selected_tiles: np.ndarray
    expansion_generation: int = 0

    def __post_init__(self):
        self.sources = np.unique(np.asarray(self.sources, np.uint32))
        self.targets = np.unique(np.asarray(self.targets, np.uint32))
        self.selected_tiles = np.unique(np.asarray(self.selected_tiles, np.uint32))

    def c(self) -> RouteQueryC:
        return RouteQueryC(self.query_id, self.expansion_generation, len(self.sources), len(self.targets),
                           _ptr(self.sources), _ptr(self.targets), len(self.selected_tiles), 0,
                           _ptr(self.selected_tiles))


@dataclass
class BatchPlannerPolicy:
    """bfnew::BatchPlannerPolicy (include/bfnew/batch_plan.hpp:27-35) + narrow_lanes."""
    lane_width: int = 32
    minimum_jaccard_numerator: int = 1
    minimum_jaccard_denominator: int = 8
    maximum_union_inflation_numerator: int = 2
    maximum_union_inflation_denominator: int = 1
    narrow_lanes: bool = False

    def c(self) -> PlannerPolicyC:
        return PlannerPolicyC(self.lane_width, self.minimum_jaccard_numerator, self.minimum_jaccard_denominator,
                              self.maximum_union_inflation_numerator, self.maximum_union_inflation_denominator,
                              int(self.narrow_lanes))


class BatchDescription:
    """Owning Python image of one bfnew::BatchDeviceDescription (device-materialized runs)."""

    def __init__(self, lane_width, valid_lane_mask, source_offsets, sources, target_offsets, targets, union_tiles,
                 tile_lane_masks, ranges, query_index_by_lane=None):
        self.lane_width = int(lane_width)
        self.valid_lane_mask = int(valid_lane_mask)
        self.source_offsets = np.ascontiguousarray(source_offsets, np.uint32)
        self.sources = np.ascontiguousarray(sources, np.uint32)
        self.target_offsets = np.ascontiguousarray(target_offsets, np.uint32)
        self.targets = np.ascontiguousarray(targets, np.uint32)
        self.union_tiles = np.ascontiguousarray(union_tiles, np.uint32)
        self.tile_lane_masks = np.ascontiguousarray(tile_lane_masks, np.uint32)
        self.ranges = np.ascontiguousarray(ranges, np.uint32).reshape(-1, 3)
        self.query_index_by_lane = query_index_by_lane

    @classmethod
    def from_c(cls, d: BatchDescriptionC, qidx=None) -> "BatchDescription":
        W = d.lane_width

        def arr(p, n, dt=np.uint32):
            return np.ctypeslib.as_array(p, shape=(n,)).copy() if n else np.zeros(0, dt)

        so = arr(d.source_offsets, W + 1)
        to = arr(d.target_offsets, W + 1)
        rg = np.ctypeslib.as_array(C.cast(d.selected_vertex_ranges, P(u32)), shape=(3 * d.range_count,)).copy()
        return cls(W, d.valid_lane_mask, so, arr(d.sources, int(so[-1])), to, arr(d.targets, int(to[-1])),
                   arr(d.union_tiles, d.union_tile_count), arr(d.tile_lane_masks, d.tile_count), rg, qidx)

    def c(self) -> BatchDescriptionC:
        """The C view (pointers into this object's arrays), rebuilt only when a
        field was replaced since the last call."""
        # the key holds the arrays themselves, so none of them can be freed
        # (and its address reused) while the view points at it
        key = (self.lane_width, self.valid_lane_mask, self.source_offsets, self.sources, self.target_offsets,
               self.targets, self.union_tiles, self.tile_lane_masks, self.ranges)
        cached = getattr(self, "_c_view", None)
        if cached is None or len(cached[0]) != len(key) or any(a is not b for a, b in zip(cached[0], key)):
            view = BatchDescriptionC(self.lane_width, self.valid_lane_mask, _ptr(self.source_offsets),
                                     _ptr(self.sources), _ptr(self.target_offsets), _ptr(self.targets),
                                     len(self.union_tiles), len(self.tile_lane_masks), _ptr(self.union_tiles),
                                     _ptr(self.tile_lane_masks), self.ranges.shape[0], 0,
                                     C.cast(_ptr(self.ranges), P(BatchVertexRange)))
            cached = (key, view)
            self._c_view = cached
        return cached[1]

    @property
    def union_vertex_count(self) -> int:
        return int((self.ranges[:, 1].astype(np.int64) - self.ranges[:, 0]).sum())


class QueryLanes:
    """A batch set as lane -> query assignments over a query list -- the input
    of device-side description preparation -- with its C image built once."""

    def __init__(self, lanes: Sequence[tuple[int, Sequence[int]]], queries: Sequence["RouteQuery"]):
        self.queries = list(queries)
        self.query_count = len(self.queries)
        self.queries_c = (RouteQueryC * self.query_count)(*[q.c() for q in self.queries])
        self._idx = [np.ascontiguousarray(np.asarray(ix, np.uint32)) for _, ix in lanes]
        self.count = len(self._idx)
        self.batches_c = (BatchLanesC * self.count)(*[BatchLanesC(w, len(a), _ptr(a))
                                                      for (w, _), a in zip(lanes, self._idx)])

    @classmethod
    def from_descriptions(cls, descriptions: Sequence["BatchDescription"], queries: Sequence["RouteQuery"]):
        """The assignment a plan's descriptions carry (valid lanes first)."""
        lanes = [(d.lane_width, [int(x) for x in d.query_index_by_lane[:bin(d.valid_lane_mask).count("1")]])
                 for d in descriptions]
        return cls(lanes, queries)


class BatchPlan:
    """make_overlapping_batch_plan + prepare_batch_device_description (libbfx)."""

    def __init__(self, layout: DeviceGraphLayout, queries: Sequence[RouteQuery], policy: BatchPlannerPolicy):
        lib = load()
        self.queries = list(queries)
        qc = (RouteQueryC * len(self.queries))(*[q.c() for q in self.queries])
        self._h = C.c_void_p()
        v = layout.view()
        tvo = np.ascontiguousarray(layout.tiles["tile_vertex_offsets"], np.uint32)
        _check(lib.bfx_plan_build(C.byref(v), _ptr(tvo), u32(len(self.queries)), qc, C.byref(policy.c()),
                                  C.byref(self._h)))
        n = u32()
        _check(lib.bfx_plan_batch_count(self._h, C.byref(n)))
        self.batch_count = n.value
        self._descs = []
        self.estimates = []
        for b in range(self.batch_count):
            d = BatchDescriptionC()
            _check(lib.bfx_plan_description(self._h, u32(b), C.byref(d)))
            qidx = (u32 * d.lane_width)()
            est = (u64 * 4)()
            _check(lib.bfx_plan_batch_info(self._h, u32(b), qidx, est))
            self._descs.append(BatchDescription.from_c(d, np.array(qidx[:], np.uint32)))
            self.estimates.append(tuple(int(x) for x in est))
        _check(lib.bfx_plan_destroy(self._h))
        self._h = None

    def descriptions(self) -> list[BatchDescription]:
        return self._descs


def make_overlapping_batch_plan(layout: DeviceGraphLayout, queries: Sequence[RouteQuery],
                                policy: BatchPlannerPolicy | None = None) -> BatchPlan:
    """bfnew::make_overlapping_batch_plan + prepare_batch_device_description (libbfx)."""
    return BatchPlan(layout, queries, policy or BatchPlannerPolicy())


# --------------------------------------------------------------------------
# Device engines
# --------------------------------------------------------------------------

class ResidentDeviceGraph:
    """bfnew::hip::ResidentDeviceGraph (include/bfnew/hip/runtime.hpp:238-270)."""

    def __init__(self, handle, layout: DeviceGraphLayout):
        self._h = handle
        self.layout = layout

    @classmethod
    def upload_once(cls, layout: DeviceGraphLayout, device: int = 0) -> "ResidentDeviceGraph":
        h = C.c_void_p()
        v = layout.view()
        _check(load().bfx_resident_graph_upload(C.byref(v), C.c_int(device), C.byref(h)))
        return cls(h, layout)

    def set_weights(self, weights_by_edge_id) -> None:
        """Replaces every edge weight on the device (array indexed by stable edge id)."""
        w = np.ascontiguousarray(weights_by_edge_id, np.float32)
        if w.shape[0] != self.layout.edge_count:
            raise ValueError("one weight per edge is required")
        _check(load().bfx_resident_graph_set_weights(self._h, _ptr(w, f32)))

    def info(self) -> dict:
        out = (u64 * 4)()
        _check(load().bfx_resident_graph_info(self._h, out))
        return {"vertices": out[0], "edges": out[1], "tiles": out[2], "device_bytes": out[3]}

    def close(self):
        if self._h is not None:
            load().bfx_resident_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        if getattr(self, "_h", None) is not None and _lib is not None:
            self.close()


class Workspace:
    """Reusable batched workspace bound to one resident graph and one CUDA stream."""

    def __init__(self, graph: ResidentDeviceGraph):
        self.graph = graph
        self._h = C.c_void_p()
        _check(load().bfx_workspace_create(graph._h, C.byref(self._h)))
        self.batch_count = 0

    @property
    def stream(self) -> int:
        s = C.c_void_p()
        _check(load().bfx_workspace_stream(self._h, C.byref(s)))
        return int(s.value or 0)

    def device_bytes(self) -> int:
        b = u64()
        _check(load().bfx_workspace_bytes(self._h, C.byref(b)))
        return b.value

    def prepare(self, batches: Sequence[BatchDescription]):
        arr = (BatchDescriptionC * len(batches))(*[b.c() for b in batches])
        self._keep = batches
        _check(load().bfx_prepare_batches(self._h, u32(len(batches)), arr))
        self.batch_count = len(batches)

    def prepare_from_queries(self, lanes, queries: Sequence["RouteQuery"] | None = None):
        """bfx_prepare_batches_from_queries: batches given as (lane width, query
        indices of the valid lanes) over `queries`, or a prebuilt QueryLanes;
        descriptions are built on the device."""
        image = lanes if isinstance(lanes, QueryLanes) else QueryLanes(lanes, queries)
        self._keep = image
        _check(load().bfx_prepare_batches_from_queries(self._h, u32(image.count), image.batches_c, u32(image.query_count),
                                                       image.queries_c))
        self.batch_count = image.count

    def prepared_description(self, batch: int) -> "BatchDescription":
        """The prepared description of a batch, read back from the device."""
        lib = load()
        counts = (u32 * 5)()
        _check(lib.bfx_fetch_prepared_description(self._h, u32(batch), counts, None, None, None, None, None, None,
                                                  None))
        W, valid, S, Tg, R = (int(x) for x in counts)
        T = self.graph.layout.tile_count
        so, to = np.zeros(W + 1, np.uint32), np.zeros(W + 1, np.uint32)
        sv, tv = np.zeros(max(S, 1), np.uint32), np.zeros(max(Tg, 1), np.uint32)
        ut, tm = np.zeros(max(R, 1), np.uint32), np.zeros(T, np.uint32)
        rg = np.zeros(3 * max(R, 1), np.uint32)
        _check(lib.bfx_fetch_prepared_description(self._h, u32(batch), counts, _ptr(so), _ptr(sv), _ptr(to), _ptr(tv),
                                                  _ptr(ut), _ptr(tm), C.cast(_ptr(rg), P(BatchVertexRange))))
        return BatchDescription(W, valid, so, sv[:S], to, tv[:Tg], ut[:R], tm, rg[:3 * R])

    def execute(self, options: GpuRunOptions):
        _check(load().bfx_execute(self._h, C.byref(options)))

    def autotune(self, batches: Sequence[BatchDescription], base: GpuRunOptions | None = None,
                 trials: int = 2) -> tuple[list[int], int]:
        """bfx_autotune: per-batch engine choice (timed, cached by batch shape);
        leaves the batches prepared for ENGINE_AUTO launches.  Returns
        (engines, batches measured)."""
        arr = (BatchDescriptionC * len(batches))(*[b.c() for b in batches])
        self._keep = batches
        out = (u32 * len(batches))()
        deltas = (f32 * len(batches))()
        measured = u32()
        _check(load().bfx_autotune(self._h, u32(len(batches)), arr, C.byref(base or GpuRunOptions()), u32(trials),
                                   out, deltas, C.byref(measured)))
        self.batch_count = len(batches)
        self.tuned_deltas = [float(x) for x in deltas]
        return list(out), measured.value

    def autotune_policy(self, layout, queries: Sequence["RouteQuery"], policies: Sequence["BatchPlannerPolicy"],
                        base: GpuRunOptions | None = None, trials: int = 2) -> tuple[int, list[float]]:
        """bfx_autotune_policy: plans, tunes and times the whole query set under each
        candidate planner policy; returns (index of the fastest, relaxation ms per
        candidate).  The workspace is left prepared and tuned with the winner;
        make_overlapping_batch_plan(layout, queries, policies[best]) rebuilds its plan."""
        v = layout.view()
        tvo = np.ascontiguousarray(layout.tiles["tile_vertex_offsets"], np.uint32)
        qs = list(queries)
        qc = (RouteQueryC * len(qs))(*[q.c() for q in qs])
        pc = (PlannerPolicyC * len(policies))(*[p.c() for p in policies])
        best = u32()
        times = (f32 * len(policies))()
        _check(load().bfx_autotune_policy(self._h, C.byref(v), _ptr(tvo), u32(len(qs)), qc, u32(len(policies)), pc,
                                          C.byref(base or GpuRunOptions()), u32(trials), C.byref(best), times))
        plan = make_overlapping_batch_plan(layout, qs, policies[best.value])
        self._keep = plan.descriptions()
        self.batch_count = plan.batch_count
        return best.value, [float(t) for t in times]

    def set_batch_deltas(self, deltas: Sequence[float]):
        """Near/far threshold steps per frontier batch (inf = plain frontier)."""
        arr = (f32 * len(deltas))(*deltas)
        _check(load().bfx_set_batch_deltas(self._h, u32(len(deltas)), arr))

    def set_register_budget(self, registers: int):
        """40 (three 512-thread blocks per SM), 64 or -- chunked layout, blocks of <= 256 threads -- 80
        registers per thread for the persistent kernel."""
        _check(load().bfx_set_register_budget(self._h, u32(registers)))

    def set_chunk_pairs(self, mode: int):
        """Chunked layout: 0 work list, 1 (vertex, lane) pair per thread (persistent control)."""
        _check(load().bfx_set_chunk_pairs(self._h, u32(mode)))

    def set_chunk_pack(self, pack: int):
        """Chunk slots per warp item of the chunked layout (1, 2, 4 or 8)."""
        _check(load().bfx_set_chunk_pack(self._h, u32(pack)))

    def chunk_pack(self) -> int:
        out = u32()
        _check(load().bfx_get_chunk_pack(self._h, C.byref(out)))
        return int(out.value)

    def set_flat_order(self, edge_major: int):
        """Flat/chunked work order: 0 entry-lane-edge, 1 entry-edge-lane."""
        _check(load().bfx_set_flat_order(self._h, u32(edge_major)))

    def set_relax_atomic(self, mode: int):
        """Flat layout: 0 pre-read + min on success, 1 returning min per relaxation."""
        _check(load().bfx_set_relax_atomic(self._h, u32(mode)))

    def set_flat_items(self, items: int):
        """Flat layout: work items per thread per iteration (2, 3 or 4)."""
        _check(load().bfx_set_flat_items(self._h, u32(items)))

    def set_frontier_layout(self, layout: int):
        """FRONTIER_GROUPS (sub-warp groups per entry), FRONTIER_FLAT (flat work list),
        FRONTIER_CHUNKED (32-vertex chunks) or FRONTIER_TILED (tile visits in shared memory)."""
        _check(load().bfx_set_frontier_layout(self._h, u32(layout)))

    def set_batch_mappings(self, mappings: Sequence[int]):
        """Tiled layout: per-batch dense-round mapping (MAPPING_TILE_VISITS or MAPPING_CHUNKS)."""
        arr = (u32 * len(mappings))(*mappings)
        _check(load().bfx_set_batch_mappings(self._h, u32(len(mappings)), arr))

    def frontier_mapping(self, count: int | None = None) -> tuple[int, list[int]]:
        """(frontier layout, per-batch mappings of the first `count` batches)."""
        n = self.batch_count if count is None else count
        layout = u32()
        arr = (u32 * max(n, 1))()
        _check(load().bfx_get_frontier_mapping(self._h, C.byref(layout), u32(n), arr))
        return layout.value, list(arr[:n])

    def set_tile_passes(self, passes: int):
        """Tiled layout: local relaxation passes per staged visit."""
        _check(load().bfx_set_tile_passes(self._h, u32(passes)))

    def set_tile_stage_min(self, lane_edges: int):
        """Tiled layout: visits with less lane-edge work relax in global memory (no staging)."""
        _check(load().bfx_set_tile_stage_min(self._h, u32(lane_edges)))

    def set_batch_engines(self, engines: Sequence[int]):
        arr = (u32 * len(engines))(*engines)
        _check(load().bfx_set_batch_engines(self._h, u32(len(engines)), arr))

    def fetch_statuses(self, controllers: bool = False):
        st = (DeviceRunStatus * self.batch_count)()
        ct = (DeviceController * self.batch_count)() if controllers else None
        _check(load().bfx_fetch_statuses(self._h, st, ct))
        return (list(st), list(ct)) if controllers else list(st)

    def download_labels(self, batch: int, lane_width: int):
        V = self.graph.layout.vertex_count
        bits = np.empty(V * lane_width, np.uint32)
        pred = np.empty(V * lane_width, np.uint32)
        _check(load().bfx_download_labels(self._h, u32(batch), _ptr(bits), _ptr(pred)))
        return bits.reshape(V, lane_width), pred.reshape(V, lane_width)

    def download_lane(self, batch: int, lane: int):
        """One lane of a batch as graph-sized (distance bits, predecessor edge ids)."""
        V = self.graph.layout.vertex_count
        bits = np.empty(V, np.uint32)
        pred = np.empty(V, np.uint32)
        _check(load().bfx_download_lane_labels(self._h, u32(batch), u32(lane), _ptr(bits), _ptr(pred)))
        return bits, pred

    def label_bounds(self) -> np.ndarray:
        """Largest finite distance bits per prepared batch (0: nothing beyond the sources)."""
        out = np.zeros(self.batch_count, np.uint32)
        _check(load().bfx_fetch_label_bounds(self._h, _ptr(out)))
        return out

    def last_launch_count(self) -> int:
        n = u64()
        _check(load().bfx_last_launch_count(self._h, C.byref(n)))
        return n.value

    def last_execute_timing(self) -> tuple[float, float]:
        """(relaxation kernels ms, whole execute ms) from the library's CUDA events."""
        out = (f32 * 2)()
        _check(load().bfx_last_execute_timing(self._h, out))
        return float(out[0]), float(out[1])

    def transfer_bytes(self) -> tuple[int, int]:
        out = (u64 * 2)()
        _check(load().bfx_workspace_transfer_bytes(self._h, out))
        return int(out[0]), int(out[1])

    def compact_paths(self, first_batch: int = 0, batch_count: int | None = None, raw: bool = False):
        """ReusableCompactPathWorkspace::reconstruct: per target (description
        order, batches [first_batch, first_batch+batch_count)) a dict with the
        summary fields and, for complete targets, vertices (source first),
        distance labels and stable edge ids.  raw=True returns the summaries
        as one structured array plus the flat payload arrays instead."""
        lib = load()
        n = (self.batch_count - first_batch) if batch_count is None else batch_count
        total = sum(self._keep[b].targets.shape[0] for b in range(first_batch, first_batch + n)) \
            if hasattr(self, "_keep") and self._keep is not None else None
        if total is None:
            raise RuntimeError("compact paths need batches prepared through this workspace")
        summ = (CompactTargetSummary * max(total, 1))()
        sizes = (u64 * 3)()
        _check(lib.bfx_compact_path_summaries(self._h, u32(first_batch), u32(n), summ, sizes))
        nv, ne = int(sizes[1]), int(sizes[2])
        verts = np.zeros(max(nv, 1), np.uint32)
        labels = np.zeros(max(nv, 1), np.float32)
        edges = np.zeros(max(ne, 1), np.uint32)
        _check(lib.bfx_compact_path_payload(self._h, _ptr(verts), _ptr(labels, f32), _ptr(edges)))
        if raw:
            return {"summaries": np.ctypeslib.as_array(summ)[:total].copy(), "vertices": verts[:nv],
                    "labels": labels[:nv], "edges": edges[:ne]}
        out, vo, eo = [], 0, 0
        for i in range(total):
            s = summ[i]
            d = {"target": s.target, "selected_source": s.selected_source, "distance": s.distance,
                 "path_length": s.path_length, "reached": s.reached, "reconstruction": s.reconstruction,
                 "has_selected_source": s.has_selected_source}
            if s.reconstruction == 0:
                L = s.path_length
                d["vertices"] = verts[vo:vo + L + 1].copy()
                d["labels"] = labels[vo:vo + L + 1].copy()
                d["edges"] = edges[eo:eo + L].copy()
                vo += L + 1
                eo += L
            out.append(d)
        return out

    def edge_usage_adjoint(self, target_grads) -> np.ndarray:
        """dL/dw (by stable edge id) for L = sum_t g_t * dist_t over the targets
        of the last compact_paths() call, in its target order."""
        g = np.ascontiguousarray(target_grads, np.float32)
        out = np.zeros(self.graph.layout.edge_count, np.float32)
        _check(load().bfx_edge_usage_adjoint(self._h, _ptr(g, f32), _ptr(out, f32)))
        return out

    WORK_KEYS = ("entries", "records", "active_pairs", "relaxations", "claims", "decreases", "min_reductions",
                 "rounds")

    def work_counters(self) -> dict:
        out = (u64 * 8)()
        _check(load().bfx_fetch_work_statistics(self._h, None, out))
        return dict(zip(self.WORK_KEYS, (int(x) for x in out)))

    def round_trace(self) -> np.ndarray:
        """(rounds, 4) array of {start ns, warp items | split batches << 32, active pairs,
        lane-edge relaxations} from the last instrumentation-2 persistent run."""
        n = u32()
        _check(load().bfx_fetch_round_trace(self._h, u32(0), None, C.byref(n)))
        out = np.zeros((max(n.value, 1), 4), np.uint64)
        _check(load().bfx_fetch_round_trace(self._h, u32(n.value), _ptr(out, u64), C.byref(n)))
        return out[:n.value]

    def engine_work(self) -> dict:
        """Work counters split by engine class: push (frontier / dense) and Jacobi pull."""
        out = (u64 * 16)()
        _check(load().bfx_fetch_engine_work(self._h, out))
        w = [int(x) for x in out]
        return {"push": dict(zip(self.WORK_KEYS[:7], w[:7])), "rounds": w[7],
                "jacobi": {"items": w[8], "records": w[9], "relaxations": w[10], "changes": w[11]},
                "split": {"entries": w[12], "lanes": w[13]},
                "tiled": {"local_relaxations": w[14], "staged_visits": w[15]}}

    def run_query(self, sources, targets, selected_tiles, options: GpuRunOptions) -> DeviceRunStatus:
        s = np.ascontiguousarray(np.unique(np.asarray(sources, np.uint32)))
        t = np.ascontiguousarray(np.unique(np.asarray(targets, np.uint32)))
        st = np.ascontiguousarray(np.unique(np.asarray(selected_tiles, np.uint32)))
        out = DeviceRunStatus()
        _check(load().bfx_run_query(self._h, u32(len(s)), _ptr(s), u32(len(t)), _ptr(t), u32(len(st)), _ptr(st),
                                    C.byref(options), C.byref(out)))
        self.batch_count = 1
        return out

    def close(self):
        if self._h is not None:
            load().bfx_workspace_destroy(self._h)
            self._h = None

    def __del__(self):
        if getattr(self, "_h", None) is not None and _lib is not None:
            self.close()


class _BatchedEngine:
    """Common shape of hip::Batched{JacobiPull,DenseChaoticPush,FrontierPush}Engine
    (include/bfnew/hip/batched_frontier_push.hpp:91-144)."""
    kind = ENGINE_FRONTIER_PUSH

    def __init__(self, graph: ResidentDeviceGraph, workspace: Workspace):
        self.graph = graph
        self.workspace = workspace

    def _opts(self, options: GpuRunOptions) -> GpuRunOptions:
        o = GpuRunOptions()
        C.memmove(C.byref(o), C.byref(options), C.sizeof(o))
        o.engine = self.kind
        return o

    def run_compact_status(self, batches, options: GpuRunOptions):
        batches = batches if isinstance(batches, (list, tuple)) else [batches]
        self.workspace.prepare(batches)
        self.workspace.execute(self._opts(options))
        return self.workspace.fetch_statuses()

    def run_status_only(self, batches, options: GpuRunOptions):
        batches = batches if isinstance(batches, (list, tuple)) else [batches]
        self.workspace.prepare(batches)
        self.workspace.execute(self._opts(options))
        return self.workspace.fetch_statuses(controllers=True)

    def run_with_distances(self, batches, options: GpuRunOptions):
        """Statuses plus per-batch (distance_bits[V, W], predecessor_edges[V, W])."""
        batches = batches if isinstance(batches, (list, tuple)) else [batches]
        st = self.run_compact_status(batches, options)
        labels = [self.workspace.download_labels(b, d.lane_width) for b, d in enumerate(batches)]
        return st, labels


class BatchedFrontierPushEngine(_BatchedEngine):
    kind = ENGINE_FRONTIER_PUSH


class BatchedJacobiPullEngine(_BatchedEngine):
    kind = ENGINE_JACOBI_PULL


class BatchedDenseChaoticPushEngine(_BatchedEngine):
    kind = ENGINE_DENSE_CHAOTIC_PUSH


def make_description(layout: DeviceGraphLayout, lanes: Sequence[RouteQuery], lane_width: int | None = None
                     ) -> BatchDescription:
    """One batch description from queries in lane order (prepare_batch_device_description
    semantics, src/batch_layout.cpp:1056-1296): lane terminals, dense tile masks, one
    vertex range per union tile."""
    W = lane_width or (1 if len(lanes) == 1 else (8 if len(lanes) <= 8 else (16 if len(lanes) <= 16 else 32)))
    if len(lanes) > W:
        raise ValueError("more queries than lanes")
    tvo = layout.tiles["tile_vertex_offsets"]
    T = tvo.shape[0] - 1
    masks = np.zeros(T, np.uint32)
    so, to, src, tgt = [0], [0], [], []
    for lane in range(W):
        if lane < len(lanes):
            q = lanes[lane]
            masks[q.selected_tiles] |= np.uint32(1 << lane)
            src.extend(q.sources.tolist())
            tgt.extend(q.targets.tolist())
        so.append(len(src))
        to.append(len(tgt))
    union = np.nonzero(masks)[0].astype(np.uint32)
    ranges = np.stack([tvo[union], tvo[union + 1], masks[union]], axis=1).astype(np.uint32)
    valid = (1 << len(lanes)) - 1 if len(lanes) < 32 else 0xFFFFFFFF
    return BatchDescription(W, valid, so, src, to, tgt, union, masks, ranges)
