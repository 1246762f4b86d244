"""GPU parity of the tiled frontier layout (BFX_FRONTIER_TILED): a thread
block visits one tile, relaxes its intra-tile edges in shared memory until no
lane of the tile is pending, and pushes inter-tile edges through global
memory.  Labels must equal the oracle's bit for bit for every tile size the
claim unit takes (fixture graphs whose tiles are smaller than or straddle a
unit, 64-vertex c1 tiles, 128-vertex c2 tiles, 256-vertex c3 tiles), every
lane width, with and without near/far thresholds, with every visit staged,
none staged, or the default mix, and in launches that mix engines."""
import numpy as np
import pytest

import bfx
from bfx import workloads
from golden_cases import fixture_paths, load_case
from oracle.oracle import Oracle
from test_gpu_engines import check_batches

pytestmark = pytest.mark.gpu

STAGE = {"staged": 0, "default": 1024, "unstaged": 1 << 30}


def run_tiled(layout, descs, stage_min=1024, deltas=None, engines=None, instr=0, max_rounds=1 << 30,
              control=bfx.CONTROL_PERSISTENT, block=256):
    res = bfx.ResidentDeviceGraph.upload_once(layout)
    ws = bfx.Workspace(res)
    ws.set_frontier_layout(bfx.FRONTIER_TILED)
    ws.set_tile_stage_min(stage_min)
    ws.prepare(descs)
    if deltas is not None:
        ws.set_batch_deltas(deltas)
    engine = bfx.ENGINE_FRONTIER_PUSH
    if engines is not None:
        ws.set_batch_engines(engines)
        engine = bfx.ENGINE_AUTO
    ws.execute(bfx.GpuRunOptions(engine=engine, instrumentation=instr, maximum_rounds=max_rounds,
                                 control_mode=control, block_size=block))
    st = ws.fetch_statuses()
    labels = [ws.download_labels(b, d.lane_width) for b, d in enumerate(descs)]
    work = ws.engine_work() if instr else None
    ws.close()
    res.close()
    return st, labels, work


@pytest.mark.parametrize("path", fixture_paths(), ids=lambda p: p.stem)
@pytest.mark.parametrize("stage", ["staged", "unstaged"])
def test_reference_fixtures_tiled(gpu, path, stage):
    case = load_case(path)
    descs = [bfx.make_description(case.layout, [gq.query], 1) for gq in case.queries]
    lanes = [[gq.query] for gq in case.queries]
    golden = {gq.query.query_id: gq.dist for gq in case.queries}
    st, labels, _ = run_tiled(case.layout, descs, STAGE[stage])
    check_batches(case.layout, descs, lanes, st, labels, Oracle.from_layout(case.layout), golden)


@pytest.fixture(scope="module")
def c1():
    return workloads.make_workload("c1")


@pytest.mark.parametrize("stage", ["staged", "default", "unstaged"])
@pytest.mark.parametrize("step", [None, 0.5, 3.0])
@pytest.mark.parametrize("instr", [0, 1])
def test_c1_full_graph_tiled(gpu, c1, stage, step, instr):
    """64-vertex tiles (claim unit 2^6), one W=8 full-graph batch, uint costs."""
    d = bfx.make_description(c1.layout, c1.queries, 8)
    st, labels, work = run_tiled(c1.layout, [d], STAGE[stage], None if step is None else [step], instr=instr)
    check_batches(c1.layout, [d], [c1.queries], st, labels, Oracle.from_layout(c1.layout))
    if instr:
        relax = work["push"]["relaxations"]
        assert relax > 0
        if stage == "staged":
            assert work["tiled"]["local_relaxations"] > 0 and work["tiled"]["staged_visits"] > 0
        if stage == "unstaged":
            assert work["tiled"]["local_relaxations"] == 0 and work["tiled"]["staged_visits"] == 0
        assert work["tiled"]["local_relaxations"] <= relax


@pytest.fixture(scope="module")
def c2_regional():
    layout, grid = workloads.build_graph("c2", scale_tiles=(32, 32))
    qs = workloads.box_queries(layout, grid, 60, 2, 16, seed=31, targets=(1, 4))
    plan = bfx.make_overlapping_batch_plan(layout, qs, bfx.BatchPlannerPolicy(32, 0, 1, 8, 1, narrow_lanes=True))
    descs = plan.descriptions()
    lanes = [[qs[i] if i != bfx.NO_EDGE else None for i in d.query_index_by_lane] for d in descs]
    return layout, descs, lanes


@pytest.mark.parametrize("stage", ["staged", "default", "unstaged"])
@pytest.mark.parametrize("step", [None, 3.0])
@pytest.mark.parametrize("block", [256, 384])
def test_regional_batches_tiled(gpu, c2_regional, stage, step, block):
    """128-vertex tiles (2^7), regional batches of widths 1..32 in one launch."""
    layout, descs, lanes = c2_regional
    assert len({d.lane_width for d in descs}) >= 2
    st, labels, _ = run_tiled(layout, descs, STAGE[stage], None if step is None else [step] * len(descs),
                              block=block)
    check_batches(layout, descs, lanes, st, labels, Oracle.from_layout(layout))


def test_regional_batches_tiled_mixed_engines(gpu, c2_regional):
    """Jacobi and dense batches share the tiled launch (one warp item per warp
    of a block item)."""
    layout, descs, lanes = c2_regional
    st, labels, _ = run_tiled(layout, descs, 0, engines=[i % 3 for i in range(len(descs))])
    check_batches(layout, descs, lanes, st, labels, Oracle.from_layout(layout))


@pytest.mark.parametrize("step", [None, 2.0])
@pytest.mark.parametrize("block", [256, 384])
def test_c3_shaped_full_graph_w32_tiled(gpu, step, block):
    """256-vertex tiles (2^8, 64 KB of staged labels at W=32): the c3
    generator on 16x16 tiles, one full-graph batch of 32 sources."""
    layout, grid = workloads.build_graph("c3", scale_tiles=(16, 16))
    qs = workloads.full_graph_queries(layout, grid, 32, seed=77)
    d = bfx.make_description(layout, qs, 32)
    wbar = float(np.mean(layout.arrays["csr_weights"]))
    st, labels, _ = run_tiled(layout, [d], 1024, None if step is None else [step * wbar], block=block)
    check_batches(layout, [d], [qs], st, labels, Oracle.from_layout(layout))


def test_round_limit_stops_tiled(gpu, c1):
    """A round-limited tiled run stops with maximum_rounds and reports pending
    lanes, like the other layouts."""
    d = bfx.make_description(c1.layout, c1.queries, 8)
    st, _, _ = run_tiled(c1.layout, [d], 0, max_rounds=2)
    assert st[0].stop_reason == bfx.STOP_MAXIMUM_ROUNDS
    assert st[0].reached_target_mask == 0 and st[0].bounding_box_miss_mask == 0
    assert st[0].active_lane_mask != 0


def test_host_poll_modes_fall_back_to_chunked(gpu, c1):
    """Host-poll control runs the chunked round kernels when the tiled layout
    is selected; results are the oracle's."""
    d = bfx.make_description(c1.layout, c1.queries, 8)
    st, labels, _ = run_tiled(c1.layout, [d], 0, control=bfx.CONTROL_CHUNKED)
    check_batches(c1.layout, [d], [c1.queries], st, labels, Oracle.from_layout(c1.layout))


@pytest.mark.parametrize("pack", [1, 4])
@pytest.mark.parametrize("step", [None, 3.0])
def test_per_batch_mappings_bit_exact(gpu, c2_regional, step, pack):
    """One tiled launch with dense rounds mapped per batch: alternating tile
    visits and chunk-slot warp items (1 or 4 chunk slots per warp item)."""
    layout, descs, lanes = c2_regional
    res = bfx.ResidentDeviceGraph.upload_once(layout)
    ws = bfx.Workspace(res)
    ws.set_frontier_layout(bfx.FRONTIER_TILED)
    ws.set_tile_stage_min(0)
    ws.set_chunk_pack(pack)
    ws.prepare(descs)
    if step is not None:
        ws.set_batch_deltas([step] * len(descs))
    mappings = [bfx.MAPPING_TILE_VISITS if b % 2 else bfx.MAPPING_CHUNKS for b in range(len(descs))]
    ws.set_batch_mappings(mappings)
    assert ws.frontier_mapping(len(descs)) == (bfx.FRONTIER_TILED, mappings)
    ws.execute(bfx.GpuRunOptions(instrumentation=1))
    st = ws.fetch_statuses()
    labels = [ws.download_labels(b, d.lane_width) for b, d in enumerate(descs)]
    check_batches(layout, descs, lanes, st, labels, Oracle.from_layout(layout))
    ws.close()
    res.close()


@pytest.mark.parametrize("start", [bfx.FRONTIER_CHUNKED, bfx.FRONTIER_TILED], ids=["from_chunked", "from_tiled"])
def test_autotuner_chooses_layout_and_mappings(gpu, c2_regional, start):
    """bfx_autotune's mapping phase: whichever of the chunked and tiled layouts
    it keeps, and whatever per-batch mappings, the AUTO launch is bit-exact."""
    layout, descs, lanes = c2_regional
    res = bfx.ResidentDeviceGraph.upload_once(layout)
    ws = bfx.Workspace(res)
    bfx.load().bfx_autotune_reset()
    ws.set_frontier_layout(start)
    engines, measured = ws.autotune(descs)
    kept, mappings = ws.frontier_mapping(len(descs))
    assert kept in (bfx.FRONTIER_CHUNKED, bfx.FRONTIER_TILED)
    assert set(mappings) <= {bfx.MAPPING_CHUNKS, bfx.MAPPING_TILE_VISITS}
    ws.execute(bfx.GpuRunOptions(engine=bfx.ENGINE_AUTO))
    st = ws.fetch_statuses()
    labels = [ws.download_labels(b, d.lane_width) for b, d in enumerate(descs)]
    check_batches(layout, descs, lanes, st, labels, Oracle.from_layout(layout))
    ws.close()
    res.close()
