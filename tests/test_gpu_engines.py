"""GPU parity: the sm_100a engines in libbfx.so against the oracle and the
reference's golden vectors.  Distances and predecessors must be bit-exact;
statuses must match the reference semantics (reached / miss lanes,
convergence, stop reason)."""
import numpy as np
import pytest

import bfx
from bfx import workloads
from golden_cases import GOLDEN, fixture_paths, load_case
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

ENGINES = [bfx.ENGINE_FRONTIER_PUSH, bfx.ENGINE_JACOBI_PULL, bfx.ENGINE_DENSE_CHAOTIC_PUSH]
ENGINE_CLASS = {bfx.ENGINE_FRONTIER_PUSH: bfx.BatchedFrontierPushEngine,
                bfx.ENGINE_JACOBI_PULL: bfx.BatchedJacobiPullEngine,
                bfx.ENGINE_DENSE_CHAOTIC_PUSH: bfx.BatchedDenseChaoticPushEngine}


def check_batches(layout, descs, lane_queries, statuses, labels, orc, golden_dist=None):
    """Every valid lane of every batch equals the oracle bit for bit."""
    for b, d in enumerate(descs):
        bits, pred = labels[b]
        st = statuses[b]
        assert st.stop_reason == bfx.STOP_CONVERGED, st.as_dict()
        assert st.converged == 1 and st.error_bits == 0
        reached = 0
        for lane in range(d.lane_width):
            if not (d.valid_lane_mask >> lane) & 1:
                assert np.all(bits[:, lane] == bfx.INF_BITS)
                continue
            q = lane_queries[b][lane]
            od, op = orc.region_sssp(q.sources, q.targets, q.selected_tiles)
            np.testing.assert_array_equal(bits[:, lane], od, err_msg=f"batch {b} lane {lane} distances")
            np.testing.assert_array_equal(pred[:, lane], op, err_msg=f"batch {b} lane {lane} predecessors")
            if golden_dist is not None:
                np.testing.assert_array_equal(bits[:, lane], golden_dist[q.query_id])
            if np.all(od[q.targets] != bfx.INF_BITS):
                reached |= 1 << lane
        assert st.reached_target_mask == reached
        assert st.bounding_box_miss_mask == d.valid_lane_mask & ~reached
        assert st.valid_lane_mask == d.valid_lane_mask
        assert st.converged_lane_mask == d.valid_lane_mask and st.active_lane_mask == 0


def run(layout, descs, engine, control=bfx.CONTROL_PERSISTENT, **kw):
    res = bfx.ResidentDeviceGraph.upload_once(layout)
    ws = bfx.Workspace(res)
    eng = ENGINE_CLASS[engine](res, ws)
    opts = bfx.GpuRunOptions(control_mode=control, **kw)
    st, labels = eng.run_with_distances(descs, opts)
    launches = ws.last_launch_count()
    ws.close()
    res.close()
    return st, labels, launches


@pytest.mark.parametrize("path", fixture_paths(), ids=lambda p: p.stem)
@pytest.mark.parametrize("engine", ENGINES, ids=["frontier", "jacobi", "dense"])
def test_reference_fixtures_single_lane(gpu, path, engine):
    case = load_case(path)
    orc = Oracle.from_layout(case.layout)
    descs = [bfx.make_description(case.layout, [gq.query], 1) for gq in case.queries]
    lanes = [[gq.query] for gq in case.queries]
    golden = {gq.query.query_id: gq.dist for gq in case.queries}
    st, labels, _ = run(case.layout, descs, engine)
    check_batches(case.layout, descs, lanes, st, labels, orc, golden)
    if case.name != "compact_paths" and len(case.queries) == 1:
        assert st[0].reached_target_mask == case.expected_reached
        assert st[0].bounding_box_miss_mask == case.expected_miss


@pytest.mark.parametrize("engine", ENGINES, ids=["frontier", "jacobi", "dense"])
@pytest.mark.parametrize("control", [bfx.CONTROL_PERSISTENT, bfx.CONTROL_CHUNKED, bfx.CONTROL_PER_ROUND],
                         ids=["persistent", "chunked", "per_round"])
def test_batched_mixed_fixture_matches_reference_engines(gpu, engine, control):
    """The five-lane overlap fixture (tests/batched_jacobi_fixture_suite.hpp:57):
    our plan equals the reference plan and our labels equal the reference's
    portable batched engines' labels, in every control mode."""
    z = dict(np.load(GOLDEN / "batched_mixed.npz"))
    case = load_case(GOLDEN / "batched_mixed.npz")
    queries = [gq.query for gq in case.queries]
    plan = bfx.make_overlapping_batch_plan(case.layout, queries, bfx.BatchPlannerPolicy(8, 0, 1, 4, 1))
    assert plan.batch_count == int(z["batch_count"]) == 1
    d = plan.descriptions()[0]
    np.testing.assert_array_equal(d.query_index_by_lane, z["B0_lane_query"])
    np.testing.assert_array_equal(d.union_tiles, z["B0_union_tiles"])
    st, labels, _ = run(case.layout, [d], engine, control, rounds_per_chunk=2)
    bits, _ = labels[0]
    for eng in (0, 1, 2):
        ref_bits = z[f"B0_E{eng}_bits"]
        np.testing.assert_array_equal(bits, ref_bits)
        ref_st = z[f"B0_E{eng}_status"]
        assert st[0].converged == ref_st[0]
        assert st[0].reached_target_mask == ref_st[1]
        assert st[0].bounding_box_miss_mask == ref_st[2]
        assert st[0].valid_lane_mask == ref_st[3]
        assert st[0].stop_reason == ref_st[6] and st[0].error_bits == ref_st[7]
    lanes = [[queries[i] if i != bfx.NO_EDGE else None for i in d.query_index_by_lane]]
    check_batches(case.layout, [d], lanes, st, labels, Oracle.from_layout(case.layout))


@pytest.fixture(scope="module")
def c1():
    return workloads.make_workload("c1")


@pytest.mark.parametrize("engine", ENGINES, ids=["frontier", "jacobi", "dense"])
def test_c1_full_graph_batch_bit_exact(gpu, c1, engine):
    """c1: 8 full-graph sources in one width-8 batch; uint costs."""
    d = bfx.make_description(c1.layout, c1.queries, 8)
    st, labels, launches = run(c1.layout, [d], engine)
    check_batches(c1.layout, [d], [c1.queries], st, labels, Oracle.from_layout(c1.layout))
    assert launches >= 3


@pytest.mark.parametrize("engine", ENGINES, ids=["frontier", "jacobi", "dense"])
def test_regional_multi_batch_one_launch(gpu, engine):
    """Uneven regional queries planned into several batches of different
    widths and relaxed in one launch (c2 recipe on a 32x32-tile grid)."""
    layout, grid = workloads.build_graph("c2", scale_tiles=(32, 32))
    qs = workloads.box_queries(layout, grid, 48, 2, 16, seed=9)
    plan = workloads.plan_batches(layout, qs, 32, narrow=True,
                                  policy=bfx.BatchPlannerPolicy(32, 0, 1, 8, 1, narrow_lanes=True))
    descs = plan.descriptions()
    assert len(descs) >= 2
    lanes = [[qs[i] if i != bfx.NO_EDGE else None for i in d.query_index_by_lane] for d in descs]
    st, labels, _ = run(layout, descs, engine)
    check_batches(layout, descs, lanes, st, labels, Oracle.from_layout(layout))


def test_plain_per_query_engine_matches(gpu, c1):
    """bfx_run_query (the plain one-query-per-launch engine) on c1 queries."""
    res = bfx.ResidentDeviceGraph.upload_once(c1.layout)
    ws = bfx.Workspace(res)
    orc = Oracle.from_layout(c1.layout)
    for q in c1.queries[:3]:
        st = ws.run_query(q.sources, q.targets, q.selected_tiles, bfx.GpuRunOptions())
        bits, pred = ws.download_labels(0, 1)
        od, op = orc.region_sssp(q.sources, q.targets, q.selected_tiles)
        np.testing.assert_array_equal(bits[:, 0], od)
        np.testing.assert_array_equal(pred[:, 0], op)
        assert st.converged == 1 and st.reached_target_mask == 1
    ws.close()
    res.close()


@pytest.mark.parametrize("engine", ENGINES, ids=["frontier", "jacobi", "dense"])
def test_round_limit_stops_without_result_masks(gpu, c1, engine):
    """maximum_rounds reached: not converged, no reached/miss bits
    (make_frontier_run_status, include/bfnew/frontier_push.hpp:270-294)."""
    d = bfx.make_description(c1.layout, c1.queries, 8)
    res = bfx.ResidentDeviceGraph.upload_once(c1.layout)
    ws = bfx.Workspace(res)
    eng = ENGINE_CLASS[engine](res, ws)
    st, ctl = eng.run_status_only([d], bfx.GpuRunOptions(maximum_rounds=2))
    s = st[0]
    assert s.stop_reason == bfx.STOP_MAXIMUM_ROUNDS and s.converged == 0
    assert s.reached_target_mask == 0 and s.bounding_box_miss_mask == 0
    assert s.rounds_completed == 2
    assert s.active_lane_mask != 0 and (s.active_lane_mask & ~d.valid_lane_mask) == 0
    assert ctl[0].done == 1 and ctl[0].stop_reason == bfx.STOP_MAXIMUM_ROUNDS
    ws.close()
    res.close()


@pytest.mark.parametrize("engine", ENGINES, ids=["frontier", "jacobi", "dense"])
def test_instrumented_counters_and_timing(gpu, c1, engine):
    """Light instrumentation fills the work counters without changing labels;
    the library's event timing brackets the relaxation launch."""
    d = bfx.make_description(c1.layout, c1.queries, 8)
    res = bfx.ResidentDeviceGraph.upload_once(c1.layout)
    ws = bfx.Workspace(res)
    eng = ENGINE_CLASS[engine](res, ws)
    st, labels = eng.run_with_distances([d], bfx.GpuRunOptions(instrumentation=1))
    w = ws.work_counters()
    k_ms, x_ms = ws.last_execute_timing()
    assert 0 < k_ms <= x_ms
    assert w["rounds"] == st[0].rounds_completed
    assert w["relaxations"] >= w["decreases"] > 0 and w["records"] > 0 and w["entries"] > 0
    if engine == bfx.ENGINE_FRONTIER_PUSH:
        # every (vertex, lane) improvement that activated a vertex was claimed once per round
        assert w["claims"] <= w["decreases"] and w["entries"] >= w["claims"]
    plain, plabels = eng.run_with_distances([d], bfx.GpuRunOptions())
    np.testing.assert_array_equal(labels[0][0], plabels[0][0])
    np.testing.assert_array_equal(labels[0][1], plabels[0][1])
    h2d, d2h = ws.transfer_bytes()
    assert h2d > 0 and d2h == 48
    ws.close()
    res.close()


def test_invalid_options_and_descriptions_rejected(gpu, c1):
    res = bfx.ResidentDeviceGraph.upload_once(c1.layout)
    ws = bfx.Workspace(res)
    d = bfx.make_description(c1.layout, c1.queries, 8)
    eng = bfx.BatchedFrontierPushEngine(res, ws)
    with pytest.raises(ValueError):
        eng.run_compact_status([d], bfx.GpuRunOptions(maximum_rounds=0))
    with pytest.raises(ValueError):
        eng.run_compact_status([d], bfx.GpuRunOptions(block_size=100))
    bad = bfx.make_description(c1.layout, c1.queries, 8)
    bad.tile_lane_masks = bad.tile_lane_masks.copy()
    bad.tile_lane_masks[bad.union_tiles[0]] ^= 1
    with pytest.raises(ValueError):
        eng.run_compact_status([bad], bfx.GpuRunOptions())
    ws.close()
    res.close()


def test_autotuned_mixed_engines_one_launch(gpu):
    """bfx_autotune picks an engine per batch; an ENGINE_AUTO launch relaxes
    every batch with its own engine in one launch, bit-exact.  A forced mix
    of all three engines checks the per-batch dispatch itself."""
    layout, grid = workloads.build_graph("c2", scale_tiles=(32, 32))
    qs = workloads.box_queries(layout, grid, 30, 2, 16, seed=19)
    plan = bfx.make_overlapping_batch_plan(layout, qs, bfx.BatchPlannerPolicy(32, 0, 1, 8, 1, narrow_lanes=True))
    descs = plan.descriptions()
    lanes = [[qs[i] if i != bfx.NO_EDGE else None for i in d.query_index_by_lane] for d in descs]
    res = bfx.ResidentDeviceGraph.upload_once(layout)
    ws = bfx.Workspace(res)
    lib = bfx.load()
    lib.bfx_autotune_reset()
    engines, measured = ws.autotune(descs)
    assert len(engines) == len(descs) and set(engines) <= {0, 1, 2} and measured >= 1
    engines2, measured2 = ws.autotune(descs)
    assert engines2 == engines and measured2 == 0  # cached by shape
    orc = Oracle.from_layout(layout)
    for mix in (engines, [i % 3 for i in range(len(descs))]):
        ws.prepare(descs)
        ws.set_batch_engines(mix)
        ws.execute(bfx.GpuRunOptions(engine=bfx.ENGINE_AUTO))
        st = ws.fetch_statuses()
        labels = [ws.download_labels(b, d.lane_width) for b, d in enumerate(descs)]
        check_batches(layout, descs, lanes, st, labels, orc)
    ws.close()
    res.close()


@pytest.mark.parametrize("step", [0.5, 3.0, 40.0])
def test_near_far_frontier_bit_exact(gpu, c1, step):
    """Near/far frontier with a threshold step (several splits on c1's uint
    costs): same labels as the oracle, fewer or equal relaxations."""
    layout = c1.layout
    d = bfx.make_description(layout, c1.queries, 8)
    layout2, grid = workloads.build_graph("c2", scale_tiles=(32, 32))
    qs = workloads.box_queries(layout2, grid, 40, 2, 16, seed=23)
    plan = bfx.make_overlapping_batch_plan(layout2, qs, bfx.BatchPlannerPolicy(32, 0, 1, 8, 1, narrow_lanes=True))
    for lay, descs, lanes in ((layout, [d], [c1.queries]),
                              (layout2, plan.descriptions(),
                               [[qs[i] if i != bfx.NO_EDGE else None for i in x.query_index_by_lane]
                                for x in plan.descriptions()])):
        res = bfx.ResidentDeviceGraph.upload_once(lay)
        ws = bfx.Workspace(res)
        ws.prepare(descs)
        ws.set_batch_deltas([step] * len(descs))
        ws.execute(bfx.GpuRunOptions(instrumentation=1))
        st = ws.fetch_statuses()
        labels = [ws.download_labels(b, x.lane_width) for b, x in enumerate(descs)]
        check_batches(lay, descs, lanes, st, labels, Oracle.from_layout(lay))
        ws.close()
        res.close()


def test_autotuner_with_near_far_candidates(gpu):
    layout, grid = workloads.build_graph("c2", scale_tiles=(32, 32))
    qs = workloads.box_queries(layout, grid, 20, 4, 20, seed=29)
    plan = bfx.make_overlapping_batch_plan(layout, qs, bfx.BatchPlannerPolicy(32, 0, 1, 8, 1, narrow_lanes=True))
    descs = plan.descriptions()
    res = bfx.ResidentDeviceGraph.upload_once(layout)
    ws = bfx.Workspace(res)
    bfx.load().bfx_autotune_reset()
    engines, _ = ws.autotune(descs)
    assert len(ws.tuned_deltas) == len(descs) and all(x > 0 for x in ws.tuned_deltas)
    ws.execute(bfx.GpuRunOptions(engine=bfx.ENGINE_AUTO))
    st = ws.fetch_statuses()
    labels = [ws.download_labels(b, x.lane_width) for b, x in enumerate(descs)]
    lanes = [[qs[i] if i != bfx.NO_EDGE else None for i in x.query_index_by_lane] for x in descs]
    check_batches(layout, descs, lanes, st, labels, Oracle.from_layout(layout))
    ws.close()
    res.close()


@pytest.mark.parametrize("regs,items,amin,order,pairs,instr", [(40, 2, 0, 0, 0, 1), (64, 2, 0, 0, 0, 1),
                                                               (64, 3, 0, 0, 0, 1), (64, 4, 0, 0, 0, 1),
                                                               (64, 2, 1, 0, 0, 1), (64, 2, 0, 1, 0, 1),
                                                               (64, 2, 0, 0, 1, 1), (64, 2, 0, 0, 0, 0),
                                                               (80, 2, 0, 0, 0, 1), (80, 2, 0, 0, 0, 0),
                                                               (80, 3, 0, 0, 0, 0), (80, 4, 0, 0, 0, 1)])
@pytest.mark.parametrize("layout_kind", [bfx.FRONTIER_FLAT, bfx.FRONTIER_GROUPS, bfx.FRONTIER_CHUNKED],
                         ids=["flat", "groups", "chunked"])
@pytest.mark.parametrize("step", [None, 3.0])
@pytest.mark.parametrize("control", [bfx.CONTROL_PERSISTENT, bfx.CONTROL_PER_ROUND], ids=["persistent", "per_round"])
def test_flat_frontier_layout_bit_exact(gpu, c1, step, control, layout_kind, regs, items, amin, order, pairs, instr):
    """The flat work-list frontier (32 entries per warp, (lane, edge) pairs
    walked 32 per step) gives the oracle's labels on full-graph W=8, regional
    multi-batch W in {1, 8, 16, 32}, plain and near/far, with the counting
    (instr 1) and the production (instr 0) kernel instantiations."""
    run_layout_case(c1, layout_kind, step, control, regs, items, amin, order, pairs, instr)


def run_layout_case(c1, layout_kind, step, control, regs, items, amin, order, pairs, instr, pack=1):
    layout = c1.layout
    d = bfx.make_description(layout, c1.queries, 8)
    layout2, grid = workloads.build_graph("c2", scale_tiles=(32, 32))
    qs = workloads.box_queries(layout2, grid, 60, 2, 16, seed=31, targets=(1, 4))
    plan = bfx.make_overlapping_batch_plan(layout2, qs, bfx.BatchPlannerPolicy(32, 0, 1, 8, 1, narrow_lanes=True))
    for lay, descs, lanes in ((layout, [d], [c1.queries]),
                              (layout2, plan.descriptions(),
                               [[qs[i] if i != bfx.NO_EDGE else None for i in x.query_index_by_lane]
                                for x in plan.descriptions()])):
        res = bfx.ResidentDeviceGraph.upload_once(lay)
        ws = bfx.Workspace(res)
        ws.set_frontier_layout(layout_kind)
        ws.set_register_budget(regs)
        ws.set_flat_items(items)
        ws.set_relax_atomic(amin)
        ws.set_flat_order(order)
        ws.set_chunk_pairs(pairs)
        ws.set_chunk_pack(pack)
        ws.prepare(descs)
        if step is not None:
            ws.set_batch_deltas([step] * len(descs))
        ws.execute(bfx.GpuRunOptions(instrumentation=instr, control_mode=control, maximum_rounds=1 << 20))
        st = ws.fetch_statuses()
        labels = [ws.download_labels(b, x.lane_width) for b, x in enumerate(descs)]
        check_batches(lay, descs, lanes, st, labels, Oracle.from_layout(lay))
        ws.close()
        res.close()


@pytest.mark.parametrize("pack", [2, 4, 8])
@pytest.mark.parametrize("regs,items,order,pairs,instr", [(80, 2, 0, 0, 0), (80, 2, 0, 0, 1), (80, 4, 0, 0, 0),
                                                          (80, 2, 1, 0, 1), (64, 2, 0, 1, 1), (64, 2, 0, 0, 0)])
@pytest.mark.parametrize("step", [None, 3.0])
@pytest.mark.parametrize("control", [bfx.CONTROL_PERSISTENT, bfx.CONTROL_PER_ROUND], ids=["persistent", "per_round"])
def test_chunk_pack_bit_exact(gpu, c1, step, control, regs, items, order, pairs, instr, pack):
    """Chunked layout with 2, 4 or 8 chunk slots per warp item (the pending
    vertices of several chunks compacted into one work list): the oracle's
    labels on the same full-graph and regional multi-batch sets."""
    run_layout_case(c1, bfx.FRONTIER_CHUNKED, step, control, regs, items, 0, order, pairs, instr, pack)


def test_chunk_pack_rejects_other_values(gpu, c1):
    res = bfx.ResidentDeviceGraph.upload_once(c1.layout)
    ws = bfx.Workspace(res)
    for bad in (0, 3, 16):
        with pytest.raises(ValueError):
            ws.set_chunk_pack(bad)
    ws.close()
    res.close()


def test_plain_query_after_autotune_ignores_batch_settings(gpu):
    """run_query (one width-1 batch) runs the options' engine even when the
    workspace holds autotuned per-batch engines and steps for a batch set."""
    layout, grid = workloads.build_graph("c2", scale_tiles=(32, 32))
    qs = workloads.box_queries(layout, grid, 12, 4, 12, seed=37)
    plan = bfx.make_overlapping_batch_plan(layout, qs, bfx.BatchPlannerPolicy(32, 0, 1, 8, 1, narrow_lanes=True))
    descs = plan.descriptions()
    res = bfx.ResidentDeviceGraph.upload_once(layout)
    ws = bfx.Workspace(res)
    ws.autotune(descs)
    orc = Oracle.from_layout(layout)
    for q in qs[:3]:
        st = ws.run_query(q.sources, q.targets, q.selected_tiles, bfx.GpuRunOptions(engine=bfx.ENGINE_FRONTIER_PUSH))
        assert st.stop_reason == bfx.STOP_CONVERGED
        d, _ = orc.region_sssp(q.sources, q.targets, q.selected_tiles)
        assert bool(st.reached_target_mask & 1) == bool(np.all(d[q.targets] != bfx.INF_BITS))
    # the tuned set is still usable after re-preparing it
    ws.prepare(descs)
    ws.execute(bfx.GpuRunOptions(engine=bfx.ENGINE_AUTO))
    assert all(s.stop_reason == bfx.STOP_CONVERGED for s in ws.fetch_statuses())
    ws.close()
    res.close()


def test_round_trace_at_debug_instrumentation(gpu, c1):
    """instrumentation 2 records one {start time, warp items | split batches,
    pairs, relaxations} record per round of a persistent launch: as many
    rounds as the work counters report, start times non-decreasing, every
    traced round with work, per-round work summing to the launch totals."""
    d = bfx.make_description(c1.layout, c1.queries, 8)
    res = bfx.ResidentDeviceGraph.upload_once(c1.layout)
    ws = bfx.Workspace(res)
    ws.prepare([d])
    ws.execute(bfx.GpuRunOptions(instrumentation=2))
    st = ws.fetch_statuses()[0]
    assert st.stop_reason == bfx.STOP_CONVERGED
    tr = ws.round_trace()
    assert tr.shape[0] == ws.work_counters()["rounds"] > 0
    assert np.all(np.diff(tr[:, 0].astype(np.int64)) >= 0)
    assert np.all((tr[:, 1] & 0xFFFFFFFF) > 0)
    assert np.all((tr[:, 1] >> 32) == 0)  # plain frontier: no split rounds
    assert ws.engine_work()["split"] == {"entries": 0, "lanes": 0}
    w = ws.work_counters()
    assert int(tr[:, 2].sum()) == w["active_pairs"] and int(tr[:, 3].sum()) == w["relaxations"]
    # near/far frontier: split rounds are marked with their batch count and
    # the split counters see the far pile
    ws.set_batch_deltas([0.5 * float(np.mean(c1.layout.arrays["csr_weights"]))])
    ws.execute(bfx.GpuRunOptions(engine=bfx.ENGINE_AUTO, instrumentation=2))
    assert ws.fetch_statuses()[0].stop_reason == bfx.STOP_CONVERGED
    tr = ws.round_trace()
    splits = tr[:, 1] >> 32
    assert np.all(splits <= 1) and splits.sum() > 0
    assert np.all((tr[:, 1] & 0xFFFFFFFF) > 0)
    sw = ws.engine_work()["split"]
    assert sw["entries"] > 0 and sw["lanes"] >= sw["entries"]
    ws.close()
    res.close()


def test_planner_policy_autotune_picks_and_prepares_the_fastest(gpu):
    """bfx_autotune_policy times the whole set under each planner policy and
    leaves the workspace prepared with the fastest plan, whose labels are the
    oracle's."""
    layout, grid = workloads.build_graph("c2", scale_tiles=(32, 32))
    qs = workloads.box_queries(layout, grid, 40, 2, 16, seed=41)
    policies = [bfx.BatchPlannerPolicy(32, 1, 8, 2, 1, narrow_lanes=True),
                bfx.BatchPlannerPolicy(32, 0, 1, 64, 1, narrow_lanes=True)]
    res = bfx.ResidentDeviceGraph.upload_once(layout)
    ws = bfx.Workspace(res)
    best, times = ws.autotune_policy(layout, qs, policies)
    assert best in (0, 1) and all(t > 0 for t in times) and times[best] == min(times)
    descs = bfx.make_overlapping_batch_plan(layout, qs, policies[best]).descriptions()
    ws.execute(bfx.GpuRunOptions(engine=bfx.ENGINE_AUTO))
    st = ws.fetch_statuses()
    labels = [ws.download_labels(b, x.lane_width) for b, x in enumerate(descs)]
    lanes = [[qs[i] if i != bfx.NO_EDGE else None for i in x.query_index_by_lane] for x in descs]
    check_batches(layout, descs, lanes, st, labels, Oracle.from_layout(layout))
    ws.close()
    res.close()
