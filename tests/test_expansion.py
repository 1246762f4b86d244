"""Expansion loop (bfx_expansion_run_with_runner) on the CPU: the host loop
driven by the oracle as the pass runner must reproduce the reference's own
run_host_batched_expansion (src/batched_expansion.cpp:1681) outcome for
outcome -- dispositions, attempts, scheduled/total expansions, fallback use,
final regions and their sizes, terminal status words -- plus the
deterministic metrics and the expansion-count histogram, for every schedule
kind and both terminal policies."""
import numpy as np
import pytest

import bfx
from bfx import expansion as ex
from bfx import workloads
from oracle.oracle import Oracle, Ref

needs_ref = pytest.mark.skipif(not Ref.available(), reason="reference library not built here (oracle/_ref)")

SCHEDULES = [
    # (kind, fixed ring, hybrid count, maximum expansions, terminal policy)
    (ex.ONE_RING, 0, 0, 3, ex.FULL_REGION_FALLBACK),
    (ex.ONE_RING, 0, 0, 2, ex.EXPLICIT_FAILURE),
    (ex.FIXED_RING, 2, 0, 2, ex.EXPLICIT_FAILURE),
    (ex.DOUBLING, 0, 0, 3, ex.FULL_REGION_FALLBACK),
    (ex.HYBRID, 0, 1, 4, ex.EXPLICIT_FAILURE),
    (ex.DOUBLING, 0, 0, 0, ex.FULL_REGION_FALLBACK),
]


def oracle_runner(layout, orc):
    """Pass runner: every valid lane of every batch solved by the oracle on
    its own selected tiles; clean statuses with reached / miss lanes."""
    T = layout.tile_count

    def run(descs):
        out = []
        for dc in descs:
            d = bfx.BatchDescription.from_c(dc)
            st = bfx.DeviceRunStatus()
            st.valid_lane_mask = d.valid_lane_mask
            st.converged = 1
            st.converged_lane_mask = d.valid_lane_mask
            st.stop_reason = bfx.STOP_CONVERGED
            masks = d.tile_lane_masks[:T]
            for lane in range(d.lane_width):
                if not (d.valid_lane_mask >> lane) & 1:
                    continue
                src = d.sources[d.source_offsets[lane]:d.source_offsets[lane + 1]]
                tgt = d.targets[d.target_offsets[lane]:d.target_offsets[lane + 1]]
                tiles = np.nonzero((masks >> np.uint32(lane)) & 1)[0].astype(np.uint32)
                dist, _ = orc.region_sssp(src, tgt, tiles)
                if np.all(dist[tgt] != np.uint32(0x7F800000)):
                    st.reached_target_mask |= 1 << lane
                else:
                    st.bounding_box_miss_mask |= 1 << lane
            out.append(st)
        return out

    return run


def rich_queries(layout, grid, seed):
    """Small boxes (many first-pass misses), targets that no edge enters
    (unreachable everywhere: expansion limit or full-region fallback), boxes
    already covering every located tile (stall), and full-graph regions."""
    rng = np.random.default_rng(seed)
    qs = workloads.box_queries(layout, grid, 40, 1, 2, seed=seed, targets=(1, 4))
    indeg = np.diff(layout.arrays["csc_column_offsets"].astype(np.int64))
    dead = np.nonzero(indeg == 0)[0]
    owner = layout.arrays["owner_tiles"]
    tvo = layout.tiles["tile_vertex_offsets"]
    xy = layout.tiles["tile_xy"]
    located = np.nonzero(layout.tiles["has_location"])[0].astype(np.uint32)
    every = np.arange(layout.tile_count, dtype=np.uint32)

    def vertex_in(tiles):
        t = int(tiles[rng.integers(0, len(tiles))])
        return int(tvo[t] + rng.integers(0, int(tvo[t + 1] - tvo[t])))

    qid = 1000
    for k, v in enumerate(dead[:10]):
        if k < 6:
            tx, ty = xy[owner[v]]
            tiles = located[(np.abs(xy[located, 0] - tx) <= 1) & (np.abs(xy[located, 1] - ty) <= 1)]
        else:
            tiles = located if k < 8 else every
        src = vertex_in(tiles)
        qs.append(bfx.RouteQuery(qid, [src], [int(v), vertex_in(tiles)], tiles))
        qid += 1
    return qs


@pytest.fixture(scope="module")
def case():
    spec = dict(workloads.GRAPHS["c1"])
    g, order, _ = bfx.synth_graph(**spec)
    layout = bfx.build_device_graph_layout(g, order)
    qs = rich_queries(layout, (spec["tiles_x"], spec["tiles_y"]), 1717)
    return g, order, layout, qs


def compare_with_reference(res, ref, qs):
    outs = ref["outcomes"]
    assert len(res["outcomes"]) == len(qs)
    tiles_at = 0
    for i, o in enumerate(res["outcomes"]):
        assert [o[f] for f in ex.OUTCOME_FIELDS] == [int(x) for x in outs[i]], (i, o, outs[i])
        n = o["final_tile_count"]
        np.testing.assert_array_equal(res["final_tiles"][i], ref["tiles"][tiles_at:tiles_at + n])
        tiles_at += n
    assert [res["metrics"][f] for f in ex.METRIC_FIELDS] == [int(x) for x in ref["metrics"]]
    assert res["histogram"] == [int(x) for x in ref["histogram"]]


@needs_ref
@pytest.mark.parametrize("sched", SCHEDULES, ids=lambda s: f"k{s[0]}r{s[1]}h{s[2]}m{s[3]}t{s[4]}")
def test_expansion_loop_equals_reference(case, sched):
    g, order, layout, qs = case
    kind, ring, hyb, mx, term = sched
    policy = bfx.BatchPlannerPolicy(32, 1, 8, 2, 1)
    opts = ex.ExpansionOptions(schedule_kind=kind, fixed_ring_size=ring, hybrid_small_expansion_count=hyb,
                               maximum_expansions=mx, terminal_policy=term, planner_policy=policy)
    res = ex.run_expansion_with_runner(oracle_runner(layout, Oracle.from_layout(layout)), layout, qs, opts)
    ref = Ref()
    h = ref.case_from_input(g, order)
    for q in qs:
        ref.query_add(h, q.query_id, q.sources, q.targets, q.selected_tiles)
    r = ref.expansion_run(h, len(qs), 2, (32, 1, 8, 2, 1), kind, ring, hyb, mx, term,
                          tile_cap=len(qs) * layout.tile_count)
    ref.free(h)
    compare_with_reference(res, r, qs)
    m = res["metrics"]
    # the workload exercises the loop: first-pass misses, retries, and
    # terminal outcomes other than reached
    assert m["initial_reached_queries"] < m["reached_queries"] < len(qs) and m["planning_passes"] >= 2


def test_expansion_options_are_validated(case):
    _, _, layout, qs = case
    run = oracle_runner(layout, Oracle.from_layout(layout))
    bad = [dict(schedule_kind=0), dict(schedule_kind=ex.FIXED_RING, fixed_ring_size=1),
           dict(schedule_kind=ex.ONE_RING, fixed_ring_size=2), dict(schedule_kind=ex.HYBRID),
           dict(schedule_kind=ex.DOUBLING, hybrid_small_expansion_count=1), dict(terminal_policy=2),
           dict(engine=7)]
    for kw in bad:
        with pytest.raises(ValueError):
            ex.run_expansion_with_runner(run, layout, qs[:4], ex.ExpansionOptions(**kw))


def test_runner_status_contract_is_enforced(case):
    """A clean status that does not partition the valid lanes is rejected."""
    _, _, layout, qs = case

    def broken(descs):
        out = []
        for dc in descs:
            st = bfx.DeviceRunStatus()
            st.valid_lane_mask = dc.valid_lane_mask
            st.converged = 1
            st.stop_reason = bfx.STOP_CONVERGED
            out.append(st)
        return out

    with pytest.raises(Exception):
        ex.run_expansion_with_runner(broken, layout, qs[:4], ex.ExpansionOptions())


def test_non_clean_batches_are_engine_failures_and_never_expand(case):
    _, _, layout, qs = case

    def round_limited(descs):
        out = []
        for dc in descs:
            st = bfx.DeviceRunStatus()
            st.valid_lane_mask = dc.valid_lane_mask
            st.stop_reason = bfx.STOP_MAXIMUM_ROUNDS
            out.append(st)
        return out

    res = ex.run_expansion_with_runner(round_limited, layout, qs[:10], ex.ExpansionOptions())
    for o in res["outcomes"]:
        assert ex.DISPOSITIONS[o["disposition"]] == "engine_failure"
        assert o["attempts"] == 1 and o["total_expansions"] == 0
        assert o["terminal_stop_reason"] == bfx.STOP_MAXIMUM_ROUNDS
    assert res["metrics"]["planning_passes"] == 1
