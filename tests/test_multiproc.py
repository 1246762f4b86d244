"""Multi-process (world size 2, gloo on CPU) coverage of the replica path:
every rank derives the same batch shard from the plan, the shards cover all
batches exactly once with balanced estimated work, per-rank status records
are gathered, and step times are max-reduced -- the only collectives the
replica design uses (no collective on the data path)."""
import os

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bfx
from bfx import replicas, workloads


def _worker(rank, world, port, queue):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        layout, grid = workloads.build_graph("c1")
        qs = workloads.box_queries(layout, grid, 60, 2, 10, seed=21)
        plan = bfx.make_overlapping_batch_plan(layout, qs, bfx.BatchPlannerPolicy(32, narrow_lanes=True))
        est = [e[3] for e in plan.estimates]
        shards = workloads.shard_batches(est, world)
        mine = shards[rank]
        # per-rank status records (48-byte DeviceRunStatus) as a rank's
        # workspace returns them: rounds_completed carries the batch index
        statuses = []
        for b in mine:
            s = bfx.DeviceRunStatus()
            s.rounds_completed = b + 1
            s.error_bits = rank
            s.stop_reason = bfx.STOP_CONVERGED
            statuses.append(s)
        gathered = replicas.gather_statuses(dist, statuses)
        recs = [[(int(s.rounds_completed), int(s.error_bits), int(s.stop_reason)) for s in g] for g in gathered]
        t = replicas.max_over_ranks(dist, 1.0 + rank)
        queue.put((rank, shards, recs, t, est))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_replica_shards_gather_and_max_timing():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = 29500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get() for _ in range(world)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    out.sort()
    shards0, shards1 = out[0][1], out[1][1]
    assert shards0 == shards1  # deterministic assignment on every rank
    flat = sorted(b for s in shards0 for b in s)
    assert flat == list(range(len(flat)))
    est = out[0][4]
    loads = [sum(est[b] for b in s) for s in shards0]
    assert max(loads) - min(loads) <= max(est)  # greedy bound
    for rank in range(world):
        recs = out[rank][2]
        assert len(recs) == world
        for r in range(world):  # rank r's records, in its shard order, tagged with r
            assert [x[0] - 1 for x in recs[r]] == shards0[r]
            assert all(x[1] == r and x[2] == bfx.STOP_CONVERGED for x in recs[r])
        assert out[rank][3] == 2.0  # max over ranks


def _shard_worker(rank, world, port, queue):
    """One rank of a sharded run: the whole query set is planned on every
    rank, this rank takes its shard of batches (balanced lane-edges), runs
    each valid lane through the oracle as the runner, and the per-query
    results are all-gathered."""
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle.oracle import Oracle
        layout, grid = workloads.build_graph("c2", scale_tiles=(16, 16))
        qs = workloads.box_queries(layout, grid, 40, 2, 8, seed=5, targets=(1, 3))
        plan = bfx.make_overlapping_batch_plan(layout, qs, bfx.BatchPlannerPolicy(32, 1, 8, 2, 1, narrow_lanes=True))
        descs = plan.descriptions()
        mine = workloads.shard_batches([e[3] for e in plan.estimates], world)[rank]
        orc = Oracle.from_layout(layout)
        results = {}
        for b in mine:
            d = descs[b]
            for lane in range(d.lane_width):
                if not (d.valid_lane_mask >> lane) & 1:
                    continue
                qi = int(d.query_index_by_lane[lane])
                q = qs[qi]
                od, op = orc.region_sssp(q.sources, q.targets, q.selected_tiles)
                tg = np.asarray(q.targets, np.int64)
                results[qi] = (od[tg].tolist(), op[tg].tolist(), int(od.astype(np.uint64).sum()), rank)
        gathered = [None] * world
        dist.all_gather_object(gathered, results)
        queue.put((rank, gathered, len(descs)))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_sharded_query_set_equals_one_rank_run():
    """bench.py --shard's split (not measured on GPUs here): two gloo ranks
    share one planned query set by shard_batches; the union of their gathered
    per-query results covers every query exactly once and equals the one-rank
    run of the whole set."""
    from oracle.oracle import Oracle
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = 30500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_shard_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get() for _ in range(world)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    out.sort(key=lambda x: x[0])
    assert out[0][1] == out[1][1]  # every rank holds the same gathered set
    merged = {}
    for part in out[0][1]:
        assert not set(part) & set(merged)  # no query on two ranks
        merged.update(part)
    assert {r for v in merged.values() for r in [v[3]]} == {0, 1}  # both ranks did work
    layout, grid = workloads.build_graph("c2", scale_tiles=(16, 16))
    qs = workloads.box_queries(layout, grid, 40, 2, 8, seed=5, targets=(1, 3))
    assert sorted(merged) == list(range(len(qs)))
    orc = Oracle.from_layout(layout)
    for qi, qq in enumerate(qs):
        od, op = orc.region_sssp(qq.sources, qq.targets, qq.selected_tiles)
        tg = np.asarray(qq.targets, np.int64)
        assert merged[qi][:3] == (od[tg].tolist(), op[tg].tolist(), int(od.astype(np.uint64).sum()))
