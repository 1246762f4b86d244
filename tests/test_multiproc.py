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
