"""Replica execution across ranks (one process per GPU).

Queries and batches are independent, so every rank holds the whole resident
graph and relaxes its own batches; the relaxation itself has no collective.
The one exchange is the final gather of the fixed-size per-batch status
records (48-byte DeviceRunStatus, gpu_api.hpp:176-187) so that one rank can
report the whole job; timing uses a max-reduction over ranks.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import DeviceRunStatus
from .workloads import shard_batches

__all__ = ["shard_batches", "gather_statuses", "max_over_ranks"]

_REC = C.sizeof(DeviceRunStatus)


def _device_for(dist, group):
    import torch
    if dist.get_backend(group) == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def gather_statuses(dist, statuses, group=None) -> list:
    """All-gather every rank's status records; returns one list of
    DeviceRunStatus per rank (rank order).  Counts may differ per rank: the
    records are padded to the largest count for the collective."""
    import torch
    dev = _device_for(dist, group)
    world = dist.get_world_size(group)
    n = torch.tensor([len(statuses)], dtype=torch.int64, device=dev)
    counts = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(counts, n, group=group)
    counts = [int(c.item()) for c in counts]
    cap = max(max(counts), 1)
    buf = np.zeros(cap * _REC, np.uint8)
    for i, s in enumerate(statuses):
        buf[i * _REC:(i + 1) * _REC] = np.frombuffer(bytes(s), np.uint8)
    mine = torch.from_numpy(buf).to(dev)
    parts = [torch.zeros_like(mine) for _ in range(world)]
    dist.all_gather(parts, mine, group=group)
    out = []
    for r in range(world):
        raw = parts[r].cpu().numpy().tobytes()
        out.append([DeviceRunStatus.from_buffer_copy(raw[i * _REC:(i + 1) * _REC]) for i in range(counts[r])])
    return out


def max_over_ranks(dist, x: float, group=None) -> float:
    """Largest value of x over all ranks (device times are reported as the max)."""
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device_for(dist, group))
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
