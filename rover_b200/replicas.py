"""Replica plumbing for multi-GPU runs: one process per GPU, each holding a
full copy of the index and searching its own queries.

Searches shard over queries with no exchange, so no collective touches the
data path.  The collectives here only coordinate measurement: a timed
region's length is the maximum over ranks, a configuration picked on rank 0
is shared with every rank, and a decision that changes which collectives
follow (time the gated form or not) is taken by all ranks together, so every
rank runs the same collective sequence.
"""
from __future__ import annotations

import datetime
import os


def init(backend: str = "nccl", timeout_s: int = 600):
    """torch.distributed for WORLD_SIZE > 1 (None for a single process)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world <= 1:
        return None
    import torch.distributed as dist
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def max_over_ranks(dist, value: float, device) -> float:
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def all_ranks(dist, flag: bool, device) -> bool:
    """True when the flag holds on every rank."""
    if dist is None:
        return bool(flag)
    import torch
    t = torch.tensor([1 if flag else 0], dtype=torch.int32, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MIN)
    return bool(t.item())


def from_rank0(dist, obj):
    """Rank 0's object on every rank (a picked configuration)."""
    if dist is None:
        return obj
    box = [obj]
    dist.broadcast_object_list(box, src=0)
    return box[0]


def throughput(queries_per_rank: int, steps: int, world: int, total_ms: float) -> float:
    """Whole-job queries per second: every rank searched queries_per_rank
    queries per step; total_ms is the max over ranks."""
    return queries_per_rank * steps * world / (total_ms / 1e3)
