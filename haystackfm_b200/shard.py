"""Multi-GPU data parallelism for the query path: index replicas + read sharding.

Reads are independent, so each rank (one process per GPU) loads its own copy of the index
and queries its contiguous share of the reads; there is no exchange step on the data
path.  The only collectives are a barrier around timed regions, a MAX reduction of the
per-rank time, and an optional gather of per-read results to rank 0 in read order.
Works with any torch.distributed backend (nccl on GPUs, gloo on CPU for tests).
"""
from __future__ import annotations

import pickle
from typing import Callable, List, Sequence

import numpy as np


def shard_range(n: int, rank: int, world: int):
    """Contiguous [start, end) share of n reads for `rank` (sizes differ by at most one)."""
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def max_over_ranks(value: float, dist=None) -> float:
    """Max of a per-rank scalar (timings are reported as the slowest rank)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return value
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64)
    if dist.get_backend() == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_in_order(per_read: Sequence, dist=None) -> List:
    """Concatenate every rank's per-read results on rank 0, in global read order."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return list(per_read)
    world = dist.get_world_size()
    out = [None] * world
    dist.all_gather_object(out, list(per_read))
    if dist.get_rank() != 0:
        return []
    res: List = []
    for part in out:
        res.extend(part)
    return res


def run_sharded(n: int, query: Callable[[int, int], Sequence], dist=None) -> List:
    """Run `query(start, end)` on this rank's share and gather the results to rank 0."""
    rank = dist.get_rank() if dist is not None and dist.is_initialized() else 0
    world = dist.get_world_size() if dist is not None and dist.is_initialized() else 1
    a, b = shard_range(n, rank, world)
    return gather_in_order(query(a, b), dist)
