"""Splitting independent transforms across GPUs (one process per GPU, no data-path collective).

Transforms of a batch are independent, so a multi-GPU run gives each rank its own share and
needs no exchange of data: `shard_batch` splits a uniform batch into contiguous ranges,
`shard_uneven` splits an uneven batch's descriptors by work (5 n log2 n per transform, largest
first onto the least-loaded rank). The only collective is the timing reduction of a benchmark,
`max_over_ranks`, which takes the slowest rank's time.
"""
from __future__ import annotations

import heapq

import numpy as np


def shard_batch(batch: int, world: int, rank: int) -> tuple[int, int]:
    """(first transform, count) of rank `rank` for `batch` transforms over `world` ranks;
    counts differ by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("invalid rank / world size")
    base, extra = divmod(batch, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def transform_cost(log2n: np.ndarray) -> np.ndarray:
    n = np.left_shift(1, np.asarray(log2n, np.int64))
    return 5.0 * n * np.maximum(np.asarray(log2n, np.float64), 1.0)


def shard_uneven(log2n, world: int) -> list[np.ndarray]:
    """Indices of the descriptors each rank runs, balancing 5 n log2 n (longest-processing-time
    first: each transform, largest first, goes to the rank with the least work so far)."""
    if world < 1:
        raise ValueError("invalid world size")
    cost = transform_cost(log2n)
    order = np.argsort(-cost, kind="stable")
    heap = [(0.0, r) for r in range(world)]
    owner = np.empty(len(cost), np.int64)
    for i in order:
        load, r = heapq.heappop(heap)
        owner[i] = r
        heapq.heappush(heap, (load + cost[i], r))
    return [np.flatnonzero(owner == r) for r in range(world)]


def max_over_ranks(seconds: float, device=None) -> float:
    """The slowest rank's time (all_reduce MAX); the value itself when not distributed."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(seconds)
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
