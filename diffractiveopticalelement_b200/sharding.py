"""Multi-GPU plumbing for batched designs and sweeps (no reference counterpart).

The work units of this path -- designs, and fields x distances of a focus sweep
-- are independent, so N GPUs run N replicas, one process per GPU
(torch.distributed over NCCL; gloo for CPU tests), each on a contiguous shard of
the global batch. Nothing is exchanged inside a design loop. The only collectives
are the final gather of per-design results to rank 0 and, when the warm-start
surrogate is trained data-parallel, the all-reduce of its gradients.
"""
from __future__ import annotations

import math

import numpy as np


def design_cost(n: int, iterations: int) -> float:
    """Relative cost of one n x n design: two FFT passes per iteration ~ n^2 log2(n^2)."""
    return float(n) * n * math.log2(max(2, n * n)) * max(1, iterations)


def shard_by_cost(costs, world: int) -> list[tuple[int, int]]:
    """Contiguous [start, end) ranges of `costs` for `world` ranks with balanced sums.

    Boundaries are placed where the running total crosses k / world of the total
    (each unit is indivisible); every rank gets a range, possibly empty.
    """
    if world < 1:
        raise ValueError("world must be >= 1")
    c = np.asarray(costs, dtype=np.float64)
    if c.ndim != 1 or np.any(c < 0):
        raise ValueError("costs must be a 1-D array of non-negative values")
    n = c.size
    if n == 0:
        return [(0, 0)] * world
    cum = np.concatenate([[0.0], np.cumsum(c)])
    total = cum[-1]
    bounds = [0]
    for k in range(1, world):
        target = total * k / world
        # the boundary whose prefix sum is closest to the target, never before the previous one
        j = int(np.searchsorted(cum, target))
        if j > 0 and abs(cum[j - 1] - target) <= abs(cum[min(j, n)] - target):
            j -= 1
        bounds.append(min(max(j, bounds[-1]), n))
    bounds.append(n)
    return [(bounds[k], bounds[k + 1]) for k in range(world)]


def my_shard(costs, rank: int, world: int) -> tuple[int, int]:
    return shard_by_cost(costs, world)[rank]


def gather_results(local, rank: int, world: int, counts, group=None):
    """Concatenate per-rank result arrays (shape [count_r, ...]) on every rank in rank order.

    `local` is a torch tensor on the rank's device (NCCL) or CPU (gloo); `counts`
    are the shard sizes of all ranks. Returns the full [sum(counts), ...] tensor.
    """
    import torch
    import torch.distributed as dist
    if world == 1:
        return local
    mx = max(counts)
    shape = tuple(local.shape[1:])
    pad = torch.zeros((mx,) + shape, dtype=local.dtype, device=local.device)
    pad[:local.shape[0]] = local
    bufs = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(bufs, pad, group=group)
    return torch.cat([b[:c] for b, c in zip(bufs, counts)])


def allreduce_mean_(t, world: int, group=None):
    """In-place average of a tensor over ranks (data-parallel gradients)."""
    import torch.distributed as dist
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        t /= world
    return t
