"""Multi-GPU use: replicas only.

Systems are independent and the integrators have no exchange step, so N GPUs
run N independent launches over disjoint contiguous system ranges (one
process per GPU).  The only collectives are host-side bookkeeping: the
max-over-ranks time of a step, the sum of substep counts, and gathering
results on one rank.  They go through torch.distributed (NCCL on GPUs, gloo
on CPU); nothing crosses NVLink on the data path.
"""
from __future__ import annotations

import numpy as np


def shard_range(nsys: int, rank: int, world: int):
    """Contiguous [begin, end) of systems owned by `rank` (sizes differ by at
    most one)."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad rank/world")
    base, extra = divmod(nsys, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def shard(workload, rank: int, world: int):
    b, e = shard_range(workload.net.nsys, rank, world)
    return workload.subset(slice(b, e))


def reduce_max(value: float, dist, device=None) -> float:
    """Max of a per-rank float over the group (step times)."""
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(value: int, dist, device=None) -> int:
    """Sum of a per-rank integer over the group (substep totals)."""
    import torch
    t = torch.tensor([value], dtype=torch.int64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return int(t.item())


def gather_states(y_local: np.ndarray, nsys: int, rank: int, world: int, dist):
    """Assemble the full [nsys, N] state on every rank from contiguous shards."""
    import torch
    n = y_local.shape[1]
    full = torch.zeros((nsys, n), dtype=torch.float64)
    b, e = shard_range(nsys, rank, world)
    full[b:e] = torch.from_numpy(y_local)
    dist.all_reduce(full, op=dist.ReduceOp.SUM)
    return full.numpy()
