"""Host-side helpers for running the engine as independent replicas, one
process per GPU.

The hash has no exchange step: rows are independent and the parameter table
is read-only, so N GPUs are N replicas that each hash a contiguous, nnz-balanced
share of the rows (the reference splits rows over devices the same way,
minhashcuda.cc:289-383, but inside one process).  Only timing needs the ranks
to agree (the slowest rank's time is the job's time).
"""
from __future__ import annotations

import numpy as np


def shard_rows(indptr, world: int, rank: int) -> tuple[int, int]:
    """Rows [r0, r1) of rank `rank` out of `world`: contiguous ranges whose nnz
    are as equal as row boundaries allow."""
    indptr = np.asarray(indptr, dtype=np.int64)
    rows = len(indptr) - 1
    if world <= 1:
        return 0, rows
    base, nnz = int(indptr[0]), int(indptr[-1] - indptr[0])

    def cut(k):
        if k <= 0:
            return 0
        if k >= world:
            return rows
        target = base + nnz * k // world
        return int(np.searchsorted(indptr, target, side="left"))

    r0, r1 = cut(rank), cut(rank + 1)
    return min(r0, rows), min(max(r1, r0), rows)


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The largest `value` over all ranks (the job's time is the slowest
    rank's); `value` itself when there is no process group."""
    if dist is None or not dist.is_initialized():
        return value
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, dist=None, device=None) -> float:
    """The sum of `value` over all ranks (the job's work is every rank's
    shard); `value` itself when there is no process group."""
    if dist is None or not dist.is_initialized():
        return value
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())

