"""Sharding a batch of independent systems over GPUs, one process per GPU.

Systems never exchange data, so the data path needs no collective.  Each rank
integrates a contiguous slice of the columns of y[N, NUM] (and of var[NUM]).
Collectives appear only at the edges:
  * `max_over_ranks` reduces a timing or a counter, for example the max over
    ranks of the device time of a step;
  * `gather_columns` assembles the slices on every rank when the results must
    meet in one place (an all-gather of equal-size padded slices).
The process group (NCCL on GPUs, gloo on CPU) belongs to the caller.
"""
from __future__ import annotations

import numpy as np


def shard_range(num: int, rank: int, world: int):
    """[lo, hi) of the systems owned by `rank`: contiguous, sizes differ by at most one."""
    if world < 1 or not 0 <= rank < world or num < 0:
        raise ValueError("bad shard arguments")
    base, extra = divmod(num, world)
    lo = rank * base + min(rank, extra)
    hi = lo + base + (1 if rank < extra else 0)
    return lo, hi


def shard_columns(y: np.ndarray, var: np.ndarray, rank: int, world: int):
    lo, hi = shard_range(y.shape[1], rank, world)
    return np.ascontiguousarray(y[:, lo:hi]), np.ascontiguousarray(var[lo:hi])


def max_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_columns(y_local: np.ndarray, num: int, device=None) -> np.ndarray:
    """All-gather the column slices of every rank into the full y[N, num]."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return y_local
    world, rank = dist.get_world_size(), dist.get_rank()
    n = y_local.shape[0]
    width = -(-num // world)
    buf = torch.zeros((n, width), dtype=torch.float64, device=device)
    lo, hi = shard_range(num, rank, world)
    buf[:, :hi - lo] = torch.from_numpy(np.ascontiguousarray(y_local)).to(buf.device)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    out = np.empty((n, num))
    for r, p in enumerate(parts):
        a, b = shard_range(num, r, world)
        out[:, a:b] = p[:, :b - a].cpu().numpy()
    return out
