"""Host logic of multi-GPU runs: one process per GPU, no collective on the
data path.

Independent instances (a batch of reconstructions) are the shard unit: every
rank solves its own contiguous share as its own block-diagonal batch, and
only timings and per-instance results cross ranks, through torch.distributed
(NCCL between GPUs, gloo on the host).  The single large SIRT is run as
independent replicas.
"""
from __future__ import annotations

import numpy as np


def shard(n_units: int, rank: int, world: int, cost=None) -> np.ndarray:
    """Contiguous indices of the units rank `rank` of `world` owns.

    With `cost` (one non-negative weight per unit, e.g. nonzeros), the cut
    points split the cumulative cost as evenly as contiguous ranges allow;
    without it every rank gets n_units // world units, the first
    n_units % world ranks one more.  Every unit belongs to exactly one rank.
    """
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must lie in 0..world-1")
    if cost is None:
        q, r = divmod(n_units, world)
        lo = rank * q + min(rank, r)
        return np.arange(lo, lo + q + (1 if rank < r else 0))
    c = np.asarray(cost, dtype=np.float64)
    if c.size != n_units or np.any(c < 0):
        raise ValueError("cost needs one non-negative weight per unit")
    cum = np.concatenate([[0.0], np.cumsum(c)])
    total = cum[-1]
    # cut k sits where the cumulative cost first reaches k/world of the total
    cuts = [0] + [int(np.searchsorted(cum, total * k / world, side="left")) for k in range(1, world)] + [n_units]
    cuts = np.maximum.accumulate(np.clip(cuts, 0, n_units))
    return np.arange(cuts[rank], cuts[rank + 1])


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of `value` over all ranks (the job's time is its slowest
    rank's); the value itself when torch.distributed is not initialised."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def gather_units(local: np.ndarray, device=None) -> np.ndarray:
    """Concatenate every rank's per-unit results (rows of `local`) in rank
    order, on every rank.  Ranks may hold different numbers of rows."""
    import torch
    import torch.distributed as dist
    local = np.ascontiguousarray(local, dtype=np.float64)
    if not (dist.is_available() and dist.is_initialized()):
        return local
    world = dist.get_world_size()
    n = torch.tensor([local.shape[0]], dtype=torch.int64, device=device)
    counts = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(counts, n)
    counts = [int(c.item()) for c in counts]
    width = int(np.prod(local.shape[1:])) if local.ndim > 1 else 1
    mx = max(counts)
    buf = torch.zeros((mx, width), dtype=torch.float64, device=device)
    if local.shape[0]:
        buf[:local.shape[0]] = torch.from_numpy(local.reshape(local.shape[0], width)).to(buf.device)
    parts = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    rows = [p[:c].cpu().numpy() for p, c in zip(parts, counts)]
    out = np.concatenate(rows, axis=0)
    return out.reshape((out.shape[0],) + local.shape[1:]) if local.ndim > 1 else out.ravel()
