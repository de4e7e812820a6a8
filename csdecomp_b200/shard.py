"""Work sharding across ranks: inflations, configurations and edges are
independent units, so each rank takes a contiguous slice and no collective is
needed on the data path (only the timing reductions of bench.py).

Slices are either equal in count (`shard_range`) or balanced by a predicted
cost per unit (`cost_balanced_ranges`): an EI-ZO inflation's cost grows with
its plant's dimension and primitive count (the sampler's face loop is
dimension-long and a check visits every pair), so equal counts would leave
the ranks that drew the two-arm scenes last to finish.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple

import numpy as np


def shard_range(n: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous [begin, end) slice of n units for `rank` of `world`; sizes differ by at most one."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    base, extra = divmod(n, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def shard(items: Sequence, rank: int, world: int):
    b, e = shard_range(len(items), rank, world)
    return items[b:e]


def cost_balanced_ranges(costs: Sequence[float], world: int) -> List[Tuple[int, int]]:
    """Contiguous [begin, end) ranges, one per rank, covering every unit once,
    with the cumulative cost cut as close as possible to r / world of the
    total at each boundary (each range non-empty when there are at least
    `world` units). Deterministic, so every rank computes the same split."""
    if world <= 0:
        raise ValueError("world must be positive")
    c = np.asarray(costs, np.float64)
    if c.ndim != 1 or (c < 0).any() or not np.isfinite(c).all():
        raise ValueError("costs must be finite and non-negative")
    n = len(c)
    if n == 0:
        return [(0, 0)] * world
    cum = np.concatenate([[0.0], np.cumsum(c)])
    total = cum[-1]
    cuts = [0]
    for r in range(1, world):
        target = total * r / world
        j = int(np.searchsorted(cum, target))          # first boundary with cum >= target
        if j > 0 and target - cum[j - 1] <= cum[min(j, n)] - target:
            j -= 1                                      # the nearer boundary
        lo = cuts[-1] + (1 if n - cuts[-1] > world - r else 0)  # keep ranges non-empty where possible
        hi = n - (world - r) if n >= world else n
        cuts.append(int(min(max(j, lo), max(hi, lo))))
    cuts.append(n)
    return [(cuts[r], cuts[r + 1]) for r in range(world)]


def reduce_timing(dist, device, dev_seconds: float, wall_seconds: float, units: float):
    """Max over ranks of the device and wall times, sum of the units processed."""
    import torch
    t = torch.tensor([dev_seconds, wall_seconds], dtype=torch.float64, device=device)
    u = torch.tensor([units], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return float(t[0]), float(t[1]), float(u[0])
