"""Work sharding across ranks: inflations, configurations and edges are
independent units, so each rank takes a contiguous slice and no collective is
needed on the data path (only the timing reductions of bench.py)."""
from __future__ import annotations

from typing import Sequence, Tuple


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


def reduce_timing(dist, device, dev_seconds: float, wall_seconds: float, units: float):
    """Max over ranks of the device and wall times, sum of the units processed."""
    import torch
    t = torch.tensor([dev_seconds, wall_seconds], dtype=torch.float64, device=device)
    u = torch.tensor([units], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return float(t[0]), float(t[1]), float(u[0])
