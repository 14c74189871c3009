"""Multi-GPU use of the substrate: one process per GPU, independent shards.

Configurations, edges, rollouts and trajectories are independent units, so a
batch is split into contiguous ranges, one per rank; each rank evaluates its
range on its own GPU with no communication on the data path. The only
collective is the optional gather of the per-rank result arrays (to every
rank, or to none when each rank consumes its own slice).
"""
from __future__ import annotations

from typing import Callable, List, Sequence, Tuple

import numpy as np


def shard_range(n: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous [lo, hi) of n units for `rank` of `world` (sizes differ by at most 1)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, rem = divmod(n, world)
    lo = rank * base + min(rank, rem)
    return lo, lo + base + (1 if rank < rem else 0)


def run_sharded(n: int, evaluate: Callable[[int, int], Sequence[np.ndarray]], group=None,
                gather: bool = True) -> List[np.ndarray]:
    """Evaluate units [lo, hi) of this rank with `evaluate(lo, hi)` (which
    returns a tuple of host arrays, one row per unit) and, if `gather`,
    all-gather the pieces so every rank holds the full arrays in unit order."""
    import torch.distributed as dist

    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    lo, hi = shard_range(n, rank, world)
    mine = [np.asarray(a) for a in evaluate(lo, hi)]
    if not gather or world == 1:
        return mine
    pieces = [None] * world
    dist.all_gather_object(pieces, mine, group=group)
    return [np.concatenate([p[k] for p in pieces]) for k in range(len(mine))]


def check_edges_sharded(robot, scene, frm, to, samples=None, params=None, gather: bool = True, group=None):
    """ps_check_edges over this rank's contiguous range of edges on the current
    GPU; returns (valid, cost) as host arrays (full arrays when gather)."""
    import torch

    from .api import check_edges

    frm = np.asarray(frm, np.float32)
    to = np.asarray(to, np.float32)
    G = None if samples is None else np.asarray(samples, np.int32)

    def evaluate(lo, hi):
        v, c, _ = check_edges(robot, scene, torch.from_numpy(frm[lo:hi]).cuda(), torch.from_numpy(to[lo:hi]).cuda(),
                              samples=None if G is None else torch.from_numpy(G[lo:hi]).cuda(), params=params)
        return v.cpu().numpy(), c.cpu().numpy()

    return run_sharded(len(frm), evaluate, group=group, gather=gather)
