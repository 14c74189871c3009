"""Multi-GPU use of the substrate: one process per GPU, independent shards.

Configurations, edges, rollouts and trajectories are independent units, so a
batch is split into contiguous ranges, one per rank; each rank evaluates its
range on its own GPU with no communication on the data path. The only
collective is the optional gather of the per-rank result arrays (to every
rank, or to none when each rank consumes its own slice).
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence, Tuple

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


def require_same_device(model_device: int, current_device: int) -> None:
    """A model's device blob lives on the GPU it was built on; every kernel
    reads it, so a rank must build its own model on its own GPU. Raises
    ValueError on a mismatch (the library returns PS_EINVAL for the same
    case, with the two ordinals in the message)."""
    if int(model_device) != int(current_device):
        raise ValueError(f"robot model was built on cuda:{model_device} but cuda:{current_device} is current; "
                         "build one model per rank on that rank's GPU")


def gpu_edge_checker(robot, scene, params=None) -> Callable[[np.ndarray, np.ndarray, Optional[np.ndarray]],
                                                             Tuple[np.ndarray, np.ndarray]]:
    """The default per-shard checker of check_edges_sharded: ps_check_edges on
    the current GPU, host arrays in and out. The robot must have been built
    on the current GPU (one model per rank)."""
    import torch

    from .api import check_edges

    require_same_device(robot.info()["device"], torch.cuda.current_device())

    def check(frm, to, G):
        dev = torch.device("cuda", torch.cuda.current_device())
        v, c, _ = check_edges(robot, scene, torch.from_numpy(frm).to(dev), torch.from_numpy(to).to(dev),
                              samples=None if G is None else torch.from_numpy(G).to(dev), params=params)
        return v.cpu().numpy(), c.cpu().numpy()

    return check


def check_edges_sharded(robot, scene, frm, to, samples=None, params=None, gather: bool = True, group=None,
                        checker=None):
    """ps_check_edges over this rank's contiguous range of edges; returns
    (valid, cost) as host arrays (the full arrays, in edge order, when
    gather). `checker(frm, to, G) -> (valid, cost)` evaluates one shard; the
    default is gpu_edge_checker(robot, scene, params) on this rank's GPU."""
    frm = np.ascontiguousarray(frm, np.float32)
    to = np.ascontiguousarray(to, np.float32)
    if frm.shape != to.shape:
        raise ValueError("from/to shapes differ")
    G = None if samples is None else np.ascontiguousarray(samples, np.int32)
    if G is not None and len(G) != len(frm):
        raise ValueError("samples must have one entry per edge")
    if checker is None:
        checker = gpu_edge_checker(robot, scene, params)

    def evaluate(lo, hi):
        return checker(frm[lo:hi], to[lo:hi], None if G is None else G[lo:hi])

    return run_sharded(len(frm), evaluate, group=group, gather=gather)
