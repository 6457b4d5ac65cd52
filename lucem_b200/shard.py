"""Splitting independent work items across ranks (one process per GPU).

The path shards naturally: blocks of a tile walk (crates/lucem-core/src/
tiling.rs:54-78) and images of a batch are independent, so each rank takes a
contiguous share of the list, balanced by an estimate of the work (pixels),
and runs it with no collective on the data path.  Only the final gather of
results (if the caller wants them on one rank) crosses processes.
"""
from __future__ import annotations

from typing import Callable, Sequence, TypeVar

T = TypeVar("T")


def split_balanced(costs: Sequence[float], world: int) -> list:
    """Boundaries [b0=0, b1, ..., b_world=len] of contiguous shares whose summed
    costs are as even as a greedy prefix split makes them."""
    n = len(costs)
    if world < 1:
        raise ValueError("world must be >= 1")
    total = float(sum(costs))
    bounds = [0]
    acc = 0.0
    i = 0
    for r in range(1, world):
        target = total * r / world
        while i < n and acc + costs[i] / 2 <= target:
            acc += costs[i]
            i += 1
        bounds.append(i)
    bounds.append(n)
    return bounds


def shard(items: Sequence[T], rank: int, world: int, cost: Callable[[T], float] = lambda _: 1.0) -> list:
    """The contiguous share of `items` that `rank` of `world` processes."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world {world}")
    b = split_balanced([cost(x) for x in items], world)
    return list(items[b[rank]:b[rank + 1]])


def block_cost(block) -> float:
    """Work estimate of one tile-walk block: its owned pixels."""
    return float(block.size[0] * block.size[1] * block.size[2])


def allreduce_psf_grad(grad, group=None):
    """Sum a PSF gradient over the ranks of the default (or given) process
    group, in place: the one collective of a data-parallel PSF fit, where each
    rank runs the reverse pass of its share of the volumes with the same PSF.
    A no-op without an initialised process group or with one rank."""
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size(group) == 1:
        return grad
    dist.all_reduce(grad, op=dist.ReduceOp.SUM, group=group)
    return grad
