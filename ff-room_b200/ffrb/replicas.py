"""Room-parallel replicas across GPUs (one process per GPU).

Rooms are independent, so N GPUs share a job without any collective on the
data path: each rank takes its own rooms (round-robin), advances them on its
GPU, and only the timing is combined (the max over ranks, the device time of
the slowest rank).  With torch.distributed the process group carries that one
reduction; the same helpers run on gloo (CPU tests) and NCCL (GPUs).
"""
from __future__ import annotations

from typing import List, Sequence, TypeVar

T = TypeVar("T")


def shard(items: Sequence[T], rank: int, world: int) -> List[T]:
    """Round-robin share of `items` for `rank` of `world` ranks."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    return [x for i, x in enumerate(items) if i % world == rank]


def max_over_ranks(value: float, dist=None, device: str = "cpu") -> float:
    """The maximum of `value` over all ranks (identity without a group)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, dist=None, device: str = "cpu") -> float:
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
