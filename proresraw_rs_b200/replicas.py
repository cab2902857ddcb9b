"""Multi-GPU replicas: frames are independent, so each rank (one process per
GPU) decodes and develops its own share of the frames and no collective is on
the data path. The only exchanges are host-side bookkeeping after the timed
region: the slowest rank's time and the total frame count.

`shard` deals a list of frames round-robin; `reduce_max` / `reduce_sum` run
over torch.distributed (NCCL on GPUs, gloo on CPU) when a process group is
up, and return the local value otherwise.
"""

from __future__ import annotations

import os
from typing import List, Sequence, Tuple, TypeVar

T = TypeVar("T")


def world() -> Tuple[int, int, int]:
    """(world size, rank, local rank) from the launcher's environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard(items: Sequence[T], rank: int, world_size: int) -> List[T]:
    """This rank's frames: every world_size-th from position rank."""
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError("rank out of range")
    return list(items[rank::world_size])


def _reduce(value: float, op: str) -> float:
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    backend = dist.get_backend()
    device = "cuda" if backend == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def reduce_max(value: float) -> float:
    """The largest value over the ranks (the slowest rank's time)."""
    return _reduce(value, "max")


def reduce_sum(value: float) -> float:
    """The sum over the ranks (frames processed by all ranks)."""
    return _reduce(value, "sum")
