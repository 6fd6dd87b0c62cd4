"""Multi-GPU plumbing for replica runs (one process per GPU).

The fused path exchanges no data between GPUs: a multi-GPU run is N independent
replicas (or N disjoint shards of independent batch jobs), and the only collective
is the max over ranks of the measured step time. The reference's MPI slab halo
exchange is not part of this path.
"""
from __future__ import annotations

from typing import List, Sequence, TypeVar

import torch

T = TypeVar("T")


def shard(items: Sequence[T], rank: int, world: int) -> List[T]:
    """Rank ``rank``'s share of independent jobs (round-robin, sizes within one)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} of {world}")
    return list(items[rank::world])


def max_over_ranks(x: float, world: int) -> float:
    """Max of a host scalar over the default process group (NCCL or gloo)."""
    if world == 1:
        return float(x)
    import torch.distributed as dist
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
