"""Multi-rank source sharding: every rank sweeps a contiguous share of the sources, then one
all-reduce sums the partial BC vectors.

Sources are independent in Brandes' algorithm (BC = 0.5 * sum_s delta_s), so the only exchange
of the multi-GPU path is that single reduction of n doubles.  Shares are contiguous in the index's
DFS-preorder source order so each rank's 32-source groups stay neighbours in the tree.
"""
from __future__ import annotations

import numpy as np


def shard_sources(order: np.ndarray, world: int, rank: int) -> np.ndarray:
    """Contiguous share `rank` of `world` of the source list `order` (as int32)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} of {world}")
    return np.ascontiguousarray(np.array_split(np.asarray(order), world)[rank], dtype=np.int32)


def all_reduce_bc(partial, group=None):
    """Sums the ranks' partial BC tensors in place (torch.distributed, any backend)."""
    import torch.distributed as dist

    dist.all_reduce(partial, op=dist.ReduceOp.SUM, group=group)
    return partial


def max_over_ranks(value: float, device=None, group=None) -> float:
    """Largest value of all ranks (timings are reported as the slowest rank)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
