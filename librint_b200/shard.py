"""Rank layout of the multi-GPU ERI sweep.

Shell quartets are independent, so N ranks (one process per GPU) each run
their own shard, drawn from a rank-specific seed, with no collective on the
data path.  The only communication is the timing: every rank's device time
is reduced with MAX so the reported throughput is that of the slowest rank.
"""
from __future__ import annotations

import os


def world_info():
    """(world size, rank, local rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard_seed(base_seed: int, rank: int) -> int:
    """Seed of a rank's quartet shard (disjoint random streams per rank)."""
    return base_seed + 1000 * rank


def max_over_ranks(x: float, device=None) -> float:
    """Maximum of x over all ranks (x itself without a process group).
    ``device`` is where the reduction tensor lives: a CUDA device for NCCL,
    None (CPU) for gloo."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
