"""Rank layout of the multi-GPU paths.

ERI sweep: shell quartets are independent, so N ranks (one process per GPU)
each run their own shard, drawn from a rank-specific seed, with no collective
on the data path.  The only communication is the timing: every rank's device
time is reduced with MAX so the reported throughput is that of the slowest
rank.

Fock build: the screened quartet candidates are enumerated in one order
fixed by the Schwarz-sorted shell pairs; rank r digests the candidates with
index r mod N into its own J/K, and one all-reduce (sum) of the n x n FP64
partial G per build gives every rank the full G (``fock_G_distributed``).
"""
from __future__ import annotations

import os

import numpy as np


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


# ------------------------------------------------------------ Fock build
def fock_G_distributed(ctx, P, tau: float = 1e-13, group=None):
    """G(P) of a Fock build split over the ranks of ``group`` (one GPU each):
    every rank digests its share of the screened quartets into a private
    n x n FP64 partial (lrb_fock_G_part_device), then one all-reduce (sum)
    of those n*n doubles gives every rank the full G.  P is this rank's
    device copy of the density (n x n float64)."""
    import torch
    import torch.distributed as dist
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    n = dist.get_world_size(group) if dist.is_initialized() else 1
    G = torch.empty_like(P)
    ctx.fock_G_part_device(P, G, tau, rank, n)
    if n > 1:
        dist.all_reduce(G, group=group)
    return G


def fock_candidates(Q, dmax: float, tau: float):
    """Host mirror of the device's candidate enumeration for the Fock build
    (k_cand_count / k_screen_sorted): shell pairs in descending Schwarz order
    (stable), and for each sorted position i the ket positions j <= i with
    Q_i Q_j 2 max|D| >= tau; candidate t = (sum of earlier counts) + j.
    Returns (t, bra pair, ket pair) arrays; rank r of N takes t = r mod N."""
    Q = np.asarray(Q, dtype=np.float64)
    order = np.argsort(-Q, kind="stable")
    Qs = Q[order]
    f = Qs * 2.0 * dmax
    cnt = np.zeros(len(Q), dtype=np.int64)
    pos = f > 0
    thr = np.where(pos, tau / np.where(pos, f, 1.0), np.inf)
    # first j in [0, i] with Qs[j] < thr (Qs is descending)
    first = np.searchsorted(-Qs, -thr, side="right")
    cnt[pos] = np.minimum(first[pos], np.arange(len(Q))[pos] + 1)
    off = np.concatenate([[0], np.cumsum(cnt)])
    i = np.repeat(np.arange(len(Q)), cnt)
    j = np.arange(off[-1]) - off[i]
    return np.arange(off[-1]), order[i], order[j]
