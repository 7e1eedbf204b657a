"""Replica and input shards over ranks (one process per GPU).

Replicas are independent (each has its own lattice and RNG stream), so a
swarm or a committor run splits across GPUs with no exchange on the data
path: every rank simulates its own shard, and the only collective steps are
the final gather of per-input results and, for timing, the maximum over ranks.
The functions take a ``torch.distributed``-like module (NCCL on GPUs, gloo for
host-side tests) or ``None`` for a single process.
"""
from __future__ import annotations

import numpy as np


def rank_and_world(dist):
    if dist is None or not dist.is_initialized():
        return 0, 1
    return dist.get_rank(), dist.get_world_size()


def shard_range(n, world, rank):
    """Contiguous, balanced shard of n items for `rank`: (start, count).  The
    first n % world ranks take one extra item."""
    if world <= 0 or not 0 <= rank < world or n < 0:
        raise ValueError(f"bad shard request n={n} world={world} rank={rank}")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, base + (1 if rank < extra else 0)


def rank_seed(seed, rank):
    """Seed of `rank`'s replica streams for a weak-scaling swarm (each rank
    runs its own replicas; rank 0 keeps the single-GPU seed)."""
    return int(seed) + 7919 * int(rank)


def _reduce(value, dist, op, device):
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(value, dist, device="cpu"):
    """max of a per-rank float (a step time: the job is as slow as its slowest rank)."""
    if rank_and_world(dist)[1] == 1:
        return float(value)
    return _reduce(value, dist, dist.ReduceOp.MAX, device)


def sum_over_ranks(value, dist, device="cpu"):
    """Sum of a per-rank float (attempts, grids processed)."""
    if rank_and_world(dist)[1] == 1:
        return float(value)
    return _reduce(value, dist, dist.ReduceOp.SUM, device)


def gather_shards(local, n_total, dist, device="cpu"):
    """Concatenate every rank's 1-D float64 shard, in rank order (shards as
    laid out by shard_range over n_total items), on every rank."""
    local = np.ascontiguousarray(local, np.float64).reshape(-1)
    rank, world = rank_and_world(dist)
    if world == 1:
        return local.copy()
    import torch
    counts = [shard_range(n_total, world, r)[1] for r in range(world)]
    if local.size != counts[rank]:
        raise ValueError(f"rank {rank} shard has {local.size} items, expected {counts[rank]}")
    width = max(counts) if counts else 0
    buf = torch.zeros(width, dtype=torch.float64, device=device)
    buf[:local.size] = torch.from_numpy(local).to(device)
    parts = [torch.zeros(width, dtype=torch.float64, device=device) for _ in range(world)]
    dist.all_gather(parts, buf)
    return np.concatenate([p[:c].cpu().numpy() for p, c in zip(parts, counts)])


def sharded_committor(inputs, shots, shoot, dist=None, device="cpu"):
    """pB of every input grid, the inputs split over the ranks.

    ``shoot(grids, shots) -> pB[len(grids)]`` runs one rank's shard (for
    example ``surrogate.shoot`` on that rank's GPU).  Returns the full pB
    array on every rank."""
    inputs = np.asarray(inputs)
    rank, world = rank_and_world(dist)
    start, count = shard_range(inputs.shape[0], world, rank)
    local = np.asarray(shoot(inputs[start:start + count], shots), np.float64) if count else \
        np.zeros(0, np.float64)
    return gather_shards(local, inputs.shape[0], dist, device)


__all__ = ["rank_and_world", "shard_range", "rank_seed", "max_over_ranks", "sum_over_ranks",
           "gather_shards", "sharded_committor"]
