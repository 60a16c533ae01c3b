"""Multi-GPU sharding: one process per GPU, instances split across ranks.

PDLP instances are independent, so a multi-GPU run partitions them -- by
instance, balanced by nonzeros for LPs of uneven sizes -- and every rank
solves its own share with no collective inside the iteration loop. The only
collectives are the max of the per-rank times and the gathering of small
per-rank summaries. A single LP is not split (replicas only): a row-block
split would need an all-gather of the primal and dual iterates on every
iteration.

Works with any torch.distributed backend (NCCL between GPUs, gloo on CPU).
"""
from __future__ import annotations

import numpy as np


def balanced_shards(weights, world: int) -> list[np.ndarray]:
    """Instance indices per rank: contiguous ranges whose weight sums (e.g.
    nonzeros) are as even as the instance granularity allows. Every instance
    is in exactly one shard; a rank may get none when there are fewer
    instances than ranks."""
    w = np.asarray(weights, dtype=np.float64)
    if world <= 0:
        raise ValueError("world must be positive")
    cum = np.concatenate([[0.0], np.cumsum(w)])
    total = cum[-1]
    bounds = [0]
    for r in range(1, world):
        bounds.append(int(np.searchsorted(cum, total * r / world, side="left")))
    bounds.append(len(w))
    bounds = np.maximum.accumulate(np.minimum(np.array(bounds), len(w)))
    return [np.arange(bounds[r], bounds[r + 1]) for r in range(world)]


def rank_seeds(rank: int, count: int, base: int = 100_000) -> list[int]:
    """Seeds of a rank's `count` instance batches, disjoint across ranks (and
    from the training seeds, which are below `base`)."""
    return [base * (rank + 1) + k for k in range(count)]


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of a per-rank value (a time) over all ranks; the value
    itself when torch.distributed is not initialised."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def weak_scaling_rate(per_rank_units: float, per_rank_seconds: float, device=None) -> float:
    """Whole-job throughput: the units all ranks processed over the slowest
    rank's time."""
    units = sum_over_ranks(per_rank_units, device)
    seconds = max_over_ranks(per_rank_seconds, device)
    return units / seconds if seconds > 0 else float("nan")


def gather_to_rank0(indices, records):
    """Per-instance records of every rank's shard, assembled in instance
    order on rank 0 (None on the other ranks). `indices` are the rank's
    instance indices, `records` one picklable summary per instance (status,
    objective, iterations -- small; solutions stay on their rank). Without
    torch.distributed the records are returned as they are."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return list(records)
    world = dist.get_world_size()
    mine = list(zip([int(i) for i in indices], records))
    parts = [None] * world if dist.get_rank() == 0 else None
    dist.gather_object(mine, parts, dst=0)
    if dist.get_rank() != 0:
        return None
    pairs = sorted((p for part in parts for p in part), key=lambda t: t[0])
    return [r for _, r in pairs]
