"""Replica plumbing for several GPUs (one process per GPU).

Queries are independent, so a multi-GPU run is a set of replicas: every rank
uploads the same timetable, runs its own shard of the query stream and
reports its times; nothing is exchanged on the data path.  Whole-job
throughput is the queries of all ranks divided by the slowest rank's time.
"""
from __future__ import annotations

from typing import List, Sequence


def query_seed(base_seed: int, rank: int) -> int:
    """Seed of rank's query shard: disjoint, reproducible streams."""
    return base_seed + 7919 * rank


def shard(n_total: int, rank: int, world: int) -> range:
    """Contiguous share of n_total items for rank (sizes differ by <= 1)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of {world}")
    base, extra = divmod(n_total, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def max_over_ranks(values: Sequence[float], group=None, device=None) -> List[float]:
    """Element-wise maximum of per-rank values over the process group (the
    timing rule for multi-GPU numbers); identity without a group."""
    if group is None:
        return list(values)
    import torch
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    group.all_reduce(t, op=group.ReduceOp.MAX)
    return t.tolist()


def from_rank0(values: Sequence[int], group=None, device=None) -> List[int]:
    """Rank 0's integers on every rank (a launch shape tuned once, so that
    every replica times the same kernels); identity without a group."""
    if group is None:
        return [int(v) for v in values]
    import torch
    t = torch.tensor([int(v) for v in values], dtype=torch.int64, device=device)
    group.broadcast(t, src=0)
    return [int(v) for v in t.tolist()]


def whole_job_throughput(units_per_rank: int, world: int, slowest_seconds: float) -> float:
    """Units all ranks processed / the slowest rank's time."""
    return units_per_rank * world / slowest_seconds
