"""Replica sharding of independent JW-step work over ranks (one process per GPU).

The JW path has no exchange step: right-hand sides are independent, and so are
the harmonic degrees of an uneven timestep, while the bands are a few KB per
size and are replicated.  Multi-GPU is therefore sharding plus timing
aggregation: each rank solves its shard with no data-path collective, and
the only collectives are the barrier and the max-over-ranks of the timed
region (NCCL on GPUs, gloo in the CPU tests).
"""
from __future__ import annotations

import heapq
from typing import List, Sequence, Tuple


def shard(total: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous balanced split of `total` systems: (start, count) of `rank`;
    counts differ by at most one, lower ranks take the remainder."""
    if world < 1 or not 0 <= rank < world or total < 0:
        raise ValueError("bad shard arguments")
    base, extra = divmod(total, world)
    start = rank * base + min(rank, extra)
    return start, base + (1 if rank < extra else 0)


def shard_weighted(weights: Sequence[float], world: int) -> List[List[int]]:
    """Assign items (e.g. harmonic degrees, weight (2l+1) * N_l) to ranks by
    longest-processing-time-first: heaviest item to the least loaded rank.
    Returns the item indices of every rank, each list in ascending order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0.0, r) for r in range(world)]
    out: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(weights)), key=lambda k: -weights[k]):
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(weights[i]), r))
    return [sorted(v) for v in out]


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank float over the default process group (the job's time
    is its slowest rank's); the value itself when no group is initialised."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(units_per_rank: float, ms_max: float, world: int) -> float:
    """Whole-job units per second under weak scaling: every rank processed
    `units_per_rank` units, the job took the slowest rank's `ms_max`."""
    return world * units_per_rank / (ms_max * 1e-3)
