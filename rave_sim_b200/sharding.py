"""Instance sharding across GPUs (one process per GPU).

Independent sources (energies x source points, each with all its phase steps)
are assigned to ranks by longest-processing-time-first on the cost
N_j * split_steps_j, so uneven field sizes balance; a source never spans
ranks (its phase steps share the in-HBM snapshot). The FP64 detector
accumulators are then summed with one all-reduce.
"""

from __future__ import annotations

import heapq
from typing import Sequence


def shard_sources(costs: Sequence[float], world: int) -> list[list[int]]:
    """Indices of the sources run by each rank (LPT greedy; deterministic:
    ties broken by source index, then by rank)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world)]
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(s) for s in out]


def reduce_detector(acc, group=None):
    """Sum the FP64 detector accumulators of all ranks in place."""
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(acc, group=group)
    return acc
