"""Multi-GPU replicas: every rank owns whole, independent problems.

The path shards by problem (batched and served workloads are independent
solves), so ranks exchange nothing on the data path: problems are assigned
greedily by cell count (largest first, to the least-loaded rank), each rank
seeds its own synthetic inputs, and only the timing is reduced (max over
ranks) for the report.
"""
from __future__ import annotations

import heapq

import numpy as np


def assign_greedy(cells, world: int) -> list[list[int]]:
    """Problem indices per rank; largest problems first to the least-loaded rank
    (ties by rank id), so every rank computes the same assignment."""
    order = sorted(range(len(cells)), key=lambda k: (-int(cells[k]), k))
    heap = [(0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for k in order:
        load, r = heapq.heappop(heap)
        out[r].append(k)
        heapq.heappush(heap, (load + int(cells[k]), r))
    return [sorted(v) for v in out]


def rank_seed(base: int, rank: int) -> int:
    return int(base) + 1000 * int(rank)


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank float over the process group (identity without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def imbalance(cells, assignment) -> float:
    loads = np.array([sum(int(cells[k]) for k in a) for a in assignment], dtype=float)
    return float(loads.max() / loads.mean()) if loads.mean() > 0 else 1.0
