"""Distribution of independent scenarios over ranks (one process per GPU).

Scenarios of a steady ensemble never exchange data, so the multi-GPU path has no
data-path collective: each rank runs its own share in one batched handle and the
ranks meet only to agree on the timing (max over ranks) and to gather per-scenario
statistics.  Shares are balanced by cell count with the longest-processing-time
rule (largest scenario first onto the least-loaded rank), which every rank computes
identically from the same sizes.
"""
from __future__ import annotations

import heapq

import numpy as np


def lpt_shards(sizes, world: int) -> list[list[int]]:
    """Indices of the scenarios each rank runs; ties go to the lower rank, and each
    share keeps the ensemble's order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0, r) for r in range(world)]
    heapq.heapify(heap)
    shares = [[] for _ in range(world)]
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i))
    for i in order:
        load, r = heapq.heappop(heap)
        shares[r].append(i)
        heapq.heappush(heap, (load + int(sizes[i]), r))
    return [sorted(s) for s in shares]


def imbalance(sizes, shares) -> float:
    """max share / mean share of the cell counts (1.0 = perfect balance)."""
    loads = np.array([sum(int(sizes[i]) for i in s) for s in shares], dtype=np.float64)
    return float(loads.max() / max(loads.mean(), 1e-30))


def combine(local: dict, dist=None) -> dict:
    """Whole-job figures from every rank's {"cell_stages", "device_ms", "scenarios",
    "converged"}: cell-stages and counts add up, the time is the slowest rank's."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return dict(local)
    gathered = [None] * dist.get_world_size()
    dist.all_gather_object(gathered, local)
    return {
        "cell_stages": float(sum(g["cell_stages"] for g in gathered)),
        "device_ms": float(max(g["device_ms"] for g in gathered)),
        "scenarios": int(sum(g["scenarios"] for g in gathered)),
        "converged": int(sum(g["converged"] for g in gathered)),
        "per_rank_ms": [float(g["device_ms"]) for g in gathered],
    }
