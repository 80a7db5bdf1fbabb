"""Host-side sharding of an ensemble of independent tissues across ranks.

Tissues never interact, so a multi-GPU run is weak-scaled sharding with no
collective on the data path: each rank uploads its shard into one context and
steps it; only timing and the final gather cross ranks.
"""
from __future__ import annotations

import heapq
from typing import List, Sequence


def shard_tissues(sizes: Sequence[int], world: int) -> List[List[int]]:
    """Longest-processing-time greedy: tissues by size, largest first, each to
    the currently lightest rank (ties -> lowest rank). Deterministic. Each
    shard is returned in ascending tissue order."""
    if world <= 0:
        raise ValueError("world must be positive")
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i))
    heap = [(0, r) for r in range(world)]
    heapq.heapify(heap)
    shards: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + int(sizes[i]), r))
    return [sorted(s) for s in shards]


def imbalance(sizes: Sequence[int], shards: Sequence[Sequence[int]]) -> float:
    """max shard load / mean shard load (1.0 = perfect balance)."""
    loads = [sum(int(sizes[i]) for i in s) for s in shards]
    mean = sum(loads) / max(len(loads), 1)
    return max(loads) / mean if mean > 0 else 1.0
