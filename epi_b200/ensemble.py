"""Host-side sharding of an ensemble of independent tissues across ranks.

Tissues never interact, so a multi-GPU run is weak-scaled sharding with no
collective on the data path: each rank uploads its shard into one context and
steps it; only timing and the final gather cross ranks.
"""
from __future__ import annotations

import heapq
from typing import Any, List, Optional, Sequence

import numpy as np


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


def split_by_tissue(arrays: Sequence[np.ndarray], sizes: Sequence[int]) -> List[tuple]:
    """Per-tissue slices of concatenated per-particle arrays (a context's
    positions are the tissues' particles back to back, in upload order)."""
    cut = np.concatenate([[0], np.cumsum(np.asarray(sizes, np.int64))])
    return [tuple(a[cut[k]:cut[k + 1]] for a in arrays) for k in range(len(sizes))]


def gather_results(mine: Sequence[int], results: Sequence[Any], dist,
                   dst: int = 0) -> Optional[List[Any]]:
    """Collects every rank's per-tissue results on rank `dst` and returns them
    in job order (result k belongs to tissue k of the whole job); other ranks
    return None. `mine` are this rank's tissue ids (its shard from
    shard_tissues), `results` its results in the same order -- positions from
    split_by_tissue, an adjoint's (loss, gradient) per tissue, ... Every rank
    must call it (it is a collective); results travel as pickled objects, off
    the timed path."""
    if len(mine) != len(results):
        raise ValueError("one result per tissue of the shard")
    rank, world = dist.get_rank(), dist.get_world_size()
    parts = [None] * world if rank == dst else None
    dist.gather_object((list(mine), list(results)), parts, dst=dst)
    if rank != dst:
        return None
    total = sum(len(ids) for ids, _ in parts)
    out: List[Any] = [None] * total
    for ids, res in parts:
        for i, r in zip(ids, res):
            if out[i] is not None:
                raise ValueError(f"tissue {i} returned by two ranks")
            out[i] = r
    if any(r is None for r in out):
        raise ValueError("a tissue of the job returned by no rank")
    return out
