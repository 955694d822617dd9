"""Split a sweep's independent cases across ranks (one process per GPU).

The cases of a `.krk` Sweep never exchange data, so each rank runs its own
subset in its own persistent launch and no collective touches the data
path; only the per-rank timings are combined (max over ranks).  Cases are
assigned longest-processing-time first on their node count N^2, which keeps
the ranks' node totals within one large case of each other.
"""
from __future__ import annotations

import heapq

import numpy as np


def shard_cases(N, world: int, rank: int) -> np.ndarray:
    """Indices of the cases (sizes N) that `rank` of `world` runs."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} of world {world}")
    N = np.asarray(N, dtype=np.int64)
    work = N * N
    order = np.argsort(-work, kind="stable")
    heap = [(0, r) for r in range(world)]
    owner = np.empty(len(N), dtype=np.int64)
    for c in order:
        load, r = heapq.heappop(heap)
        owner[c] = r
        heapq.heappush(heap, (load + int(work[c]), r))
    return np.flatnonzero(owner == rank)


def shard_loads(N, world: int) -> list[int]:
    """Node total per rank under shard_cases."""
    N = np.asarray(N, dtype=np.int64)
    return [int(np.sum(N[shard_cases(N, world, r)] ** 2)) for r in range(world)]
