"""Host-side helpers of the batched form: cost model and a size-balanced
partition of a batch over ranks (one process per GPU; independent matrices
need no collective -- every rank solves its shard with
gjx_hypJacL2_batched and writes its own outputs)."""

from __future__ import annotations

import heapq

import numpy as np


def cost(nrow: int, ncol: int, full: bool = True) -> float:
    """Work of one sweep of an nrow x ncol decomposition (block pairs x rows,
    w = 32): P_sweep (4 M w^2 + [V] 2 N w^2), P_sweep = n1 (n1 - 1) / 2."""
    n1 = ncol // 16
    p = n1 * (n1 - 1) / 2.0
    return p * (4.0 * nrow * 1024.0 + (2.0 * ncol * 1024.0 if full else 0.0))


def partition(nrows, ncols, world: int, full: bool = True):
    """Longest-processing-time-first assignment of matrices to `world` ranks:
    returns a list of index arrays (each sorted), deterministic for equal
    inputs on every rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    c = np.array([cost(int(m), int(n), full) for m, n in zip(nrows, ncols)])
    order = sorted(range(len(c)), key=lambda i: (-c[i], i))
    heap = [(0.0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + c[i], r))
    return [np.array(sorted(o), dtype=np.int64) for o in out]


def imbalance(parts, nrows, ncols, full: bool = True) -> float:
    """max load / mean load of a partition."""
    loads = [sum(cost(int(nrows[i]), int(ncols[i]), full) for i in p) for p in parts]
    return max(loads) / (sum(loads) / len(loads))
