"""Host-side sharding of a batch of independent matrices across ranks.

A batched expm has no data-path exchange: every matrix is independent, so a
batch is partitioned across the ranks of a job (one process per GPU) and each
rank runs its shard through ``calaman_expm_batched_*`` on its own GPU. The
partition balances the algorithmic work of each matrix,
(pi_m + s) * 2 n^3 + (2/3) n^3 + 2 n^3 (pi_m = 2, 3, 4, 5, 6 for m = 3 .. 13),
with the longest-processing-time rule: matrices in decreasing cost, each to the
currently lightest rank (ties to the lower rank, so every rank computes the
same partition without communication).
"""
from __future__ import annotations

import heapq

_PI = {3: 2, 5: 3, 7: 4, 9: 5, 13: 6}


def expm_cost(n: int, m: int, s: int) -> float:
    """Algorithmic flops of one real expm of order n with plan (m, s)."""
    return (_PI[m] + s) * 2.0 * n ** 3 + (2.0 / 3.0) * n ** 3 + 2.0 * n ** 3


def partition(costs, world: int) -> list[list[int]]:
    """Indices of `costs` split into `world` shards of near-equal total cost.
    Deterministic: the same input gives every rank the same partition."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    shards: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(s) for s in shards]


def shard_of(costs, world: int, rank: int) -> list[int]:
    return partition(costs, world)[rank]
