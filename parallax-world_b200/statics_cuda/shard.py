"""Splitting one batch of pieces across GPUs (one process per GPU).

Pieces are independent (each has its own hierarchy and its own conjugate gradients), so
a batch shards with no exchange on the data path: each rank solves its share with one
batched solve, and only the per-piece statistics meet at the end. The reference solves
one structure per `motions` call on one host (statics/src/bodies.rs:429, threads only
inside it, bodies.rs:51-69); this split is the multi-GPU form of its many calls.

The share is chosen by longest processing time first, with a piece's unknowns (6 per
free face node) as its weight: pieces in decreasing weight, each given to the rank whose
load is least so far (the lowest rank on ties). Its largest load is at most 4/3 of the
best possible split, and never more than the mean load plus the heaviest piece.
"""
from __future__ import annotations

import heapq


def lpt_split(weights, ranks: int) -> list[list[int]]:
    """Indices of `weights` for each of `ranks` ranks (each list in increasing order)."""
    if ranks < 1:
        raise ValueError("ranks must be at least 1")
    order = sorted(range(len(weights)), key=lambda i: (-weights[i], i))
    heap = [(0, r) for r in range(ranks)]  # (load, rank)
    share: list[list[int]] = [[] for _ in range(ranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        share[r].append(i)
        heapq.heappush(heap, (load + weights[i], r))
    return [sorted(s) for s in share]


def loads(weights, share) -> list:
    """Each rank's total weight under a split."""
    return [sum(weights[i] for i in s) for s in share]
