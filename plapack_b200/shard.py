"""Splitting a batched factor-and-solve across GPUs (one process per GPU).

The instances of a batch are independent, so the batch shards by instance with
no data-path collective: every rank computes the same deterministic split
(longest-processing-time first, by the instances' flop counts), factors and
solves its share with one PLA_Batch_plan on its own GPU, and the only exchange
is a final gather of the per-instance info words.
"""
from __future__ import annotations

import heapq
from typing import Sequence


def instance_flops(n: int, kind: int, nrhs: int) -> float:
    """LU 2/3 n^3, Cholesky 1/3 n^3 (TEST/test_lu.c:144, TEST/test_chol.c:140),
    plus 2 n^2 per right-hand side for the two triangular solves."""
    return (2.0 / 3.0 if kind == 0 else 1.0 / 3.0) * n ** 3 + 2.0 * n * n * nrhs


def partition(ns: Sequence[int], kinds: Sequence[int], nrhs: Sequence[int],
              world: int) -> list[list[int]]:
    """Instance ids per rank, balanced by flops (greedy LPT, ties by id)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    work = [instance_flops(n, k, r) for n, k, r in zip(ns, kinds, nrhs)]
    order = sorted(range(len(work)), key=lambda i: (-work[i], i))
    heap = [(0.0, rank) for rank in range(world)]
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, rank = heapq.heappop(heap)
        parts[rank].append(i)
        heapq.heappush(heap, (load + work[i], rank))
    for p in parts:
        p.sort()
    return parts


def gather_info(local_ids: Sequence[int], local_info: Sequence[int], count: int, dist,
                group=None) -> list[int]:
    """All ranks' info words, in instance order (the one collective)."""
    world = dist.get_world_size(group)
    gathered: list = [None] * world
    dist.all_gather_object(gathered, (list(local_ids), list(local_info)), group=group)
    out = [0] * count
    for ids, infos in gathered:
        for i, v in zip(ids, infos):
            out[i] = v
    return out
