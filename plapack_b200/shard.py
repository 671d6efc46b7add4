"""Splitting a batched factor-and-solve across GPUs (one process per GPU).

The instances of a batch are independent, so the batch shards by instance with
no data-path collective: every rank computes the same deterministic split
(longest-processing-time first, by the instances' flop counts), factors and
solves its share with one PLA_Batch_plan on its own GPU, and the only exchange
is a final gather of the per-instance info words.

    parts = partition(ns, kinds, nrhs, world)          # the same on every rank
    share = RankBatch(lib, MPI_DOUBLE, records, info)  # this rank's instances
    share.execute()
    info_all = gather_info(parts[rank], share.info(), count, dist)

The reference has no batched form; its only parallel layout is the 2-D mesh
of TEMPLATE/PLA_Init.c, which a batch of independent systems does not need.
"""
from __future__ import annotations

import ctypes
import heapq
from typing import Callable, Sequence


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
    """All ranks' info words, in instance order (the one collective).  Every
    rank must call it, in the same order relative to its other collectives."""
    if dist is None:
        out = [0] * count
        for i, v in zip(local_ids, local_info):
            out[i] = int(v)
        return out
    world = dist.get_world_size(group)
    gathered: list = [None] * world
    dist.all_gather_object(gathered, (list(map(int, local_ids)), list(map(int, local_info))),
                           group=group)
    out = [0] * count
    seen = 0
    for ids, infos in gathered:
        for i, v in zip(ids, infos):
            out[i] = v
        seen += len(ids)
    if seen != count:
        raise RuntimeError(f"gathered {seen} info words for {count} instances")
    return out


def solve_sharded(ns: Sequence[int], kinds: Sequence[int], nrhs: Sequence[int],
                  solve_share: Callable[[list[int]], Sequence[int]], rank: int, world: int,
                  dist=None, group=None) -> list[int]:
    """Partition the instances, solve this rank's share with
    ``solve_share(ids) -> info words`` and return every instance's info word.
    On a GPU ``solve_share`` runs one RankBatch; the CPU tests pass the
    oracle's per-instance factor-and-solve."""
    parts = partition(ns, kinds, nrhs, world)
    mine = parts[rank]
    info = list(solve_share(mine))
    if len(info) != len(mine):
        raise RuntimeError("solve_share returned the wrong number of info words")
    return gather_info(mine, info, len(ns), dist, group)


class RankBatch:
    """One rank's instances as one PLA_Batch_plan (persistent launch replayed
    from a CUDA graph).  `records` is a ctypes array of PLA_Batch_instance
    (pla.BatchInstance) for this rank's instances only; `info_ptr` a device
    int array of the same length."""

    def __init__(self, lib, datatype: int, records, info_ptr: int, autotune: int = 1):
        from . import pla
        self.lib = lib
        self.count = len(records)
        self.plan = ctypes.c_void_p()
        self.info_ptr = int(info_ptr)
        if self.count:
            pla.check(lib.PLA_Batch_plan_create(datatype, self.count, records,
                                                ctypes.c_void_p(self.info_ptr), autotune,
                                                ctypes.byref(self.plan)),
                      "PLA_Batch_plan_create")

    def execute(self) -> None:
        from . import pla
        if self.count:
            pla.check(self.lib.PLA_Batch_plan_execute(self.plan), "PLA_Batch_plan_execute")

    def free(self) -> None:
        if self.plan.value:
            self.lib.PLA_Batch_plan_free(ctypes.byref(self.plan))
