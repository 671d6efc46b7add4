"""Sharding of the batched path across ranks, on CPU with two gloo processes."""
import os

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from plapack_b200 import shard


def batch(count=2000, seed=3):
    rng = np.random.default_rng(seed)
    ns = np.round(np.exp(rng.uniform(np.log(8), np.log(512), count))).astype(int).tolist()
    kinds = [i % 2 for i in range(count)]
    nrhs = rng.integers(1, 5, count).tolist()
    return ns, kinds, nrhs


def test_partition_is_complete_disjoint_and_balanced():
    ns, kinds, nrhs = batch()
    for world in (1, 2, 3, 8):
        parts = shard.partition(ns, kinds, nrhs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(ns)))
        loads = [sum(shard.instance_flops(ns[i], kinds[i], nrhs[i]) for i in p) for p in parts]
        biggest = max(shard.instance_flops(n, k, r) for n, k, r in zip(ns, kinds, nrhs))
        assert max(loads) - min(loads) <= biggest


def _instance(seed, i, n, kind):
    """Instance i of the test batch: LU on uniform[-1, 1] (every 7th one with a
    zero column, so exactly singular) or Cholesky on G G'/n + I (every 5th one
    with a negative diagonal entry, so not SPD)."""
    rng = np.random.default_rng(seed * 100003 + i)
    if kind == 0:
        A = rng.uniform(-1, 1, (n, n))
        if i % 7 == 3:
            A[:, n // 2] = 0.0
    else:
        G = rng.standard_normal((n, n))
        A = G @ G.T / n + np.eye(n)
        if i % 5 == 1:
            A[n - 1, n - 1] = -1.0
    return np.asfortranarray(A)


def _oracle_info(restated, seed, i, n, kind):
    """The info word of one instance from the CPU oracle: LU (PLA_dlu,
    SOLVERS/LU/PLA_seq_lu.c:21-46) -> first exact zero pivot, 1-based;
    Cholesky (PLA_dchol, SOLVERS/Cholesky/PLA_Local_chol.c:103-143) -> the
    failing column, 1-based; 0 when the factorization succeeds."""
    A = _instance(seed, i, n, kind)
    if kind == 0:
        LU, _ = restated.lu_unblocked(A)
        z = np.nonzero(np.diagonal(LU) == 0.0)[0]
        return int(z[0]) + 1 if len(z) else 0
    _, info = restated.chol_blocked(A, 32)
    return int(info)


def _rank_main(rank, world, port, ret):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle.oracle import Restated
        restated = Restated()
        ns, kinds, nrhs = batch(count=80, seed=5)
        ns = [min(n, 96) for n in ns]              # keep the CPU solves short

        def solve_share(ids):
            return [_oracle_info(restated, 5, i, ns[i], kinds[i]) for i in ids]

        out = shard.solve_sharded(ns, kinds, nrhs, solve_share, rank, world, dist)
        ret[rank] = (out, shard.partition(ns, kinds, nrhs, world)[rank])
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_solve_their_shares_and_gather_info(restated):
    """Two gloo ranks each factor their flop-balanced share with the CPU oracle;
    the gathered info words equal a serial pass over all instances."""
    world = 2
    port = 29500 + os.getpid() % 1000
    mgr = mp.get_context("spawn").Manager()
    ret = mgr.dict()
    mp.start_processes(_rank_main, args=(world, port, ret), nprocs=world, start_method="spawn",
                       join=True)
    ns, kinds, nrhs = batch(count=80, seed=5)
    ns = [min(n, 96) for n in ns]
    expect = [_oracle_info(restated, 5, i, ns[i], kinds[i]) for i in range(80)]
    assert any(v != 0 for v in expect) and any(v == 0 for v in expect)
    assert ret[0][0] == expect and ret[1][0] == expect
    assert sorted(ret[0][1] + ret[1][1]) == list(range(80))
    assert ret[0][1] and ret[1][1]


def test_single_rank_needs_no_process_group(restated):
    ns, kinds, nrhs = batch(count=20, seed=6)
    ns = [min(n, 64) for n in ns]
    out = shard.solve_sharded(ns, kinds, nrhs,
                              lambda ids: [_oracle_info(restated, 6, i, ns[i], kinds[i])
                                           for i in ids], 0, 1)
    assert out == [_oracle_info(restated, 6, i, ns[i], kinds[i]) for i in range(20)]
