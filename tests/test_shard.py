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


def _rank_main(rank, world, port, ret):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ns, kinds, nrhs = batch(count=300, seed=5)
        parts = shard.partition(ns, kinds, nrhs, world)
        mine = parts[rank]
        # stand-in for the per-rank batched solve: info = id + 1 on odd ids
        info = [(i + 1) if i % 2 else 0 for i in mine]
        out = shard.gather_info(mine, info, len(ns), dist)
        ret[rank] = out
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_split_and_gather():
    world = 2
    port = 29500 + os.getpid() % 1000
    mgr = mp.get_context("spawn").Manager()
    ret = mgr.dict()
    mp.start_processes(_rank_main, args=(world, port, ret), nprocs=world, start_method="spawn",
                       join=True)
    expect = [(i + 1) if i % 2 else 0 for i in range(300)]
    assert ret[0] == expect and ret[1] == expect
