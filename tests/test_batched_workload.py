"""The batched benchmark's instance mix, generated on the CPU.

20,000 instances in the benchmark; 2,000 here: orders log-uniform in [8, 512],
even instances LU on uniform[-1, 1] matrices and odd ones Cholesky on
G G'/n + I, 1 to 4 right-hand sides, every instance's pointers inside its
order's tensors, and the flop count the benchmark reports.
"""
import ctypes
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_batched_instance_mix():
    torch = pytest.importorskip("torch")
    from plapack_b200 import pla
    from plapack_b200.workloads import batched_workload
    count = 2000
    arr, groups, piv, flops, ids = batched_workload(torch, pla, torch.device("cpu"),
                                                    torch.float64, count, 3)
    assert ids.tolist() == list(range(count))
    ns = np.array([arr[k].n for k in range(count)])
    assert ns.min() >= 8 and ns.max() <= 512
    assert 40 < np.median(ns) < 100                # log-uniform: median near 64
    assert [arr[k].kind for k in range(8)] == [0, 1] * 4
    nrhs = np.array([arr[k].nrhs for k in range(count)])
    assert set(nrhs.tolist()) == {1, 2, 3, 4}
    expect = sum((2.0 / 3.0 if arr[k].kind == 0 else 1.0 / 3.0) * arr[k].n ** 3
                 + 2.0 * arr[k].n ** 2 * arr[k].nrhs for k in range(count))
    assert flops == pytest.approx(expect)
    assert piv.numel() == ns.sum()
    for g in groups:
        n, A = g["n"], g["A"]
        lo, hi = A.data_ptr(), A.data_ptr() + A.numel() * 8
        for j, k in enumerate(g["order"]):
            assert arr[k].n == n and lo <= arr[k].A < hi
            if k % 25:
                continue                            # spectra on a sample of instances
            M = A[j].numpy()
            if arr[k].kind == 1:
                assert np.allclose(M, M.T) and np.linalg.eigvalsh(M).min() >= 1.0 - 1e-9
            else:
                assert np.abs(M).max() <= 1.0
        assert torch.equal(g["A0"], A) and torch.equal(g["B0"], g["B"])


def test_rank_subset_builds_the_same_instances():
    """A rank that builds only its share (select=...) gets bitwise the matrices
    and right-hand sides the full build gives those instances."""
    torch = pytest.importorskip("torch")
    from plapack_b200 import pla, shard
    from plapack_b200.workloads import batched_orders, batched_workload
    count = 600
    ns, nrhs, kinds = batched_orders(count, 3)
    full, gfull, _, ffull, _ = batched_workload(torch, pla, torch.device("cpu"), torch.float64,
                                                count, 3)
    parts = shard.partition(ns.tolist(), kinds.tolist(), nrhs.tolist(), 3)
    flops = 0.0
    for part in parts:
        sub, gsub, _, fsub, ids = batched_workload(torch, pla, torch.device("cpu"),
                                                   torch.float64, count, 3, select=part)
        flops += fsub
        assert ids.tolist() == part
        for q, k in enumerate(ids):
            n = sub[q].n
            assert (n, sub[q].nrhs, sub[q].kind) == (full[k].n, full[k].nrhs, full[k].kind)
            a = np.ctypeslib.as_array(ctypes.cast(sub[q].A, ctypes.POINTER(ctypes.c_double)),
                                      (n * n,))
            b = np.ctypeslib.as_array(ctypes.cast(full[k].A, ctypes.POINTER(ctypes.c_double)),
                                      (n * n,))
            assert np.array_equal(a, b)
    assert flops == pytest.approx(ffull)
