"""Batched factor-and-solve on the B200 through the C ABI.

Uneven orders (log-uniform in [1, 300]), LU and Cholesky mixed, 1-4
right-hand sides, FP64 and FP32: every instance's pivots equal the CPU
oracle's unblocked LU (PLA_dlu order), factors and solutions agree within
rounding, info reports exact zero pivots and non-positive Cholesky pivots,
and the per-instance launch loop gives the same solutions.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from plapack_b200 import pla
    s = pla.Session()
    yield s, torch, pla
    s.close()


def make_batch(torch, pla, count, dtype, seed, nmax=300):
    rng = np.random.default_rng(seed)
    ns = np.round(np.exp(rng.uniform(np.log(1), np.log(nmax), count))).astype(int)
    host, dev = [], []
    arr = (pla.BatchInstance * count)()
    tdt = torch.float64 if dtype == np.float64 else torch.float32
    for k, n in enumerate(ns):
        kind = k % 2
        nrhs = int(rng.integers(1, 5))
        if kind == 0:
            A = rng.uniform(-1, 1, (n, n))
        else:
            G = rng.standard_normal((n, n))
            A = G @ G.T / max(n, 1) + np.eye(n)
        B = rng.standard_normal((n, nrhs))
        A = np.asfortranarray(A.astype(dtype))
        B = np.asfortranarray(B.astype(dtype))
        tA = torch.from_numpy(A.T.copy()).to("cuda", tdt)   # row-major A' = column-major A
        tB = torch.from_numpy(B.T.copy()).to("cuda", tdt)
        tp = torch.zeros(max(n, 1), dtype=torch.int32, device="cuda")
        arr[k].n, arr[k].nrhs, arr[k].kind = int(n), nrhs, kind
        arr[k].A, arr[k].B = tA.data_ptr(), tB.data_ptr()
        arr[k].pivots = ctypes.cast(tp.data_ptr(), ctypes.POINTER(ctypes.c_int))
        host.append((A, B, kind))
        dev.append((tA, tB, tp))
    return arr, host, dev


def check_results(host, dev, info, restated, dtype):
    eps = np.finfo(dtype).eps
    for k, ((A, B, kind), (tA, tB, tp)) in enumerate(zip(host, dev)):
        n = A.shape[0]
        F = tA.cpu().numpy().T.astype(np.float64)
        X = tB.cpu().numpy().T.astype(np.float64)
        assert info[k] == 0, (k, n, kind, info[k])
        if n == 0:
            continue
        if kind == 0:
            LUo, pivo = restated.lu_unblocked(A)
            assert np.array_equal(tp.cpu().numpy()[:n], pivo), (k, n)
            assert np.abs(F - LUo).max() <= 8 * n * eps * max(1.0, np.abs(LUo).max()), (k, n)
        else:
            L = np.linalg.cholesky(A.astype(np.float64))
            assert np.abs(np.tril(F) - L).max() <= 8 * n * eps * max(1.0, np.abs(L).max()), (k, n)
        Xr = np.linalg.solve(A.astype(np.float64), B.astype(np.float64))
        cond = np.linalg.cond(A.astype(np.float64))
        assert np.abs(X - Xr).max() <= 16 * n * eps * cond * max(1.0, np.abs(Xr).max()), (k, n)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("autotune", [0, 1])
def test_batched_matches_oracle(env, restated, dtype, autotune):
    s, torch, pla = env
    count = 160
    arr, host, dev = make_batch(torch, pla, count, dtype, 3 + autotune)
    info = torch.full((count,), -1, dtype=torch.int32, device="cuda")
    dt = pla.MPI_DOUBLE if dtype == np.float64 else pla.MPI_FLOAT
    plan = ctypes.c_void_p()
    pla.check(s.lib.PLA_Batch_plan_create(dt, count, arr, info.data_ptr(), autotune,
                                          ctypes.byref(plan)), "plan_create")
    pla.check(s.lib.PLA_Batch_plan_execute(plan), "plan_execute")
    torch.cuda.synchronize()
    check_results(host, dev, info.cpu().numpy(), restated, dtype)
    s.lib.PLA_Batch_plan_free(ctypes.byref(plan))


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_batched_large_orders_blocked(env, restated, dtype):
    """Orders up to 512 go through the blocked global-memory form; its pivots
    and factors are those of the column algorithm (the oracle's PLA_dlu)."""
    s, torch, pla = env
    count = 40
    arr, host, dev = make_batch(torch, pla, count, dtype, 17, nmax=512)
    info = torch.full((count,), -1, dtype=torch.int32, device="cuda")
    dt = pla.MPI_DOUBLE if dtype == np.float64 else pla.MPI_FLOAT
    pla.check(s.lib.PLA_Batched_factor_solve(dt, count, arr, info.data_ptr()), "batched")
    torch.cuda.synchronize()
    check_results(host, dev, info.cpu().numpy(), restated, dtype)


def test_batched_reports_failures(env):
    s, torch, pla = env
    arr = (pla.BatchInstance * 3)()
    A0 = np.eye(40)
    A0[:, 17] = 0.0                     # exact zero pivot at column 18
    A1 = np.eye(200)
    A1[150, 150] = -2.0                 # not positive definite at column 151
    A2 = np.eye(20)
    A2[3, 3] = 0.0                      # Cholesky fails at column 4 (warp path)
    keep = []
    for k, (A, kind) in enumerate([(A0, 0), (A1, 1), (A2, 1)]):
        n = A.shape[0]
        tA = torch.from_numpy(A.T.copy()).cuda()
        tB = torch.ones(1, n, dtype=torch.float64, device="cuda")
        tp = torch.zeros(n, dtype=torch.int32, device="cuda")
        arr[k].n, arr[k].nrhs, arr[k].kind = n, 1, kind
        arr[k].A, arr[k].B = tA.data_ptr(), tB.data_ptr()
        arr[k].pivots = ctypes.cast(tp.data_ptr(), ctypes.POINTER(ctypes.c_int))
        keep.append((tA, tB, tp))
    info = torch.full((3,), -1, dtype=torch.int32, device="cuda")
    pla.check(s.lib.PLA_Batched_factor_solve(pla.MPI_DOUBLE, 3, arr, info.data_ptr()), "batched")
    assert info.cpu().tolist() == [18, 151, 4]


def test_loop_baseline_same_solutions(env, restated):
    s, torch, pla = env
    count = 24
    arr, host, dev = make_batch(torch, pla, count, np.float64, 9, nmax=200)
    pla.check(s.lib.PLA_Batched_factor_solve_loop(pla.MPI_DOUBLE, count, arr), "loop")
    torch.cuda.synchronize()
    check_results(host, dev, np.zeros(count, dtype=np.int32), restated, np.float64)
