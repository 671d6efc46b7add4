"""LINPACK-style LU, the LINPACK driver's solve sequence, and the BLAS1 calls it uses.

- PLA_LU_linpack (SOLVERS/LINPACK/PLA_LU_linpack.c:13-208) is the blocked LU
  whose row interchanges skip the columns left of each panel (:145 applies
  them to A_BR only).  Against the oracle's restatement (itself pinned bit
  for bit to the compiled reference in test_oracle.py): pivots equal, factors
  within a rounding tolerance, over square, rectangular and augmented shapes,
  with and without the lookahead panel.
- SOLVERS/LINPACK/driver.c:100-150: factor the augmented [A b] with PLA_LU,
  solve U x = y with PLA_Trsv on the n x n view, then PLA_Axpy(-1, x_true,
  x) and PLA_Nrm2.  The same sequence with PLA_LU_linpack gives the same U
  and the same last column, so the same solution.
- PLA_Axpy (BLAS1/PLA_Axpy.c:13), PLA_Nrm2 (BLAS1/PLA_Nrm2.c:13; scaled as
  dnrm2: no overflow at 1e200, no underflow at 1e-200, NaN propagates) and
  PLA_Shift (UTIL/PLA_Shift.c:15, TEST/test_chol.c:127's diagonal shift)
  against numpy.
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    from plapack_b200 import pla
    s = pla.Session(nb_distr=64, nb_alg=64)
    yield s, pla, orc.Restated()
    s.close()


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("m,n,nb", [(1000, 1000, 64), (2100, 2101, 128), (600, 450, 64),
                                    (450, 600, 32)])
def test_lu_linpack_matches_oracle(env, dt, m, n, nb):
    s, pla, oracle = env
    rng = np.random.default_rng(m + n)
    A = rng.uniform(-1, 1, (m, n)).astype(dt)
    a = s.matrix(m, n, dt)
    piv = s.mvector(min(m, n), 1, np.int32)
    s.put(a, A)
    pla.check(s.lib.PLA_LU_linpack_right(nb, a, piv), "PLA_LU_linpack_right")
    LU = s.get(a)
    p = s.get(piv)[:, 0]
    ref, ref_piv = oracle.lu_linpack(A, nb)
    assert np.array_equal(p, ref_piv)
    eps = np.finfo(dt).eps
    tol = 4 * max(m, n) * eps * max(1.0, np.abs(ref).max())
    assert np.abs(LU.astype(np.float64) - ref).max() <= tol
    # the standard LU: same pivots and U, L rows in a different order
    std, std_piv = oracle.lu_blocked(A, nb)
    assert np.array_equal(p, std_piv)
    k = min(m, n)
    assert np.abs(np.triu(LU[:k]) - np.triu(std[:k])).max() <= tol
    s.free(a, piv)


def test_lu_linpack_reads_nb_alg_from_the_environment(env):
    s, pla, oracle = env
    n = 700
    A = np.random.default_rng(3).standard_normal((n, n))
    a = s.matrix(n, n)
    piv = s.mvector(n, 1, np.int32)
    s.put(a, A)
    s.set_nb_alg(96)
    try:
        pla.check(s.lib.PLA_LU_linpack(a, piv), "PLA_LU_linpack")
    finally:
        s.set_nb_alg(64)
    ref, ref_piv = oracle.lu_linpack(A, 96)
    assert np.array_equal(s.get(piv)[:, 0], ref_piv)
    assert np.abs(s.get(a) - ref).max() <= 4 * n * np.finfo(float).eps * np.abs(ref).max()
    s.free(a, piv)


@pytest.mark.parametrize("linpack", [False, True])
def test_linpack_driver_sequence(env, linpack):
    s, pla, _ = env
    lib = s.lib
    n = 1500
    rng = np.random.default_rng(9)
    A = rng.uniform(-1, 1, (n, n))
    x_true = rng.uniform(-1, 1, n)
    b = A @ x_true
    a_app = s.matrix(n, n + 1)                        # A with b appended (driver.c:100-102)
    piv = s.mvector(n, 1, np.int32)
    x = s.mvector(n)
    bvec = s.mvector(n)
    bnorm = s.scalar(0.0)
    minus_one = s.scalar(-1.0)
    s.put(a_app, np.hstack([A, b[:, None]]))
    s.put(x, x_true)
    a_view, rhs = ctypes.c_void_p(), ctypes.c_void_p()
    pla.check(lib.PLA_Obj_vert_split_2(a_app, -1, ctypes.byref(a_view), ctypes.byref(rhs)), "split")
    factor = lib.PLA_LU_linpack if linpack else lib.PLA_LU
    pla.check(factor(a_app, piv), "factor")
    pla.check(lib.PLA_Copy(rhs, bvec), "PLA_Copy")
    pla.check(lib.PLA_Trsv(pla.PLA_UPPER_TRIANGULAR, pla.PLA_NO_TRANSPOSE, pla.PLA_NONUNIT_DIAG,
                           a_view, bvec), "PLA_Trsv")
    x_hat = s.get(bvec)[:, 0]
    assert np.abs(x_hat - np.linalg.solve(A, b)).max() <= 1e-10 * np.abs(x_true).max() * n
    pla.check(lib.PLA_Axpy(minus_one, x, bvec), "PLA_Axpy")   # b <- b - x
    pla.check(lib.PLA_Nrm2(bvec, bnorm), "PLA_Nrm2")
    err = s.get(bnorm)[0, 0]
    assert err == pytest.approx(np.linalg.norm(x_hat - x_true), rel=1e-12, abs=1e-300)
    assert err < 1e-9
    s.free(a_view, rhs, a_app, piv, x, bvec, bnorm, minus_one)


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_axpy_nrm2_shift(env, dt):
    s, pla, _ = env
    lib = s.lib
    rng = np.random.default_rng(17)
    eps = np.finfo(dt).eps
    # PLA_Axpy on matrices of one shape, and x a row against a column y
    X, Y = rng.standard_normal((300, 70)).astype(dt), rng.standard_normal((300, 70)).astype(dt)
    x, y = s.matrix(300, 70, dt), s.matrix(300, 70, dt)
    s.put(x, X)
    s.put(y, Y)
    alpha = s.scalar(-2.5, dt)
    pla.check(lib.PLA_Axpy(alpha, x, y), "PLA_Axpy")
    assert np.abs(s.get(y) - (Y - 2.5 * X)).max() <= 8 * eps * np.abs(Y - 2.5 * X).max()
    row, col = ctypes.c_void_p(), ctypes.c_void_p()
    pla.check(lib.PLA_Obj_view(x, 1, 70, 4, 0, ctypes.byref(row)), "row view")
    col_v = s.mvector(70, 1, dt)
    C = rng.standard_normal(70).astype(dt)
    s.put(col_v, C)
    pla.check(lib.PLA_Axpy(alpha, row, col_v), "PLA_Axpy row->col")
    assert np.abs(s.get(col_v)[:, 0] - (C - 2.5 * X[4])).max() <= 8 * eps * 10
    # PLA_Nrm2: a column, a row view, scaled extremes, zeros, NaN
    nrm = s.scalar(0.0, dt)
    v = s.mvector(5000, 1, dt)
    V = rng.standard_normal(5000).astype(dt)
    s.put(v, V)
    pla.check(lib.PLA_Nrm2(v, nrm), "PLA_Nrm2")
    assert s.get(nrm)[0, 0] == pytest.approx(np.linalg.norm(V.astype(np.float64)), rel=4 * eps)
    pla.check(lib.PLA_Nrm2(row, nrm), "PLA_Nrm2 row")
    assert s.get(nrm)[0, 0] == pytest.approx(np.linalg.norm(X[4].astype(np.float64)), rel=4 * eps)
    scales = [1e200, 1e-200] if dt == np.float64 else [1e30, 1e-30]
    for sc in scales:
        s.set(v, (V * dt(sc)).astype(dt))
        pla.check(lib.PLA_Nrm2(v, nrm), "PLA_Nrm2 scaled")
        want = np.linalg.norm(V.astype(np.float64)) * sc  # numpy's own sum of squares overflows
        assert np.isfinite(s.get(nrm)[0, 0]) and s.get(nrm)[0, 0] == pytest.approx(want, rel=8 * eps)
    s.set(v, np.zeros(5000, dt))
    pla.check(lib.PLA_Nrm2(v, nrm), "PLA_Nrm2 zeros")
    assert s.get(nrm)[0, 0] == 0.0
    W = V.copy()
    W[1234] = np.nan
    s.set(v, W)
    pla.check(lib.PLA_Nrm2(v, nrm), "PLA_Nrm2 nan")
    assert np.isnan(s.get(nrm)[0, 0])
    # PLA_Shift: the diagonal of a square and of a wide matrix, value of the other type
    for (m, n) in [(200, 200), (150, 260)]:
        M = rng.standard_normal((m, n)).astype(dt)
        a = s.matrix(m, n, dt)
        s.put(a, M)
        if dt == np.float64:
            val, vt = ctypes.c_float(3.5), pla.MPI_FLOAT
        else:
            val, vt = ctypes.c_double(3.5), pla.MPI_DOUBLE
        pla.check(lib.PLA_Shift(a, vt, ctypes.byref(val)), "PLA_Shift")
        want = M.copy()
        k = min(m, n)
        want[np.arange(k), np.arange(k)] += dt(3.5)
        assert np.array_equal(s.get(a), want)
        s.free(a)
    s.free(row, x, y, alpha, col_v, nrm, v)
