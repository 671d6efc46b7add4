"""Entry points the reference's callers reach directly, beside PLA_LU and PLA_Gemm.

- PLA_LU_right(nb_alg, A, pivots) (SOLVERS/LU/PLA_LU.c:37): the blocked LU
  with the caller's block size, against the oracle's blocked LU (pivots
  equal, factors within rounding).
- PLA_LU_right_mv(A_mv, A_11_msc, pivots_msc) (SOLVERS/LU/PLA_LU_mv.c:13):
  the panel factorization on a multivector; pivots equal to the oracle's
  column loop, the factors within rounding, and A_11_msc a copy of the
  factored top block (PLA_Apply_pivots_new.c:274 copies each pivot row).
- PLA_Gemm_x (BLAS3/PLA_Gemm_x.c:13): every version gives PLA_Gemm's bits;
  an unknown version is an error.
- PLA_Timings_initialize / print / average (OBJ/PLA_Timings.c): they switch
  on, print and keep the phase timers.
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


@pytest.mark.parametrize("m,n,nb", [(900, 900, 48), (1300, 700, 96)])
def test_lu_right_with_block_size(env, m, n, nb):
    s, pla, oracle = env
    A = np.random.default_rng(m).standard_normal((m, n))
    a, piv = s.matrix(m, n), s.mvector(min(m, n), 1, np.int32)
    s.put(a, A)
    pla.check(s.lib.PLA_LU_right(nb, a, piv), "PLA_LU_right")
    ref, ref_piv = oracle.lu_blocked(A, nb)
    assert np.array_equal(s.get(piv)[:, 0], ref_piv)
    assert np.abs(s.get(a) - ref).max() <= 4 * max(m, n) * np.finfo(float).eps * np.abs(ref).max()
    assert s.lib.PLA_LU_right(0, a, piv) == pla.PLA_ERROR
    s.free(a, piv)


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("r,w", [(2000, 64), (500, 128), (40, 40)])
def test_lu_right_mv(env, dt, r, w):
    s, pla, oracle = env
    A = np.random.default_rng(r + w).standard_normal((r, w)).astype(dt)
    a_mv = s.mvector(r, w, dt)
    a11 = ctypes.c_void_p()
    pla.check(s.lib.PLA_Mscalar_create(pla.MPI_DOUBLE if dt == np.float64 else pla.MPI_FLOAT,
                                       pla.PLA_ALL_ROWS, pla.PLA_ALL_COLS, w, w, s.templ,
                                       ctypes.byref(a11)), "A_11_msc")
    piv = ctypes.c_void_p()
    pla.check(s.lib.PLA_Mscalar_create(pla.MPI_INT, pla.PLA_ALL_ROWS, pla.PLA_ALL_COLS, w, 1,
                                       s.templ, ctypes.byref(piv)), "pivots_msc")
    s.put(a_mv, A)
    pla.check(s.lib.PLA_LU_right_mv(a_mv, a11, piv), "PLA_LU_right_mv")
    LU, p, top = s.get(a_mv), s.get(piv)[:, 0], s.get(a11)
    ref, ref_piv = oracle.lu_unblocked(A)
    assert np.array_equal(p, ref_piv)
    eps = np.finfo(dt).eps
    assert np.abs(LU.astype(np.float64) - ref).max() <= 8 * w * eps * max(1.0, np.abs(ref).max())
    assert np.array_equal(top, LU[:w])
    s.free(a_mv, a11, piv)


def test_gemm_x_versions(env):
    s, pla, _ = env
    rng = np.random.default_rng(2)
    A, B, C = (rng.standard_normal(sh) for sh in [(300, 200), (200, 250), (300, 250)])
    a, b = s.matrix(300, 200), s.matrix(200, 250)
    s.put(a, A)
    s.put(b, B)
    alpha, beta = s.scalar(1.5), s.scalar(-0.5)
    outs = []
    for version in (None, pla.PLA_VERSION_A, pla.PLA_VERSION_B, pla.PLA_VERSION_C):
        c = s.matrix(300, 250)
        s.put(c, C)
        if version is None:
            pla.check(s.lib.PLA_Gemm(pla.PLA_NO_TRANSPOSE, pla.PLA_NO_TRANSPOSE, alpha, a, b,
                                     beta, c), "PLA_Gemm")
        else:
            pla.check(s.lib.PLA_Gemm_x(version, pla.PLA_NO_TRANSPOSE, pla.PLA_NO_TRANSPOSE, alpha,
                                       a, b, beta, c), "PLA_Gemm_x")
        outs.append(s.get(c))
        s.free(c)
    for o in outs[1:]:
        assert np.array_equal(o, outs[0])
    assert np.abs(outs[0] - (1.5 * A @ B - 0.5 * C)).max() <= 1e-12 * 200
    c = s.matrix(300, 250)
    assert s.lib.PLA_Gemm_x(7, pla.PLA_NO_TRANSPOSE, pla.PLA_NO_TRANSPOSE, alpha, a, b, beta,
                            c) == pla.PLA_ERROR
    s.free(a, b, c, alpha, beta)


def test_timings(env, capfd):
    s, pla, _ = env
    n = 1024
    a, piv = s.matrix(n, n), s.mvector(n, 1, np.int32)
    s.put(a, np.random.default_rng(0).standard_normal((n, n)))
    assert s.lib.PLA_Timings_initialize() == 0
    pla.check(s.lib.PLA_LU(a, piv), "PLA_LU")
    assert s.lib.PLA_Timings_average() == 0
    assert s.lib.PLA_Timings_print() == 0
    ctypes.CDLL(None).fflush(None)              # the library's printf buffer
    out = capfd.readouterr().out
    assert "panel   time =" in out and "update  time =" in out
    s.lib.PLA_B200_set_phase_timing(0)
    s.free(a, piv)
