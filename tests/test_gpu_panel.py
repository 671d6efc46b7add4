"""The panel kernel against the oracle, at the sizes and edge cases the solvers meet.

pla_k_lu_panel_ex factors an r x w panel with partial pivoting on at most
max_ctas CTAs.  This is the per-column loop of PLA_LU_right_mv
(SOLVERS/LU/PLA_LU_mv.c:52-82).  The oracle's unblocked LU restates the same
loop (SOLVERS/LU/PLA_seq_lu.c:21-46) on the CPU.  The checks: pivots equal to
the oracle's, and factors within a rounding tolerance of them (the kernel
fuses the rank-1 update into one fma per element).  The cases cover:
- CTA caps (72 CTAs beside a trailing update; one CTA per SM), and 57 to
  911 panel rows per CTA;
- a leading dimension larger than r, and widths below 32;
- equal candidates in different CTAs: the smaller row index wins
  (BLAS1/PLA_Iamax.c:108-111, the first index of idamax);
- an exactly zero pivot, whose 1-based column comes back through zero_info;
- a column of NaNs, where no row is a candidate and the row stays its own
  pivot.
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
    s = pla.Session(nb_distr=128, nb_alg=128)
    lib = s.lib
    lib.pla_k_lu_panel_ex.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                      ctypes.c_long, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_void_p]
    lib.pla_k_lu_panel_ex.restype = ctypes.c_int
    yield s, torch, pla, orc.Restated()
    s.close()


def run_panel(env, A, ld, max_ctas, row_base=0):
    s, torch, pla, _ = env
    r, w = A.shape
    mpi = pla.MPI_DOUBLE if A.dtype == np.float64 else pla.MPI_FLOAT
    buf = np.zeros((w, ld), dtype=A.dtype)     # column-major r x w with leading dimension ld
    buf[:, :r] = A.T
    a = torch.from_numpy(buf).cuda()
    piv = torch.full((w,), -7, dtype=torch.int32, device="cuda")
    status = torch.zeros(4, dtype=torch.int32, device="cuda")
    zinfo = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = s.lib.pla_k_lu_panel_ex(mpi, r, w, a.data_ptr(), ld, piv.data_ptr(), status.data_ptr(),
                                 zinfo.data_ptr(), row_base, max_ctas, None)
    assert rc == 0
    torch.cuda.synchronize()
    assert int(status[0].item()) == 0
    return a.cpu().numpy()[:, :r].T.copy(), piv.cpu().numpy(), int(zinfo[0].item())


def check_factors(LU, ref, A, w):
    eps = np.finfo(A.dtype).eps
    finite = np.isfinite(ref)
    assert np.array_equal(finite, np.isfinite(LU))
    tol = 8 * w * eps * max(1.0, np.nanmax(np.abs(A))) * max(1.0, np.abs(ref[finite]).max())
    assert np.abs(LU[finite].astype(np.float64) - ref[finite]).max() <= tol


CASES = [
    # (dtype, r, w, ld, max_ctas)
    (np.float32, 32768, 32, 32768, 72),   # the first sub-panel of the n = 32768 mixed LU
    (np.float32, 32768, 32, 32800, 0),
    (np.float32, 15000, 32, 15000, 24),
    (np.float32, 20000, 32, 20003, 24),
    (np.float32, 3000, 17, 3000, 0),
    (np.float32, 40, 32, 40, 0),          # one CTA
    (np.float64, 20000, 32, 20000, 48),   # a sub-panel of the FP64 LU beside its DGEMM
    (np.float64, 5000, 32, 5001, 0),
    (np.float64, 1000, 7, 1000, 0),
]


@pytest.mark.parametrize("dt,r,w,ld,max_ctas", CASES)
def test_panel_matches_oracle(env, dt, r, w, ld, max_ctas):
    oracle = env[3]
    rng = np.random.default_rng(r + w)
    A = rng.standard_normal((r, w)).astype(dt)
    LU, piv, zinfo = run_panel(env, A, ld, max_ctas)
    ref, ref_piv = oracle.lu_unblocked(A)
    assert np.array_equal(piv, ref_piv)
    assert zinfo == 0
    check_factors(LU, ref, A, w)


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("case", ["ties", "zero", "nan"])
def test_panel_ties_zero_and_nan_columns(env, dt, case):
    oracle = env[3]
    r, w = 9000, 32
    rng = np.random.default_rng(5)
    A = rng.standard_normal((r, w)).astype(dt)
    if case == "ties":
        A[:, 0] = 1.0             # every row a candidate of the same size: row 0 wins
        A[4000, 1] = 50.0         # a clear winner far from the diagonal
    elif case == "zero":
        A[:, 5] = 0.0             # stays zero under the updates: an exact zero pivot at 5
    else:
        A[:, 9] = np.nan          # no candidate anywhere: row 9 stays its own pivot
    LU, piv, zinfo = run_panel(env, A, r, 0, row_base=1000)
    ref, ref_piv = oracle.lu_unblocked(A)
    assert np.array_equal(piv, ref_piv)
    if case == "ties":
        assert piv[0] == 0 and piv[1] == 3999 and zinfo == 0
    elif case == "zero":
        assert zinfo == 1000 + 5 + 1
    else:
        assert piv[9] == 0 and zinfo == 0
    # the columns before the zero or NaN column are finite and match
    good = {"ties": w, "zero": 5, "nan": 9}[case]
    check_factors(LU[:, :good], ref[:, :good], A[:, :good], w)


def test_panel_wait_runs_out_and_the_next_call_succeeds(env):
    """The timeout path of the panel's exchange: one CTA publishes nothing and
    every poll is limited to a few hundred tries, so every CTA gives up.  The
    launch must return with status PLA_K_TIMEOUT (1), and the next panel on
    the same stream must run normally and match the oracle."""
    s, torch, pla, rs = env
    lib = s.lib
    lib.pla_k_panel_test_timeout.argtypes = [ctypes.c_long, ctypes.c_int]
    lib.pla_k_panel_test_timeout.restype = None
    rng = np.random.default_rng(77)
    r, w = 4096, 32
    A = rng.standard_normal((r, w))
    a = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
    piv = torch.zeros(w, dtype=torch.int32, device="cuda")
    status = torch.zeros(4, dtype=torch.int32, device="cuda")
    lib.pla_k_panel_test_timeout(300, 1)           # CTA 1 of 4 or more stays silent
    rc = lib.pla_k_lu_panel_ex(pla.MPI_DOUBLE, r, w, a.data_ptr(), r, piv.data_ptr(),
                               status.data_ptr(), None, 0, 4, None)
    assert rc == 0
    torch.cuda.synchronize()
    assert int(status[0].item()) == 1              # PLA_K_TIMEOUT
    # the hook applies to one launch only: the same panel again, fresh status
    a = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
    status.zero_()
    rc = lib.pla_k_lu_panel_ex(pla.MPI_DOUBLE, r, w, a.data_ptr(), r, piv.data_ptr(),
                               status.data_ptr(), None, 0, 4, None)
    assert rc == 0
    torch.cuda.synchronize()
    assert int(status[0].item()) == 0
    LUo, pivo = rs.lu_unblocked(A)
    assert np.array_equal(piv.cpu().numpy(), pivo)
    LU = a.cpu().numpy().T
    assert np.abs(LU - LUo).max() <= 4 * r * 2.0 ** -52 * np.abs(LUo).max()
