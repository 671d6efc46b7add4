"""Tournament-pivoted fp32 panel (the mixed LU's sub-panels) against its CPU model.

pla_k_lu_panel_tslu factors an r x w fp32 panel (w <= 32) with tournament
pivoting: every block of rows picks w candidate rows by partial pivoting on
its own, the candidate sets are merged up a tree, the root's rows become the
pivots, and the rest of the panel is solved against their U.  The reference
has no such panel (its pivots are partial pivoting's), so the check is twofold:
- bit for bit against the oracle's C model of the same tree and arithmetic
  (oracle_slu_tournament): pivots and factors identical, NaN where it has NaN;
- as an LU: P A = L U to fp32 rounding, |L| bounded, pivots a valid
  sequence of interchanges.
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
    lib.pla_k_lu_panel_tslu.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                        ctypes.c_long, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    lib.pla_k_lu_panel_tslu.restype = ctypes.c_int
    yield s, torch, pla, orc.Restated()
    s.close()


def run_tslu(env, A, ld, max_ctas, row_base=0):
    s, torch, pla, _ = env
    r, w = A.shape
    buf = np.zeros((w, ld), dtype=np.float32)   # column-major r x w, leading dimension ld
    buf[:, :r] = A.T
    a = torch.from_numpy(buf).cuda()
    piv = torch.full((w,), -7, dtype=torch.int32, device="cuda")
    zinfo = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = s.lib.pla_k_lu_panel_tslu(r, w, a.data_ptr(), ld, piv.data_ptr(), zinfo.data_ptr(),
                                   row_base, max_ctas, None)
    assert rc == 0
    torch.cuda.synchronize()
    out = a.cpu().numpy()
    assert np.array_equal(out[:, r:], buf[:, r:])   # rows past r untouched
    return out[:, :r].T, piv.cpu().numpy(), int(zinfo.item())


CASES = [(1000, 32, 4), (5000, 32, 72), (32768, 32, 72), (32768, 32, 148), (300, 17, 3),
         (64, 32, 1), (100, 32, 2), (1500, 32, 148), (2000, 8, 16), (40, 32, 148),
         (33, 32, 1), (9000, 32, 1)]


@pytest.mark.parametrize("r,w,ctas", CASES)
def test_tslu_matches_its_model_bit_for_bit(env, r, w, ctas):
    rs = env[3]
    A = np.random.default_rng(r * 7 + w).standard_normal((r, w)).astype(np.float32)
    LU, piv, zinfo = run_tslu(env, A, r + 3, ctas)
    LUo, pivo = rs.slu_tournament(A, ctas)
    assert np.array_equal(piv, pivo)
    assert np.array_equal(LU, LUo)
    assert zinfo == 0


@pytest.mark.parametrize("r,w,ctas", [(4096, 32, 72), (777, 20, 8)])
def test_tslu_is_an_lu_factorization(env, r, w, ctas):
    A = np.random.default_rng(5).standard_normal((r, w)).astype(np.float32)
    LU, piv, _ = run_tslu(env, A, r, ctas)
    assert np.all(piv >= 0) and np.all(np.arange(w) + piv < r)
    perm = np.arange(r)
    for j in range(w):
        p = j + piv[j]
        perm[[j, p]] = perm[[p, j]]
    L = np.tril(LU.astype(np.float64), -1)[:, :w] + np.eye(r, w)
    U = np.triu(LU[:w].astype(np.float64))
    res = np.abs(A[perm].astype(np.float64) - L @ U).max() / np.abs(A).max()
    assert res < 16 * w * 2.0 ** -24
    assert np.abs(L).max() < 8.0                   # tournament growth stays small here


def test_tslu_ties_zero_and_nan_columns(env):
    """Equal candidates in different blocks (the smaller row wins), an exactly
    zero column (first zero pivot reported, 1-based + row_base, as the
    partial-pivoting panel does) and a NaN: all as the model has them."""
    rs = env[3]
    r, w = 3000, 32
    A = np.random.default_rng(9).standard_normal((r, w)).astype(np.float32)
    A[:, 0] = np.where(np.arange(r) % 2, 1.0, -1.0)    # every |a| equal in column 0
    A[:, 5] = 0.0
    A[17, 9] = np.nan
    LU, piv, zinfo = run_tslu(env, A, r, 72, row_base=100)
    LUo, pivo = rs.slu_tournament(A, 72)
    assert piv[0] == 0                               # row 0 is the first of the maximal rows
    assert np.array_equal(piv, pivo)
    assert np.array_equal(LU, LUo, equal_nan=True)
    assert zinfo == 100 + 6


def test_mixed_solve_with_either_panel_pivoting(env):
    """The fp16 mixed LU-IR solve reaches FP64 backward error with tournament
    (the default) and with partial pivoting of its fp32 panels."""
    s, torch, pla, _ = env
    lib = s.lib
    n = 3000
    rng = np.random.default_rng(12)
    M = np.asfortranarray(rng.standard_normal((n, n)))
    B = M @ rng.standard_normal((n, 1))
    for pivoting in (pla.PLA_B200_PIVOT_TOURNAMENT, pla.PLA_B200_PIVOT_PARTIAL):
        m, b = s.matrix(n, n), s.matrix(n, 1)
        s.set(m, M)
        s.set(b, B)
        prm, rep = pla.MixedParams(), pla.MixedReport()
        lib.PLA_Mixed_params_default(ctypes.byref(prm))
        assert prm.panel_pivoting == pla.PLA_B200_PIVOT_TOURNAMENT
        prm.panel_pivoting = pivoting
        prm.nb = 256
        pla.check(lib.PLA_General_solve_mixed(m, b, ctypes.byref(prm), ctypes.byref(rep)),
                  "PLA_General_solve_mixed")
        X = s.get(b)
        eta = np.abs(B - M @ X).max() / (np.abs(M).sum(axis=1).max() * np.abs(X).max() +
                                         np.abs(B).max())
        assert rep.converged == 1 and eta <= n * 2.0 ** -53, (pivoting, eta)
        assert rep.precision_used == pla.PLA_B200_PREC_FP16
        s.free(m, b)


@pytest.mark.parametrize("n", [32, 64, 96, 128, 160, 224, 256])
def test_unit_lower_inverse(env, n):
    """inv(L11) of the mixed LU's unit-lower diagonal block (pla_k_trtri_unit_lower:
    independent 32-column block columns, diagonal blocks inverted by warps):
    equal to the inverse to fp32 rounding, unit diagonal, strictly upper part
    zero; only L's strictly lower part is read (the upper part holds U)."""
    import scipy.linalg as sl
    s, torch, pla, _ = env
    lib = s.lib
    lib.pla_k_trtri_unit_lower.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_long,
                                           ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p,
                                           ctypes.c_void_p]
    lib.pla_k_trtri_unit_lower.restype = ctypes.c_int
    rng = np.random.default_rng(n)
    ld = n + 5
    L = sl.lu(rng.standard_normal((n, n)))[1]         # a unit-lower factor of a pivoted LU
    Lbuf = np.zeros((n, ld), dtype=np.float32)      # column-major n x n, leading dimension ld
    Lbuf[:, :n] = (L + np.triu(rng.standard_normal((n, n)), 0) * 1e3).T   # U above, ignored
    tL = torch.from_numpy(Lbuf).cuda()
    tD = torch.full((n, n), 7.0, dtype=torch.float32, device="cuda")
    assert lib.pla_k_trtri_unit_lower(n, tL.data_ptr(), ld, tD.data_ptr(), n, None, None) == 0
    torch.cuda.synchronize()
    D = tD.cpu().numpy().T.astype(np.float64)
    assert np.all(np.triu(D, 1) == 0.0) and np.all(np.diag(D) == 1.0)
    Dref = np.linalg.inv(L.astype(np.float32).astype(np.float64))
    assert np.abs(D - Dref).max() <= 64 * n * 2.0 ** -24 * np.abs(Dref).max()


@pytest.mark.parametrize("m,w,ncols", [(32768, 32, 224), (1000, 20, 37), (32, 32, 100),
                                       (33, 32, 480), (5000, 32, 16), (300, 7, 1)])
def test_panel_update(env, m, w, ncols):
    """The fp32 panel's sub-panel step after its interchanges (pla_k_panel_update):
    U12 = inv(L11) A12 over A12 and A22 -= L21 U12, one launch, to fp32 rounding;
    the sub-panel itself and the rows past m untouched.  Launched twice so the
    per-group counters are seen reset."""
    import scipy.linalg as sl
    s, torch, pla, _ = env
    lib = s.lib
    lib.pla_k_panel_update.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                       ctypes.c_long, ctypes.c_void_p]
    lib.pla_k_panel_update.restype = ctypes.c_int
    ld = m + 3
    for rep in range(2):
        rng = np.random.default_rng(m + w + ncols + rep)
        buf = rng.standard_normal((w + ncols, ld)).astype(np.float32)   # column-major, ld
        buf[:w, :w] = (np.tril(rng.uniform(-1, 1, (w, w)), -1) + np.triu(np.full((w, w), 9.0))).T
        t = torch.from_numpy(buf).cuda()
        assert lib.pla_k_panel_update(m, w, ncols, t.data_ptr(), ld, None) == 0
        torch.cuda.synchronize()
        out = t.cpu().numpy()
        A = buf[:, :m].T.astype(np.float64)                             # m x (w + ncols)
        L11 = np.tril(A[:w, :w], -1) + np.eye(w)
        U12 = sl.solve_triangular(L11, A[:w, w:], lower=True, unit_diagonal=True)
        A22 = A[w:, w:] - A[w:, :w] @ U12
        got = out[:, :m].T.astype(np.float64)
        assert np.array_equal(out[:w], buf[:w])                          # the sub-panel
        assert np.array_equal(out[:, m:], buf[:, m:])                    # rows past m
        tol = 8 * w * 2.0 ** -24
        assert np.abs(got[:w, w:] - U12).max() <= tol * max(1.0, np.abs(U12).max())
        if m > w:
            scale = np.abs(A[w:, w:]).max() + np.abs(A[w:, :w]).max() * np.abs(U12).max() * w
            assert np.abs(got[w:, w:] - A22).max() <= tol * scale


@pytest.mark.parametrize("r,b,pivoting", [(4096, 256, 1), (4096, 256, 0), (700, 96, 1),
                                          (256, 256, 1)])
def test_blocked_panel_is_an_lu_factorization(env, r, b, pivoting):
    """The mixed LU's whole r x b fp32 panel (pla_k_panel_lu_blocked: 32-column
    sub-panels, each followed by its interchanges and pla_k_panel_update):
    P A = L U to fp32 rounding, with tournament (1) and partial (0) pivoting."""
    s, torch, pla, _ = env
    lib = s.lib
    lib.pla_k_panel_lu_blocked.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p,
                                           ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_void_p]
    lib.pla_k_panel_lu_blocked.restype = ctypes.c_int
    A = np.random.default_rng(r + b + pivoting).standard_normal((r, b)).astype(np.float32)
    t = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
    piv = torch.full((b,), -7, dtype=torch.int32, device="cuda")
    zinfo = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert lib.pla_k_panel_lu_blocked(pla.MPI_FLOAT, r, b, t.data_ptr(), r, piv.data_ptr(),
                                      zinfo.data_ptr(), 72, pivoting, None) == 0
    torch.cuda.synchronize()
    LU = t.cpu().numpy().T.astype(np.float64)
    p = piv.cpu().numpy()
    assert np.all(p >= 0) and np.all(np.arange(b) + p < r) and int(zinfo.item()) == 0
    perm = np.arange(r)
    for j in range(b):
        q = j + p[j]
        perm[[j, q]] = perm[[q, j]]
    L = np.tril(LU, -1)[:, :b] + np.eye(r, b)
    U = np.triu(LU[:b])
    res = np.abs(A[perm].astype(np.float64) - L @ U).max() / np.abs(A).max()
    assert res < 4 * b * 2.0 ** -24
