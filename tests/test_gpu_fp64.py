"""Parity of the B200 FP64 path with the reference, through the C ABI.

Every case calls the library exactly as a PLAPACK driver would (PLA_Matrix_create,
PLA_API_axpy_matrix_to_global, PLA_LU / PLA_Chol / PLA_Trsm / PLA_Gemm, ...)
and compares with the golden outputs of the upstream PLAPACK (tests/golden)
or with the CPU oracle on the same inputs:
  - pivots: identical integers;
  - factors and solutions: within n * eps64 * ||A||,
    scaled by the size of the compared quantity.
"""
import ctypes

import numpy as np
import pytest

import inputs
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

EPS = np.finfo(np.float64).eps


@pytest.fixture(scope="module")
def pla_session():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from plapack_b200 import pla
    s = pla.Session(nb_distr=64, nb_alg=64)
    yield s
    s.close()


def pla_lu(s, A, nb):
    from plapack_b200 import pla
    s.set_nb_alg(nb)
    m, n = A.shape
    a = s.matrix(m, n, A.dtype)
    p = s.mvector(min(m, n), 1, np.int32)
    s.put(a, A)
    info = ctypes.c_int(-1)
    pla.check(s.lib.PLA_LU_info(a, p, ctypes.byref(info)), "PLA_LU")
    LU, piv = s.get(a), s.get(p)[:, 0]
    s.free(a, p)
    return LU, piv, info.value


def tol_factor(A, LU_ref):
    n = max(A.shape)
    eps = np.finfo(A.dtype).eps
    return 4 * n * eps * max(1.0, np.abs(A).max()) * max(1.0, np.abs(LU_ref).max())


def test_lu_golden_pivots_and_factors(pla_session, golden, restated):
    manifest, arrays = golden
    for name, e in manifest.items():
        if e["kind"] != "lu":
            continue
        A = inputs.build(restated, e["spec"])
        LU, piv, info = pla_lu(pla_session, A, e["nb_alg"])
        assert np.array_equal(piv, arrays[name + "__piv"]), name
        if name.startswith("lu_singular"):
            assert info == A.shape[1], name      # the zero pivot in the last column
            continue
        LUo, _ = restated.lu_blocked(A, e["nb_alg"])
        assert np.abs(LU - LUo).max() <= tol_factor(A, LUo), name
        d = arrays[name + "__diag"]
        assert np.abs(np.diag(LU) - d).max() <= tol_factor(A, LUo), name


def test_lu_ties_first_index(pla_session, golden, restated):
    """Every |a_ij| = 1: the first-index tie-break decides every pivot."""
    manifest, arrays = golden
    e = manifest["lu_ties_48_nb16"]
    A = inputs.build(restated, e["spec"])
    _, piv, _ = pla_lu(pla_session, A, 16)
    assert np.array_equal(piv, arrays["lu_ties_48_nb16__piv"])


def test_lu_zero_column_nan_fill(pla_session):
    """An exact zero pivot early on turns the rest of the matrix into NaN (as
    the reference does: no detection, 1/0 scaling).  Pivot searches over NaN
    columns must still name rows of the matrix, and info reports the column."""
    rng = np.random.default_rng(4)
    for n, nb in [(100, 32), (300, 128)]:
        A = np.asfortranarray(rng.standard_normal((n, n)))
        A[:, 5] = 0.0
        LU, piv, info = pla_lu(pla_session, A, nb)
        assert info == 6
        assert np.all(piv >= 0) and np.all(piv + np.arange(n) < n)
        assert np.isnan(LU[10:, 10:]).all()


@pytest.mark.parametrize("n,nb", [(1000, 64), (2048, 128), (1537, 96)])
def test_lu_vs_oracle_random(pla_session, restated, n, nb):
    rng = np.random.default_rng(n)
    A = np.asfortranarray(rng.standard_normal((n, n)))
    LU, piv, _ = pla_lu(pla_session, A, nb)
    LUo, pivo = restated.lu_blocked(A, nb)
    assert np.array_equal(piv, pivo)
    assert np.abs(LU - LUo).max() <= tol_factor(A, LUo)


def test_lu_residual_large(pla_session):
    """Size-independent check at n = 8192: ||P A - L U|| / ||A|| and pivots vs LAPACK."""
    import scipy.linalg as sl
    n = 8192
    rng = np.random.default_rng(1)
    A = np.asfortranarray(rng.standard_normal((n, n)))
    LU, piv, _ = pla_lu(pla_session, A, 128)
    _, ipiv = sl.lu_factor(A, check_finite=False)
    assert np.array_equal(piv, ipiv - np.arange(n))
    import torch
    L = torch.tril(torch.from_numpy(LU), -1).cuda() + torch.eye(n, dtype=torch.float64, device="cuda")
    U = torch.triu(torch.from_numpy(LU)).cuda()
    PA = torch.from_numpy(A).cuda()
    perm = np.arange(n)
    for i in range(n):
        p = i + piv[i]
        perm[[i, p]] = perm[[p, i]]
    PA = PA[torch.from_numpy(perm).cuda()]
    res = (torch.linalg.matrix_norm(L @ U - PA) / torch.linalg.matrix_norm(PA)).item()
    assert res < 64 * EPS * np.sqrt(n)


def test_chol_golden(pla_session, golden, restated):
    from plapack_b200 import pla
    manifest, arrays = golden
    s = pla_session
    for name, e in manifest.items():
        if e["kind"] != "chol":
            continue
        A = inputs.build(restated, e["spec"])
        s.set_nb_alg(e["nb_alg"])
        a = s.matrix(*A.shape)
        s.put(a, A)
        ret = pla.check(s.lib.PLA_Chol(pla.PLA_LOWER_TRIANGULAR, a), "PLA_Chol")
        assert ret == e["ret"], name
        if ret == 0:
            L = np.tril(s.get(a))
            Lo, _ = restated.chol_blocked(A, e["nb_alg"])
            Lo = np.tril(Lo)
            assert np.abs(L - Lo).max() <= tol_factor(A, Lo), name
            assert np.abs(np.diag(L) - arrays[name + "__diag"]).max() <= tol_factor(A, Lo)
            # the strict upper triangle is never written
            assert np.array_equal(np.triu(s.get(a), 1), np.triu(A, 1)), name
        s.free(a)


@pytest.mark.parametrize("n,nb", [(2600, 512), (2100, 384)])
def test_chol_wide_block_columns(pla_session, restated, n, nb):
    """Block columns of 384 and 512 (factored in 128-column steps, with the
    lookahead on) against the restated PLA_Chol at the same nb_alg, and the
    failing column of an indefinite matrix."""
    from plapack_b200 import pla
    s = pla_session
    rng = np.random.default_rng(nb)
    G = rng.standard_normal((n, n))
    A = np.asfortranarray(G @ G.T / n + np.eye(n))
    s.set_nb_alg(nb)
    a = s.matrix(n, n)
    s.put(a, A)
    assert pla.check(s.lib.PLA_Chol(pla.PLA_LOWER_TRIANGULAR, a), "PLA_Chol") == 0
    Lo, info = restated.chol_blocked(A, nb)
    assert info == 0
    assert np.abs(np.tril(s.get(a)) - np.tril(Lo)).max() <= tol_factor(A, Lo)
    A[n - 700, n - 700] = -1.0                 # indefinite at 1-based column n - 699
    s.put(a, A)
    assert s.lib.PLA_Chol(pla.PLA_LOWER_TRIANGULAR, a) == restated.chol_blocked(A, nb)[1]
    s.free(a)


def test_general_and_pos_def_solve_golden(pla_session, golden, restated):
    from plapack_b200 import pla
    manifest, arrays = golden
    s = pla_session
    for name, e in manifest.items():
        if e["kind"] not in ("general_solve", "pos_def_solve"):
            continue
        A = inputs.build(restated, e["spec"])
        B = A @ np.ones((A.shape[0], 1)) if "rhs_spec" not in e else inputs.build(restated, e["rhs_spec"])
        s.set_nb_alg(e["nb_alg"])
        a = s.matrix(*A.shape)
        s.put(a, A)
        b = s.mvector(B.shape[0], 1) if B.shape[1] == 1 else s.matrix(*B.shape)
        s.put(b, B)
        if e["kind"] == "general_solve":
            p = s.mvector(A.shape[0], 1, np.int32)
            pla.check(s.lib.PLA_General_solve(a, p, b), "General_solve")
            assert np.array_equal(s.get(p)[:, 0], arrays[name + "__piv"]), name
            s.free(p)
        else:
            assert pla.check(s.lib.PLA_Pos_def_solve(a, b), "Pos_def_solve") == 0
        X = s.get(b)
        Xr = arrays[name + "__X"].reshape(X.shape)
        cond = np.linalg.cond(A, 1)
        assert np.abs(X - Xr).max() <= 16 * A.shape[0] * EPS * cond * max(1.0, np.abs(Xr).max()), name
        s.free(a, b)


def test_trsv_trsm_golden(pla_session, golden, restated):
    from plapack_b200 import pla
    manifest, arrays = golden
    s = pla_session
    for name, e in manifest.items():
        if e["kind"] not in ("trsv", "trsm"):
            continue
        T = inputs.build(restated, e["spec"])
        B = inputs.build(restated, e["rhs_spec"])
        a = s.matrix(*T.shape)
        s.put(a, T)
        if e["kind"] == "trsv":
            x = s.mvector(B.shape[0], 1)
            s.put(x, B)
            pla.check(s.lib.PLA_Trsv(e["uplo"], e["trans"], e["diag"], a, x), "Trsv")
            X, ref = s.get(x)[:, 0], arrays[name + "__x"]
        else:
            x = s.matrix(*B.shape)
            s.put(x, B)
            al = s.scalar(e["alpha"])
            pla.check(s.lib.PLA_Trsm(e["side"], e["uplo"], e["trans"], e["diag"], al, a, x), "Trsm")
            s.free(al)
            X, ref = s.get(x), arrays[name + "__X"]
        assert np.abs(X - ref).max() <= 1e-11 * np.abs(ref).max(), name
        s.free(a, x)


@pytest.mark.parametrize("m,n,k", [(37, 29, 17), (300, 200, 128), (513, 257, 96), (1, 1, 1)])
@pytest.mark.parametrize("alpha,beta", [(-1.0, 0.5), (1.0, 1.0), (0.75, -0.5), (-1.0, 0.0)])
def test_gemm_all_transposes(pla_session, m, n, k, alpha, beta):
    """alpha = +-1 starts the accumulators from beta C, other alphas read C in
    the epilogue; beta = 0 must not read C at all (C is NaN there)."""
    from plapack_b200 import pla
    s = pla_session
    rng = np.random.default_rng(m * 7 + n)
    for ta in (pla.PLA_NO_TRANSPOSE, pla.PLA_TRANSPOSE):
        for tb in (pla.PLA_NO_TRANSPOSE, pla.PLA_TRANSPOSE):
            A = rng.standard_normal((m, k) if ta == pla.PLA_NO_TRANSPOSE else (k, m))
            B = rng.standard_normal((k, n) if tb == pla.PLA_NO_TRANSPOSE else (n, k))
            C = rng.standard_normal((m, n)) if beta != 0.0 else np.full((m, n), np.nan)
            a, b, c = s.matrix(*A.shape), s.matrix(*B.shape), s.matrix(m, n)
            s.put(a, A), s.put(b, B), s.put(c, C)
            al, be = s.scalar(alpha), s.scalar(beta)
            pla.check(s.lib.PLA_Gemm(ta, tb, al, a, b, be, c), "Gemm")
            opA = A if ta == pla.PLA_NO_TRANSPOSE else A.T
            opB = B if tb == pla.PLA_NO_TRANSPOSE else B.T
            ref = alpha * (opA @ opB) + (beta * C if beta != 0.0 else 0.0)
            got = s.get(c)
            assert np.isfinite(got).all()
            scale = (np.abs(opA) @ np.abs(opB)).max() + abs(beta) * np.nan_to_num(np.abs(C)).max()
            assert np.abs(got - ref).max() <= 4 * k * EPS * scale + 1e-15
            s.free(a, b, c, al, be)


def test_gemm_golden(pla_session, golden, restated):
    from plapack_b200 import pla
    manifest, arrays = golden
    s = pla_session
    for name, e in manifest.items():
        if e["kind"] != "gemm":
            continue
        A, B, C = (inputs.build(restated, e[k]) for k in ("A_spec", "B_spec", "C_spec"))
        a, b, c = s.matrix(*A.shape), s.matrix(*B.shape), s.matrix(*C.shape)
        s.put(a, A), s.put(b, B), s.put(c, C)
        al, be = s.scalar(e["alpha"]), s.scalar(e["beta"])
        pla.check(s.lib.PLA_Gemm(e["transa"], e["transb"], al, a, b, be, c), "Gemm")
        assert np.abs(s.get(c) - arrays[name + "__C"]).max() <= 1e-13, name
        s.free(a, b, c, al, be)


def test_views_and_local_blas(pla_session):
    """Views share the device buffer; Local BLAS wrappers act on views."""
    from plapack_b200 import pla
    s = pla_session
    rng = np.random.default_rng(5)
    A = rng.standard_normal((40, 30))
    a = s.matrix(40, 30)
    s.put(a, A)
    tl, tr, bl, br = (ctypes.c_void_p() for _ in range(4))
    pla.check(s.lib.PLA_Obj_split_4(a, 10, 12, ctypes.byref(tl), ctypes.byref(tr),
                                    ctypes.byref(bl), ctypes.byref(br)), "split_4")
    assert np.array_equal(s.get(br), A[10:, 12:])
    two = s.scalar(2.0)
    pla.check(s.lib.PLA_Local_scal(two, br), "scal")
    assert np.array_equal(s.get(a)[10:, 12:], 2 * A[10:, 12:])
    pla.check(s.lib.PLA_Local_inv_scal(two, br), "inv_scal")
    assert np.allclose(s.get(a), A, rtol=0, atol=1e-15)
    # iamax on a column view: first index of the largest magnitude
    col = ctypes.c_void_p()
    pla.check(s.lib.PLA_Obj_view(a, 40, 1, 0, 3, ctypes.byref(col)), "view")
    idx = ctypes.c_int()
    val = ctypes.c_double()
    pla.check(s.lib.PLA_Local_iamax(col, ctypes.byref(idx), ctypes.byref(val)), "iamax")
    assert idx.value == int(np.argmax(np.abs(A[:, 3]))) and val.value == A[idx.value, 3]
    # negative split sizes count from the bottom / right
    top, bot = ctypes.c_void_p(), ctypes.c_void_p()
    pla.check(s.lib.PLA_Obj_horz_split_2(a, -7, ctypes.byref(top), ctypes.byref(bot)), "split")
    assert np.array_equal(s.get(bot), A[-7:, :])
    s.free(tl, tr, bl, br, two, col, top, bot, a)


def test_api_axpy_accumulates(pla_session):
    s = pla_session
    A = np.arange(12.0).reshape(4, 3, order="F")
    a = s.matrix(6, 5)
    s.put(a, A, 1, 2)
    s.put(a, A, 1, 2)
    out = s.get(a)
    exp = np.zeros((6, 5))
    exp[1:5, 2:5] = 2 * A
    assert np.array_equal(out, exp)
    s.free(a)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("n", [1024, 3001])
def test_trsv_single_launch(pla_session, dtype, n):
    """PLA_Trsv of order >= 1024 runs the single-launch solve (inverse diagonal
    blocks of 64 in FP64, 128 in fp32): all four triangle / transpose cases,
    unit and non-unit diagonals, against LAPACK's triangular solve."""
    from scipy.linalg import solve_triangular
    from plapack_b200 import pla
    s = pla_session
    rng = np.random.default_rng(n)
    M = rng.standard_normal((n, n)) / np.sqrt(n)
    M[np.diag_indices(n)] = 1.0 + rng.random(n)
    cases = [(pla.PLA_LOWER_TRIANGULAR, pla.PLA_NO_TRANSPOSE, pla.PLA_UNIT_DIAG),
             (pla.PLA_UPPER_TRIANGULAR, pla.PLA_NO_TRANSPOSE, pla.PLA_NONUNIT_DIAG),
             (pla.PLA_LOWER_TRIANGULAR, pla.PLA_TRANSPOSE, pla.PLA_NONUNIT_DIAG),
             (pla.PLA_UPPER_TRIANGULAR, pla.PLA_TRANSPOSE, pla.PLA_UNIT_DIAG)]
    eps = np.finfo(dtype).eps
    for uplo, trans, diag in cases:
        A = np.asfortranarray(M.astype(dtype))
        b = rng.standard_normal((n, 1)).astype(dtype)
        a = s.matrix(n, n, dtype)
        x = s.mvector(n, 1, dtype)
        s.put(a, A)
        s.put(x, b)
        pla.check(s.lib.PLA_Trsv(uplo, trans, diag, a, x), "PLA_Trsv")
        got = s.get(x)[:, 0].astype(np.float64)
        ref = solve_triangular(A.astype(np.float64), b[:, 0].astype(np.float64),
                               lower=uplo == pla.PLA_LOWER_TRIANGULAR,
                               trans=0 if trans == pla.PLA_NO_TRANSPOSE else 1,
                               unit_diagonal=diag == pla.PLA_UNIT_DIAG)
        assert np.abs(got - ref).max() <= 64 * n * eps * np.abs(ref).max(), (uplo, trans, diag)
        s.free(a, x)


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("b", [1, 7, 64, 100, 128])
def test_potrf_diagonal_block(pla_session, dt, b):
    """pla_k_potrf_lower, the Cholesky's diagonal-block kernel, against
    LAPACK's Cholesky; the strict upper triangle is never written; a block
    that is not positive definite at column c reports base + c and
    PLA_K_NOT_SPD and leaves the block unwritten (PLA_Chol.c:181-185)."""
    import torch
    from plapack_b200 import pla
    lib = pla_session.lib
    f = lib.pla_k_potrf_lower
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    f.restype = ctypes.c_int
    mpi = pla.MPI_DOUBLE if dt == np.float64 else pla.MPI_FLOAT
    rng = np.random.default_rng(b)
    G = rng.standard_normal((b, b))
    A = (G @ G.T / b + np.eye(b)).astype(dt)
    A[np.triu_indices(b, 1)] = 7.0               # the upper triangle must stay as it is
    lda = b + 3
    buf = np.full((b, lda), -1.0, dtype=dt)      # column-major b x b, leading dimension lda
    buf[:, :b] = A.T
    a = torch.from_numpy(buf).cuda()
    st = torch.zeros(4, dtype=torch.int32, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert f(mpi, b, a.data_ptr(), lda, st.data_ptr(), info.data_ptr(), 0, None) == 0
    torch.cuda.synchronize()
    out = a.cpu().numpy()[:, :b].T
    assert int(st[0]) == 0 and int(info[0]) == 0
    Lr = np.linalg.cholesky(np.tril(A).astype(np.float64) + np.tril(A, -1).T)
    eps = np.finfo(dt).eps
    assert np.abs(np.tril(out) - Lr).max() <= 8 * b * eps * np.abs(Lr).max()
    assert np.array_equal(np.triu(out, 1), np.triu(A, 1))
    assert np.all(a.cpu().numpy()[:, b:] == -1.0)
    if b < 7:
        return
    c = b // 2                                   # make column c + 1 (1-based) fail
    A2 = A.copy()
    A2[c, c] = -1.0
    buf[:, :b] = A2.T
    a = torch.from_numpy(buf).cuda()
    assert f(mpi, b, a.data_ptr(), lda, st.data_ptr(), info.data_ptr(), 500, None) == 0
    torch.cuda.synchronize()
    assert int(info[0]) == 500 + c + 1 and int(st[0]) != 0
    assert np.array_equal(a.cpu().numpy()[:, :b].T, A2)


def test_phase_times_count_interchanges(pla_session):
    """With phase timing on, PLA_Phase_times.interchanges counts the LU's row
    interchanges that moved rows (pivot offset != 0), summed over calls."""
    from plapack_b200 import pla
    lib = pla_session.lib
    A = np.asfortranarray(np.random.default_rng(4).standard_normal((700, 700)))
    lib.PLA_B200_set_phase_timing(1)
    try:
        lib.PLA_B200_reset_phase_times()
        _, piv1, _ = pla_lu(pla_session, A, 64)
        _, piv2, _ = pla_lu(pla_session, np.asfortranarray(np.eye(700)), 64)
        ph = pla.PhaseTimes()
        lib.PLA_B200_phase_times(ctypes.byref(ph))
    finally:
        lib.PLA_B200_set_phase_timing(0)
    assert np.count_nonzero(piv2) == 0
    assert ph.interchanges == np.count_nonzero(piv1) > 600
    assert ph.update_launches > 0
