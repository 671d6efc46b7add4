"""Mixed-precision path on the B200, through the C ABI.

 - the tensor-core trailing update (tcgen05, bf16/fp16 operands, fp32
   accumulation, TMA reduce-add into fp32 C) against a plain PyTorch fp32
   product of the same rounded operands;
 - PLA_General_solve_mixed / PLA_Pos_def_solve_mixed reach FP64 backward
   error (<= n * 2^-53) and agree with an FP64 LAPACK solve.
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
    s = pla.Session(nb_distr=128, nb_alg=128)
    yield s, torch, pla
    s.close()


def tc_update(lib, torch, prec, M, N, K, L, U, C, row0, col0, lower=0):
    fn = lib.pla_k_tc_update
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_int] * 4 + [ctypes.c_float, ctypes.c_void_p, ctypes.c_long,
                                        ctypes.c_long, ctypes.c_void_p, ctypes.c_long,
                                        ctypes.c_long, ctypes.c_void_p, ctypes.c_long,
                                        ctypes.c_long, ctypes.c_long, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    status = torch.zeros(4, dtype=torch.int32, device="cuda")
    ldc, ccols = C.shape[1], C.shape[0]   # C stored as a transposed torch tensor (column-major)
    rc = fn(prec, M, N, K, -1.0, L.data_ptr(), L.shape[1], L.shape[0], U.data_ptr(), U.shape[1],
            U.shape[0], C.data_ptr(), ldc, ldc, ccols, row0, col0, lower, status.data_ptr(), None)
    torch.cuda.synchronize()
    assert rc == 0
    assert status[0].item() == 0


@pytest.mark.parametrize("prec,dt", [(1001, "bfloat16"), (1002, "float16")])
@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (300, 257, 128), (1000, 777, 256), (64, 200, 192),
                                   (4096, 3000, 128), (2100, 2100, 256)])
def test_tc_update_matches_fp32_product(env, prec, dt, M, N, K):
    s, torch, pla = env
    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    tdt = getattr(torch, dt)
    rows, cols = M + 8, N + 12
    L = torch.randn(M, K, device="cuda", generator=g).to(tdt).contiguous()
    U = torch.randn(N, K, device="cuda", generator=g).to(tdt).contiguous()
    ld = (rows + 31) // 32 * 32
    Cc = torch.randn(cols, ld, device="cuda", generator=g)   # column-major rows x cols, ld
    ref = Cc.clone()
    r0, c0 = 4, 12
    tc_update(s.lib, torch, prec, M, N, K, L, U, Cc, r0, c0)
    prod = (L.float() @ U.float().T)          # M x N
    ref[c0:c0 + N, r0:r0 + M] -= prod.T
    err = (Cc - ref).abs().max().item()
    assert err <= 1e-5 * K * max(1.0, prod.abs().max().item())
    # everything outside the updated block is untouched
    mask = torch.ones_like(Cc, dtype=torch.bool)
    mask[c0:c0 + N, r0:r0 + M] = False
    assert torch.equal(Cc[mask], ref[mask])


def test_tc_update_lower_tiles(env):
    s, torch, pla = env
    M = N = 512
    K = 128
    g = torch.Generator(device="cuda").manual_seed(3)
    L = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16).contiguous()
    Cc = torch.zeros(N, M, device="cuda")
    tc_update(s.lib, torch, 1001, M, N, K, L, L, Cc, 0, 0, lower=1)
    full = -(L.float() @ L.float().T)
    got = Cc.T
    low = torch.tril(torch.ones(M, N, device="cuda", dtype=torch.bool))
    assert (got[low] - full[low]).abs().max().item() <= 1e-4 * K


@pytest.mark.parametrize("uplo,trans,diag", [("L", "N", "U"), ("U", "N", "N"), ("L", "N", "N"),
                                             ("L", "T", "N")])
@pytest.mark.parametrize("n", [1, 100, 128, 1000, 3001])
def test_single_launch_trsv(env, uplo, trans, diag, n):
    """Ticket-ordered single-kernel solve vs a plain FP64 PyTorch triangular solve."""
    s, torch, pla = env
    lib = s.lib
    g = torch.Generator(device="cuda").manual_seed(n)
    ld = (n + 31) // 32 * 32
    M = torch.randn(n, ld, device="cuda", generator=g) * (0.5 / max(n, 1) ** 0.5)
    M[:, :n] += 2.0 * torch.eye(n, device="cuda")   # well conditioned; memory: column-major A = M'
    Acm = M[:, :n].t()                               # the column-major matrix A as a torch view
    ldd = (n + 127) // 128 * 128
    Dinv = torch.zeros(128, ldd, device="cuda")
    b = torch.randn(n, device="cuda", generator=g)
    x = b.clone()
    status = torch.zeros(4, dtype=torch.int32, device="cuda")
    c = ctypes.c_char
    vp = ctypes.c_void_p
    lib.pla_k_trsv_inv_blocks.argtypes = [ctypes.c_int, c, c, c, ctypes.c_int, vp, ctypes.c_long,
                                          vp, ctypes.c_long, vp]
    lib.pla_k_trsv_ticket.argtypes = [ctypes.c_int, c, c, ctypes.c_int, vp, ctypes.c_long, vp,
                                      ctypes.c_long, vp, vp, vp, vp]
    assert lib.pla_k_trsv_inv_blocks(pla.MPI_FLOAT, uplo.encode(), trans.encode(), diag.encode(),
                                     n, M.data_ptr(), ld, Dinv.data_ptr(), ldd, None) == 0
    assert lib.pla_k_trsv_ticket(pla.MPI_FLOAT, uplo.encode(), trans.encode(), n, M.data_ptr(),
                                 ld, Dinv.data_ptr(), ldd, x.data_ptr(), x.data_ptr(),
                                 status.data_ptr(), None) == 0
    torch.cuda.synchronize()
    assert status[0].item() == 0
    T = torch.tril(Acm) if uplo == "L" else torch.triu(Acm)
    if diag == "U":
        T = T - torch.diag(torch.diag(T)) + torch.eye(n, device="cuda")
    if trans == "T":
        T = T.t()
    ref = torch.linalg.solve_triangular(T.double(), b.double()[:, None],
                                        upper=(uplo == "U") != (trans == "T"))[:, 0]
    err = (x.double() - ref).abs().max().item()
    assert err <= 1e-4 * max(1.0, ref.abs().max().item())


@pytest.mark.parametrize("uplo,trans,diag", [("L", "N", "U"), ("U", "N", "N"), ("L", "N", "N"),
                                             ("L", "T", "N")])
@pytest.mark.parametrize("n", [1, 100, 128, 1000, 3001, 8192])
def test_single_launch_trsv_link_blocks(env, uplo, trans, diag, n):
    """The solve with link blocks (G_i = op(A)(i, p) inv(D_p): the successor of a
    block reads its y before the inverse-block product) against an FP64 solve,
    in place, every triangle and transpose the preconditioner uses."""
    s, torch, pla = env
    lib = s.lib
    g = torch.Generator(device="cuda").manual_seed(n + 7)
    ld = (n + 31) // 32 * 32
    M = torch.randn(n, ld, device="cuda", generator=g) * (0.5 / max(n, 1) ** 0.5)
    M[:, :n] += 2.0 * torch.eye(n, device="cuda")
    Acm = M[:, :n].t()
    ldd = (n + 127) // 128 * 128
    Dinv = torch.zeros(128, ldd, device="cuda")
    G = torch.full((128, ldd), float("nan"), device="cuda")
    b = torch.randn(n, device="cuda", generator=g)
    x = b.clone()
    status = torch.zeros(4, dtype=torch.int32, device="cuda")
    c = ctypes.c_char
    vp = ctypes.c_void_p
    lg = ctypes.c_long
    lib.pla_k_trsv_inv_blocks.argtypes = [ctypes.c_int, c, c, c, ctypes.c_int, vp, lg, vp, lg, vp]
    lib.pla_k_trsv_link_blocks.argtypes = [c, c, ctypes.c_int, vp, lg, vp, lg, vp, vp]
    lib.pla_k_trsv_ticket_link.argtypes = [c, c, ctypes.c_int, vp, lg, vp, lg, vp, vp, vp, vp, vp]
    assert lib.pla_k_trsv_inv_blocks(pla.MPI_FLOAT, uplo.encode(), trans.encode(), diag.encode(),
                                     n, M.data_ptr(), ld, Dinv.data_ptr(), ldd, None) == 0
    assert lib.pla_k_trsv_link_blocks(uplo.encode(), trans.encode(), n, M.data_ptr(), ld,
                                      Dinv.data_ptr(), ldd, G.data_ptr(), None) == 0
    for _ in range(2):   # twice: the second solve reuses the flags and the y buffer
        x.copy_(b)
        assert lib.pla_k_trsv_ticket_link(uplo.encode(), trans.encode(), n, M.data_ptr(), ld,
                                          Dinv.data_ptr(), ldd, G.data_ptr(), x.data_ptr(),
                                          x.data_ptr(), status.data_ptr(), None) == 0
        torch.cuda.synchronize()
        assert status[0].item() == 0
    T = torch.tril(Acm) if uplo == "L" else torch.triu(Acm)
    if diag == "U":
        T = T - torch.diag(torch.diag(T)) + torch.eye(n, device="cuda")
    if trans == "T":
        T = T.t()
    ref = torch.linalg.solve_triangular(T.double(), b.double()[:, None],
                                        upper=(uplo == "U") != (trans == "T"))[:, 0]
    err = (x.double() - ref).abs().max().item()
    assert err <= 1e-4 * max(1.0, ref.abs().max().item())


def solve_mixed(s, pla, A, B, kind, prec, ref, nb=0):
    n = A.shape[0]
    a = s.matrix(n, n)
    s.set(a, A)
    b = s.matrix(*B.shape)
    s.set(b, B)
    p = pla.MixedParams()
    s.lib.PLA_Mixed_params_default(ctypes.byref(p))
    p.precision, p.refinement, p.nb = prec, ref, nb
    rep = pla.MixedReport()
    fn = s.lib.PLA_General_solve_mixed if kind == "lu" else s.lib.PLA_Pos_def_solve_mixed
    rc = pla.check(fn(a, b, ctypes.byref(p), ctypes.byref(rep)), "solve_mixed")
    X = s.get(b)
    A_after = s.get(a)
    s.free(a, b)
    return rc, X, rep, A_after


def backward_error(A, X, B):
    R = B - A @ X
    return (np.abs(R).max(axis=0) /
            (np.abs(A).sum(axis=1).max() * np.abs(X).max(axis=0) + np.abs(B).max(axis=0))).max()


@pytest.mark.parametrize("prec", [1, 2, 3])
@pytest.mark.parametrize("ref", [1, 2])
def test_general_solve_mixed(env, prec, ref):
    """GMRES-IR on a Gaussian matrix (kappa ~ 1e4); classic LU-IR needs
    kappa * u_factor < 1, so it gets a kappa = 10 matrix of the C3 family."""
    s, torch, pla = env
    n = 1536
    rng = np.random.default_rng(prec * 10 + ref)
    if ref == 2:
        A = np.asfortranarray(rng.standard_normal((n, n)))
    else:
        A = c3_matrix(n, 10.0, prec)
    B = np.asfortranarray(rng.standard_normal((n, 3)))
    rc, X, rep, A_after = solve_mixed(s, pla, A, B, "lu", prec, ref)
    assert rc == 0 and rep.converged == 1, (rep.iterations, rep.backward_error)
    assert np.array_equal(A_after, A)              # A is read, never overwritten
    eta = backward_error(A, X, B)
    assert eta <= n * 2.0 ** -53
    assert abs(eta - rep.backward_error) <= 0.5 * max(eta, rep.backward_error) + 1e-18
    Xr = np.linalg.solve(A, B)
    assert np.abs(X - Xr).max() <= 1e-10 * np.abs(Xr).max() * np.linalg.cond(A) ** 0.5


def c3_matrix(n, kappa, seed):
    """A = U diag(sigma) V' with sigma geometric 1 -> 1/kappa and U, V products of
    8 Householder reflectors with seeded Gaussian vectors."""
    rng = np.random.default_rng(seed)
    sigma = kappa ** (-np.arange(n) / (n - 1))
    A = np.diag(sigma)
    for _ in range(8):
        v = rng.standard_normal(n)
        A -= (2.0 / (v @ v)) * np.outer(v, v @ A)
    for _ in range(8):
        v = rng.standard_normal(n)
        A -= (2.0 / (v @ v)) * np.outer(A @ v, v)
    return np.asfortranarray(A)


@pytest.mark.parametrize("kappa", [1e2, 1e6])
def test_gmres_ir_c3_family(env, kappa):
    s, torch, pla = env
    n = 2048
    A = c3_matrix(n, kappa, 7)
    x_true = np.random.default_rng(8).standard_normal((n, 1))
    B = A @ x_true
    rc, X, rep, _ = solve_mixed(s, pla, A, B, "lu", 2, 2)
    assert rep.converged == 1, (rep.iterations, rep.backward_error)
    assert backward_error(A, X, B) <= n * 2.0 ** -53


@pytest.mark.parametrize("prec", [1, 2])
def test_pos_def_solve_mixed(env, prec):
    s, torch, pla = env
    n = 1280
    rng = np.random.default_rng(prec)
    G = rng.standard_normal((n, n))
    A = np.asfortranarray(G @ G.T / n + np.eye(n))
    B = np.asfortranarray(rng.standard_normal((n, 2)))
    rc, X, rep, _ = solve_mixed(s, pla, A, B, "chol", prec, 2)
    assert rc == 0 and rep.converged == 1, (rep.iterations, rep.backward_error)
    assert backward_error(A, X, B) <= n * 2.0 ** -53


def test_pos_def_mixed_reports_not_spd(env):
    s, torch, pla = env
    n = 256
    A = np.asfortranarray(np.eye(n))
    A[100, 100] = -1.0
    B = np.ones((n, 1), order="F")
    rc, X, rep, _ = solve_mixed(s, pla, A, B, "chol", 2, 1)
    assert rc == 101 and rep.info == 101


def solve_mixed_params(s, pla, A, B, kind, **kw):
    n = A.shape[0]
    a = s.matrix(n, n)
    s.set(a, A)
    b = s.matrix(*B.shape)
    s.set(b, B)
    p = pla.MixedParams()
    s.lib.PLA_Mixed_params_default(ctypes.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    rep = pla.MixedReport()
    fn = s.lib.PLA_General_solve_mixed if kind == "lu" else s.lib.PLA_Pos_def_solve_mixed
    rc = fn(a, b, ctypes.byref(p), ctypes.byref(rep))
    X = s.get(b)
    s.free(a, b)
    return rc, X, rep


def haar_matrix(n, kappa, seed):
    """A = Q1 diag(sigma) Q2' with Q1, Q2 dense orthogonal (QR of Gaussian
    matrices): unlike the C3 family, its LU factors' diagonal spreads over
    only about sqrt(kappa), so the diagonal-range rule does not fire."""
    rng = np.random.default_rng(seed)
    q1 = np.linalg.qr(rng.standard_normal((n, n)))[0]
    q2 = np.linalg.qr(rng.standard_normal((n, n)))[0]
    sigma = kappa ** (-np.arange(n) / (n - 1))
    return np.asfortranarray((q1 * sigma) @ q2.T)


@pytest.mark.parametrize("prec", [1, 2])
def test_kappa_1e10_escalates_to_split_factors(env, prec):
    """kappa = 1e10 is out of reach of bf16/fp16 factors (kappa * u_f >> 1).
    The C3 family's factors show it on their diagonal (range about kappa), so
    the solver refactors with bf16 x 6 operands at once, without refining
    the first factors, and ends at FP64 backward error; the forward error is
    checked against the FP64 LAPACK solution."""
    s, torch, pla = env
    n = 2048
    A = c3_matrix(n, 1e10, 11)
    x_true = np.random.default_rng(12).standard_normal((n, 1))
    B = A @ x_true
    rc, X, rep = solve_mixed_params(s, pla, A, B, "lu", precision=prec, refinement=2)
    assert rc == 0 and rep.converged == 1, (rep.iterations, rep.backward_error)
    assert (rep.precision_used, rep.factorizations) == (pla.PLA_B200_PREC_BF16X6, 2), \
        (rep.precision_used, rep.factorizations, rep.iterations, rep.inner_iterations)
    assert rep.inner_iterations <= 60, rep.inner_iterations
    assert backward_error(A, X, B) <= n * 2.0 ** -53
    Xr = np.linalg.solve(A, B)
    fwd = np.abs(X - Xr).max() / np.abs(Xr).max()
    assert fwd <= 1e10 * n * 2.0 ** -53, fwd


@pytest.mark.parametrize("refinement,max_steps", [(1, 2), (2, 1)])
def test_stagnation_rule_per_refinement(env, refinement, max_steps):
    """How many non-halving steps escalate: one GMRES-IR step (a whole restart
    cycle), two classic LU-IR steps.  A dense-orthogonal kappa = 1e10 matrix
    passes the diagonal-range rule with fp16 factors but stagnates at once,
    so the fp16 attempt ends after max_steps corrections and higher
    factors (bf16 x 6, then FP64 if those stagnate too) finish the solve."""
    s, torch, pla = env
    n = 1024
    A = haar_matrix(n, 1e10, 17)
    B = A @ np.random.default_rng(18).standard_normal((n, 1))
    rc, X, rep = solve_mixed_params(s, pla, A, B, "lu", precision=2, refinement=refinement)
    assert rc == 0 and rep.converged == 1
    assert rep.factorizations >= 2
    assert rep.precision_used in (pla.PLA_B200_PREC_BF16X6, pla.PLA_B200_PREC_FP64)
    # the fp16 attempt takes at most max_steps corrections, the later ones a few
    assert rep.iterations <= max_steps + 2 * 3, rep.iterations
    if refinement == 2:  # one restart cycle of fp16 GMRES (30), then short cycles
        assert rep.inner_iterations <= 30 + 40, rep.inner_iterations
    assert backward_error(A, X, B) <= n * 2.0 ** -53


def test_bf16x6_factors(env):
    """bf16 x 6 factors requested: fp32-level preconditioner, a few GMRES
    iterations at kappa = 1e6 where fp16 factors need a dozen or more."""
    s, torch, pla = env
    n = 3000
    A = c3_matrix(n, 1e6, 21)
    B = A @ np.random.default_rng(22).standard_normal((n, 2))
    rc, X, rep = solve_mixed_params(s, pla, A, B, "lu", precision=pla.PLA_B200_PREC_BF16X6,
                                    refinement=2, nb=256)
    assert rc == 0 and rep.converged == 1 and rep.factorizations == 1
    assert rep.precision_used == pla.PLA_B200_PREC_BF16X6
    assert rep.inner_iterations <= 2 * 6, rep.inner_iterations
    assert backward_error(A, X, B) <= n * 2.0 ** -53


@pytest.mark.parametrize("kind", ["lu", "chol"])
def test_bf16x3_factors(env, kind):
    """bf16 x 3 factors (operands split two ways, three part products): FP64
    backward error with fewer GMRES iterations than fp16 factors need."""
    s, torch, pla = env
    n = 3000
    A = c3_matrix(n, 1e6, 23) if kind == "lu" else spd_family(n, 1e5, 24)
    B = np.asfortranarray(A @ np.random.default_rng(24).standard_normal((n, 2)))
    its = {}
    for prec in (pla.PLA_B200_PREC_FP16, pla.PLA_B200_PREC_BF16X3):
        rc, X, rep = solve_mixed_params(s, pla, A, B, kind, precision=prec, refinement=2)
        assert rc == 0 and rep.converged == 1, (prec, rep.iterations, rep.backward_error)
        assert rep.precision_used == prec and rep.factorizations == 1
        assert backward_error(A, X, B) <= n * 2.0 ** -53
        its[prec] = rep.inner_iterations
    assert its[pla.PLA_B200_PREC_BF16X3] < its[pla.PLA_B200_PREC_FP16], its


@pytest.mark.parametrize("kappa", [1e3, 1e7])
def test_bf16x6_cholesky(env, kappa):
    s, torch, pla = env
    n = 2048
    A = spd_family(n, kappa, 33)
    B = np.asfortranarray(A @ np.random.default_rng(34).standard_normal((n, 4)))
    rc, X, rep = solve_mixed_params(s, pla, A, B, "chol", precision=pla.PLA_B200_PREC_BF16X6,
                                    refinement=2)
    assert rc == 0 and rep.converged == 1, (rep.iterations, rep.backward_error)
    assert rep.precision_used in (pla.PLA_B200_PREC_BF16X6, pla.PLA_B200_PREC_FP64)
    if kappa == 1e3:
        assert rep.precision_used == pla.PLA_B200_PREC_BF16X6
    assert backward_error(A, X, B) <= n * 2.0 ** -53


def pack_split(lib, torch, X, nseg, code):
    """pla_k_pack_split_ex of the column-major m x k float32 tensor X (stored
    as X' row-major), rows of nseg k-wide segments."""
    fn = lib.pla_k_pack_split_ex
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_long, ctypes.c_long,
                   ctypes.c_void_p, ctypes.c_long, ctypes.c_int, ctypes.c_uint, ctypes.c_int,
                   ctypes.c_void_p]
    k, m = X.shape
    out = torch.zeros(m, nseg * k, dtype=torch.bfloat16, device="cuda")
    assert fn(m, k, X.data_ptr(), 1, m, out.data_ptr(), nseg * k, nseg, code, 0, None) == 0
    torch.cuda.synchronize()
    return out


def test_pack_split_three_parts(env):
    """x = p0 + p1 + p2 in bf16 parts, to within fp32 rounding; segment codes
    place the parts."""
    s, torch, pla = env
    g = torch.Generator(device="cuda").manual_seed(5)
    m, k = 300, 70
    X = (torch.randn(k, m, device="cuda", generator=g) *
         torch.exp(torch.randn(k, m, device="cuda", generator=g) * 4))
    out = pack_split(s.lib, torch, X, 3, 0 | (1 << 2) | (2 << 4)).float()
    x = X.t()                                                  # m x k, element (i, kk)
    p0, p1, p2 = out[:, :k], out[:, k:2 * k], out[:, 2 * k:]
    assert torch.equal(p0, x.to(torch.bfloat16).float())
    assert torch.equal(p1, (x - p0).to(torch.bfloat16).float())
    rec = (p0.double() + p1.double()) + p2.double()
    assert ((rec - x.double()).abs() <= x.double().abs() * 2.0 ** -24).all()
    six = pack_split(s.lib, torch, X, 6, 0x910).float()       # [0 0 1 0 1 2]
    for seg, part in enumerate([p0, p0, p1, p0, p1, p2]):
        assert torch.equal(six[:, seg * k:(seg + 1) * k], part)


def test_tc_update_bf16x6_is_fp32_accurate(env):
    """One K = 6b tensor-core product of bf16 x 6 split operands against the
    float64 product of the fp32 operands: within a few fp32 roundings, far
    inside what bf16 operands alone give."""
    s, torch, pla = env
    g = torch.Generator(device="cuda").manual_seed(7)
    M, N, b = 1000, 900, 256
    Lf = torch.randn(b, M, device="cuda", generator=g)          # column-major M x b
    Uf = torch.randn(b, N, device="cuda", generator=g)          # U' column-major N x b
    La = pack_split(s.lib, torch, Lf, 6, 0x124)                # [0 1 2 0 1 0]
    Ub = pack_split(s.lib, torch, Uf, 6, 0x46)                 # [2 1 0 1 0 0]
    ld = (M + 31) // 32 * 32
    Cc = torch.zeros(N, ld, device="cuda")
    tc_update(s.lib, torch, 1001, M, N, 6 * b, La, Ub, Cc, 0, 0)
    ref = -(Lf.t().double() @ Uf.double())                     # M x N
    err = (Cc[:, :M].t().double() - ref).abs().max().item()
    assert err <= 8 * b * 2.0 ** -24 * (Lf.abs().max() * Uf.abs().max()).item(), err
    lo = -(Lf.t().to(torch.bfloat16).double() @ Uf.to(torch.bfloat16).double())
    assert err < 0.01 * (lo - ref).abs().max().item()


def test_no_escalation_reports_stagnation(env):
    s, torch, pla = env
    n = 1024
    A = c3_matrix(n, 1e10, 13)
    B = A @ np.ones((n, 1))
    rc, X, rep = solve_mixed_params(s, pla, A, B, "lu", precision=1, refinement=1, escalate=0,
                                    max_iterations=6)
    assert rc == 0 and rep.factorizations == 1 and rep.precision_used == 1
    assert rep.converged == 0 and rep.iterations <= 6


@pytest.mark.parametrize("kind", ["lu", "chol"])
def test_fp64_precision_requested(env, kind):
    s, torch, pla = env
    n = 777
    rng = np.random.default_rng(14)
    G = rng.standard_normal((n, n))
    A = np.asfortranarray(G if kind == "lu" else G @ G.T / n + np.eye(n))
    B = np.asfortranarray(rng.standard_normal((n, 2)))
    rc, X, rep = solve_mixed_params(s, pla, A, B, kind, precision=pla.PLA_B200_PREC_FP64)
    assert rc == 0 and rep.converged == 1 and rep.precision_used == pla.PLA_B200_PREC_FP64
    assert backward_error(A, X, B) <= n * 2.0 ** -53


@pytest.mark.parametrize("prec", [1, 2])
def test_sixteen_right_hand_sides(env, prec):
    s, torch, pla = env
    n = 1024
    A = c3_matrix(n, 1e6, 15)
    Xt = np.random.default_rng(16).standard_normal((n, 16))
    B = np.asfortranarray(A @ Xt)
    rc, X, rep = solve_mixed_params(s, pla, A, B, "lu", precision=prec, refinement=2)
    assert rc == 0 and rep.converged == 1, (rep.iterations, rep.backward_error)
    assert backward_error(A, X, B) <= n * 2.0 ** -53
    Xr = np.linalg.solve(A, B)
    assert np.abs(X - Xr).max() / np.abs(Xr).max() <= 1e6 * n * 2.0 ** -53


def fp8_pack(lib, torch, X, si_rows=True):
    """Pack the rows of X (fp32, m x k) with pla_k_pack_fp8; returns (bytes
    m x k uint8, inverse scales per 128 rows)."""
    m, k = X.shape
    Xc = X.t().contiguous() if si_rows else X.contiguous()  # column-major or row-major source
    si, sk = (1, m) if si_rows else (k, 1)
    dst = torch.zeros(m, k, dtype=torch.uint8, device="cuda")
    inv = torch.zeros((m + 127) // 128, dtype=torch.float32, device="cuda")
    fn = lib.pla_k_pack_fp8
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_long, ctypes.c_long,
                   ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p, ctypes.c_void_p]
    assert fn(m, k, Xc.data_ptr(), si, sk, dst.data_ptr(), k, inv.data_ptr(), None) == 0
    torch.cuda.synchronize()
    return dst, inv


@pytest.mark.parametrize("si_rows", [True, False])
def test_fp8_pack_scales_and_bytes(env, si_rows):
    s, torch, pla = env
    g = torch.Generator(device="cuda").manual_seed(21)
    m, k = 300, 128
    X = torch.randn(m, k, device="cuda", generator=g) * torch.logspace(-3, 3, m, device="cuda")[:, None]
    q, inv = fp8_pack(s.lib, torch, X, si_rows)
    for b in range(inv.numel()):
        blk = X[128 * b:128 * b + 128]
        scale = 1.0 / inv[b].item()
        assert scale == 2.0 ** round(np.log2(scale))           # a power of two
        amax = blk.abs().max().item()
        assert amax * scale <= 448.0 < 2 * amax * scale        # the largest that fits
        want = (blk * scale).to(torch.float8_e4m3fn).view(torch.uint8)
        assert torch.equal(q[128 * b:128 * b + 128], want)     # round to nearest even


@pytest.mark.parametrize("M,N,K", [(128, 128, 128), (1000, 777, 256), (4096, 3000, 128)])
def test_tc_update_fp8_matches_dequantized_product(env, M, N, K):
    s, torch, pla = env
    g = torch.Generator(device="cuda").manual_seed(M + N)
    L = torch.randn(M, K, device="cuda", generator=g) * 3.0
    U = torch.randn(N, K, device="cuda", generator=g) * 0.01
    Lq, il = fp8_pack(s.lib, torch, L)
    Uq, iu = fp8_pack(s.lib, torch, U)
    deq = lambda q, inv: q.view(torch.float8_e4m3fn).float() * inv.repeat_interleave(128)[:q.shape[0], None]
    ld = (M + 8 + 31) // 32 * 32
    Cc = torch.randn(N + 12, ld, device="cuda", generator=g)
    ref = Cc.clone()
    r0, c0 = 4, 12
    status = torch.zeros(4, dtype=torch.int32, device="cuda")
    fn = s.lib.pla_k_tc_update_fp8
    fn.restype = ctypes.c_int
    vp, lg, i = ctypes.c_void_p, ctypes.c_long, ctypes.c_int
    fn.argtypes = [i, i, i, ctypes.c_float, vp, lg, lg, vp, vp, lg, lg, vp, vp, lg, lg, lg, i, i,
                   i, vp, vp]
    rc = fn(M, N, K, -1.0, Lq.data_ptr(), K, M, il.data_ptr(), Uq.data_ptr(), K, N, iu.data_ptr(),
            Cc.data_ptr(), ld, ld, N + 12, r0, c0, 0, status.data_ptr(), None)
    torch.cuda.synchronize()
    assert rc == 0 and status[0].item() == 0
    prod = deq(Lq, il) @ deq(Uq, iu).T
    ref[c0:c0 + N, r0:r0 + M] -= prod.T
    assert (Cc - ref).abs().max().item() <= 1e-5 * K * max(1.0, prod.abs().max().item())
    mask = torch.ones_like(Cc, dtype=torch.bool)
    mask[c0:c0 + N, r0:r0 + M] = False
    assert torch.equal(Cc[mask], ref[mask])


def spd_family(n, kappa, seed):
    """A = Q diag(lambda) Q' with lambda log-uniform in [1/kappa, 1] and Q a
    product of 8 Householder reflectors with seeded Gaussian vectors."""
    rng = np.random.default_rng(seed)
    lam = np.exp(rng.uniform(np.log(1.0 / kappa), 0.0, n))
    lam[0], lam[-1] = 1.0, 1.0 / kappa
    A = np.diag(lam)
    for _ in range(8):
        v = rng.standard_normal(n)
        A -= (2.0 / (v @ v)) * np.outer(v, v @ A)
        A -= (2.0 / (v @ v)) * np.outer(A @ v, v)
    return np.asfortranarray((A + A.T) / 2)


@pytest.mark.parametrize("kappa", [1e3, 1e7])
def test_fp8_cholesky_ir(env, kappa):
    """FP8 E4M3 trailing updates with per-tile scaling and diagonal scaling,
    8 right-hand sides: FP64 backward error, forward error against LAPACK;
    the solver may escalate past FP8 (reported in precision_used)."""
    s, torch, pla = env
    n = 2048
    A = spd_family(n, kappa, 31)
    Xt = np.random.default_rng(32).standard_normal((n, 8))
    B = np.asfortranarray(A @ Xt)
    rc, X, rep = solve_mixed_params(s, pla, A, B, "chol", precision=pla.PLA_B200_PREC_FP8,
                                    refinement=2)
    assert rc == 0 and rep.converged == 1, (rep.iterations, rep.backward_error)
    assert rep.precision_used in (pla.PLA_B200_PREC_FP8, 1, 3, 4, pla.PLA_B200_PREC_BF16X6)
    assert backward_error(A, X, B) <= n * 2.0 ** -53
    Xr = np.linalg.solve(A, B)
    assert np.abs(X - Xr).max() / np.abs(Xr).max() <= kappa * n * 2.0 ** -53


def test_fp8_lu_ir(env):
    s, torch, pla = env
    n = 1536
    A = c3_matrix(n, 1e2, 33)
    B = np.asfortranarray(A @ np.random.default_rng(34).standard_normal((n, 2)))
    rc, X, rep = solve_mixed_params(s, pla, A, B, "lu", precision=pla.PLA_B200_PREC_FP8,
                                    refinement=2)
    assert rc == 0 and rep.converged == 1, (rep.iterations, rep.backward_error)
    assert backward_error(A, X, B) <= n * 2.0 ** -53


@pytest.mark.parametrize("prec,nb", [(2, 256), (5, 128), (2, 64)])   # 64: split first group
def test_streamed_solve_from_host(env, prec, nb):
    """PLA_General_solve_mixed_host copies A from host memory while the
    factorization runs: FP64 backward error, A copied into the device object,
    and a bitwise-identical solution whether the copy overlaps (page-locked
    memory) or not (pageable memory), because each column group replays the
    steps it missed in order."""
    s, torch, pla = env
    n = 8192
    A = c3_matrix(n, 1e3, 41)
    Xt = np.random.default_rng(42).standard_normal((n, 1))
    B = np.asfortranarray(A @ Xt)
    pinned = torch.empty((n, n), dtype=torch.float64, pin_memory=True)
    pinned.numpy()[:] = A.T          # row-major view of the column-major matrix
    pageable = np.ascontiguousarray(A.T)
    sols = []
    for host in (pinned.data_ptr(), pageable.ctypes.data):
        a = s.matrix(n, n)
        b = s.matrix(n, 1)
        s.set(b, B)
        p = pla.MixedParams()
        s.lib.PLA_Mixed_params_default(ctypes.byref(p))
        p.precision, p.refinement, p.nb = prec, 2, nb
        rep = pla.MixedReport()
        rc = s.lib.PLA_General_solve_mixed_host(a, ctypes.c_void_p(host), n, b, ctypes.byref(p),
                                                ctypes.byref(rep))
        assert rc == 0 and rep.converged == 1, (rep.iterations, rep.backward_error)
        assert np.array_equal(s.get(a), A)
        X = s.get(b)
        assert backward_error(A, X, B) <= n * 2.0 ** -53
        sols.append(X)
        s.free(a, b)
    assert np.array_equal(sols[0], sols[1])


def test_streamed_solve_small_order_copies_first(env):
    s, torch, pla = env
    n = 1000
    A = c3_matrix(n, 1e2, 43)
    B = np.asfortranarray(A @ np.ones((n, 2)))
    host = np.ascontiguousarray(A.T)
    a, b = s.matrix(n, n), s.matrix(n, 2)
    s.set(b, B)
    p = pla.MixedParams()
    s.lib.PLA_Mixed_params_default(ctypes.byref(p))
    rep = pla.MixedReport()
    rc = s.lib.PLA_General_solve_mixed_host(a, ctypes.c_void_p(host.ctypes.data), n, b,
                                            ctypes.byref(p), ctypes.byref(rep))
    assert rc == 0 and rep.converged == 1
    assert backward_error(A, s.get(b), B) <= n * 2.0 ** -53
    s.free(a, b)


@pytest.mark.parametrize("uplo,trans,diag", [("L", "N", "U"), ("U", "N", "N"), ("L", "N", "N"),
                                             ("L", "T", "N")])
@pytest.mark.parametrize("n,ld,nrhs", [(3001, 3008, 16), (2048, 2048, 3), (1500, 1501, 8)])
def test_trsv_ticket_multi(env, uplo, trans, diag, n, ld, nrhs):
    """The single-launch solve for several fp32 right-hand sides (the GMRES-IR
    preconditioner of a multi-rhs solve) against an FP64 solve of the same
    data: every triangle and transpose the preconditioner uses, ragged orders,
    a leading dimension that rules out the vector loads, and in-place use."""
    s, torch, pla = env
    lib = s.lib
    for name, args in (("pla_k_trsv_inv_blocks", [ctypes.c_int, ctypes.c_char, ctypes.c_char,
                                                  ctypes.c_char, ctypes.c_int, ctypes.c_void_p,
                                                  ctypes.c_long, ctypes.c_void_p, ctypes.c_long,
                                                  ctypes.c_void_p]),
                       ("pla_k_trsv_ticket_multi", [ctypes.c_char, ctypes.c_char, ctypes.c_int,
                                                    ctypes.c_int, ctypes.c_void_p, ctypes.c_long,
                                                    ctypes.c_void_p, ctypes.c_long,
                                                    ctypes.c_void_p, ctypes.c_long,
                                                    ctypes.c_void_p, ctypes.c_long,
                                                    ctypes.c_void_p, ctypes.c_void_p])):
        getattr(lib, name).argtypes = args
        getattr(lib, name).restype = ctypes.c_int
    g = torch.Generator(device="cuda").manual_seed(n + nrhs)
    M = torch.randn(n, n, device="cuda", generator=g, dtype=torch.float64) * (0.5 / n ** 0.5)
    T = torch.tril(M, -1) if uplo == "L" else torch.triu(M, 1)
    T.diagonal().copy_(1.0 + torch.rand(n, device="cuda", generator=g, dtype=torch.float64))
    T32 = T.float()
    # column-major n x n with leading dimension ld: row-major (n, ld) of the transpose
    Acm = torch.zeros(n, ld, device="cuda", dtype=torch.float32)
    Acm[:, :n] = T32.t()
    ldd = (n + 127) // 128 * 128
    dinv = torch.zeros(128, ldd, device="cuda", dtype=torch.float32)
    st = torch.zeros(4, dtype=torch.int32, device="cuda")
    assert lib.pla_k_trsv_inv_blocks(pla.MPI_FLOAT, uplo.encode(), trans.encode(), diag.encode(), n,
                                     Acm.data_ptr(), ld, dinv.data_ptr(), ldd, None) == 0
    B = torch.randn(nrhs, n, device="cuda", generator=g, dtype=torch.float32)  # column-major n x nrhs
    X = B.clone()
    assert lib.pla_k_trsv_ticket_multi(uplo.encode(), trans.encode(), n, nrhs, Acm.data_ptr(), ld,
                                       dinv.data_ptr(), ldd, X.data_ptr(), n, X.data_ptr(), n,
                                       st.data_ptr(), None) == 0
    torch.cuda.synchronize()
    assert st[0].item() == 0
    Td = T32.double()
    if diag == "U":
        Td.diagonal().fill_(1.0)
    op = Td.t() if trans == "T" else Td
    ref = torch.linalg.solve_triangular(op, B.double().t(), upper=(uplo == "U") != (trans == "T"))
    err = (X.double().t() - ref).abs().max().item()
    assert err <= 64 * n * np.finfo(np.float32).eps * ref.abs().max().item(), err


@pytest.mark.parametrize("uplo,trans,diag", [("L", "N", "U"), ("U", "N", "N"), ("L", "N", "N"),
                                             ("L", "T", "N")])
@pytest.mark.parametrize("n,ld,nrhs", [(1000, 1000, 1), (4096, 4096, 8), (777, 781, 16)])
def test_trsv_ticket_multi_f64(env, uplo, trans, diag, n, ld, nrhs):
    """The FP64 form on an fp32 triangle (the preconditioner of bf16 x 6
    factors): FP64 right-hand sides, FP64 inverse diagonal blocks and
    arithmetic, so the result matches an FP64 solve with the same fp32 values
    to FP64 rounding, not fp32."""
    s, torch, pla = env
    lib = s.lib
    for name, args in (("pla_k_trsv_inv_blocks_f64", [ctypes.c_char, ctypes.c_char, ctypes.c_char,
                                                      ctypes.c_int, ctypes.c_void_p, ctypes.c_long,
                                                      ctypes.c_void_p, ctypes.c_long,
                                                      ctypes.c_void_p]),
                       ("pla_k_trsv_ticket_multi_f64", [ctypes.c_char, ctypes.c_char, ctypes.c_int,
                                                        ctypes.c_int, ctypes.c_void_p,
                                                        ctypes.c_long, ctypes.c_void_p,
                                                        ctypes.c_long, ctypes.c_void_p,
                                                        ctypes.c_long, ctypes.c_void_p,
                                                        ctypes.c_long, ctypes.c_void_p,
                                                        ctypes.c_void_p])):
        getattr(lib, name).argtypes = args
        getattr(lib, name).restype = ctypes.c_int
    g = torch.Generator(device="cuda").manual_seed(n + nrhs + 1)
    M = torch.randn(n, n, device="cuda", generator=g, dtype=torch.float64) * (0.5 / n ** 0.5)
    T = torch.tril(M, -1) if uplo == "L" else torch.triu(M, 1)
    T.diagonal().copy_(1.0 + torch.rand(n, device="cuda", generator=g, dtype=torch.float64))
    T32 = T.float()
    Acm = torch.zeros(n, ld, device="cuda", dtype=torch.float32)
    Acm[:, :n] = T32.t()
    ldd = (n + 127) // 128 * 128
    dinv = torch.zeros(128, ldd, device="cuda", dtype=torch.float64)
    st = torch.zeros(4, dtype=torch.int32, device="cuda")
    assert lib.pla_k_trsv_inv_blocks_f64(uplo.encode(), trans.encode(), diag.encode(), n,
                                         Acm.data_ptr(), ld, dinv.data_ptr(), ldd, None) == 0
    B = torch.randn(nrhs, n, device="cuda", generator=g, dtype=torch.float64)
    X = B.clone()
    assert lib.pla_k_trsv_ticket_multi_f64(uplo.encode(), trans.encode(), n, nrhs, Acm.data_ptr(),
                                           ld, dinv.data_ptr(), ldd, X.data_ptr(), n, X.data_ptr(),
                                           n, st.data_ptr(), None) == 0
    torch.cuda.synchronize()
    assert st[0].item() == 0
    Td = T32.double()
    if diag == "U":
        Td.diagonal().fill_(1.0)
    op = Td.t() if trans == "T" else Td
    ref = torch.linalg.solve_triangular(op, B.t(), upper=(uplo == "U") != (trans == "T"))
    err = (X.t() - ref).abs().max().item()
    assert err <= 64 * n * np.finfo(np.float64).eps * ref.abs().max().item(), err
