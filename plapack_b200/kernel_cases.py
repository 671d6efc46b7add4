"""Run one kernel of the library at a stated size, through its C ABI, for
profiling and timing.  Every case allocates its operands with torch on
cuda:0, launches the kernel `--reps` times after `--warmup` launches, and
prints the mean CUDA-event time per launch with the kernel's algorithmic
bytes or flops and the rate they imply.

    python -m plapack_b200.kernel_cases dgemm --m 16384 --n 16384 --k 128
    python -m plapack_b200.kernel_cases tc_update --m 8192 --n 8192 --k 256
    python -m plapack_b200.kernel_cases tc_update_fp8 --m 8192 --n 8192 --k 256
    python -m plapack_b200.kernel_cases panel --m 32768 --k 32 [--dtype f64]
    python -m plapack_b200.kernel_cases laswp --m 32768 --n 32768 --k 256
    python -m plapack_b200.kernel_cases trsv --n 32768
    python -m plapack_b200.kernel_cases residual --n 32768
    python -m plapack_b200.kernel_cases batched --count 2000
    python -m plapack_b200.kernel_cases potrf --k 128 --dtype f64
    python -m plapack_b200.kernel_cases trsm_small --side R --m 32768 --k 128 --dtype f64
    python -m plapack_b200.kernel_cases sgemm --m 32768 --n 224 --k 32
    python -m plapack_b200.kernel_cases panel_blocked --m 32768 --n 256 --ctas 72
    python -m plapack_b200.kernel_cases panel_update --m 32768 --n 224 --k 32
    python -m plapack_b200.kernel_cases trtri --m 32768 --k 256

The cases mirror the calls the solvers make (the trailing update of one LU
step, one 32-column sub-panel, the row interchanges of one panel, the
single-launch triangular solve and the FP64 residual of the refinement, one
batched factor-and-solve).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import sys

import numpy as np

from . import pla

vp, lg, i32, f32, f64 = ctypes.c_void_p, ctypes.c_long, ctypes.c_int, ctypes.c_float, ctypes.c_double
ch = ctypes.c_char


def _fn(lib, name, argtypes):
    f = getattr(lib, name)
    f.argtypes = argtypes
    f.restype = ctypes.c_int
    return f


def _time(torch, launch, warmup, reps):
    for _ in range(warmup):
        rc = launch()
        assert rc == 0, rc
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        launch()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3 / reps


def case_dgemm(torch, lib, a):
    m, n, k = a.m, a.n, a.k
    A = torch.randn(k, m, dtype=torch.float64, device="cuda")   # column-major m x k
    B = torch.randn(n, k, dtype=torch.float64, device="cuda")   # column-major k x n
    C = torch.randn(n, m, dtype=torch.float64, device="cuda")   # column-major m x n
    g = _fn(lib, "pla_k_gemm", [i32] * 6 + [f64, vp, lg, vp, lg, f64, vp, lg, i32, vp, vp])
    t = _time(torch, lambda: g(pla.MPI_DOUBLE, pla.PLA_NO_TRANSPOSE, pla.PLA_NO_TRANSPOSE, m, n, k,
                               -1.0, A.data_ptr(), m, B.data_ptr(), k, 1.0, C.data_ptr(), m, 0,
                               None, None), a.warmup, a.reps)
    fl = 2.0 * m * n * k
    return {"case": f"FP64 trailing update C -= A B, m={m} n={n} k={k}", "s": t,
            "tflops": fl / t / 1e12}


def _tc(torch, lib, a, fp8):
    m, n, k = a.m, a.n, a.k
    ld = (m + 31) // 32 * 32
    C = torch.randn(n, ld, dtype=torch.float32, device="cuda")
    st = torch.zeros(4, dtype=torch.int32, device="cuda")
    if fp8:
        L = torch.randint(0, 120, (m, k), dtype=torch.uint8, device="cuda")
        U = torch.randint(0, 120, (n, k), dtype=torch.uint8, device="cuda")
        il = torch.full(((m + 127) // 128,), 2.0 ** -8, device="cuda")
        iu = torch.full(((n + 127) // 128,), 2.0 ** -8, device="cuda")
        g = _fn(lib, "pla_k_tc_update_fp8", [i32, i32, i32, f32, vp, lg, lg, vp, vp, lg, lg, vp, vp,
                                             lg, lg, lg, i32, i32, i32, vp, vp])
        launch = lambda: g(m, n, k, -1.0, L.data_ptr(), k, m, il.data_ptr(), U.data_ptr(), k, n,
                           iu.data_ptr(), C.data_ptr(), ld, ld, n, 0, 0, 0, st.data_ptr(), None)
        esz = 1
    else:
        L = torch.randn(m, k, device="cuda").half()
        U = torch.randn(n, k, device="cuda").half()
        g = _fn(lib, "pla_k_tc_update", [i32] * 4 + [f32, vp, lg, lg, vp, lg, lg, vp, lg, lg, lg,
                                                     i32, i32, i32, vp, vp])
        launch = lambda: g(1002, m, n, k, -1.0, L.data_ptr(), k, m, U.data_ptr(), k, n,
                           C.data_ptr(), ld, ld, n, 0, 0, 0, st.data_ptr(), None)
        esz = 2
    t = _time(torch, launch, a.warmup, a.reps)
    assert st[0].item() == 0
    byt = m * n * 8.0 + (m + n) * k * esz
    return {"case": f"tensor-core trailing update ({'fp8 e4m3' if fp8 else 'fp16'}), m={m} n={n} "
                    f"k={k}", "s": t, "algorithmic_bytes": byt, "gbs": byt / t / 1e9,
            "tflops": 2.0 * m * n * k / t / 1e12}


def case_tc_update(torch, lib, a):
    return _tc(torch, lib, a, False)


def case_tc_update_fp8(torch, lib, a):
    return _tc(torch, lib, a, True)


def case_panel(torch, lib, a):
    r, w = a.m, a.k
    dt = pla.MPI_DOUBLE if a.dtype == "f64" else pla.MPI_FLOAT
    tdt = torch.float64 if a.dtype == "f64" else torch.float32
    A0 = torch.randn(w, r, dtype=tdt, device="cuda")
    A = A0.clone()
    piv = torch.zeros(w, dtype=torch.int32, device="cuda")
    st = torch.zeros(4, dtype=torch.int32, device="cuda")
    g = _fn(lib, "pla_k_lu_panel_ex", [i32, i32, i32, vp, lg, vp, vp, vp, i32, i32, vp])

    def launch():
        A.copy_(A0)
        return g(dt, r, w, A.data_ptr(), r, piv.data_ptr(), st.data_ptr(), None, 0, a.ctas, None)

    t = _time(torch, launch, a.warmup, a.reps)
    assert st[0].item() == 0
    es = 8 if dt == pla.MPI_DOUBLE else 4
    return {"case": f"panel LU {r} x {w} ({a.dtype}), at most {a.ctas or 'one per SM'} CTAs, "
                    f"copy of the panel included", "s": t,
            "us_per_column": t / w * 1e6, "bytes_read_written": 2.0 * r * w * es,
            "gbs": 2.0 * r * w * es / t / 1e9}


def case_tslu(torch, lib, a):
    """The tournament-pivoted fp32 panel (select + apply launches)."""
    r, w = a.m, a.k
    A0 = torch.randn(w, r, dtype=torch.float32, device="cuda")
    A = A0.clone()
    piv = torch.zeros(w, dtype=torch.int32, device="cuda")
    g = _fn(lib, "pla_k_lu_panel_tslu", [i32, i32, vp, lg, vp, vp, i32, i32, vp])

    def launch():
        A.copy_(A0)
        return g(r, w, A.data_ptr(), r, piv.data_ptr(), None, 0, a.ctas, None)

    t = _time(torch, launch, a.warmup, a.reps)
    return {"case": f"tournament panel LU {r} x {w} (f32), at most {a.ctas or 'one per SM'} "
                    f"CTAs, copy of the panel included", "s": t,
            "us_per_column": t / w * 1e6, "bytes_read_written": 2.0 * r * w * 4,
            "gbs": 2.0 * r * w * 4 / t / 1e9}


def case_panel_blocked(torch, lib, a):
    """The mixed LU's whole r x b fp32 panel (--m x --n): 32-column sub-panels
    with tournament pivoting, each followed by its row interchanges,
    triangular solve and rank-32 update (pla_k_panel_lu_blocked)."""
    r, b = a.m, a.n
    st = torch.cuda.Stream()
    A0 = torch.randn(b, r, dtype=torch.float32, device="cuda")
    A = A0.clone()
    piv = torch.zeros(b, dtype=torch.int32, device="cuda")
    g = _fn(lib, "pla_k_panel_lu_blocked", [i32, i32, i32, vp, lg, vp, vp, i32, i32, vp])

    def launch():
        A.copy_(A0)
        return g(pla.MPI_FLOAT, r, b, A.data_ptr(), r, piv.data_ptr(), None, a.ctas, 1,
                 st.cuda_stream)

    with torch.cuda.stream(st):
        t = _time(torch, launch, a.warmup, a.reps)
    return {"case": f"blocked tournament panel {r} x {b} (f32), 32-column sub-panels, at most "
                    f"{a.ctas or 'one per SM'} CTAs, copy of the panel included",
            "s": t, "us_per_subpanel": t / ((b + 31) // 32) * 1e6}


def case_trtri(torch, lib, a):
    """inv(L11) of the mixed LU's unit-lower diagonal block (n = --k), L11 at
    the top of an --m-row column-major panel as the factorization has it."""
    n, ld = a.k, max(a.m, a.k)
    P = torch.randn(n, ld, dtype=torch.float32, device="cuda") * (1.0 / n)
    D = torch.empty(n, n, dtype=torch.float32, device="cuda")
    g = _fn(lib, "pla_k_trtri_unit_lower", [i32, vp, lg, vp, lg, vp, vp])
    t = _time(torch, lambda: g(n, P.data_ptr(), ld, D.data_ptr(), n, None, None), a.warmup,
              a.reps)
    flops = n ** 3 / 3.0
    return {"case": f"unit-lower triangular inverse, n={n} (f32), leading dimension {ld}",
            "s": t, "us": t * 1e6, "gflops": flops / t / 1e9}


def case_laswp(torch, lib, a):
    m, n, npiv = a.m, a.n, a.k
    A = torch.randn(n, m, dtype=torch.float64, device="cuda")
    rng = np.random.default_rng(1)
    piv = torch.from_numpy(np.array([rng.integers(0, m - i) for i in range(npiv)], dtype=np.int32)).cuda()
    g = _fn(lib, "pla_k_laswp", [i32, vp, lg, i32, vp, i32, i32, i32, i32, vp])
    t = _time(torch, lambda: g(pla.MPI_DOUBLE, A.data_ptr(), m, npiv, piv.data_ptr(), 0, 0, npiv,
                               n, None), a.warmup, a.reps)
    byt = 2.0 * 2 * npiv * (n - npiv) * 8
    return {"case": f"row interchanges of one panel: {npiv} pivots over {n - npiv} columns (FP64)",
            "s": t, "algorithmic_bytes": byt, "gbs": byt / t / 1e9}


def case_trsv(torch, lib, a):
    n = a.n
    ld = (n + 31) // 32 * 32
    M = torch.randn(n, ld, device="cuda") * 0.01
    M.diagonal()[:n] += 1.0
    ldd = (n + 127) // 128 * 128
    Dinv = torch.zeros(128, ldd, device="cuda")
    b = torch.randn(n, device="cuda")
    x = torch.empty_like(b)
    st = torch.zeros(4, dtype=torch.int32, device="cuda")
    inv = _fn(lib, "pla_k_trsv_inv_blocks", [i32, ch, ch, ch, i32, vp, lg, vp, lg, vp])
    assert inv(pla.MPI_FLOAT, b"L", b"N", b"U", n, M.data_ptr(), ld, Dinv.data_ptr(), ldd, None) == 0
    g = _fn(lib, "pla_k_trsv_ticket", [i32, ch, ch, i32, vp, lg, vp, lg, vp, vp, vp, vp])
    t = _time(torch, lambda: g(pla.MPI_FLOAT, b"L", b"N", n, M.data_ptr(), ld, Dinv.data_ptr(),
                               ldd, b.data_ptr(), x.data_ptr(), st.data_ptr(), None),
              a.warmup, a.reps)
    byt = 4.0 * n * n / 2
    return {"case": f"single-launch unit-lower triangular solve, n={n} (fp32 factor)", "s": t,
            "algorithmic_bytes": byt, "gbs": byt / t / 1e9}

def case_trsv_link(torch, lib, a):
    """The single-column solve with link blocks (pla_k_trsv_ticket_link), the
    link blocks formed once beforehand as the refinement does per factor."""
    n = a.n
    ld = (n + 31) // 32 * 32
    M = torch.randn(n, ld, device="cuda") * 0.01
    M.diagonal()[:n] += 1.0
    ldd = (n + 127) // 128 * 128
    Dinv = torch.zeros(128, ldd, device="cuda")
    G = torch.zeros(128, ldd, device="cuda")
    b = torch.randn(n, device="cuda")
    x = torch.empty_like(b)
    st = torch.zeros(4, dtype=torch.int32, device="cuda")
    inv = _fn(lib, "pla_k_trsv_inv_blocks", [i32, ch, ch, ch, i32, vp, lg, vp, lg, vp])
    assert inv(pla.MPI_FLOAT, b"L", b"N", b"U", n, M.data_ptr(), ld, Dinv.data_ptr(), ldd, None) == 0
    lk = _fn(lib, "pla_k_trsv_link_blocks", [ch, ch, i32, vp, lg, vp, lg, vp, vp])
    assert lk(b"L", b"N", n, M.data_ptr(), ld, Dinv.data_ptr(), ldd, G.data_ptr(), None) == 0
    g = _fn(lib, "pla_k_trsv_ticket_link", [ch, ch, i32, vp, lg, vp, lg, vp, vp, vp, vp, vp])
    t = _time(torch, lambda: g(b"L", b"N", n, M.data_ptr(), ld, Dinv.data_ptr(), ldd,
                               G.data_ptr(), b.data_ptr(), x.data_ptr(), st.data_ptr(), None),
              a.warmup, a.reps)
    assert st[0].item() == 0
    byt = 4.0 * n * n / 2
    return {"case": f"single-launch unit-lower triangular solve with link blocks, n={n} "
                    f"(fp32 factor)", "s": t, "algorithmic_bytes": byt, "gbs": byt / t / 1e9}


def case_trsv_multi(torch, lib, a):
    """pla_k_trsv_ticket_multi: --k right-hand sides (at most 16) in one launch,
    on an fp32 factor; with --dtype f64 the FP64 form (pla_k_trsv_ticket_multi_f64:
    FP64 right-hand sides and arithmetic, the bf16 x 6 preconditioner)."""
    n, nrhs = a.n, min(a.k, 16)
    f64 = a.dtype == "f64"
    vt = torch.float64 if f64 else torch.float32
    ld = (n + 31) // 32 * 32
    M = torch.randn(n, ld, device="cuda") * 0.01
    M.diagonal()[:n] += 1.0
    ldd = (n + 127) // 128 * 128
    Dinv = torch.zeros(128, ldd, device="cuda", dtype=vt)
    B = torch.randn(nrhs, n, device="cuda", dtype=vt)
    X = torch.empty_like(B)
    st = torch.zeros(4, dtype=torch.int32, device="cuda")
    if f64:
        inv = _fn(lib, "pla_k_trsv_inv_blocks_f64", [ch, ch, ch, i32, vp, lg, vp, lg, vp])
        assert inv(b"L", b"N", b"U", n, M.data_ptr(), ld, Dinv.data_ptr(), ldd, None) == 0
        g = _fn(lib, "pla_k_trsv_ticket_multi_f64", [ch, ch, i32, i32, vp, lg, vp, lg, vp, lg, vp,
                                                     lg, vp, vp])
    else:
        inv = _fn(lib, "pla_k_trsv_inv_blocks", [i32, ch, ch, ch, i32, vp, lg, vp, lg, vp])
        assert inv(pla.MPI_FLOAT, b"L", b"N", b"U", n, M.data_ptr(), ld, Dinv.data_ptr(), ldd,
                   None) == 0
        g = _fn(lib, "pla_k_trsv_ticket_multi", [ch, ch, i32, i32, vp, lg, vp, lg, vp, lg, vp, lg,
                                                 vp, vp])
    t = _time(torch, lambda: g(b"L", b"N", n, nrhs, M.data_ptr(), ld, Dinv.data_ptr(), ldd,
                               B.data_ptr(), n, X.data_ptr(), n, st.data_ptr(), None),
              a.warmup, a.reps)
    assert st[0].item() == 0
    es = 8 if f64 else 4
    byt = 4.0 * n * n / 2 + 2 * es * n * nrhs
    return {"case": f"single-launch unit-lower triangular solve, n={n}, {nrhs} rhs (fp32 factor, "
                    f"{'FP64' if f64 else 'fp32'} right-hand sides and arithmetic)",
            "s": t, "algorithmic_bytes": byt, "gbs": byt / t / 1e9,
            "gflops": 2.0 * n * n / 2 * nrhs / t / 1e9}


def case_basis(torch, lib, a):
    """The lockstep GMRES's batched basis kernels at --n rows, --k columns (at
    most 16) and --count basis vectors: CGS coefficients, update, norms, scale."""
    n, nrhs, j = a.n, min(a.k, 16), min(a.count, 30)
    m = 30
    ldv = n * (m + 1)
    V = torch.randn(nrhs, m + 1, n, dtype=torch.float64, device="cuda")
    tmp = torch.zeros(nrhs * (m + 1), dtype=torch.float64, device="cuda")
    dots = _fn(lib, "pla_k_basis_dots", [i32, i32, vp, lg, i32, i32, i32, ctypes.c_uint, vp, i32,
                                         vp])
    upd = _fn(lib, "pla_k_basis_update", [i32, i32, vp, lg, i32, i32, vp, i32, ctypes.c_uint, vp])
    scl = _fn(lib, "pla_k_basis_scale", [i32, i32, vp, lg, i32, ctypes.POINTER(ctypes.c_double),
                                         ctypes.c_uint, vp])
    active = (1 << nrhs) - 1
    scales = (ctypes.c_double * 16)(*([0.5] * 16))

    def one_pass():
        dots(n, nrhs, V.data_ptr(), ldv, 0, j, j, active, tmp.data_ptr(), m + 1, None)
        upd(n, nrhs, V.data_ptr(), ldv, j, j, tmp.data_ptr(), m + 1, active, None)
        dots(n, nrhs, V.data_ptr(), ldv, j, 1, j, active, tmp.data_ptr(), 1, None)
        return scl(n, nrhs, V.data_ptr(), ldv, j, scales, active, None)

    t = _time(torch, one_pass, a.warmup, a.reps)
    byt = 8.0 * n * nrhs * (2 * (j + 1) + j + 3)   # dots, update (read j, r/w one), norms, scale
    return {"case": f"GMRES basis kernels, n={n}, {nrhs} columns, {j} basis vectors: one CGS "
                    "pass + norms + scale", "s": t, "algorithmic_bytes": byt,
            "gbs": byt / t / 1e9}


def case_residual(torch, lib, a):
    n = a.n
    A = torch.randn(n, n, dtype=torch.float64, device="cuda")
    X = torch.randn(n, dtype=torch.float64, device="cuda")
    B = torch.randn(n, dtype=torch.float64, device="cuda")
    R = torch.empty_like(B)
    wk = _fn(lib, "pla_k_residual_work", [i32, i32, i32])
    wk.restype = ctypes.c_size_t
    work = torch.empty(wk(n, n, 1) // 8 + 64, dtype=torch.float64, device="cuda")
    g = _fn(lib, "pla_k_residual", [i32, i32, i32, vp, lg, vp, lg, vp, lg, vp, lg, i32, vp, vp])
    t = _time(torch, lambda: g(n, n, 1, A.data_ptr(), n, X.data_ptr(), n, B.data_ptr(), n,
                               R.data_ptr(), n, 0, work.data_ptr(), None), a.warmup, a.reps)
    byt = 8.0 * n * n
    return {"case": f"FP64 residual b - A x, n={n}", "s": t, "algorithmic_bytes": byt,
            "gbs": byt / t / 1e9}


def case_potrf(torch, lib, a):
    """pla_k_potrf_lower on one --k x --k diagonal block (k <= 128): the
    Cholesky's diagonal factorization, one CTA, latency-bound."""
    b = a.k
    dt = pla.MPI_DOUBLE if a.dtype == "f64" else pla.MPI_FLOAT
    tdt = torch.float64 if a.dtype == "f64" else torch.float32
    G = torch.randn(b, b, dtype=torch.float64, device="cuda")
    A0 = (G @ G.t() / b + torch.eye(b, dtype=torch.float64, device="cuda")).to(tdt)
    A = A0.clone()
    st = torch.zeros(4, dtype=torch.int32, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    g = _fn(lib, "pla_k_potrf_lower", [i32, i32, vp, lg, vp, vp, i32, vp])

    def launch():
        A.copy_(A0)
        return g(dt, b, A.data_ptr(), b, st.data_ptr(), info.data_ptr(), 0, None)

    t = _time(torch, launch, a.warmup, a.reps)
    assert st[0].item() == 0 and info.item() == 0
    flops = b ** 3 / 3.0
    return {"case": f"diagonal block Cholesky {b} x {b} ({a.dtype}), copy of the block included",
            "s": t, "flops": flops, "gflops": flops / t / 1e9}


def case_trsm_small(torch, lib, a):
    """pla_k_trsm_small as the solvers call it: --side L solves the --k x --n
    block to the right of a unit-lower --k x --k diagonal block (the LU's
    sub-panel and U12 solves); --side R solves the --m x --k block column
    below a lower --k x --k block, A21 inv(L11)' (the Cholesky)."""
    dt = pla.MPI_DOUBLE if a.dtype == "f64" else pla.MPI_FLOAT
    tdt = torch.float64 if a.dtype == "f64" else torch.float32
    es = 8 if a.dtype == "f64" else 4
    b = a.k
    L = torch.randn(b, b, dtype=tdt, device="cuda") * 0.05      # column-major b x b
    L.diagonal().add_(1.0)
    st = torch.zeros(4, dtype=torch.int32, device="cuda")
    g = _fn(lib, "pla_k_trsm_small", [i32, ch, ch, ch, ch, i32, i32, f64, vp, lg, vp, lg, vp, vp])
    if a.side == "L":
        other = a.n
        B0 = torch.randn(other, b, dtype=tdt, device="cuda")       # column-major b x other
        args = (b"L", b"L", b"N", b"U")
        what = f"unit-lower {b} x {b} solve of a {b} x {other} block (left)"
        ldb = b
    else:
        other = a.m
        B0 = torch.randn(b, other, dtype=tdt, device="cuda")       # column-major other x b
        args = (b"R", b"L", b"T", b"N")
        what = f"A21 inv(L11)' for a {other} x {b} block column (right, lower, transposed)"
        ldb = other
    B = B0.clone()

    def launch():
        B.copy_(B0)
        return g(dt, *args, b, other, 1.0, L.data_ptr(), b, B.data_ptr(), ldb, st.data_ptr(), None)

    t = _time(torch, launch, a.warmup, a.reps)
    assert st[0].item() == 0
    flops = float(b) * b * other
    byt = 2.0 * b * other * es
    return {"case": f"{what} ({a.dtype}), copy of the block included", "s": t, "flops": flops,
            "gflops": flops / t / 1e9, "algorithmic_bytes": byt, "gbs": byt / t / 1e9}


def case_sgemm(torch, lib, a):
    """pla_k_gemm in fp32 as the mixed LU's sub-panel update calls it:
    C (m x n) -= A (m x k) B (k x n), k = 32."""
    m, n, k = a.m, a.n, a.k
    A = torch.randn(k, m, device="cuda")
    B = torch.randn(n, k, device="cuda")
    C = torch.randn(n, m, device="cuda")
    g = _fn(lib, "pla_k_gemm", [i32, i32, i32, i32, i32, i32, f64, vp, lg, vp, lg, f64, vp, lg,
                                i32, vp, vp])
    t = _time(torch, lambda: g(pla.MPI_FLOAT, pla.PLA_NO_TRANSPOSE, pla.PLA_NO_TRANSPOSE, m, n, k,
                               -1.0, A.data_ptr(), m, B.data_ptr(), k, 1.0, C.data_ptr(), m, 0,
                               None, None), a.warmup, a.reps)
    flops = 2.0 * m * n * k
    byt = 4.0 * (2.0 * m * n + m * k + k * n)
    return {"case": f"fp32 update C -= A B, {m} x {n} x {k}", "s": t,
            "tflops": flops / t / 1e12, "algorithmic_bytes": byt, "gbs": byt / t / 1e9}


def case_panel_update(torch, lib, a):
    """pla_k_panel_update as the fp32 panel calls it after a sub-panel's
    interchanges: U12 = inv(L11) A12 and A22 -= L21 U12 for the --m x --k
    sub-panel (k <= 32) and --n columns right of it, one launch."""
    m, n, w = a.m, a.n, a.k
    P0 = torch.randn(w + n, m, device="cuda")
    P0[:w, :w] = torch.eye(w, device="cuda") + 0.1 * torch.randn(w, w, device="cuda").tril(-1).t()
    P = P0.clone()
    g = _fn(lib, "pla_k_panel_update", [i32, i32, i32, vp, lg, vp])

    def launch():
        return g(m, w, n, P.data_ptr(), m, None)

    t = _time(torch, launch, a.warmup, a.reps)
    flops = 2.0 * (m - w) * n * w + float(w) * w * n
    byt = 4.0 * (2.0 * m * n + m * w)
    return {"case": f"fp32 sub-panel step: U12 solve and A22 -= L21 U12, {m} x {n} x {w}",
            "s": t, "tflops": flops / t / 1e12, "algorithmic_bytes": byt, "gbs": byt / t / 1e9}


def case_batched(torch, lib, a):
    """The batched workload's instance mix (n log-uniform in [8, 512], LU and
    Cholesky), optionally only the orders in [--nmin, --nmax], planned with
    (--tune 1) or without the autotuner."""
    from .workloads import batched_orders, batched_workload
    dtype = torch.float64 if a.dtype == "f64" else torch.float32
    ns, _, _ = batched_orders(a.count, 3)
    sel = [i for i in range(a.count) if a.nmin <= ns[i] <= a.nmax]
    arr, groups, piv, flops, ids = batched_workload(torch, pla, torch.device("cuda", 0), dtype,
                                                    a.count, 3, select=sel)
    info = torch.zeros(max(1, len(ids)), dtype=torch.int32, device="cuda")
    dt = pla.MPI_DOUBLE if a.dtype == "f64" else pla.MPI_FLOAT
    plan = ctypes.c_void_p()
    pla.check(lib.PLA_Batch_plan_create(dt, len(ids), arr, ctypes.c_void_p(info.data_ptr()),
                                        a.tune, ctypes.byref(plan)), "plan")

    def launch():
        for gr in groups:
            gr["A"].copy_(gr["A0"])
            gr["B"].copy_(gr["B0"])
        return lib.PLA_Batch_plan_execute(plan)

    t = _time(torch, launch, a.warmup, a.reps)
    lib.PLA_Batch_plan_free(ctypes.byref(plan))
    return {"case": f"batched factor-and-solve, {len(ids)} of {a.count} instances (orders "
                    f"{a.nmin}..{a.nmax}, {a.dtype}, autotune {a.tune}), input restore "
                    "included", "s": t, "gflops": flops / t / 1e9}


CASES = {k[5:]: v for k, v in globals().items() if k.startswith("case_")}


def main(argv=None):
    p = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    p.add_argument("case", choices=sorted(CASES))
    p.add_argument("--m", type=int, default=16384)
    p.add_argument("--n", type=int, default=16384)
    p.add_argument("--k", type=int, default=128)
    p.add_argument("--count", type=int, default=2000)
    p.add_argument("--nmin", type=int, default=0, help="batched: smallest order kept")
    p.add_argument("--nmax", type=int, default=1 << 30, help="batched: largest order kept")
    p.add_argument("--tune", type=int, default=1, help="batched: autotune the plan")
    p.add_argument("--dtype", choices=["f32", "f64"], default="f32")
    p.add_argument("--warmup", type=int, default=2)
    p.add_argument("--reps", type=int, default=3)
    p.add_argument("--ctas", type=int, default=0, help="panel: CTA cap (0: one per SM)")
    p.add_argument("--side", choices=["L", "R"], default="L", help="trsm_small: side")
    a = p.parse_args(argv)
    import torch
    torch.cuda.set_device(0)
    lib = pla.lib()
    print(json.dumps(CASES[a.case](torch, lib, a)))
    return 0


if __name__ == "__main__":
    sys.exit(main())
