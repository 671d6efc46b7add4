"""Pin the CPU oracle against the reference's own outputs (CPU only).

The golden fixtures were produced by the upstream PLAPACK sources compiled in
this repository's oracle/ recipe (tests/golden/make_golden.py).  These tests
check that the C restatement (oracle/pla_oracle.c) reproduces them: pivots
exactly, LU and Cholesky factors bit for bit (SHA-256), solves to rounding.
When the compiled reference is present (oracle/_ref), it is also compared
with the restatement directly on fresh inputs.
"""
import hashlib
import os

import numpy as np
import pytest

import inputs
from oracle import oracle as orc


def sha(a):
    return hashlib.sha256(np.asfortranarray(a).tobytes(order="F")).hexdigest()


def cases(golden, kind):
    manifest, _ = golden
    return [k for k, v in manifest.items() if v["kind"] == kind]


def test_fixture_inventory(golden):
    manifest, arrays = golden
    kinds = {v["kind"] for v in manifest.values()}
    assert {"lu", "chol", "general_solve", "pos_def_solve", "trsv", "trsm", "gemm",
            "apply_pivots"} <= kinds
    assert manifest["chol_fail_60_nb16"]["ret"] == 37      # k + local index, PLA_Chol.c:181-185
    assert arrays["c1_lu_n1000_nb64__piv"].shape == (1000,)


@pytest.mark.parametrize("blocked", [True, False])
def test_lu_bitexact_vs_reference(golden, restated, blocked):
    manifest, arrays = golden
    for name in cases(golden, "lu"):
        e = manifest[name]
        A = inputs.build(restated, e["spec"])
        if blocked:
            LU, piv = restated.lu_blocked(A, e["nb_alg"])
        else:
            LU, piv = restated.lu_unblocked(A)
        assert np.array_equal(piv, arrays[name + "__piv"]), name
        if blocked or A.dtype == np.float64:
            # unblocked and blocked orders coincide element-wise for this loop nest
            assert sha(LU) == e["factor_sha256"], name


def test_chol_bitexact_vs_reference(golden, restated):
    manifest, arrays = golden
    for name in cases(golden, "chol"):
        e = manifest[name]
        A = inputs.build(restated, e["spec"])
        L, info = restated.chol_blocked(A, e["nb_alg"])
        assert info == e["ret"], name
        if e["ret"] == 0:
            assert sha(np.tril(L)) == e["lower_sha256"], name


def test_general_solve(golden, restated):
    manifest, arrays = golden
    for name in cases(golden, "general_solve"):
        e = manifest[name]
        A = inputs.build(restated, e["spec"])
        B = A @ np.ones((A.shape[0], 1)) if "rhs_spec" not in e else inputs.build(restated, e["rhs_spec"])
        LU, piv = restated.lu_blocked(A, e["nb_alg"])
        assert np.array_equal(piv, arrays[name + "__piv"])
        X = restated.solve_lu(LU, piv, B)
        Xr = arrays[name + "__X"].reshape(X.shape)
        n = A.shape[0]
        tol = n * np.finfo(np.float64).eps * np.abs(A).max() * max(1.0, np.abs(Xr).max()) * 10
        assert np.abs(X - Xr).max() <= tol * np.linalg.cond(A, 1) ** 0.5


def test_pos_def_solve(golden, restated):
    manifest, arrays = golden
    for name in cases(golden, "pos_def_solve"):
        e = manifest[name]
        A = inputs.build(restated, e["spec"])
        B = inputs.build(restated, e["rhs_spec"])
        L, info = restated.chol_blocked(A, e["nb_alg"])
        assert info == 0
        L = np.tril(L)
        X = np.empty_like(B)
        for j in range(B.shape[1]):
            y = restated.trsv("L", "N", "N", L, B[:, j])
            X[:, j] = restated.trsv("L", "T", "N", L, y)
        assert np.allclose(X, arrays[name + "__X"].reshape(X.shape), rtol=0, atol=1e-13)


def test_trsv_trsm(golden, restated):
    manifest, arrays = golden
    tr = {orc.PLA_LOWER_TRIANGULAR: "L", orc.PLA_UPPER_TRIANGULAR: "U",
          orc.PLA_NO_TRANSPOSE: "N", orc.PLA_TRANSPOSE: "T",
          orc.PLA_UNIT_DIAG: "U", orc.PLA_NONUNIT_DIAG: "N"}
    for name in cases(golden, "trsv") + cases(golden, "trsm"):
        e = manifest[name]
        T = inputs.build(restated, e["spec"])
        B = inputs.build(restated, e["rhs_spec"])
        X = np.stack([restated.trsv(tr[e["uplo"]], tr[e["trans"]], tr[e["diag"]], T, B[:, j])
                      for j in range(B.shape[1])], axis=1)
        ref = arrays[name + ("__x" if e["kind"] == "trsv" else "__X")].reshape(X.shape)
        # summation order differs from the reference's blocked dot form
        # (BLAS2/PLA_Trsv_ln.c:54-79); bound the difference normwise
        assert np.abs(X - ref).max() <= 1e-11 * np.abs(ref).max(), name


def test_gemm_and_pivots(golden, restated):
    manifest, arrays = golden
    for name in cases(golden, "gemm"):
        e = manifest[name]
        A = inputs.build(restated, e["A_spec"])
        B = inputs.build(restated, e["B_spec"])
        C = inputs.build(restated, e["C_spec"])
        opA = A if e["transa"] == orc.PLA_NO_TRANSPOSE else A.T
        opB = B if e["transb"] == orc.PLA_NO_TRANSPOSE else B.T
        ref = e["alpha"] * opA @ opB + e["beta"] * C
        assert np.allclose(arrays[name + "__C"], ref, rtol=0, atol=1e-13), name
    e = manifest["apply_pivots_12x3"]
    B = inputs.build(restated, e["spec"])
    out = restated.apply_pivots(arrays["apply_pivots_12x3__piv"], B)
    assert np.array_equal(out, arrays["apply_pivots_12x3__B"])


def test_c1_accuracy(golden, restated):
    """C1: ||LU - PA|| / ||A|| and the solution error of the reference run."""
    manifest, arrays = golden
    A = inputs.build(restated, manifest["c1_lu_n1000_nb64"]["spec"])
    LU, piv = restated.lu_blocked(A, 64)
    L = np.tril(LU, -1) + np.eye(1000)
    U = np.triu(LU)
    PA = restated.apply_pivots(piv, A)
    assert np.linalg.norm(L @ U - PA) / np.linalg.norm(A) < 1000 * np.finfo(float).eps
    x = arrays["c1_general_solve_n1000_nb64__X"]
    assert np.abs(x - 1.0).max() < 1e-9


_REF = os.path.join(orc.REF_DIR, "libplapack_ref.so")


@pytest.mark.skipif(not os.path.exists(_REF), reason="compiled reference not built here")
def test_restatement_matches_compiled_reference_fresh_inputs(restated):
    ref = orc.Reference("netlib", nb_distr=64, nb_alg=64)
    rng = np.random.default_rng(11)
    for (m, n, nb) in [(77, 77, 8), (200, 120, 24), (33, 90, 7)]:
        A = np.asfortranarray(rng.standard_normal((m, n)))
        ref.set_nb_alg(nb)
        LUr, pr, _, _ = ref.lu(A)
        LUo, po = restated.lu_blocked(A, nb)
        assert np.array_equal(pr, po)
        assert np.array_equal(LUr, LUo)


@pytest.mark.skipif(not os.path.exists(_REF), reason="compiled reference not built here")
def test_linpack_restatement_matches_compiled_reference(restated):
    # SOLVERS/LINPACK/PLA_LU_linpack.c compiled from the reference sources
    ref = orc.Reference("netlib", nb_distr=64, nb_alg=64)
    rng = np.random.default_rng(12)
    for (m, n, nb) in [(77, 78, 8), (200, 120, 24), (90, 140, 16)]:
        A = np.asfortranarray(rng.standard_normal((m, n)))
        ref.set_nb_alg(nb)
        LUr, pr, rc, _ = ref.lu_linpack(A)
        LUo, po = restated.lu_linpack(A, nb)
        assert rc == 0
        assert np.array_equal(pr, po)
        assert np.array_equal(LUr, LUo)
        # and it differs from PLA_LU only below the diagonal (L's row order)
        LUs, ps, _, _ = ref.lu(A)
        assert np.array_equal(ps, pr)
        assert np.array_equal(np.triu(LUs), np.triu(LUr))
    ref.set_nb_alg(64)


def test_tournament_panel_model_is_an_lu(restated):
    """The C model of the library's tournament-pivoted fp32 panel (checked bit
    for bit against the GPU kernel in test_gpu_tslu.py) is itself an LU with
    interchanges: P A = L U to fp32 rounding, whatever the tree's shape."""
    for r, w, ctas in [(1000, 32, 1), (1000, 32, 4), (5000, 32, 72), (300, 17, 3), (64, 32, 1)]:
        A = np.random.default_rng(r + w).standard_normal((r, w)).astype(np.float32)
        LU, piv = restated.slu_tournament(A, ctas)
        perm = np.arange(r)
        for j in range(w):
            p = j + piv[j]
            assert j <= p < r
            perm[[j, p]] = perm[[p, j]]
        L = np.tril(LU.astype(np.float64), -1)[:, :w] + np.eye(r, w)
        U = np.triu(LU[:w].astype(np.float64))
        assert np.abs(A[perm] - L @ U).max() <= 16 * w * 2.0 ** -24 * np.abs(A).max()
        # the first pivot is the largest |a| of column 0 (smallest row on ties)
        assert perm[0] == int(np.argmax(np.abs(A[:, 0])))
