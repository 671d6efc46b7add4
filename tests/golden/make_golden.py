"""Generate the golden fixtures in tests/golden/ by running the UPSTREAM PLAPACK.

The reference sources are compiled unchanged into oracle/_ref/libplapack_ref.so
(`make -C oracle ref`: single-rank MPI stand-in + restated netlib BLAS, gcc
-ffp-contract=off) and driven through PLA_LU / PLA_Chol / PLA_General_solve /
PLA_Pos_def_solve / PLA_Trsv / PLA_Trsm / PLA_Gemm / PLA_Apply_pivots_to_rows
on a 1x1 template.  This script runs only where the reference tree exists;
what it writes is committed, so tests never need the reference at run time.

Inputs are stored as specs (tests/golden/inputs.py rebuilds them); outputs are
stored as pivots, solution vectors, factor diagonals and the SHA-256 of each
full factor (bit-exact: the restated oracle reproduces it).

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from oracle import oracle as orc  # noqa: E402
import inputs  # noqa: E402


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.asfortranarray(a).tobytes(order="F")).hexdigest()


def main():
    orc.build()
    rs = orc.Restated()
    ref = orc.Reference("netlib", nb_distr=64, nb_alg=64, error_checking=0)
    manifest, arrays = {}, {}

    def add(name, entry, **outs):
        manifest[name] = entry
        for k, v in outs.items():
            arrays[f"{name}__{k}"] = v

    # ---- LU (PLA_LU) ---------------------------------------------------------
    lu_specs = [("c1_lu_n1000_nb64", {"m": 1000, "n": 1000, "seed": 0}, 64)]
    shapes = [(1, 1, 64), (2, 2, 1), (5, 3, 2), (3, 5, 2), (65, 65, 64), (130, 130, 64),
              (150, 100, 32), (100, 150, 32), (129, 129, 128), (64, 64, 64), (97, 97, 16),
              (300, 300, 128)]
    for i, (m, n, nb) in enumerate(shapes):
        lu_specs.append((f"lu_{m}x{n}_nb{nb}", {"m": m, "n": n, "seed": 100 + i}, nb))
    lu_specs += [
        ("lu_ties_48_nb16", {"m": 48, "n": 48, "seed": 7, "mod": "sign"}, 16),
        ("lu_singular_last_40_nb16", {"m": 40, "n": 40, "seed": 8, "mod": "zero_last_col"}, 16),
        ("lu_f32_200_nb32", {"m": 200, "n": 200, "seed": 9, "dtype": "float32"}, 32),
    ]
    for name, spec, nb in lu_specs:
        A = inputs.build(rs, spec)
        ref.set_nb_alg(nb)
        LU, piv, ret, _ = ref.lu(A)
        add(name, {"kind": "lu", "spec": spec, "nb_alg": nb, "ret": int(ret),
                   "factor_sha256": sha(LU)},
            piv=piv, diag=np.diag(LU).copy())

    # C1 solve: b = A @ ones (EXAMPLES/LU/driver.c:194-211 forms b = A x)
    A = inputs.build(rs, {"m": 1000, "n": 1000, "seed": 0})
    ref.set_nb_alg(64)
    _, x, piv, ret, _ = ref.general_solve(A, A @ np.ones(1000))
    add("c1_general_solve_n1000_nb64",
        {"kind": "general_solve", "spec": {"m": 1000, "n": 1000, "seed": 0},
         "rhs": "A @ ones", "nrhs": 1, "nb_alg": 64, "ret": int(ret)},
        X=x, piv=piv)

    # ---- Cholesky (PLA_Chol(PLA_LOWER_TRIANGULAR)) --------------------------
    for (n, nb) in [(20, 4), (1, 64), (64, 64), (100, 64), (257, 64), (130, 32)]:
        spec = {"m": n, "n": n, "seed": 200 + n, "mod": "shift_n"}
        A = inputs.build(rs, spec)
        ref.set_nb_alg(nb)
        L, ret, _ = ref.chol(A)
        add(f"chol_{n}_nb{nb}", {"kind": "chol", "spec": spec, "nb_alg": nb, "ret": int(ret),
                                 "lower_sha256": sha(np.tril(L))},
            diag=np.diag(L).copy())
    spec = {"m": 60, "n": 60, "seed": 300, "mod": "shift_n_neg", "at": 36}
    ref.set_nb_alg(16)
    _, ret, _ = ref.chol(inputs.build(rs, spec))
    add("chol_fail_60_nb16", {"kind": "chol", "spec": spec, "nb_alg": 16, "ret": int(ret)})

    # ---- solves ---------------------------------------------------------------
    ref.set_nb_alg(32)
    sa, sb = {"m": 150, "n": 150, "seed": 400}, {"m": 150, "n": 16, "seed": 401}
    _, X, piv, ret, _ = ref.general_solve(inputs.build(rs, sa), inputs.build(rs, sb))
    add("general_solve_150_16rhs_nb32", {"kind": "general_solve", "spec": sa, "rhs_spec": sb,
                                         "nrhs": 16, "nb_alg": 32, "ret": int(ret)},
        X=X, piv=piv)
    ss = {"m": 140, "n": 140, "seed": 402, "mod": "shift_n_sym"}
    for nrhs, seed in ((1, 403), (8, 404)):
        sb = {"m": 140, "n": nrhs, "seed": seed}
        _, X, ret, _ = ref.pos_def_solve(inputs.build(rs, ss), inputs.build(rs, sb))
        add(f"pos_def_solve_140_{nrhs}rhs_nb32",
            {"kind": "pos_def_solve", "spec": ss, "rhs_spec": sb, "nrhs": nrhs,
             "nb_alg": 32, "ret": int(ret)}, X=X)

    # ---- triangular solves ------------------------------------------------------
    st = {"m": 130, "n": 130, "seed": 500, "mod": "shift_n"}
    sv = {"m": 130, "n": 1, "seed": 501}
    T, v = inputs.build(rs, st), inputs.build(rs, sv)[:, 0]
    L_, U_, N_, Tr_ = orc.PLA_LOWER_TRIANGULAR, orc.PLA_UPPER_TRIANGULAR, orc.PLA_NO_TRANSPOSE, orc.PLA_TRANSPOSE
    UD, ND = orc.PLA_UNIT_DIAG, orc.PLA_NONUNIT_DIAG
    for (u, t, d, tag) in [(L_, N_, UD, "ln_unit"), (U_, N_, ND, "un_nonunit"),
                           (L_, Tr_, ND, "lt_nonunit"), (L_, N_, ND, "ln_nonunit")]:
        x, ret = ref.trsv(u, t, d, T, v)
        add(f"trsv_{tag}_130", {"kind": "trsv", "spec": st, "rhs_spec": sv, "uplo": u,
                                "trans": t, "diag": d, "ret": int(ret)}, x=x)
    sB = {"m": 130, "n": 16, "seed": 502}
    B = inputs.build(rs, sB)
    for (u, t, d, tag) in [(L_, N_, UD, "lln_unit"), (U_, N_, ND, "lun"), (L_, Tr_, ND, "llt")]:
        X, ret = ref.trsm(orc.PLA_SIDE_LEFT, u, t, d, 1.0, T, B)
        add(f"trsm_{tag}_130x16", {"kind": "trsm", "spec": st, "rhs_spec": sB,
                                   "side": orc.PLA_SIDE_LEFT, "uplo": u, "trans": t,
                                   "diag": d, "alpha": 1.0, "ret": int(ret)}, X=X)

    # ---- general GEMM, every transpose pair ------------------------------------
    m, n, k = 37, 29, 17
    for ta in (N_, Tr_):
        for tb in (N_, Tr_):
            sA = {"m": m if ta == N_ else k, "n": k if ta == N_ else m, "seed": 600 + ta}
            sB2 = {"m": k if tb == N_ else n, "n": n if tb == N_ else k, "seed": 610 + tb}
            sC = {"m": m, "n": n, "seed": 620}
            C, ret = ref.gemm(ta, tb, -1.0, inputs.build(rs, sA), inputs.build(rs, sB2), 0.5,
                              inputs.build(rs, sC))
            add(f"gemm_{ta}_{tb}", {"kind": "gemm", "transa": ta, "transb": tb, "alpha": -1.0,
                                    "beta": 0.5, "A_spec": sA, "B_spec": sB2, "C_spec": sC,
                                    "ret": int(ret)}, C=C)

    # ---- pivot application to a block of right-hand sides -----------------------
    piv = np.array([3, 0, 5, 1, 0, 2, 0, 0], dtype=np.int32)
    sP = {"m": 12, "n": 3, "seed": 700}
    add("apply_pivots_12x3", {"kind": "apply_pivots", "spec": sP, "ret": 0},
        piv=piv, B=ref.apply_pivots(piv, inputs.build(rs, sP)))

    np.savez_compressed(os.path.join(HERE, "golden.npz"), **arrays)
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py",
                   "reference": "upstream PLAPACK R3.0 hot-path sources compiled with gcc "
                                "-O2 -ffp-contract=off, single-rank MPI stand-in, restated "
                                "netlib BLAS (oracle/refshim)",
                   "cases": manifest}, f, indent=1, sort_keys=True)
    print(f"wrote {len(manifest)} cases, {sum(a.nbytes for a in arrays.values())} bytes")


if __name__ == "__main__":
    main()
