"""CPU oracle bindings — TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py
import this module, and only as the checker (or, for the baseline, as the thing
timed on the host cores).  The product package never imports it.

Two CPU implementations are exposed, both column-major float64/float32:

* ``Restated``  — ``liboracle.so``, the plain-C restatement in pla_oracle.c of
  the reference's LU (SOLVERS/LU/PLA_LU.c, PLA_LU_mv.c, PLA_seq_lu.c),
  Cholesky (SOLVERS/Cholesky/PLA_Chol.c, PLA_Local_chol.c), pivot application
  (SOLVERS/LU/PLA_Apply_pivots_new.c), TRSV/TRSM/GEMM.
* ``Reference`` — ``_ref/libplapack_ref*.so``, the upstream PLAPACK sources
  compiled unchanged with a single-rank MPI stand-in and either the restated
  netlib BLAS (bit-reproducible) or OpenBLAS (for timing).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

# PLAPACK constants (INCLUDE/PLA_define.h)
PLA_NO_TRANSPOSE = 21
PLA_TRANSPOSE = 22
PLA_SIDE_LEFT = 43
PLA_SIDE_RIGHT = 44
PLA_UPPER_TRIANGULAR = 51
PLA_LOWER_TRIANGULAR = 52
PLA_UNIT_DIAG = 101
PLA_NONUNIT_DIAG = 102

_vp = ctypes.c_void_p
_i = ctypes.c_int


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_vp)


def build(reference_root: str | None = None) -> None:
    """Build liboracle.so, and the compiled reference when its sources exist.

    The reference tree is the Makefile's REFERENCE (overridden by the
    argument or the PLA_REFERENCE_ROOT environment variable); where it is
    absent, as on a machine that only runs the prebuilt files, the
    `ref-if-present` target does nothing."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    root = reference_root or os.environ.get("PLA_REFERENCE_ROOT")
    extra = [f"REFERENCE={root}"] if root else []
    subprocess.run(["make", "-s", "-j8", "-C", HERE, *extra, "ref-if-present"], check=True)


class Restated:
    """ctypes view of liboracle.so (pla_oracle.c)."""

    def __init__(self, path: str | None = None):
        path = path or os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        self.lib = ctypes.CDLL(path)

    @staticmethod
    def _dt(a):
        return "d" if a.dtype == np.float64 else "s"

    def drand48_matrix(self, m: int, n: int, seed: int = 0) -> np.ndarray:
        """TEST/create_problem.c:31,49-51: srand48(seed), drand48()*2-1, column-major."""
        out = np.empty(m * n, dtype=np.float64)
        self.lib.oracle_fill_drand48(ctypes.c_long(seed), ctypes.c_long(m * n), _ptr(out))
        return out.reshape((m, n), order="F")

    def lu_unblocked(self, A: np.ndarray):
        A = np.asfortranarray(A.copy())
        m, n = A.shape
        piv = np.zeros(min(m, n), dtype=np.int32)
        getattr(self.lib, f"oracle_{self._dt(A)}lu_unblocked")(m, n, _ptr(A), m, _ptr(piv))
        return A, piv

    def lu_blocked(self, A: np.ndarray, nb: int):
        A = np.asfortranarray(A.copy())
        m, n = A.shape
        piv = np.zeros(min(m, n), dtype=np.int32)
        getattr(self.lib, f"oracle_{self._dt(A)}lu_blocked")(m, n, nb, _ptr(A), m, _ptr(piv))
        return A, piv

    def lu_linpack(self, A: np.ndarray, nb: int):
        """Blocked LU whose pivots skip the factored L columns (PLA_LU_linpack.c:145)."""
        A = np.asfortranarray(A.copy())
        m, n = A.shape
        piv = np.zeros(min(m, n), dtype=np.int32)
        getattr(self.lib, f"oracle_{self._dt(A)}lu_linpack")(m, n, nb, _ptr(A), m, _ptr(piv))
        return A, piv

    def slu_tournament(self, A: np.ndarray, max_ctas: int):
        """Model of the library's own tournament-pivoted fp32 panel (no
        reference counterpart): pivots and L \\ U of the r x w float32 panel."""
        A = np.asfortranarray(A.astype(np.float32, copy=True))
        r, w = A.shape
        piv = np.zeros(w, dtype=np.int32)
        self.lib.oracle_slu_tournament(r, w, max_ctas, _ptr(A), r, _ptr(piv))
        return A, piv

    def chol_blocked(self, A: np.ndarray, nb: int):
        A = np.asfortranarray(A.copy())
        n = A.shape[0]
        info = getattr(self.lib, f"oracle_{self._dt(A)}chol_blocked")(n, nb, _ptr(A), n)
        return A, info

    def apply_pivots(self, piv: np.ndarray, B: np.ndarray) -> np.ndarray:
        B = np.asfortranarray(B.copy())
        if B.ndim == 1:
            B = B.reshape(-1, 1, order="F")
        piv = np.ascontiguousarray(piv, dtype=np.int32)
        getattr(self.lib, f"oracle_{self._dt(B)}apply_pivots")(
            len(piv), _ptr(piv), _ptr(B), B.shape[0], 0, B.shape[1])
        return B

    def trsv(self, uplo: str, trans: str, diag: str, A: np.ndarray, x: np.ndarray):
        A = np.asfortranarray(A)
        x = np.ascontiguousarray(x.copy())
        fn = getattr(self.lib, f"oracle_{self._dt(A)}trsv")
        fn(ctypes.c_char(uplo.encode()), ctypes.c_char(trans.encode()),
           ctypes.c_char(diag.encode()), A.shape[0], _ptr(A), A.shape[0], _ptr(x))
        return x

    def solve_lu(self, LU: np.ndarray, piv: np.ndarray, b: np.ndarray) -> np.ndarray:
        """P b, then L (unit) and U solves: the PLA_General_solve sequence."""
        x = self.apply_pivots(piv, b)
        out = np.empty_like(x)
        for j in range(x.shape[1]):
            y = self.trsv("L", "N", "U", LU, x[:, j])
            out[:, j] = self.trsv("U", "N", "N", LU, y)
        return out


def _preload_openblas_deps() -> None:
    """The OpenBLAS build used for timing ships beside its own libgfortran and
    libquadmath; load those first so the dynamic linker finds them."""
    import glob
    import sys
    for d in sys.path:
        libs = os.path.join(d, "opencv_python_headless.libs")
        if os.path.isdir(libs):
            for pat in ("libquadmath-*.so*", "libgfortran-*.so*"):
                for f in sorted(glob.glob(os.path.join(libs, pat))):
                    ctypes.CDLL(f, mode=ctypes.RTLD_GLOBAL)
            return


class Reference:
    """ctypes view of the upstream PLAPACK compiled from its sources."""

    def __init__(self, blas: str = "netlib", nb_distr: int = 64, nb_alg: int = 64,
                 error_checking: int = 0):
        name = "libplapack_ref.so" if blas == "netlib" else "libplapack_ref_openblas.so"
        path = os.path.join(REF_DIR, name)
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (make -C oracle ref)")
        if blas != "netlib":
            _preload_openblas_deps()
        self.lib = ctypes.CDLL(path)
        self.lib.ref_trsm.argtypes = [_i] * 6 + [ctypes.c_double, _i, _vp, _i, _vp, _i]
        self.lib.ref_gemm.argtypes = [_i] * 5 + [ctypes.c_double, _i, _vp, _i, _vp, _i,
                                                 ctypes.c_double, _vp, _i]
        self.lib.ref_init(nb_distr, nb_alg, error_checking)

    def set_nb_alg(self, nb_alg: int) -> None:
        self.lib.ref_set_nb_alg(nb_alg)

    @staticmethod
    def _code(a):
        return 1 if a.dtype == np.float64 else 0

    def lu(self, A: np.ndarray):
        A = np.asfortranarray(A.copy())
        m, n = A.shape
        piv = np.zeros(min(m, n), dtype=np.int32)
        t = ctypes.c_double()
        r = self.lib.ref_lu(m, n, self._code(A), _ptr(A), m, _ptr(piv), ctypes.byref(t))
        return A, piv, r, t.value

    def lu_linpack(self, A: np.ndarray):
        A = np.asfortranarray(A.copy())
        m, n = A.shape
        piv = np.zeros(min(m, n), dtype=np.int32)
        t = ctypes.c_double()
        r = self.lib.ref_lu_linpack(m, n, self._code(A), _ptr(A), m, _ptr(piv),
                                    ctypes.byref(t))
        return A, piv, r, t.value

    def chol(self, A: np.ndarray):
        A = np.asfortranarray(A.copy())
        n = A.shape[0]
        t = ctypes.c_double()
        r = self.lib.ref_chol(n, self._code(A), _ptr(A), n, ctypes.byref(t))
        return A, r, t.value

    def general_solve(self, A: np.ndarray, B: np.ndarray):
        A = np.asfortranarray(A.copy())
        B = np.asfortranarray(B.copy().reshape(A.shape[0], -1))
        n, nrhs = B.shape
        piv = np.zeros(n, dtype=np.int32)
        t = ctypes.c_double()
        r = self.lib.ref_general_solve(n, nrhs, self._code(A), _ptr(A), n, _ptr(B), n,
                                       _ptr(piv), ctypes.byref(t))
        return A, B, piv, r, t.value

    def pos_def_solve(self, A: np.ndarray, B: np.ndarray):
        A = np.asfortranarray(A.copy())
        B = np.asfortranarray(B.copy().reshape(A.shape[0], -1))
        n, nrhs = B.shape
        t = ctypes.c_double()
        r = self.lib.ref_pos_def_solve(n, nrhs, self._code(A), _ptr(A), n, _ptr(B), n,
                                       ctypes.byref(t))
        return A, B, r, t.value

    def trsv(self, uplo: int, trans: int, diag: int, A: np.ndarray, x: np.ndarray):
        A = np.asfortranarray(A)
        x = np.ascontiguousarray(x.copy())
        r = self.lib.ref_trsv(uplo, trans, diag, A.shape[0], self._code(A), _ptr(A),
                              A.shape[0], _ptr(x))
        return x, r

    def trsm(self, side, uplo, trans, diag, alpha, A, B):
        A = np.asfortranarray(A)
        B = np.asfortranarray(B.copy())
        m, n = B.shape
        r = self.lib.ref_trsm(side, uplo, trans, diag, m, n, float(alpha), self._code(A),
                              _ptr(A), A.shape[0], _ptr(B), m)
        return B, r

    def gemm(self, transa, transb, alpha, A, B, beta, C):
        A = np.asfortranarray(A)
        B = np.asfortranarray(B)
        C = np.asfortranarray(C.copy())
        m, n = C.shape
        k = A.shape[1] if transa == PLA_NO_TRANSPOSE else A.shape[0]
        r = self.lib.ref_gemm(transa, transb, m, n, k, float(alpha), self._code(A),
                              _ptr(A), A.shape[0], _ptr(B), B.shape[0], float(beta),
                              _ptr(C), m)
        return C, r

    def apply_pivots(self, piv: np.ndarray, B: np.ndarray):
        B = np.asfortranarray(B.copy())
        if B.ndim == 1:
            B = B.reshape(-1, 1, order="F")
        piv = np.ascontiguousarray(piv, dtype=np.int32)
        self.lib.ref_apply_pivots(B.shape[0], B.shape[1], self._code(B), _ptr(B),
                                  B.shape[0], _ptr(piv), len(piv))
        return B
