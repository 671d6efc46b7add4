"""FP64 PLA_LU at the large sizes: pivots identical to the upstream PLAPACK's.

The fixtures under tests/golden/c2/ come from the compiled reference
(tests/golden/make_c2_pivots.py: upstream PLA_LU, nb_alg = 128, on the seed-1
i.i.d. N(0, 1) matrix, with the restated netlib BLAS and with OpenBLAS; both
builds give the same pivots where both exist).  Here the library factors the
same matrix -- rebuilt with the same numpy generator -- through the C ABI,
with the reference's block size and with the benchmark's (512), and must
return exactly the reference's pivot vector (SOLVERS/LU/PLA_LU.c:103-192,
first-index tie-break BLAS1/PLA_Iamax.c:108-115).  The factor is checked
through size-independent figures of U's diagonal and the factor's norm,
against the reference's, to a relative 1e-10.
"""
import ctypes
import hashlib
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "c2")


def fixtures(n):
    with open(os.path.join(HERE, "manifest.json")) as f:
        man = json.load(f)
    out = []
    for blas in ("netlib", "openblas"):
        key = f"lu_n{n}_{blas}"
        if key in man:
            piv = np.load(os.path.join(HERE, f"{key}.npz"))["pivots"]
            assert hashlib.sha256(np.ascontiguousarray(piv).tobytes()).hexdigest() == \
                man[key]["pivots_sha256"]
            out.append((blas, man[key], piv))
    return out


@pytest.fixture(scope="module")
def env():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    from plapack_b200 import pla
    s = pla.Session(nb_distr=128, nb_alg=128, error_checking=0)
    yield s, torch, pla
    s.close()


_MATRICES = {}


def c2(n):
    from plapack_b200.workloads import c2_matrix
    if n not in _MATRICES:
        _MATRICES.clear()
        _MATRICES[n] = c2_matrix(n)
    return _MATRICES[n]


@pytest.mark.parametrize("n,nb", [(16384, 128), (16384, 512), (32768, 128), (32768, 512)])
def test_pla_lu_pivots_equal_the_reference(env, n, nb):
    s, torch, pla = env
    refs = fixtures(n)
    if not refs:
        pytest.skip(f"no reference fixture for n={n}")
    lib = s.lib
    A = c2(n)
    a = s.matrix(n, n)
    p = s.mvector(n, 1, np.int32)
    try:
        s.set(a, A)
        s.set_nb_alg(nb)
        info = ctypes.c_int(-1)
        pla.check(lib.PLA_LU_info(a, p, ctypes.byref(info)), "PLA_LU")
        assert info.value == 0
        piv = s.get(p)[:, 0]
        for blas, man, ref in refs:
            bad = np.nonzero(piv != ref)[0]
            assert bad.size == 0, (f"pivots differ from the reference ({blas}) first at column "
                                   f"{bad[0]}: {piv[bad[0]]} vs {ref[bad[0]]}")
        # the factor, on the device: U's diagonal and the Frobenius norm
        T = torch.empty((n, n), dtype=torch.float64, device="cuda")
        pla.check(lib.PLA_Obj_get_local_contents_device(a, ctypes.c_void_p(T.data_ptr()), n),
                  "get factor")
        d = torch.diagonal(T).abs()
        fro = float(torch.linalg.matrix_norm(T))
        slog = float(torch.log(d).sum())
        del T
        for blas, man, _ in refs:
            assert slog == pytest.approx(man["sum_log_abs_diag_u"], rel=1e-10)
            assert fro == pytest.approx(man["factor_fro"], rel=1e-10)
            assert float(d.min()) == pytest.approx(man["min_abs_diag_u"], rel=1e-9)
            assert float(d.max()) == pytest.approx(man["max_abs_diag_u"], rel=1e-9)
    finally:
        s.free(a, p)
        torch.cuda.empty_cache()
