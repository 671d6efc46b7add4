"""Out-of-core matrices and PLA_OOC_Chol against the oracle.

The matrix lives in a file: PLA_OOC_Matrix_create_without_fd, PLA_File_create,
PLA_Obj_attach_fd (OBJ/PLA_Obj_ooc.c:50, IO/PLA_File.c:25,
OBJ/PLA_Obj_management.c:146), filled tile by tile through PLA_Copy from
in-core tiles the way POOCLAPACK/TEST/create_problem_ooc_spd.c does (random
tiles, the diagonal tiles shifted by n so that the matrix its lower triangle
defines is positive definite).  PLA_OOC_Chol (the left-looking tile
algorithm of POOCLAPACK/OOC_Cholesky/PLA_OOC_Chol.c) then overwrites the
lower triangle with L.  The oracle is the restated PLA_Chol (pinned bit for
bit to the compiled reference in test_oracle.py) on the same symmetric
matrix: the Cholesky factor is unique, so the out-of-core factor must match
it within a rounding tolerance whatever the tile and panel sizes.  The
upper triangle in the file must be left as written.  Cases: ragged last
tiles, one tile, the L10 block resident in HBM and streamed with L20
(PLA_B200_OOC_RESIDENT_BYTES=0), FP64 and fp32, a failing column reported
as PLA_Chol reports it, and the IO counters.
"""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import oracle as orc

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def env():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    from plapack_b200 import pla
    s = pla.Session(nb_distr=128, nb_alg=128)
    yield s, pla, orc.Restated()
    s.close()


def make_ooc(s, pla, path, n, dt, nb_tile, rng):
    """An n x n out-of-core matrix in file `path`, filled as create_problem_ooc_spd."""
    lib = s.lib
    a = ctypes.c_void_p()
    pla.check(lib.PLA_OOC_Matrix_create_without_fd(pla.MPI_DOUBLE if dt == np.float64
                                                   else pla.MPI_FLOAT, n, n, s.templ,
                                                   pla.PLA_ALIGN_FIRST, pla.PLA_ALIGN_FIRST,
                                                   ctypes.byref(a)), "OOC create")
    fd = ctypes.c_int()
    pla.check(lib.PLA_File_create(path.encode(), pla.MPI_DOUBLE if dt == np.float64
                                  else pla.MPI_FLOAT, n * n, ctypes.byref(fd)), "File_create")
    pla.check(lib.PLA_Obj_attach_fd(a, fd.value, n, 1), "attach_fd")
    full = np.empty((n, n), dtype=dt)
    shift = ctypes.c_double(float(n))
    for j0 in range(0, n, nb_tile):
        for i0 in range(0, n, nb_tile):
            m, w = min(nb_tile, n - i0), min(nb_tile, n - j0)
            tile = rng.uniform(-1, 1, (m, w)).astype(dt)
            t_in = s.matrix(m, w, dt)
            s.put(t_in, tile)
            if i0 == j0:
                pla.check(lib.PLA_Shift(t_in, pla.MPI_DOUBLE, ctypes.byref(shift)), "Shift")
                tile[np.arange(min(m, w)), np.arange(min(m, w))] += dt(n)
            view = ctypes.c_void_p()
            pla.check(lib.PLA_Obj_view(a, m, w, i0, j0, ctypes.byref(view)), "view")
            pla.check(lib.PLA_Copy(t_in, view), "Copy to file")
            full[i0:i0 + m, j0:j0 + w] = tile
            s.free(t_in, view)
    return a, fd.value, full


def read_back(s, pla, a, n, dt):
    m = s.matrix(n, n, dt)
    pla.check(s.lib.PLA_Copy(a, m), "Copy from file")
    out = s.get(m)
    s.free(m)
    return out


def sym_from_lower(A):
    return np.tril(A) + np.tril(A, -1).T


@pytest.mark.parametrize("dt,n,nb_tile,nb_ooc", [
    (np.float64, 3000, 1024, 128),   # tiles 1024, 1024, 952
    (np.float64, 2500, 2500, 64),    # one tile: the in-core Cholesky
    (np.float64, 2100, 512, 96),     # five tile columns, ragged 52
    (np.float32, 2600, 1024, 128),
])
def test_ooc_chol_matches_oracle(env, tmp_path, dt, n, nb_tile, nb_ooc):
    s, pla, oracle = env
    rng = np.random.default_rng(n + nb_tile)
    path = str(tmp_path / "A.bin")
    a, fd, A = make_ooc(s, pla, path, n, dt, nb_tile, rng)
    assert np.array_equal(read_back(s, pla, a, n, dt), A)     # the file holds what was copied
    assert s.lib.PLA_File_stats_start() == 0
    rc = s.lib.PLA_OOC_Chol(nb_ooc, nb_tile, a)
    assert rc == 0, pla.last_error()
    got = read_back(s, pla, a, n, dt)
    ref, info = oracle.chol_blocked(sym_from_lower(A.astype(np.float64)).astype(dt), 128)
    assert info == 0
    eps = np.finfo(dt).eps
    L, Lr = np.tril(got).astype(np.float64), np.tril(ref).astype(np.float64)
    assert np.abs(L - Lr).max() <= 8 * n * eps * np.abs(Lr).max()
    assert np.array_equal(np.triu(got, 1), np.triu(A, 1))       # upper triangle untouched
    v = [ctypes.c_double() for _ in range(4)]
    s.lib.PLA_B200_file_stats(*[ctypes.byref(x) for x in v])
    assert v[0].value >= n * n * np.dtype(dt).itemsize / 2     # at least the lower triangle read
    assert v[2].value >= n * n * np.dtype(dt).itemsize / 2     # and written back
    s.lib.PLA_File_close(fd)
    s.free(a)


def test_ooc_chol_reports_the_failing_column(env, tmp_path):
    s, pla, oracle = env
    n, nb_tile = 2000, 512
    rng = np.random.default_rng(4)
    a, fd, A = make_ooc(s, pla, str(tmp_path / "B.bin"), n, np.float64, nb_tile, rng)
    # make the matrix indefinite at global column 1301 (1-based)
    bad = s.matrix(1, 1)
    s.put(bad, np.array([[-5.0 * n]]))
    view = ctypes.c_void_p()
    pla.check(s.lib.PLA_Obj_view(a, 1, 1, 1300, 1300, ctypes.byref(view)), "view")
    pla.check(s.lib.PLA_Copy(bad, view), "Copy")
    A[1300, 1300] = -5.0 * n
    rc = s.lib.PLA_OOC_Chol(128, nb_tile, a)
    _, info = oracle.chol_blocked(sym_from_lower(A), 128)
    assert info == 1301
    assert rc == info
    s.lib.PLA_File_close(fd)
    s.free(view, bad, a)


def test_ooc_chol_with_l10_streamed(env, tmp_path):
    # a child process, so that the budget variable is read fresh
    code = r'''
import ctypes, os, sys
import numpy as np
sys.path.insert(0, %r)
sys.path.insert(0, os.path.join(%r, "tests"))
import test_gpu_ooc as t
from oracle import oracle as orc
from plapack_b200 import pla
s = pla.Session(nb_distr=128, nb_alg=128)
n, nb_tile = 2300, 768
a, fd, A = t.make_ooc(s, pla, %r, n, np.float64, nb_tile, np.random.default_rng(8))
assert s.lib.PLA_OOC_Chol(100, nb_tile, a) == 0, pla.last_error()
got = t.read_back(s, pla, a, n, np.float64)
ref, info = orc.Restated().chol_blocked(t.sym_from_lower(A), 128)
assert info == 0
err = np.abs(np.tril(got) - np.tril(ref)).max()
assert err <= 8 * n * np.finfo(float).eps * np.abs(ref).max(), err
print("ok", err)
''' % (ROOT, ROOT, str(tmp_path / "C.bin"))
    envv = dict(os.environ, PLA_B200_OOC_RESIDENT_BYTES="0")
    r = subprocess.run([sys.executable, "-c", code], env=envv, capture_output=True, text=True,
                       timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ok" in r.stdout


def test_ooc_objects_are_refused_where_data_is_needed(env, tmp_path):
    s, pla, _ = env
    a, fd, _ = make_ooc(s, pla, str(tmp_path / "D.bin"), 300, np.float64, 300,
                        np.random.default_rng(1))
    piv = s.mvector(300, 1, np.int32)
    assert s.lib.PLA_LU(a, piv) != 0                      # no device data to factor
    buf = ctypes.c_void_p(1)
    assert s.lib.PLA_Obj_local_buffer(a, ctypes.byref(buf)) == 0 and not buf.value
    s.lib.PLA_File_close(fd)
    s.free(piv, a)
