"""The allocation-free panel factorization, through the C ABI.

PLA_B200_lu_panel_noalloc serves callers that cannot let the library call
cudaMalloc (their GPU memory belongs to another allocator, or allocation is
forbidden while they run): its workspace is a fixed device array.  This test
calls it twice in a row on different panels and checks each result against
the existing entry points: bit for bit against the panel kernel with library-
allocated workspace (pla_k_lu_panel), and pivots plus factors within the
tolerance of the other GPU tests against PLA_LU.  It also checks that a panel
wider than the fixed workspace allows is rejected with an error, that an
exactly singular panel reports its first zero pivot in status[1] as
PLA_LU_info does, and that a call whose tag sequence repeats an earlier
call's (the 24-bit sequence wrapped) still gets its own data, because the
array is cleared at each wrap.

The file name makes pytest collect it last.
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
    torch.cuda.set_device(0)
    from plapack_b200 import pla
    s = pla.Session(nb_distr=128, nb_alg=128)
    lib = s.lib
    lib.PLA_B200_lu_panel_noalloc.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                              ctypes.c_void_p, ctypes.c_void_p]
    lib.PLA_B200_lu_panel_noalloc.restype = ctypes.c_int
    lib.pla_k_lu_panel.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                   ctypes.c_long, ctypes.c_void_p, ctypes.c_void_p,
                                   ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    lib.pla_k_lu_panel.restype = ctypes.c_int
    yield s, torch, pla
    s.close()


def panel_on_gpu(torch, A, dtype):
    """Column-major A (m x w) as the memory of a row-major (w x m) tensor."""
    return torch.from_numpy(np.ascontiguousarray(A.T)).to("cuda", dtype)


@pytest.mark.parametrize("dt", ["float64", "float32"])
def test_noalloc_panel_matches_existing_entry_points(env, dt):
    s, torch, pla = env
    lib = s.lib
    tdt = getattr(torch, dt)
    mpi = pla.MPI_DOUBLE if dt == "float64" else pla.MPI_FLOAT
    rng = np.random.default_rng(21 if dt == "float64" else 22)
    for (m, w) in [(3000, 96), (777, 128)]:          # two calls in a row
        A = rng.standard_normal((m, w))
        a_new = panel_on_gpu(torch, A, tdt)
        a_old = panel_on_gpu(torch, A, tdt)
        p_new = torch.zeros(w, dtype=torch.int32, device="cuda")
        p_old = torch.zeros(w, dtype=torch.int32, device="cuda")
        st_new = torch.zeros(4, dtype=torch.int32, device="cuda")
        st_old = torch.zeros(4, dtype=torch.int32, device="cuda")
        rc = lib.PLA_B200_lu_panel_noalloc(mpi, m, w, a_new.data_ptr(), m, p_new.data_ptr(),
                                           st_new.data_ptr(), None)
        assert rc == pla.PLA_SUCCESS, pla.last_error()
        assert lib.pla_k_lu_panel(mpi, m, w, a_old.data_ptr(), m, p_old.data_ptr(),
                                  st_old.data_ptr(), None, 0, None) == 0
        torch.cuda.synchronize()
        assert st_new[0].item() == 0 and st_old[0].item() == 0
        # the same kernel with a different workspace: identical results
        assert torch.equal(p_new, p_old)
        assert torch.equal(a_new, a_old)
        # PLA_LU on the same m x w matrix (one panel, nb_alg >= w)
        obj = s.matrix(m, w, np.dtype(dt))
        piv = s.mvector(w, 1, np.int32)
        s.put(obj, A.astype(dt))
        pla.check(lib.PLA_LU(obj, piv), "PLA_LU")
        LU = s.get(obj)
        assert np.array_equal(s.get(piv)[:, 0], p_new.cpu().numpy())
        eps = np.finfo(np.dtype(dt)).eps
        tol = 4 * m * eps * max(1.0, np.abs(A).max()) * max(1.0, np.abs(LU).max())
        assert np.abs(a_new.cpu().numpy().T - LU).max() <= tol
        s.free(obj, piv)


def test_noalloc_rejects_panels_beyond_its_workspace(env):
    s, torch, pla = env
    a = torch.zeros(129, 200, dtype=torch.float64, device="cuda")
    p = torch.zeros(129, dtype=torch.int32, device="cuda")
    st = torch.zeros(4, dtype=torch.int32, device="cuda")
    rc = s.lib.PLA_B200_lu_panel_noalloc(pla.MPI_DOUBLE, 200, 129, a.data_ptr(), 200,
                                         p.data_ptr(), st.data_ptr(), None)
    assert rc == pla.PLA_ERROR
    assert "128" in pla.last_error()
    s.lib.PLA_Clear_error()


def test_noalloc_reports_the_first_zero_pivot(env):
    s, torch, pla = env
    lib = s.lib
    rng = np.random.default_rng(23)
    m, w = 900, 40
    A = rng.standard_normal((m, w))
    A[:, 6] = 0.0                                  # exactly singular: pivot 7 is zero
    a = panel_on_gpu(torch, A, torch.float64)
    p = torch.zeros(w, dtype=torch.int32, device="cuda")
    st = torch.zeros(2, dtype=torch.int32, device="cuda")
    rc = lib.PLA_B200_lu_panel_noalloc(pla.MPI_DOUBLE, m, w, a.data_ptr(), m, p.data_ptr(),
                                       st.data_ptr(), None)
    assert rc == pla.PLA_SUCCESS, pla.last_error()
    torch.cuda.synchronize()
    obj = s.matrix(m, w)
    piv = s.mvector(w, 1, np.int32)
    s.put(obj, A)
    info = ctypes.c_int(-1)
    pla.check(lib.PLA_LU_info(obj, piv, ctypes.byref(info)), "PLA_LU_info")
    assert int(st[0].item()) == 0
    assert int(st[1].item()) == info.value == 7
    assert np.array_equal(s.get(piv)[:6, 0], p.cpu().numpy()[:6])
    s.free(obj, piv)


def test_noalloc_after_the_tag_sequence_wraps(env):
    s, torch, pla = env
    lib = s.lib
    lib.pla_k_panel_sequence.restype = ctypes.c_uint
    lib.pla_k_panel_set_sequence.argtypes = [ctypes.c_uint]
    lib.pla_k_panel_set_sequence.restype = None
    rng = np.random.default_rng(24)
    # a tall, wide call fills much of the array with its tagged words
    m0, w0 = 6000, 128
    a0 = panel_on_gpu(torch, rng.standard_normal((m0, w0)), torch.float64)
    p0 = torch.zeros(w0, dtype=torch.int32, device="cuda")
    st0 = torch.zeros(2, dtype=torch.int32, device="cuda")
    assert lib.PLA_B200_lu_panel_noalloc(pla.MPI_DOUBLE, m0, w0, a0.data_ptr(), m0,
                                         p0.data_ptr(), st0.data_ptr(), None) == 0
    torch.cuda.synchronize()
    seq = lib.pla_k_panel_sequence()
    # 2^24 launches on: the next call's tags repeat the ones just written
    lib.pla_k_panel_set_sequence((seq + (1 << 24) - 1) & 0xffffffff)
    m, w = 1500, 64
    A = rng.standard_normal((m, w))
    a_new, a_old = panel_on_gpu(torch, A, torch.float64), panel_on_gpu(torch, A, torch.float64)
    p_new = torch.zeros(w, dtype=torch.int32, device="cuda")
    p_old = torch.zeros(w, dtype=torch.int32, device="cuda")
    st_new = torch.zeros(2, dtype=torch.int32, device="cuda")
    st_old = torch.zeros(2, dtype=torch.int32, device="cuda")
    assert lib.PLA_B200_lu_panel_noalloc(pla.MPI_DOUBLE, m, w, a_new.data_ptr(), m,
                                         p_new.data_ptr(), st_new.data_ptr(), None) == 0
    assert lib.pla_k_lu_panel(pla.MPI_DOUBLE, m, w, a_old.data_ptr(), m, p_old.data_ptr(),
                              st_old.data_ptr(), None, 0, None) == 0
    torch.cuda.synchronize()
    assert lib.pla_k_panel_sequence() >> 24 == ((seq + (1 << 24)) & 0xffffffff) >> 24
    assert int(st_new[0].item()) == 0 and int(st_old[0].item()) == 0
    assert torch.equal(p_new, p_old) and torch.equal(a_new, a_old)
