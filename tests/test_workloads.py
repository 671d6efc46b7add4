"""The benchmark's synthetic inputs have the spectra its JSON line states.

bench.py builds the C3 matrices as U diag(sigma) V' with sigma geometric from
1 to 1/kappa and U, V products of 8 Householder reflectors, and the C4 SPD
matrices as Q diag(lambda) Q' with lambda log-uniform in [1/kappa, 1].  These
run the same generators on the CPU at a small order and check the singular
values (C3), the eigenvalues and symmetry (C4), and b = A x_true.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


@pytest.fixture(scope="module")
def bench():
    from plapack_b200 import workloads
    return workloads


@pytest.mark.parametrize("kappa", [1e2, 1e6, 1e10])
def test_c3_host_spectrum(bench, kappa):
    n = 300
    A, x, b = bench.c3_host(n, kappa, 5)
    sigma = kappa ** (-np.arange(n) / (n - 1))
    sv = np.linalg.svd(A, compute_uv=False)
    assert np.allclose(sv, sigma, rtol=1e-9, atol=1e-13)
    assert np.allclose(b, A @ x, rtol=0, atol=1e-13)
    assert A.flags.f_contiguous


@pytest.mark.parametrize("kappa", [1e2, 1e6])
def test_c3_device_generator_on_cpu(bench, kappa):
    torch = pytest.importorskip("torch")
    n = 256
    T, x, b = bench.c3_device(n, kappa, 9, torch, torch.device("cpu"))
    A = T.t().numpy()                           # T holds A' (column-major A)
    sigma = kappa ** (-np.arange(n) / (n - 1))
    assert np.allclose(np.linalg.svd(A, compute_uv=False), sigma, rtol=1e-9, atol=1e-13)
    assert np.allclose(b.numpy(), A @ x.numpy(), rtol=0, atol=1e-12)


@pytest.mark.parametrize("kappa", [1e3, 1e7])
def test_spd_generator_on_cpu(bench, kappa):
    torch = pytest.importorskip("torch")
    n = 256
    A = bench.spd_device(n, kappa, 41, torch, torch.device("cpu")).numpy()
    assert np.array_equal(A, A.T)
    ev = np.linalg.eigvalsh(A)
    assert ev.min() == pytest.approx(1.0 / kappa, rel=1e-6)
    assert ev.max() == pytest.approx(1.0, rel=1e-9)
    assert np.all(ev > 0)
