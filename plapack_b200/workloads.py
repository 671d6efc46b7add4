"""Seeded synthetic systems of the dense-solve configurations.

* ``c2_matrix``   -- FP64 LU input: i.i.d. N(0, 1) entries (numpy PCG64, seed 1).
* ``c3_device`` / ``c3_host`` -- A = U diag(sigma) V' with sigma geometric from
  1 to 1/kappa and U, V products of 8 Householder reflectors with seeded
  Gaussian vectors, and b = A x_true, x_true ~ N(0, 1).
* ``spd_device``  -- SPD A = Q diag(lambda) Q', lambda log-uniform in
  [1/kappa, 1], Q a product of 8 Householder reflectors.
* ``batched_workload`` -- independent instances of order log-uniform in
  [8, 512]: even ones LU on uniform[-1, 1], odd ones Cholesky on G G'/n + I,
  1 to 4 right-hand sides each, described as ``PLA_Batch_instance`` records.

Every generator is deterministic for its seed; the device generators use a
torch.Generator on the given device, the host ones numpy.
"""
from __future__ import annotations

import ctypes

import numpy as np


def c2_matrix(n: int, seed: int = 1) -> np.ndarray:
    """Column-major n x n FP64 matrix of i.i.d. standard normal entries."""
    return np.asfortranarray(np.random.default_rng(seed).standard_normal((n, n)))


def c3_device(n, kappa, seed, torch, device):
    """Column-major A = U diag(sigma) V' as the memory of a row-major tensor T
    (T = A'), built by 16 seeded Householder reflections of diag(sigma).
    Returns (T, x_true, b = A x_true)."""
    g = torch.Generator(device=device).manual_seed(seed)
    sigma = kappa ** (-torch.arange(n, dtype=torch.float64, device=device) / max(n - 1, 1))
    T = torch.diag(sigma)
    for _ in range(8):                      # T <- H T
        v = torch.randn(n, dtype=torch.float64, device=device, generator=g)
        w = v @ T
        T.addr_(v, w, alpha=-2.0 / float(v @ v))
    for _ in range(8):                      # T <- T H
        v = torch.randn(n, dtype=torch.float64, device=device, generator=g)
        w = T @ v
        T.addr_(w, v, alpha=-2.0 / float(v @ v))
    x = torch.randn(n, 1, dtype=torch.float64, device=device, generator=g)
    b = T.t() @ x                            # b = A x_true
    return T, x, b


def c3_host(n, kappa, seed):
    """The same family on the host (numpy): A (column-major), x_true, b = A x_true.

    Each reflection is one matrix-vector product and one in-place rank-1
    update (BLAS dger on the Fortran-ordered array), so the n = 32768 matrix
    needs no temporaries of its size."""
    from scipy.linalg import blas
    rng = np.random.default_rng(seed)
    sigma = kappa ** (-np.arange(n) / max(n - 1, 1))
    A = np.zeros((n, n), order="F")
    A[np.diag_indices(n)] = sigma
    for _ in range(8):                       # A <- (I - 2 v v'/v'v) A
        v = rng.standard_normal(n)
        A = blas.dger(-2.0 / (v @ v), v, A.T @ v, a=A, overwrite_a=1)
    for _ in range(8):                       # A <- A (I - 2 v v'/v'v)
        v = rng.standard_normal(n)
        A = blas.dger(-2.0 / (v @ v), A @ v, v, a=A, overwrite_a=1)
    x = rng.standard_normal((n, 1))
    return A, x, A @ x


def spd_device(n, kappa, seed, torch, device):
    """A = Q diag(lambda) Q' with lambda log-uniform in [1/kappa, 1] and Q a
    product of 8 Householder reflectors with seeded Gaussian vectors."""
    g = torch.Generator(device=device).manual_seed(seed)
    u = torch.rand(n, dtype=torch.float64, device=device, generator=g)
    lam = torch.exp(u * -np.log(kappa))
    lam[0], lam[-1] = 1.0, 1.0 / kappa
    A = torch.diag(lam)
    for _ in range(8):                      # A <- H A H
        v = torch.randn(n, dtype=torch.float64, device=device, generator=g)
        c = -2.0 / float(v @ v)
        A.addr_(v, v @ A, alpha=c)
        A.addr_(A @ v, v, alpha=c)
    A.add_(A.t().clone()).mul_(0.5)
    return A


def batched_orders(count, seed):
    """Orders, right-hand-side counts and kinds (0 LU, 1 Cholesky) of the
    batched workload: n = round(exp(U(ln 8, ln 512)))."""
    rng = np.random.default_rng(seed)
    ns = np.round(np.exp(rng.uniform(np.log(8), np.log(512), count))).astype(int)
    nrhs = rng.integers(1, 5, count)
    kinds = np.arange(count) % 2
    return ns, nrhs, kinds


def instance_flops(n, kind, nrhs):
    """2/3 n^3 (LU) or 1/3 n^3 (Cholesky) plus 2 n^2 per right-hand side."""
    return (2.0 / 3.0 if kind == 0 else 1.0 / 3.0) * n ** 3 + 2.0 * n * n * nrhs


def batched_workload(torch, pla, device, dtype, count, seed, select=None):
    """The batched instances as PLA_Batch_instance records.

    Matrices of one order share a tensor; `A0`/`B0` keep copies to restore
    them.  With `select` (instance ids, e.g. one rank's share) only those
    instances are materialised; the records keep the global numbering of the
    full workload, so every instance is the same matrix whichever subset it
    is built in.  Returns (records, groups, pivots, flops, ids)."""
    ns, nrhs, kinds = batched_orders(count, seed)
    ids = np.arange(count) if select is None else np.sort(np.asarray(select, dtype=int))
    pos = {int(k): j for j, k in enumerate(ids)}
    es = 8 if dtype == torch.float64 else 4
    arr = (pla.BatchInstance * len(ids))()
    groups = []
    piv = torch.zeros(max(1, int(ns[ids].sum())), dtype=torch.int32, device=device)
    poff = np.concatenate([[0], np.cumsum(ns[ids])[:-1]]).astype(int)
    flops = 0.0
    for n in np.unique(ns):
        n = int(n)
        # one generator per order, seeded from (seed, n): an instance's matrix
        # does not depend on which other instances are built
        gen = torch.Generator(device=device)
        gen.manual_seed(seed * 1000003 + n)
        idx = np.nonzero(ns == n)[0]
        lu = idx[kinds[idx] == 0]
        ch = idx[kinds[idx] == 1]
        A = torch.empty((len(idx), n, n), dtype=dtype, device=device)
        if len(lu):
            A[:len(lu)] = torch.rand((len(lu), n, n), generator=gen, device=device,
                                     dtype=torch.float64).mul_(2).sub_(1).to(dtype)
        if len(ch):
            G = torch.randn((len(ch), n, n), generator=gen, device=device, dtype=torch.float64)
            S = torch.bmm(G, G.transpose(1, 2)).div_(n)
            S.diagonal(dim1=1, dim2=2).add_(1.0)
            A[len(lu):] = S.to(dtype)
            del G, S
        B = torch.randn((len(idx), 4, n), generator=gen, device=device,
                        dtype=torch.float64).to(dtype)
        order = np.concatenate([lu, ch])
        keep = np.array([k in pos for k in order], dtype=bool)
        if not keep.any():
            continue
        sel = np.nonzero(keep)[0]
        A, B = A[sel].contiguous(), B[sel].contiguous()
        order = order[keep]
        for j, k in enumerate(order):
            k = int(k)
            q = pos[k]
            arr[q].n, arr[q].nrhs, arr[q].kind = n, int(nrhs[k]), int(kinds[k])
            arr[q].A = int(A.data_ptr() + j * n * n * es)
            arr[q].B = int(B.data_ptr() + j * 4 * n * es)
            arr[q].pivots = ctypes.cast(int(piv.data_ptr() + int(poff[q]) * 4),
                                        ctypes.POINTER(ctypes.c_int))
            flops += instance_flops(n, int(kinds[k]), int(nrhs[k]))
        groups.append({"n": n, "order": order, "A": A, "B": B,
                       "A0": A.clone(), "B0": B.clone()})
    return arr, groups, piv, flops, ids


def batched_backward_error(torch, groups, nrhs_of):
    """max over instances of ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf),
    A and b the pristine inputs, x the solution left in B (in float64).
    `nrhs_of` maps a (global) instance id to its right-hand-side count."""
    worst = 0.0
    for gr in groups:
        A0 = gr["A0"].double()                 # row-major storage = A' of the column-major A
        X = gr["B"].double()                   # [cnt, 4, n]: column c of instance j is X[j, c]
        B0 = gr["B0"].double()
        R = B0 - torch.bmm(X, A0)              # (A x)' = x' A'
        mask = torch.tensor([[c < nrhs_of[int(k)] for c in range(4)] for k in gr["order"]],
                            device=X.device)
        a_inf = A0.abs().sum(dim=1).max(dim=1).values   # max row sum of A = max col sum of A'
        num = R.abs().amax(dim=2)
        den = a_inf[:, None] * X.abs().amax(dim=2) + B0.abs().amax(dim=2)
        eta = torch.where(mask, num / den, torch.zeros_like(num))
        worst = max(worst, float(eta.max()))
    return worst
