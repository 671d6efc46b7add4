"""Deterministic inputs of the golden cases, rebuilt from a small spec.

Every matrix is drand48-based exactly like TEST/create_problem.c:31,49-51
(srand48(seed), then drand48()*2-1 in column-major order), optionally followed
by a documented modification.  The generator is the C library's drand48
(POSIX 48-bit LCG), reached through the oracle's fill routine, so this module
is used by tests/ and by make_golden.py only.
"""
from __future__ import annotations

import numpy as np


def build(rs, spec: dict) -> np.ndarray:
    """Return the matrix described by ``spec`` (keys: m, n, seed, [mod], [dtype])."""
    A = rs.drand48_matrix(spec["m"], spec["n"], spec["seed"])
    mod = spec.get("mod")
    if mod == "shift_n":            # TEST/test_chol.c:121-128: A + n*I
        A = A + spec["n"] * np.eye(spec["n"])
    elif mod == "sign":             # every |a_ij| = 1: ties in every pivot search
        A = np.where(A >= 0, 1.0, -1.0)
    elif mod == "zero_last_col":    # exactly singular, zero final pivot
        A[:, -1] = 0.0
    elif mod == "shift_n_neg":      # SPD shift, then one negative diagonal entry
        A = A + spec["n"] * np.eye(spec["n"])
        A[spec["at"], spec["at"]] = -1000.0
    elif mod == "shift_n_sym":      # symmetric positive definite
        A = A + spec["n"] * np.eye(spec["n"])
        A = np.tril(A) + np.tril(A, -1).T
    elif mod is not None:
        raise ValueError(mod)
    A = np.asfortranarray(A)
    if spec.get("dtype") == "float32":
        A = np.asfortranarray(A.astype(np.float32))
    return A
