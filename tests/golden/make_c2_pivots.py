"""Reference pivot fixtures at the large FP64 LU sizes (n = 16384, 32768).

Runs the UPSTREAM PLA_LU (compiled from the reference sources into
oracle/_ref, nb_alg = nb_distr = 128, error checking off, 1x1 template) on the
seed-1 i.i.d. N(0,1) matrix

    A = np.asfortranarray(np.random.default_rng(1).standard_normal((n, n)))

once with the restated netlib BLAS (the bit-reproducible build the golden
fixtures come from) and once with OpenBLAS 0.3.15, and writes per case

    tests/golden/c2/lu_n<n>_<blas>.npz   pivots (int32, PLAPACK offsets)
    tests/golden/c2/manifest.json        SHA-256 of the pivot vector and of
                                          diag(U), ||factor||_F, sum log|u_ii|,
                                          min/max |u_ii|, seconds

The GPU parity test rebuilds A with the same numpy generator on the box and
compares PLA_LU's pivots with these.  The reference tree is needed only here:

    python tests/golden/make_c2_pivots.py --n 16384 32768 --blas netlib openblas

Each (n, blas) case runs in its own process: the netlib build is
single-threaded (about 15 min at n = 16384, 2 h at 32768 on one core), the
OpenBLAS one uses OPENBLAS_NUM_THREADS threads.  Memory: the matrix plus the
reference object's own copy (17 GB at n = 32768).
"""
from __future__ import annotations

import argparse
import ctypes
import hashlib
import json
import os
import subprocess
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "c2")
sys.path.insert(0, ROOT)


def c2_matrix(n: int) -> np.ndarray:
    """The C2 LU input: i.i.d. standard normal entries from numpy's PCG64 seeded with 1."""
    return np.asfortranarray(np.random.default_rng(1).standard_normal((n, n)))


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def run_case(n: int, blas: str, nb: int) -> dict:
    from oracle import oracle as orc
    ref = orc.Reference(blas, nb_distr=nb, nb_alg=nb, error_checking=0)
    A = c2_matrix(n)
    piv = np.zeros(n, dtype=np.int32)
    t = ctypes.c_double()
    vp = ctypes.c_void_p
    r = ref.lib.ref_lu(n, n, 1, A.ctypes.data_as(vp), n, piv.ctypes.data_as(vp),
                       ctypes.byref(t))
    d = np.ascontiguousarray(np.diagonal(A))
    colnorm = np.sqrt(np.einsum("ij,ij->j", A, A))
    os.makedirs(OUT, exist_ok=True)
    np.savez_compressed(os.path.join(OUT, f"lu_n{n}_{blas}.npz"), pivots=piv)
    return {"n": n, "blas": blas, "nb_alg": nb, "nb_distr": nb, "ret": int(r),
            "seconds": t.value,
            "threads": int(os.environ.get("OPENBLAS_NUM_THREADS", "1")) if blas != "netlib" else 1,
            "pivots_sha256": sha(piv), "diag_u_sha256": sha(d),
            "factor_fro": float(np.sqrt((colnorm ** 2).sum())),
            "sum_log_abs_diag_u": float(np.log(np.abs(d)).sum()),
            "min_abs_diag_u": float(np.abs(d).min()), "max_abs_diag_u": float(np.abs(d).max()),
            "generator": "np.asfortranarray(np.random.default_rng(1).standard_normal((n, n)))"}


def record(entry: dict) -> None:
    """Add one case to manifest.json (under a lock: cases may finish concurrently)."""
    import fcntl
    path = os.path.join(OUT, "manifest.json")
    with open(os.path.join(OUT, ".lock"), "w") as lock:
        fcntl.flock(lock, fcntl.LOCK_EX)
        man = {}
        if os.path.exists(path):
            with open(path) as f:
                man = json.load(f)
        man[f"lu_n{entry['n']}_{entry['blas']}"] = entry
        with open(path + ".tmp", "w") as f:
            json.dump(man, f, indent=1, sort_keys=True)
        os.replace(path + ".tmp", path)


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--n", type=int, nargs="+", default=[16384])
    p.add_argument("--blas", nargs="+", default=["netlib", "openblas"])
    p.add_argument("--nb", type=int, default=128)
    p.add_argument("--one", action="store_true", help="run one (n, blas) case in this process")
    a = p.parse_args()
    if a.one:
        e = run_case(a.n[0], a.blas[0], a.nb)
        record(e)
        print(json.dumps(e))
        return
    for n in a.n:
        for blas in a.blas:
            t0 = time.time()
            subprocess.run([sys.executable, __file__, "--one", "--n", str(n), "--blas", blas,
                            "--nb", str(a.nb)], check=True)
            print(f"n={n} {blas}: {time.time() - t0:.0f} s", flush=True)


if __name__ == "__main__":
    main()
