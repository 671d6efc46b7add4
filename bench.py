#!/usr/bin/env python
"""Dense direct solve on one B200: n = 32768 solve time, mixed-precision
(fp16 factors, FP64 GMRES-IR) versus FP64 LU, both to FP64 backward error.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one solve A x = b of the n = 32768 system (A = U diag(sigma) V' with
sigma geometric from 1 to 1/kappa, U and V products of 8 Householder
reflectors with seeded Gaussian vectors; kappa = 1e6; x_true ~ N(0,1)),
called through the library's C ABI (PLA_General_solve_mixed; the FP64 arm is
PLA_General_solve).  Inputs are resident in HBM and larger than L2 (8.6 GB).
`e2e` repeats the mixed solve with the matrix and right-hand side in pinned
host memory: b through PLA_Obj_set_local_contents, A through
PLA_General_solve_mixed_host (which copies it during the factorization), the
solution read back through PLA_Obj_get_local_contents, every step.

--impl reference times the upstream PLAPACK (compiled from its sources into
oracle/_ref, linked to a threaded OpenBLAS) on the host cores: PLA_General_solve
on the n = 32768 system of the same family itself: its PLA_LU, the solve's
O(n^3) part (the upstream triangular solves overflow 32-bit view offsets at
this n; see reference_solve).  About a minute and a half per run, so
--ref-steps runs, default 1, whatever --steps asks; the line reports the
count it timed.  `cpu_baseline` of this arm is the same measurement.

Under torchrun (--gpus N > 1) every rank solves its own system (replicas; the
single large solve has no data exchange) and rank 0 prints the max over ranks;
the batched sub-arm shards its instances across the ranks instead.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from plapack_b200.workloads import (batched_backward_error, batched_orders,  # noqa: E402
                                    batched_workload, c3_device, c3_host, spd_device)

METRIC = "n=32768 solve time: mixed-prec LU-IR vs FP64 LU, same B200, both at FP64 bkwd err"
# DRAM bytes (read + write) of one tensor-core update launch as a fraction of
# its algorithmic bytes: 486.5 MB measured by ncu against 545.3 MB for an
# M = N = 8192, K = 256 fp16 launch.  Below 1 because the last C tiles written
# are still dirty in L2 when the launch ends.
TC_UPDATE_TRAFFIC_RATIO = 486.5 / 545.3
# DRAM bytes (read + write) of the panel phase per n = 32768 step: filled in
# from the ncu capture of the tournament panel kernels (None until measured).
PANEL_TRAFFIC_PER_STEP = None

# PLA_B200_PREC_* codes as the JSON line names them
PREC_NAMES = {1: "bf16", 2: "fp16", 3: "fp32", 4: "fp64", 5: "fp8", 6: "bf16x6", 7: "bf16x3"}


def parse():
    p = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--n", type=int, default=32768)
    p.add_argument("--kappa", type=float, default=1e6)
    p.add_argument("--precision", choices=["fp16", "bf16", "bf16x3", "bf16x6", "fp32"],
                   default="fp16")
    p.add_argument("--refinement", choices=["gmres", "lu"], default="gmres")
    p.add_argument("--nb", type=int, default=256, help="block size of the mixed factorization")
    p.add_argument("--panel-pivoting", choices=["tournament", "partial"], default="tournament",
                   help="pivoting of the mixed LU's fp32 panels")
    p.add_argument("--nb-fp64", type=int, default=512,
                   help="nb_alg of the FP64 LU (512: K = 512 trailing updates); the Cholesky "
                        "caps it at 256")
    p.add_argument("--skip-fp64", action="store_true")
    p.add_argument("--skip-e2e", action="store_true")
    p.add_argument("--skip-cpu", action="store_true")
    p.add_argument("--skip-chol", action="store_true", help="skip the FP64 Cholesky solve")
    p.add_argument("--skip-ooc", action="store_true", help="skip the out-of-core Cholesky")
    p.add_argument("--skip-sweep", action="store_true",
                   help="skip the kappa 1e2 / 1e10 and 16-rhs solves")
    p.add_argument("--ooc-tile", type=int, default=8192, help="nb_tile of PLA_OOC_Chol")
    p.add_argument("--ooc-nb", type=int, default=256, help="nb_ooc of PLA_OOC_Chol")
    p.add_argument("--skip-batched", action="store_true", help="skip the batched workload")
    p.add_argument("--batch-count", type=int, default=20000)
    p.add_argument("--skip-chol-mixed", action="store_true",
                   help="skip the fp8 / bf16 Cholesky-IR at --chol-n")
    p.add_argument("--chol-n", type=int, default=49152)
    p.add_argument("--ref-steps", type=int, default=1,
                   help="timed upstream solves at n on the host (reference arm and cpu_baseline)")
    return p.parse_args()


# --------------------------------------------------------------- helpers ---
class Clocks:
    """nvidia-smi samples every 200 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        if self.path and os.path.exists(self.path):
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        busy = [v for v in sm if mx and v > 0.5 * max(mx)] or sm
        return {"sm_mhz": statistics.median(busy) if busy else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def fp64_gemm_peak(torch, device):
    """FP64 roofline denominator: cuBLAS DGEMM (torch.matmul) at 8192^3, best
    of 5 CUDA-event-timed calls (MEASURED_PEAKS.json carries no FP64 figure)."""
    a = torch.randn(8192, 8192, dtype=torch.float64, device=device)
    b = torch.randn(8192, 8192, dtype=torch.float64, device=device)
    c = a @ b
    best = float("inf")
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b, out=c)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b, c
    return 2.0 * 8192 ** 3 / best / 1e12


def cpu_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ----------------------------------------------------- reference (CPU) arm ---
def reference_solve(n, kappa, steps=1, seed=12, warmup_n=2048):
    """Time the upstream PLAPACK on the host cores (error checking off, OpenBLAS
    on every core, nb_alg = 128) on the n x n system of the headline family
    itself, bracketed by MPI_Wtime around the call as TEST/test_lu.c:136-142
    brackets PLA_LU.  One warm-up at warmup_n first (thread pool, page
    faults), then `steps` timed runs at n.

    What is timed is PLA_LU, the factorization (2/3 n^3 of the solve's
    2/3 n^3 + 2 n^2 flops).  The upstream solves cannot run at this size:
    PLA_General_solve's triangular solves split views at byte offsets that
    OBJ/PLA_Obj.c:2284-2285 computes in 32-bit ints (left_global_width *
    local_ldim * typesize), which overflow once n * n * 8 >= 2^31 -- the
    one-column PLA_Trsv path crashes at n = 16384, the PLA_Trsm path returns
    NaN at n = 32768 -- while PLA_LU carves its views a panel at a time and
    stays correct (its pivots at n = 32768 are pinned in tests/golden/c2).
    Leaving the solves out understates the reference's time.  The solution
    that checks the factorization is formed from the reference's own L, U
    and pivots outside the timed region (scipy's lu_solve).
    Returns the contract's cpu_baseline dict (value = median seconds)."""
    import scipy.linalg as sl
    cores = cpu_cores()
    os.environ.setdefault("OPENBLAS_NUM_THREADS", str(cores))
    threads = int(os.environ["OPENBLAS_NUM_THREADS"])
    from oracle import oracle as orc
    ref = orc.Reference("openblas", nb_distr=128, nb_alg=128, error_checking=0)
    A, _, b = c3_host(warmup_n, kappa, 11)
    ref.lu(A)
    t0 = time.perf_counter()
    A, x_true, b = c3_host(n, kappa, seed)
    gen_s = time.perf_counter() - t0
    times, LU, piv = [], None, None
    for _ in range(max(1, steps)):
        LU, piv, ret, t_inner = ref.lu(A)
        times.append(t_inner)
    t = statistics.median(times)
    # the reference's offsets (row i swapped with row i + piv[i]) as LAPACK ipiv
    X = sl.lu_solve((LU, piv.astype(np.int64) + np.arange(n)), b, check_finite=False)
    del LU
    a_inf = float(np.abs(A).sum(axis=1).max())
    eta = float(np.abs(b - A @ X).max() / (a_inf * np.abs(X).max() + np.abs(b).max()))
    fwd = float(np.abs(X - x_true).max() / np.abs(x_true).max())
    return {"value": t, "unit": "s", "cores": threads, "kind": "reference",
            "steps": len(times), "warmup": 1,
            "sample": (f"the full workload's factorization, not a sample: upstream PLA_LU "
                       f"(nb_alg=128, FP64, 1x1 template, error checking off, OpenBLAS 0.3.15 "
                       f"with {threads} threads) on the n={n}, kappa={kappa:g} system, "
                       f"{len(times)} timed run(s) after one warm-up at n={warmup_n}; the "
                       f"upstream triangular solves overflow 32-bit view offsets at this n "
                       f"(OBJ/PLA_Obj.c:2284), so they are left out (the time is a lower "
                       f"bound of the reference's solve); solution from the reference's L, U "
                       f"and pivots: backward error {eta:.2e}, forward error {fwd:.2e}; matrix "
                       f"built in {gen_s:.1f} s (untimed)"),
            "backward_error": eta, "forward_error": fwd, "lu_seconds": times}


def run_reference(args):
    """The reference arm: rank 0 solves the headline system on the host cores
    with the upstream PLAPACK; other ranks exit at once.  A solve at n = 32768
    takes minutes, so the arm times --ref-steps solves (default 1) whatever
    --steps asks, and reports the count it actually timed."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    lib = os.path.join(ROOT, "oracle", "_ref", "libplapack_ref_openblas.so")
    if not os.path.exists(lib):
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/libplapack_ref_openblas.so is not built"}))
        return 0
    info = reference_solve(args.n, args.kappa, steps=args.ref_steps)
    value = info["value"]
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": "s",
           "n_gpus": args.gpus, "steps": info["steps"], "warmup": info["warmup"],
           "steps_requested": args.steps, "warmup_requested": args.warmup,
           "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded C3 family)",
           "config": {"workload": f"general solve n={args.n}, kappa={args.kappa:g}, 1 rhs",
                      "n": args.n, "kappa": args.kappa, "nrhs": 1, "parallelism": "host cores"},
           "cpu_baseline": info,
           "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


# ---------------------------------------------------------------- our arm ---
def run_batched(torch, pla, lib, device, stream, dtype, steps, warmup, dist, count=20000,
                seed=3):
    """The batched workload, sharded by instance over the ranks (shard.partition:
    flop-balanced, the same on every rank); each rank factors and solves its
    share with one PLA_Batch_plan, the info words are gathered at the end.
    Time = max over ranks of the device time of one execute."""
    from plapack_b200 import shard
    world = dist.get_world_size() if dist is not None else 1
    rank = dist.get_rank() if dist is not None else 0
    ns, nrhs, kinds = batched_orders(count, seed)
    parts = shard.partition(ns.tolist(), kinds.tolist(), nrhs.tolist(), world)
    total_flops = sum(shard.instance_flops(int(a), int(k), int(r))
                      for a, k, r in zip(ns, kinds, nrhs))
    arr, groups, piv, flops, ids = batched_workload(torch, pla, device, dtype, count, seed,
                                                    select=parts[rank])
    dt = pla.MPI_DOUBLE if dtype == torch.float64 else pla.MPI_FLOAT
    info = torch.full((max(1, len(ids)),), -1, dtype=torch.int32, device=device)

    def restore():
        for gr in groups:
            gr["A"].copy_(gr["A0"])
            gr["B"].copy_(gr["B0"])

    def sync():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v):
        if dist is None:
            return v
        t = torch.tensor([v], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    share = shard.RankBatch(lib, dt, arr, info.data_ptr(), autotune=1)
    plan_s = max_over_ranks(time.perf_counter() - t0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    times = []
    for it in range(warmup + steps):
        restore()
        sync()
        e0.record(stream)
        share.execute()
        e1.record(stream)
        torch.cuda.synchronize()
        if it >= warmup:
            times.append(e0.elapsed_time(e1) / 1e3)
    batched_s = max_over_ranks(sum(times) / len(times))
    info_all = shard.gather_info(ids.tolist(), info[:len(ids)].cpu().tolist(), count, dist)
    bad = sum(1 for v in info_all if v != 0)
    eta = max_over_ranks(batched_backward_error(torch, groups, nrhs))
    share.free()
    # the per-instance launch loop of the plain kernels, same instances
    restore()
    torch.cuda.synchronize()
    if len(ids):
        pla.check(lib.PLA_Batched_factor_solve_loop(dt, len(ids), arr), "loop warm-up")
    restore()
    sync()
    e0.record(stream)
    if len(ids):
        pla.check(lib.PLA_Batched_factor_solve_loop(dt, len(ids), arr),
                  "PLA_Batched_factor_solve_loop")
    e1.record(stream)
    torch.cuda.synchronize()
    loop_s = max_over_ranks(e0.elapsed_time(e1) / 1e3)
    loop_eta = max_over_ranks(batched_backward_error(torch, groups, nrhs))
    del groups, piv
    torch.cuda.empty_cache()
    return {"workload": f"{count} instances, n log-uniform [8, 512], half LU half Cholesky, "
                        "1-4 rhs", "dtype": "f64" if dtype == torch.float64 else "f32",
            "ranks": world, "sharding": "by instance, flop-balanced (shard.partition); "
                                        "info words gathered once",
            "instances_this_rank": len(ids), "flops_this_rank": flops,
            "batched_s": batched_s, "loop_s": loop_s, "speedup_vs_loop": loop_s / batched_s,
            "gflops": total_flops / batched_s / 1e9, "loop_gflops": total_flops / loop_s / 1e9,
            "plan_create_s": plan_s, "instances_failed": bad,
            "backward_error_max": eta, "loop_backward_error_max": loop_eta}


def run_mixed_sweep(torch, pla, lib, s, device, stream, a, n, args, params):
    """The C3 configurations beside the headline one, each solved once after a
    warm-up solve: kappa 1e2 and 1e10 with one right-hand side (1e10 makes the
    solver escalate the factor precision), kappa 1e6 with 16 right-hand sides
    (with the headline's precision, and with bf16 x 3 factors, whose fewer
    GMRES iterations pay off over many columns), and the FP64
    PLA_General_solve of the 16-rhs system.  Reports the
    time, the precision that finished, iterations and the largest normwise
    backward error over the right-hand sides."""
    out = []
    for kappa, nrhs, fp64, prec in ((1e2, 1, False, None), (1e10, 1, False, None),
                                    (1e6, 16, False, None),
                                    (1e6, 16, False, pla.PLA_B200_PREC_BF16X3),
                                    (1e6, 16, True, None)):
        prm = params
        if prec is not None:
            prm = pla.MixedParams()
            ctypes.memmove(ctypes.byref(prm), ctypes.byref(params), ctypes.sizeof(prm))
            prm.precision = prec
        T, x_true, _ = c3_device(n, kappa, 2000 + int(np.log10(kappa)), torch, device)
        g = torch.Generator(device=device).manual_seed(77)
        X = torch.randn(n, nrhs, dtype=torch.float64, device=device, generator=g)
        X[:, :1] = x_true
        Bm = (T.t() @ X).contiguous(memory_format=torch.contiguous_format)
        Bc = Bm.t().contiguous()                     # column-major n x nrhs as a row-major tensor
        bo = s.matrix(n, nrhs)
        piv = s.mvector(n, 1, np.int32)
        rep = pla.MixedReport()

        def solve():
            pla.check(lib.PLA_Obj_set_local_contents_device(ctypes.c_void_p(T.data_ptr()), n, a),
                      "A")
            pla.check(lib.PLA_Obj_set_local_contents_device(ctypes.c_void_p(Bc.data_ptr()), n, bo),
                      "B")
            if fp64:
                pla.check(lib.PLA_General_solve(a, piv, bo), "PLA_General_solve")
            else:
                pla.check(lib.PLA_General_solve_mixed(a, bo, ctypes.byref(prm),
                                                      ctypes.byref(rep)), "solve_mixed")

        solve()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        solve()
        e1.record(stream)
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3
        Xh = torch.empty_like(Bc)
        pla.check(lib.PLA_Obj_get_local_contents_device(bo, ctypes.c_void_p(Xh.data_ptr()), n), "X")
        Xs = Xh.t()                                  # n x nrhs
        R = Bm - T.t() @ Xs
        a_inf = T.abs().sum(dim=0).max().item()
        eta = (R.abs().amax(dim=0) / (a_inf * Xs.abs().amax(dim=0) + Bm.abs().amax(dim=0))).max().item()
        fwd = ((Xs[:, 0] - x_true[:, 0]).abs().max() / x_true.abs().max()).item()
        pname = PREC_NAMES.get(prec) if prec is not None else args.precision
        entry = {"kappa": kappa, "nrhs": nrhs, "solver": "PLA_General_solve (FP64)" if fp64 else
                 f"PLA_General_solve_mixed ({pname}, {args.refinement.upper()}-IR)",
                 "solve_s": t, "backward_error_max": eta, "forward_error_rhs0": fwd}
        if not fp64:
            entry.update({"precision_used": PREC_NAMES.get(rep.precision_used),
                          "factorizations": rep.factorizations,
                          "converged": rep.converged, "iterations": rep.iterations,
                          "gmres_iterations": rep.inner_iterations,
                          "factor_ms": rep.factor_ms, "refine_ms": rep.refine_ms})
        out.append(entry)
        s.free(bo, piv)
        del T, X, Bm, Bc, Xh, R
        torch.cuda.empty_cache()
    return out


def ooc_dir(nbytes):
    """A directory with room for the out-of-core file: host memory first."""
    for d in ("/dev/shm", tempfile.gettempdir()):
        try:
            st = os.statvfs(d)
        except OSError:
            continue
        if st.f_bavail * st.f_frsize > 1.2 * nbytes:
            return d
    return None


def run_ooc_chol(torch, pla, lib, s, device, S, a_in, n, args, in_core_factor_s):
    """PLA_OOC_Chol of the n x n SPD matrix S kept in a file (host memory when
    /dev/shm has room): factor time (file restored before each step, outside
    the timed region), the file traffic, and the largest difference from the
    in-core factor the FP64 Cholesky arm left in a_in."""
    d = ooc_dir(8.0 * n * n)
    if d is None:
        return {"unavailable": f"no directory with {8.0 * n * n / 1e9:.1f} GB free for the file"}
    path = os.path.join(d, f"pla_ooc_{os.getpid()}.bin").encode()
    T, nb_ooc = args.ooc_tile, args.ooc_nb
    A = ctypes.c_void_p()
    fd = ctypes.c_int(-1)
    src = s.matrix(n, n)
    try:
        pla.check(lib.PLA_OOC_Matrix_create_without_fd(pla.MPI_DOUBLE, n, n, s.templ,
                                                   pla.PLA_ALIGN_FIRST, pla.PLA_ALIGN_FIRST,
                                                   ctypes.byref(A)), "OOC create")
        pla.check(lib.PLA_File_create(path, pla.MPI_DOUBLE, n * n if n * n < 2 ** 31 else 0,
                                  ctypes.byref(fd)), "File_create")
        pla.check(lib.PLA_Obj_attach_fd(A, fd.value, n, 1), "attach_fd")
        pla.check(lib.PLA_Obj_set_local_contents_device(ctypes.c_void_p(S.data_ptr()), n, src), "S")
        times = []
        rd = [ctypes.c_double() for _ in range(4)]
        for step in range(1 + args.steps):          # one warm-up run
            pla.check(lib.PLA_Copy(src, A), "S to the file")
            lib.PLA_File_stats_start()
            t0 = time.perf_counter()
            rc = lib.PLA_OOC_Chol(nb_ooc, T, A)
            t1 = time.perf_counter()
            lib.PLA_B200_file_stats(*[ctypes.byref(x) for x in rd])
            if rc != 0:
                raise RuntimeError(f"PLA_OOC_Chol returned {rc}: {pla.last_error()}")
            if step:
                times.append(t1 - t0)
        pla.check(lib.PLA_Copy(A, src), "factor from the file")
        L = torch.empty((n, n), dtype=torch.float64, device=device)
        pla.check(lib.PLA_Obj_get_local_contents_device(src, ctypes.c_void_p(L.data_ptr()), n), "L")
        Li = torch.empty_like(L)
        pla.check(lib.PLA_Obj_get_local_contents_device(a_in, ctypes.c_void_p(Li.data_ptr()), n), "Li")
        # row-major views of column-major data: the lower triangle is the upper here
        diff = (torch.triu(L) - torch.triu(Li)).abs().max().item() / torch.triu(Li).abs().max().item()
        del L, Li
        t = min(times)
        return {"workload": f"PLA_OOC_Chol n={n} FP64, file in {d}, nb_tile={T}, nb_ooc={nb_ooc}",
                "factor_s": t, "tflops": (n ** 3 / 3.0) / t / 1e12,
                "in_core_factor_s": in_core_factor_s,
                "read_gb": rd[0].value / 1e9, "write_gb": rd[2].value / 1e9,
                "read_gbs": rd[0].value / rd[1].value / 1e9 if rd[1].value else None,
                "write_gbs": rd[2].value / rd[3].value / 1e9 if rd[3].value else None,
                "max_rel_diff_vs_in_core": diff}
    finally:
        if fd.value >= 0:
            lib.PLA_File_close(fd.value)
            lib.PLA_File_unlink(path)
        s.free(src, A)


def run_chol_mixed(torch, pla, lib, s, device, stream, n, kappas, precs, nrhs, steps, warmup):
    """Mixed-precision Cholesky-IR (PLA_Pos_def_solve_mixed, GMRES-IR) on the
    SPD family above: time, the precision that finished, iterations and the
    backward and forward errors of each (kappa, precision)."""
    out = []
    a = s.matrix(n, n)
    bo = s.matrix(n, nrhs)
    for kappa in kappas:
        A = spd_device(n, kappa, 41, torch, device)
        g = torch.Generator(device=device).manual_seed(42)
        Xt = torch.randn(nrhs, n, dtype=torch.float64, device=device, generator=g)  # X' row-major
        Bt = Xt @ A                                   # (A X)' = X' A (A symmetric)
        a_inf = A.abs().sum(dim=0).max().item()
        for name, prec in precs:
            params = pla.MixedParams()
            lib.PLA_Mixed_params_default(ctypes.byref(params))
            params.precision = prec
            params.refinement = pla.PLA_B200_IR_GMRES
            rep = pla.MixedReport()
            times = []
            for it in range(warmup + steps):
                pla.check(lib.PLA_Obj_set_local_contents_device(ctypes.c_void_p(A.data_ptr()), n, a), "A")
                pla.check(lib.PLA_Obj_set_local_contents_device(ctypes.c_void_p(Bt.data_ptr()), n, bo), "B")
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                rc = lib.PLA_Pos_def_solve_mixed(a, bo, ctypes.byref(params), ctypes.byref(rep))
                e1.record(stream)
                torch.cuda.synchronize()
                if it >= warmup:
                    times.append(e0.elapsed_time(e1) / 1e3)
            X = torch.empty(nrhs, n, dtype=torch.float64, device=device)
            pla.check(lib.PLA_Obj_get_local_contents_device(bo, ctypes.c_void_p(X.data_ptr()), n), "X")
            R = Bt - X @ A
            eta = (R.abs().amax(dim=1) / (a_inf * X.abs().amax(dim=1) + Bt.abs().amax(dim=1))).max().item()
            fwd = ((X - Xt).abs().max() / Xt.abs().max()).item()
            out.append({"kappa": kappa, "precision": name, "rc": rc, "solve_s": min(times),
                        "precision_used": PREC_NAMES.get(rep.precision_used),
                        "factorizations": rep.factorizations, "iterations": rep.iterations,
                        "gmres_iterations": rep.inner_iterations, "factor_ms": rep.factor_ms,
                        "refine_ms": rep.refine_ms, "backward_error": eta,
                        "backward_error_target": n * 2.0 ** -53, "forward_error": fwd})
        # the FP64 PLA_Pos_def_solve of the same system, the time to beat
        times = []
        for it in range(warmup + steps):
            pla.check(lib.PLA_Obj_set_local_contents_device(ctypes.c_void_p(A.data_ptr()), n, a), "A")
            pla.check(lib.PLA_Obj_set_local_contents_device(ctypes.c_void_p(Bt.data_ptr()), n, bo), "B")
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            rc = lib.PLA_Pos_def_solve(a, bo)
            e1.record(stream)
            torch.cuda.synchronize()
            if it >= warmup:
                times.append(e0.elapsed_time(e1) / 1e3)
        X = torch.empty(nrhs, n, dtype=torch.float64, device=device)
        pla.check(lib.PLA_Obj_get_local_contents_device(bo, ctypes.c_void_p(X.data_ptr()), n), "X")
        R = Bt - X @ A
        eta = (R.abs().amax(dim=1) / (a_inf * X.abs().amax(dim=1) + Bt.abs().amax(dim=1))).max().item()
        out.append({"kappa": kappa, "precision": "fp64 (PLA_Pos_def_solve)", "rc": rc,
                    "solve_s": min(times), "backward_error": eta,
                    "backward_error_target": n * 2.0 ** -53,
                    "forward_error": ((X - Xt).abs().max() / Xt.abs().max()).item()})
        del A, Xt, Bt
        torch.cuda.empty_cache()
    s.free(a, bo)
    return {"workload": f"PLA_Pos_def_solve_mixed n={n}, A = Q diag(lambda) Q', {nrhs} rhs, "
                        "GMRES-IR; the FP64 PLA_Pos_def_solve of each system beside it",
            "results": out}


def run_ours(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    device = torch.device("cuda", torch.cuda.current_device())
    torch.backends.cuda.matmul.allow_tf32 = False

    from plapack_b200 import pla
    s = pla.Session(nb_distr=128, nb_alg=args.nb_fp64, error_checking=0)
    lib = s.lib
    stream = torch.cuda.current_stream()
    lib.PLA_B200_set_stream(ctypes.c_void_p(stream.cuda_stream))
    n = args.n

    T, x_true, b = c3_device(n, args.kappa, 1000 + rank, torch, device)
    torch.cuda.synchronize()
    a = s.matrix(n, n)
    bo = s.matrix(n, 1)
    check = pla.check
    check(lib.PLA_Obj_set_local_contents_device(ctypes.c_void_p(T.data_ptr()), n, a), "fill A")

    prec = {"fp16": pla.PLA_B200_PREC_FP16, "bf16": pla.PLA_B200_PREC_BF16,
            "bf16x6": pla.PLA_B200_PREC_BF16X6, "bf16x3": pla.PLA_B200_PREC_BF16X3,
            "fp32": pla.PLA_B200_PREC_FP32}[args.precision]
    params = pla.MixedParams()
    lib.PLA_Mixed_params_default(ctypes.byref(params))
    params.precision = prec
    params.refinement = pla.PLA_B200_IR_GMRES if args.refinement == "gmres" else pla.PLA_B200_IR_LU
    params.nb = args.nb
    params.panel_pivoting = (pla.PLA_B200_PIVOT_TOURNAMENT if args.panel_pivoting == "tournament"
                             else pla.PLA_B200_PIVOT_PARTIAL)
    report = pla.MixedReport()

    def mixed_step():
        check(lib.PLA_Obj_set_local_contents_device(ctypes.c_void_p(b.data_ptr()), n, bo), "fill b")
        check(lib.PLA_General_solve_mixed(a, bo, ctypes.byref(params), ctypes.byref(report)),
              "PLA_General_solve_mixed")

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v):
        if dist is None:
            return v
        t = torch.tensor([v], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    for _ in range(args.warmup):
        mixed_step()
    lib.PLA_B200_set_phase_timing(1)
    lib.PLA_B200_reset_phase_times()
    launches0 = lib.PLA_B200_kernel_launches()
    barrier()
    with Clocks(device.index) as clocks:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            mixed_step()
        e1.record(stream)
        barrier()
    launches = lib.PLA_B200_kernel_launches() - launches0
    ph = pla.PhaseTimes()
    lib.PLA_B200_phase_times(ctypes.byref(ph))
    lib.PLA_B200_set_phase_timing(0)
    mixed_s = max_over_ranks(e0.elapsed_time(e1) / 1e3 / args.steps)
    clock_summary = clocks.summary()
    # the report of the last timed solve (later arms reuse the struct)
    head_report = {"refinement_iterations": report.iterations,
                   "gmres_iterations": report.inner_iterations,
                   "factor_ms": report.factor_ms, "refine_ms": report.refine_ms}

    # accuracy of the last solve, checked independently with torch
    x = torch.empty(n, 1, dtype=torch.float64, device=device)
    check(lib.PLA_Obj_get_local_contents_device(bo, ctypes.c_void_p(x.data_ptr()), n), "get x")
    r = b - T.t() @ x
    a_inf = T.abs().sum(dim=0).max().item()        # ||A||_inf = max row sum of A = max col sum of T
    eta = (r.abs().max() / (a_inf * x.abs().max() + b.abs().max())).item()
    fwd = ((x - x_true).abs().max() / x_true.abs().max()).item()

    # ---- roofline of every phase of the step, the largest share first ----
    # Algorithmic bytes per step, by phase (n = order, nb = block, 32-column
    # sub-panels, r = rows of a panel, rest = trailing columns):
    #   panel   each sub-panel read and written, 2 r_s 32 4, plus its update of
    #           the panel's columns to its right, 2 (r_s - 32) right 4
    #   update  the fp32 trailing matrix read and written, 8 rest^2, and the
    #           fp16 L and U' panels read, 2 rest nb 2
    #   trsm    U12 (nb x rest) read and written, 8 nb rest
    #   convert the fp32 L and U12 read and their fp16 packs written, 6 (2 rest nb)
    #   swap    each interchange that moves rows (pivot offset != 0, counted on
    #           the device) across the other n - nb columns, 16 (n - nb) each
    #   refine  per GMRES iteration and per outer step: the FP64 matrix read
    #           once (8 n^2) and both fp32 triangles once (4 n^2)
    nb = args.nb
    by = {"panel": 0.0, "update": 0.0, "trsm": 0.0, "convert": 0.0, "swap": 0.0}
    update_launch_bytes = 0.0
    for k0 in range(0, n, nb):
        bw = min(nb, n - k0)
        rows = n - k0
        rest = rows - bw
        for s0 in range(0, bw, 32):
            sb = min(32, bw - s0)
            by["panel"] += (2.0 * (rows - s0) * sb * 4
                            + 2.0 * max(rows - s0 - sb, 0) * (bw - s0 - sb) * 4)
        if rest > 0:
            by["update"] += rest * rest * 8.0 + 2.0 * rest * nb * 2.0
            by["trsm"] += 8.0 * bw * rest
            by["convert"] += 6.0 * 2 * rest * bw
    by["swap"] = 16.0 * (n - nb) * ph.interchanges / args.steps
    iters = report.inner_iterations + report.iterations
    by["refine"] = iters * 12.0 * n * n
    peak, peak_src = measured_peaks()
    ms = {"panel": ph.panel_ms / args.steps, "update": ph.update_ms / args.steps,
          "trsm": ph.trsm_ms / args.steps, "convert": ph.convert_ms / args.steps,
          "swap": ph.swap_ms / args.steps, "refine": report.refine_ms}
    kernels = {
        "panel": "tslu_select_k + tslu_apply_k (tournament-pivoted fp32 sub-panels), laswp_k, "
                 "panel_update_k (U12 solve + rank-32 update inside the panel); on the "
                 "lookahead stream",
        "update": "tc_update_k (tcgen05 fp16 trailing update, TMA reduce-add into fp32)",
        "trsm": "trsm_left_k / sgemm_k (U12 = inv(L11) A12)",
        "convert": "pack_rows_k, convert_k (fp32 -> fp16 operand packs)",
        "swap": "laswp_k (row interchanges outside the panel)",
        "refine": "gemv_slices_k + gemv_reduce_k (FP64 residual), trsv_ticket_k (fp32 factors), "
                  "basis kernels (GMRES)"}
    step_ms = mixed_s * 1e3
    phases = []
    for key in sorted(ms, key=lambda q: -ms[q]):
        ach = by[key] / (ms[key] / 1e3) / 1e9 if ms[key] > 0 else None
        phases.append({"phase": key, "kernels": kernels[key], "ms_per_step": ms[key],
                       "share_of_step": ms[key] / step_ms if step_ms else None,
                       "algorithmic_bytes_per_step": by[key], "achieved_gbs": ach,
                       "frac": (ach / peak) if ach else None})
    top = phases[0]
    upd_launches = max(1, ph.update_launches // max(1, args.steps))
    update_launch_bytes = by["update"] / upd_launches
    roofline = {"bound": "hbm", "kernel": top["kernels"], "phase": top["phase"],
                "achieved": top["achieved_gbs"], "peak": peak, "peak_source": peak_src,
                "unit": "GB/s", "frac": top["frac"],
                "traffic": (PANEL_TRAFFIC_PER_STEP if top["phase"] == "panel" else
                            update_launch_bytes * TC_UPDATE_TRAFFIC_RATIO
                            if top["phase"] == "update" else None),
                "traffic_note": ("DRAM bytes per step of the panel phase, scaled from one ncu "
                                 "capture of tslu_select_k + tslu_apply_k" if
                                 top["phase"] == "panel" else
                                 "DRAM bytes of one tc_update_k launch (ncu)"),
                "phases": phases,
                "update_launches_per_step": ph.update_launches / args.steps,
                "interchanges_per_step": ph.interchanges / args.steps,
                "update_algorithmic_bytes_per_launch": update_launch_bytes,
                "update_traffic_per_launch": update_launch_bytes * TC_UPDATE_TRAFFIC_RATIO}

    # ---- FP64 LU arm (PLA_General_solve), restoring A every step ----
    fp64_s = None
    fp64_eta = None
    fp64_detail = None
    fp64_peak = fp64_gemm_peak(torch, device) if not (args.skip_fp64 and args.skip_chol) else None
    if not args.skip_fp64:
        s.set_nb_alg(args.nb_fp64)
        piv = s.mvector(n, 1, np.int32)

        def fp64_step():
            check(lib.PLA_Obj_set_local_contents_device(ctypes.c_void_p(T.data_ptr()), n, a), "A")
            check(lib.PLA_Obj_set_local_contents_device(ctypes.c_void_p(b.data_ptr()), n, bo), "b")
            check(lib.PLA_General_solve(a, piv, bo), "PLA_General_solve")

        for _ in range(args.warmup):
            fp64_step()
        lib.PLA_B200_set_phase_timing(1)
        lib.PLA_B200_reset_phase_times()
        barrier()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(args.steps):
            fp64_step()
        f1.record(stream)
        barrier()
        fp64_s = max_over_ranks(f0.elapsed_time(f1) / 1e3 / args.steps)
        ph64 = pla.PhaseTimes()
        lib.PLA_B200_phase_times(ctypes.byref(ph64))
        lib.PLA_B200_set_phase_timing(0)
        nbf = args.nb_fp64
        gemm_flops = sum(2.0 * (n - k - nbf) ** 2 * nbf for k in range(0, n, nbf) if n - k - nbf > 0)
        fp64_detail = {k: getattr(ph64, k) / args.steps for k in
                       ("panel_ms", "swap_ms", "trsm_ms", "update_ms", "solve_ms")}
        fp64_detail["dgemm_tflops"] = (gemm_flops * args.steps / (ph64.update_ms / 1e3) / 1e12
                                       if ph64.update_ms > 0 else None)
        fp64_detail["lu_tflops_effective"] = (2.0 / 3.0 * n ** 3) / fp64_s / 1e12
        # the factorization alone: the solve phase (timed on the same stream,
        # never overlapped) taken out of the step
        lu_factor_s = fp64_s - ph64.solve_ms / args.steps / 1e3
        fp64_detail["lu_factor_s"] = lu_factor_s
        fp64_detail["lu_factor_tflops"] = (2.0 / 3.0 * n ** 3) / lu_factor_s / 1e12
        fp64_detail["fp64_peak_tflops"] = fp64_peak
        fp64_detail["fp64_peak_source"] = "cuBLAS DGEMM 8192^3 measured in this run"
        fp64_detail["lu_frac_of_peak"] = fp64_detail["lu_tflops_effective"] / fp64_peak
        fp64_detail["lu_factor_frac_of_peak"] = fp64_detail["lu_factor_tflops"] / fp64_peak
        if fp64_detail["dgemm_tflops"]:
            fp64_detail["dgemm_frac_of_peak"] = fp64_detail["dgemm_tflops"] / fp64_peak
        check(lib.PLA_Obj_get_local_contents_device(bo, ctypes.c_void_p(x.data_ptr()), n), "x")
        r = b - T.t() @ x
        fp64_eta = (r.abs().max() / (a_inf * x.abs().max() + b.abs().max())).item()
        s.free(piv)
        # leave A as it was for the end-to-end arm
        check(lib.PLA_Obj_set_local_contents_device(ctypes.c_void_p(T.data_ptr()), n, a), "A")

    # ---- FP64 Cholesky arm (PLA_Pos_def_solve) on A = G G'/n + I ----
    chol = None
    ooc = None
    if not args.skip_chol:
        g = torch.Generator(device=device).manual_seed(2 + 1000 * rank)
        G = torch.randn((n, n), dtype=torch.float64, device=device, generator=g)
        S = G @ G.t()
        del G
        S.div_(n)
        S.diagonal().add_(1.0)
        xs = torch.randn(n, 1, dtype=torch.float64, device=device, generator=g)
        bs = S @ xs                               # S is symmetric: row- and column-major agree
        s.set_nb_alg(args.nb_fp64)

        def chol_step():
            check(lib.PLA_Obj_set_local_contents_device(ctypes.c_void_p(S.data_ptr()), n, a), "A")
            check(lib.PLA_Obj_set_local_contents_device(ctypes.c_void_p(bs.data_ptr()), n, bo), "b")
            check(lib.PLA_Pos_def_solve(a, bo), "PLA_Pos_def_solve")

        for _ in range(args.warmup):
            chol_step()
        lib.PLA_B200_set_phase_timing(1)
        lib.PLA_B200_reset_phase_times()
        barrier()
        c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c0.record(stream)
        for _ in range(args.steps):
            chol_step()
        c1.record(stream)
        barrier()
        chol_s = max_over_ranks(c0.elapsed_time(c1) / 1e3 / args.steps)
        phc = pla.PhaseTimes()
        lib.PLA_B200_phase_times(ctypes.byref(phc))
        lib.PLA_B200_set_phase_timing(0)
        nbf = args.nb_fp64
        syrk_flops = sum(float(n - k - nbf) * (n - k - nbf + 1) * nbf
                         for k in range(0, n, nbf) if n - k - nbf > 0)
        check(lib.PLA_Obj_get_local_contents_device(bo, ctypes.c_void_p(x.data_ptr()), n), "x")
        rc = bs - S @ x
        s_inf = S.abs().sum(dim=0).max().item()
        chol = {"workload": f"PLA_Pos_def_solve n={n}, A = G G'/n + I, 1 rhs, nb={nbf}",
                "solve_s": chol_s,
                "chol_tflops_effective": (n ** 3 / 3.0) / chol_s / 1e12,
                "chol_frac_of_peak": (n ** 3 / 3.0) / chol_s / 1e12 / fp64_peak,
                "chol_factor_s": chol_s - phc.solve_ms / args.steps / 1e3,
                "chol_factor_frac_of_peak": (n ** 3 / 3.0)
                / (chol_s - phc.solve_ms / args.steps / 1e3) / 1e12 / fp64_peak,
                "update_tflops": (syrk_flops * args.steps / (phc.update_ms / 1e3) / 1e12
                                  if phc.update_ms > 0 else None),
                "phase_ms_per_step": {k: getattr(phc, k) / args.steps for k in
                                      ("panel_ms", "trsm_ms", "update_ms", "solve_ms")},
                "backward_error": (rc.abs().max() / (s_inf * x.abs().max() + bs.abs().max())).item()}
        # ---- out-of-core Cholesky (PLA_OOC_Chol) of the same S from a file in host memory ----
        # one GPU only: N replicas would each keep an 8.6 GB file in the host's memory
        if not args.skip_ooc and world == 1:
            ooc = run_ooc_chol(torch, pla, lib, s, device, S, a, n, args, chol["chol_factor_s"])
        del S, bs, xs, rc
        torch.cuda.empty_cache()
        check(lib.PLA_Obj_set_local_contents_device(ctypes.c_void_p(T.data_ptr()), n, a), "A")

    # ---- batched factor-and-solve: one persistent graph launch vs a launch loop ----
    batched = None
    if not args.skip_batched:
        batched = [run_batched(torch, pla, lib, device, stream, dt, args.steps, args.warmup, dist,
                               count=args.batch_count, seed=3)
                   for dt in (torch.float64, torch.float32)]

    # ---- mixed-precision Cholesky-IR: fp8 E4M3 vs bf16 trailing updates ----
    chol_mixed = None
    if not args.skip_chol_mixed:
        chol_mixed = run_chol_mixed(torch, pla, lib, s, device, stream, args.chol_n, (1e3, 1e7),
                                    (("fp8", pla.PLA_B200_PREC_FP8),
                                     ("bf16", pla.PLA_B200_PREC_BF16),
                                     ("bf16x6", pla.PLA_B200_PREC_BF16X6)), 8, 1, 1)

    # ---- end to end: host buffers in, host solution out ----
    e2e = None
    if not args.skip_e2e:
        # page-locked host buffers (8.6 GB per rank); should the host refuse to
        # lock that much (N replicas on one node), pageable memory still works:
        # the copy of A then completes before the factorization starts
        try:
            Th = torch.empty((n, n), dtype=torch.float64, pin_memory=True)
            pinned = True
        except RuntimeError:
            Th = torch.empty((n, n), dtype=torch.float64)
            pinned = False
        Th.copy_(T)
        bh = torch.empty((n, 1), dtype=torch.float64, pin_memory=pinned)
        bh.copy_(b)
        xh = torch.empty((n, 1), dtype=torch.float64, pin_memory=pinned)
        NT = pla.PLA_NO_TRANSPOSE

        def e2e_step():
            check(lib.PLA_Obj_set_local_contents(NT, n, 1, ctypes.c_void_p(bh.data_ptr()), n, 1, bo),
                  "set b")
            # A travels from pinned host memory during the factorization
            check(lib.PLA_General_solve_mixed_host(a, ctypes.c_void_p(Th.data_ptr()), n, bo,
                                                   ctypes.byref(params), ctypes.byref(report)),
                  "solve")
            check(lib.PLA_Obj_get_local_contents(bo, NT, None, None, ctypes.c_void_p(xh.data_ptr()),
                                                 n, 1), "get x")

        e2e_step()
        barrier()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        for _ in range(args.steps):
            e2e_step()
        g1.record(stream)
        barrier()
        e2e = {"value": max_over_ranks(g0.elapsed_time(g1) / 1e3 / args.steps), "unit": "s",
               "h2d_bytes_per_step": n * n * 8 + n * 8, "d2h_bytes_per_step": n * 8,
               "path": "PLA_Obj_set_local_contents (b, pinned host) -> "
                       "PLA_General_solve_mixed_host (A from pinned host, copied during the "
                       "factorization) -> PLA_Obj_get_local_contents",
               "pinned": max_over_ranks(0.0 if pinned else 1.0) == 0.0,
               "factor_ms": report.factor_ms, "refine_ms": report.refine_ms}
        del Th

    # ---- the other C3 configurations at full size: kappa 1e2 and 1e10, and 16 rhs ----
    sweep = None
    if not args.skip_sweep:
        del T
        torch.cuda.empty_cache()
        sweep = run_mixed_sweep(torch, pla, lib, s, device, stream, a, n, args, params)

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        try:
            cpu = reference_solve(n, args.kappa, steps=args.ref_steps)
        except Exception as exc:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "s", "cores": cpu_cores(), "kind": "reference",
                   "sample": f"unavailable: {exc}"}

    if rank == 0:
        out = {"metric": METRIC, "value": mixed_s, "unit": "s", "n_gpus": world,
               "steps": args.steps, "warmup": args.warmup, "ms_per_step": mixed_s * 1e3,
               "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
               "dtype": "f16 tensor-core factors, f32 panels, f64 refinement",
               "data": "synthetic: seeded A = U diag(sigma) V', U,V = 8 Householder reflectors each",
               "config": {"workload": f"general solve n={n}, kappa={args.kappa:g}, 1 rhs, "
                                      f"{args.precision} factors + {args.refinement.upper()}-IR",
                          "n": n, "nrhs": 1, "kappa": args.kappa, "precision": args.precision,
                          "refinement": args.refinement, "nb": args.nb, "nb_fp64": args.nb_fp64,
                          "panel_pivoting": args.panel_pivoting,
                          "l2": "inputs larger than L2 (8.6 GB FP64 matrix)",
                          "parallelism": f"replicas x{world}"},
               "fp64_lu_solve_s": fp64_s, "fp64_phase_ms_per_step": fp64_detail,
               "speedup_vs_fp64": (fp64_s / mixed_s) if fp64_s else None,
               "backward_error": eta, "backward_error_fp64": fp64_eta,
               "backward_error_target": n * 2.0 ** -53, "forward_error": fwd,
               **head_report,
               "mixed_sweep": sweep,
               "fp64_cholesky": chol, "ooc_cholesky": ooc, "batched": batched,
               "cholesky_mixed": chol_mixed,
               "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
               "clocks": clock_summary, "gpu_launches": launches}
        print(json.dumps(out))
    s.free(a, bo)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
