"""Benchmark: LDL^T factor + solve of the 100^3 complex-symmetric Helmholtz
operator (PML, 10 points per wavelength, smoothed random velocity, 4 complex
N(0,1) right-hand sides), FP32 fronts + FP64 iterative refinement to relative
residual <= 1e-10, against the plain FP64 factor + solve on the same GPU.

One step = assemble the fronts from A's values, multifrontal LDL^T, and the
refined solve, all on the device through the C ABI (libcliqgpu.so).  The
factor arena (10 GB for CFP32, 20 GB for CFP64) is far larger than the 126 MB
L2, so consecutive steps cannot hit in L2 without a flush.

Usage: python bench.py [--gpus N --steps K --warmup W --impl ours|reference]
Multi-GPU (torchrun): every rank solves its own independent copy (replicas;
the single-GPU path has no exchange step), timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "LDL^T factor+solve s, FP32+IR vs FP64 on 1 B200, 100^3 Helmholtz, resid<=1e-10"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference", "cpu-sample"])
    p.add_argument("--grid", dest="n", type=int, default=100, help="grid points per axis")
    p.add_argument("--nrhs", type=int, default=4)
    p.add_argument("--cutoff", type=int, default=128)
    p.add_argument("--tol", type=float, default=1e-10)
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--no-fp64", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end pass (a second FP32 plan)")
    p.add_argument("--operator", default="helmholtz", choices=["helmholtz", "laplacian"])
    p.add_argument("--ordering", default="natural", choices=["natural", "graph"],
                   help="natural nested dissection (the reference's default) or the general-graph one")
    p.add_argument("--cpu-budget", type=float, default=20.0, help="seconds of CPU work for the baseline sample")
    p.add_argument("--ref-steps", type=int, default=1, help="full-size steps of the reference arm")
    p.add_argument("--autotune", type=int, default=0,
                   help="reps of the per-launch kernel-choice autotuner run on the FP32 plan before the warm-up (0: off)")
    return p.parse_args()


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""
    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def rank_env():
    """(rank, world, local_rank) from the torchrun environment (1 process when absent)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def dist_init(backend):
    """Process group for a multi-rank launch (None for one process).  Every rank
    solves its own replica; the group carries only barriers and the timing max."""
    _, world, _ = rank_env()
    if world == 1:
        return None
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group(backend, timeout=timedelta(seconds=600))
    return dist


def barrier(dist):
    if dist is not None:
        dist.barrier()


def max_over_ranks(value, dist, device="cpu"):
    """Slowest rank's value: the job's time is set by its last replica."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return json.load(f)
    except Exception:
        return None


def workload(n, nrhs, seed, operator="helmholtz"):
    """(A, B, description): the seeded synthetic operator and right-hand sides."""
    from clique_b200 import operators as ops
    if operator == "laplacian":
        A = ops.laplacian_3d(n, n, n, 6.1)
        B = ops.random_rhs(A.n, nrhs, seed=seed + 1, complex_=False)
        return A, B, f"{n}^3 real 7-point Laplacian + shift (diagonal 6.1)"
    A, omega, c = ops.helmholtz_workload_3d(n, seed=seed)
    B = ops.random_rhs(A.n, nrhs, seed=seed + 1, complex_=True)
    return A, B, f"{n}^3 complex-symmetric Helmholtz PML (omega={omega:.2f}, 10 ppw)"


# ---------------------------------------------------------------------------
# reference arm / CPU baseline: the oracle (C restatement of Clique's path,
# OpenBLAS-backed dense kernels, all host cores).  These run in processes
# that load only the oracle library and OpenBLAS, never libcliqgpu.so: the
# workload generator is plain numpy and the flop model is evaluated on the
# oracle's own symbolic analysis.
# ---------------------------------------------------------------------------
def host_cpu():
    """(logical cores usable by this process, CPU model name)."""
    try:
        cores = len(os.sched_getaffinity(0))
    except Exception:
        cores = os.cpu_count() or 1
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    model = ln.split(":", 1)[1].strip()
                    break
    except Exception:
        pass
    return cores, model


def native_libs():
    """Shared objects of this repository mapped into the current process."""
    libs = set()
    try:
        with open("/proc/self/maps") as f:
            for ln in f:
                parts = ln.split()
                if len(parts) >= 6 and parts[-1].endswith(".so") and parts[-1].startswith(ROOT):
                    libs.add(os.path.relpath(parts[-1], ROOT))
    except Exception:
        pass
    return sorted(libs)


def oracle_flops(S):
    """Clique's FactorizationWork model (dist_symm_front_tree/impl.hpp:560-585,
    x4 complex) on the oracle's symbolic analysis."""
    k = S.size.astype(np.float64)
    m = k + S.n_lower.astype(np.float64)
    return 4.0 * float(np.sum(k ** 3 / 3 + (m - k) * k * k + (m - k) ** 2 * k))


def cpu_run(n, nrhs, cutoff, seed, threads):
    """One oracle factor + solve of the n^3 Helmholtz workload: returns a dict
    with assembly, factor and solve seconds, residuals and the flop count."""
    from clique_b200 import operators as ops
    from oracle import oracle as O
    O.enable_blas(threads)
    A, omega, _ = ops.helmholtz_workload_3d(n, seed=seed)
    B = ops.random_rhs(A.n, nrhs, seed=seed + 1, complex_=True)
    S = O.Symbolic(n, n, n, A.rowptr, A.colind, cutoff=cutoff)
    t0 = time.perf_counter()
    F = O.Fronts(S, A.values, is_complex=True)
    t1 = time.perf_counter()
    bad = F.ldl(96)
    t2 = time.perf_counter()
    X = F.solve(B.copy(order="F"))
    t3 = time.perf_counter()
    del F
    As = A.to_scipy()
    R = As @ X - B
    relres = float(np.max(np.linalg.norm(R, axis=0) / np.linalg.norm(B, axis=0)))
    anorm = float(np.abs(As).sum(axis=1).max())
    berr = float(np.max(np.abs(R).max(axis=0) / (anorm * np.abs(X).max(axis=0) + np.abs(B).max(axis=0))))
    return {"n": n, "assemble_s": t1 - t0, "factor_s": t2 - t1, "solve_s": t3 - t2, "total_s": t3 - t0,
            "relres": relres, "backward_error": berr, "zero_pivot": int(bad), "flops": oracle_flops(S)}


def cpu_sample_estimate(args, target_n, threads):
    """Bounded sample: the largest grid whose oracle run fits about
    args.cpu_budget seconds, scaled to target_n^3 by the oracle's flop model.
    An estimate (BLAS efficiency grows with front size, so the scaling tends
    to overstate the full-size time); the measured full-size figure is the
    reference arm's."""
    from clique_b200 import operators as ops
    from oracle import oracle as O
    n0 = min(30, target_n)
    r0 = cpu_run(n0, args.nrhs, args.cutoff, args.seed, threads)
    rate = r0["flops"] / r0["total_s"]

    def flops_of(n):
        A = ops.laplacian_3d(n, n, n)
        return oracle_flops(O.Symbolic(n, n, n, A.rowptr, A.colind, cutoff=args.cutoff))
    f_target = flops_of(target_n)
    n = int(target_n * min(1.0, (args.cpu_budget * rate / f_target)) ** (1.0 / 6.0))
    n = max(n0, min(target_n, n))
    r = cpu_run(n, args.nrhs, args.cutoff, args.seed, threads)
    scale = f_target / r["flops"]
    return r, scale


def cpu_baseline_child(args):
    """Entry of the child process that times the CPU baseline sample (prints one JSON line)."""
    threads, model = host_cpu()
    r, scale = cpu_sample_estimate(args, args.n, threads)
    out = {"value": r["total_s"] * scale, "unit": "s", "cores": threads, "kind": "port", "estimate": True,
           "cpu_model": model,
           "sample": f"oracle (C restatement, OpenBLAS {threads} threads, nb=96) complex FP64 assemble+factor+solve of "
                     f"the {r['n']}^3 Helmholtz workload ({args.nrhs} RHS) in {r['total_s']:.2f} s (factor "
                     f"{r['factor_s']:.2f} s, solve {r['solve_s']:.2f} s, residual {r['relres']:.1e}), scaled to "
                     f"{args.n}^3 by Clique's FactorizationWork flop model on the oracle's own analysis (x{scale:.1f}); "
                     f"the reference arm measures {args.n}^3 itself",
           "sample_n": r["n"], "sample_s": r["total_s"], "native_so_loaded": native_libs()}
    print(json.dumps(out), flush=True)


def cpu_baseline(args):
    """Runs the bounded CPU sample in a child process (oracle + OpenBLAS only)."""
    cmd = [sys.executable, os.path.abspath(__file__), "--impl", "cpu-sample", "--grid", str(args.n), "--nrhs",
           str(args.nrhs), "--cutoff", str(args.cutoff), "--seed", str(args.seed), "--cpu-budget", str(args.cpu_budget)]
    env = dict(os.environ)
    env.pop("RANK", None)
    env.pop("WORLD_SIZE", None)
    r = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=1800)
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    if r.returncode != 0 or not lines:
        raise RuntimeError(f"cpu baseline child failed: {r.stderr[-400:]}")
    return json.loads(lines[-1])


def run_reference(args):
    """The reference's CPU path (the oracle restatement; Clique itself cannot be
    built here) on the full workload.  Each step is one whole assemble +
    factor + solve; the run does args.ref_steps steps (default 1: one step
    takes minutes) and no warm-up, and says so in steps / warmup.  Rank 0 alone
    runs; other ranks of a torchrun launch exit 0 without work."""
    if rank_env()[0] != 0:
        return
    threads, model = host_cpu()
    runs = [cpu_run(args.n, args.nrhs, args.cutoff, args.seed, threads) for _ in range(max(1, args.ref_steps))]
    v = statistics.median(r["total_s"] for r in runs)
    last = runs[-1]
    cb = {"value": v, "unit": "s", "cores": threads, "kind": "port", "cpu_model": model,
          "sample": f"full {args.n}^3 workload, {len(runs)} step(s): oracle (C restatement of Clique's LocalLDL / "
                    f"FrontLDL / Solve, OpenBLAS {threads} threads, nb=96), complex FP64 assemble+factor+solve"}
    line = {"metric": METRIC, "value": v, "unit": "s", "n_gpus": args.gpus, "steps": len(runs), "warmup": 0,
            "steps_requested": args.steps, "warmup_requested": args.warmup,
            "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "c128", "data": "synthetic", "impl": "reference",
            "config": {"workload": f"{args.n}^3 complex-symmetric Helmholtz PML (10 ppw), {args.nrhs} RHS, "
                                   f"natural ND cutoff {args.cutoff}",
                       "parallelism": f"cpu{threads}", "cpu_model": model},
            "phases_s": {"assemble": last["assemble_s"], "factor": last["factor_s"], "solve": last["solve_s"]},
            "factor_gflop": last["flops"] / 1e9, "factor_gflops_rate": last["flops"] / last["factor_s"] / 1e9,
            "relres": last["relres"], "backward_error": last["backward_error"],
            "native_so_loaded": native_libs(),
            "cpu_baseline": cb, "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def host_residuals(As, X, B):
    """Max over columns of ||b - A x||_2 / ||b||_2 and of the normwise backward
    error ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf), in FP64 on the host."""
    X = X.reshape(B.shape)
    R = As @ X - B
    anorm = float(np.abs(As).sum(axis=1).max())
    rr = np.linalg.norm(R, axis=0) / np.linalg.norm(B, axis=0)
    be = np.abs(R).max(axis=0) / (anorm * np.abs(X).max(axis=0) + np.abs(B).max(axis=0))
    return {"relres": float(rr.max()), "backward_error": float(be.max())}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(args):
    import torch
    import clique_b200 as cliq

    rank, world, local = rank_env()
    torch.cuda.set_device(local)
    dist = dist_init("nccl")

    A, B, wdesc = workload(args.n, args.nrhs, args.seed, args.operator)
    cplx = np.iscomplexobj(A.values)
    n = args.n
    stream = torch.cuda.current_stream()
    if args.ordering == "graph":
        map_, sep, info = cliq.NestedDissection(A, args.cutoff)
    else:
        map_, sep, info = cliq.NaturalNestedDissection(n, n, n, A, args.cutoff)
    vals_d = torch.from_numpy(A.values).cuda()
    B_d = torch.from_numpy(B).cuda().t().contiguous().t()

    L32 = cliq.DistSymmFrontTree(A, map_, sep, info, precision="single", stream=stream.cuda_stream)
    free0, total_hbm = torch.cuda.mem_get_info()
    memory = {"fp32_plan_bytes": L32.query(3), "hbm_total_bytes": total_hbm, "hbm_used_max_bytes": total_hbm - free0}
    phase_ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    tuned = None
    if args.autotune > 0:   # one-time set-up, outside the timed region
        L32.Initialize(vals_d)
        rep = np.zeros(5)
        cliq._capi.check(cliq._capi.load().cliqgpu_autotune(L32._h, args.autotune, rep.ctypes.data_as(C.c_void_p)), "autotune")
        tuned = {"tensor_ms": rep[0], "cuda_core_ms": rep[1], "chosen_ms": rep[2], "moved_to_cuda_cores": int(rep[3]),
                 "switchable": int(rep[4])}

    def step32():
        phase_ev[0].record()
        L32.Initialize(vals_d)
        cliq.LDL(info, L32)
        phase_ev[1].record()
        X, it, rr = cliq.RefinedSolve(L32, B_d, args.tol, 30)
        phase_ev[2].record()
        return it, rr

    for _ in range(args.warmup):
        it, rr = step32()
    torch.cuda.synchronize()
    barrier(dist)
    launches0 = L32.total_launches()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        barrier(dist)
        ev0.record()
        its, rrs = [], []
        for _ in range(args.steps):
            it, rr = step32()
            its.append(it); rrs.append(rr)
        ev1.record()
        torch.cuda.synchronize()
    barrier(dist)
    ms = ev0.elapsed_time(ev1) / args.steps
    ms = max_over_ranks(ms, dist, "cuda")
    factor_flops = L32.FactorizationWork()
    launches = (L32.total_launches() - launches0) // args.steps
    factor_phase_ms = phase_ev[0].elapsed_time(phase_ev[1])   # last timed step
    solve_phase_ms = phase_ev[1].elapsed_time(phase_ev[2])
    # per-kernel breakdown from one more step with CUDA events around every
    # factorization launch (outside the timed region)
    L32.set_profiling(True)
    step32()
    torch.cuda.synchronize()
    prof = L32.profile()
    L32.set_profiling(False)
    peaks = measured_peaks()
    upd_ms = prof["trail_ms"] + prof["schur_ms"]
    upd_flops = prof["trail_flops"] + prof["schur_flops"]
    achieved = upd_flops / (upd_ms * 1e-3) / 1e12 if upd_ms > 0 else 0.0
    f16 = os.environ.get("CLIQGPU_SPLIT", "f16") != "tf32"
    bf16 = peaks["bf16_tflops"] if peaks else 1590.0
    # dense FP16 runs at the BF16 rate, dense TF32 at half of it
    peak = bf16 if f16 else bf16 / 2.0
    roofline = {"kernel": "tc_gemm_kernel (tcgen05 kind::f16, 2xFP16 split; Schur, outer and in-panel updates)"
                          if f16 else "tc_gemm_kernel (tcgen05 kind::tf32, 3xTF32 split)",
                "bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "peak_source": ("measured bf16 burst" + ("" if f16 else " / 2") + ", MEASURED_PEAKS.json (of measured)")
                if peaks else "fallback 1.59 PFLOP/s bf16" + ("" if f16 else " / 2") + " (of fallback)",
                "numerator": "Clique FactorizationWork counting (complex x4) of the update GEMMs over their CUDA-event "
                             "time (GEMM kernel only; operand packing is pack_ms); the three split products per real "
                             "product count against the fraction, not in the numerator (frac <= 1/3)",
                "traffic": 580e6,
                "traffic_note": "DRAM read+write bytes of one Schur-update launch (60^3, tree level 2, 1653 CTAs of "
                                "128x128; ncu --set full); its algorithmic bytes (packed operands read once, update "
                                "read and written once) are 582 MB"}

    # end-to-end through the C ABI with host buffers (pinned): matrix values
    # and right-hand sides copied in, the solution copied out, every step
    As = A.to_scipy()
    e2e = None
    if args.no_e2e:
        # the solution of the last device step, checked on the host
        Xd, _, _ = cliq.RefinedSolve(L32, B_d, args.tol, 30)
        host_check = {"fp32ir": host_residuals(As, Xd.cpu().numpy(), B)}
    else:
        L32h = cliq.DistSymmFrontTree(A, map_, sep, info, precision="single")
        vals_h = torch.from_numpy(A.values).pin_memory().numpy()
        nrhs_h = B.shape[1]
        hdt = torch.complex128 if cplx else torch.float64
        B_h = torch.empty((nrhs_h, B.shape[0]), dtype=hdt, pin_memory=True).numpy().T
        B_h[...] = B
        X_h = torch.empty((nrhs_h, B.shape[0]), dtype=hdt, pin_memory=True).numpy().T

        def step_host():
            L32h.Initialize(vals_h)
            cliq.LDL(info, L32h)
            return cliq.RefinedSolve(L32h, B_h, args.tol, 30, X=X_h)
        step_host()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            Xh, ith, rrh = step_host()
        e2e_s = (time.perf_counter() - t0) / args.steps
        e2e_s = max_over_ranks(e2e_s, dist, "cuda")
        memory["hbm_used_max_bytes"] = max(memory["hbm_used_max_bytes"], total_hbm - torch.cuda.mem_get_info()[0])
        del L32h
        e2e = {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": int(A.values.nbytes + B.nbytes),
               "d2h_bytes_per_step": int(B.nbytes)}
        # the returned solution checked on the host (scipy FP64 product)
        host_check = {"fp32ir": host_residuals(As, np.asarray(Xh), B)}

    fp64 = None
    if not args.no_fp64:
        # the FP32 plan's numbers are taken: free it before the FP64 plan (at
        # 160^3 the two do not fit in HBM together)
        del L32
        torch.cuda.synchronize()
        L64 = cliq.DistSymmFrontTree(A, map_, sep, info, precision="double", stream=stream.cuda_stream)
        X64 = torch.zeros_like(B_d)
        memory["fp64_plan_bytes"] = L64.query(3)

        def step64():
            L64.Initialize(vals_d)
            cliq.LDL(info, L64)
            X64.copy_(B_d)
            cliq.Solve(info, L64, X64)
        for _ in range(max(1, args.warmup)):
            step64()
        torch.cuda.synchronize()
        L64.set_profiling(True)
        ev0.record()
        for _ in range(args.steps):
            step64()
        ev1.record()
        torch.cuda.synchronize()
        memory["hbm_used_max_bytes"] = max(memory["hbm_used_max_bytes"], total_hbm - torch.cuda.mem_get_info()[0])
        fp64_ms = ev0.elapsed_time(ev1) / args.steps
        fp64_ms = max_over_ranks(fp64_ms, dist, "cuda")
        Xc = X64.cpu().numpy()
        res64 = float(np.linalg.norm(As @ Xc - B) / np.linalg.norm(B))
        host_check["fp64"] = host_residuals(As, Xc, B)
        p64 = L64.profile()
        fp64 = {"fp64_plain_s": fp64_ms / 1e3, "fp64_residual": res64,
                "speedup_vs_fp64": fp64_ms / ms,
                "fp64_factor_profile_ms": {k: v for k, v in p64.items() if k.endswith("_ms")},
                "fp64_update_tflops": (p64["trail_flops"] + p64["schur_flops"]) /
                                      max(1e-9, (p64["trail_ms"] + p64["schur_ms"]) * 1e-3) / 1e12}
        del L64

    line = {"metric": METRIC, "value": ms / 1e3, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "c64+c128-IR" if cplx else "f32+f64-IR", "data": "synthetic",
            "config": {"workload": f"{wdesc}, {args.nrhs} RHS, {args.ordering} ND cutoff {args.cutoff}",
                       "precision": ("CFP32" if cplx else "FP32") + " fronts, FP64 pivots, FP64 refinement",
                       "tol": args.tol,
                       "parallelism": f"replicas{world}", "l2": "inputs larger than L2 (factor arena >> 126 MB)"},
            "refine_iters": its, "relres": max(rrs), "factor_gflop": factor_flops / 1e9,
            "factor_tflops_effective": factor_flops / (ms / 1e3) / 1e12,
            "gpu_launches": launches,
            "autotune": tuned,
            "phases_ms": {"assemble+factor": factor_phase_ms, "refined_solve": solve_phase_ms},
            "factor_profile_ms": {k: v for k, v in prof.items() if k.endswith("_ms")},
            "roofline": roofline,
            "e2e": e2e,
            "clocks": clk.summary()}
    line["host_check"] = host_check
    line["memory"] = memory
    line["backward_error"] = host_check["fp32ir"]["backward_error"]
    if fp64:
        line.update(fp64)
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            line["cpu_baseline"] = cpu_baseline(args)
        except Exception as e:  # the baseline must not hide the GPU number
            line["cpu_baseline"] = {"error": str(e)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.impl == "cpu-sample":
        cpu_baseline_child(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
