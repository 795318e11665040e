"""Batch workload (run by hand on a GPU box; pytest does not collect this file).

512 independent 2D Helmholtz-PML problems (examples/HelmholtzPML2D.cpp form,
omega for 10 points per wavelength at each problem's slowest speed, smoothed
random velocity), side lengths drawn uniformly from 32..256 and 1..64 complex
N(0,1) right-hand sides per problem (seeded), in one forest plan: complex
FP32 fronts + FP64 refinement to a per-problem relative residual <= 1e-10.
The right-hand-side block has as many columns as the largest count; a
problem's further columns are zero.  Steps: build + one autotuning of the
update kernels, then runs of cliqgpu_batch_run (the first direct, the second
recorded as a CUDA graph, the rest replays), each timed with CUDA events;
every problem's residual is checked again on the host.  Prints one JSON line.

Usage: python tests/cfg3_batch.py [--count 512] [--runs 5]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--count", type=int, default=512)
    ap.add_argument("--lo", type=int, default=32)
    ap.add_argument("--hi", type=int, default=256)
    ap.add_argument("--rhs-hi", type=int, default=64)
    ap.add_argument("--runs", type=int, default=5)
    ap.add_argument("--steps", type=int, default=6)
    ap.add_argument("--max-extra", type=int, default=2)
    ap.add_argument("--cutoff", type=int, default=64)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--precision", default="single", choices=["single", "double"])
    ap.add_argument("--check-worst", type=int, default=0,
                    help="re-solve this many of the worst problems alone (FP64 and FP32 plans) and report them")
    args = ap.parse_args()
    import torch
    from clique_b200 import operators as ops
    from clique_b200.batch import BatchSolver
    rng = np.random.default_rng(args.seed)
    sides = rng.integers(args.lo, args.hi + 1, args.count)
    nrhs = rng.integers(1, args.rhs_hi + 1, args.count)
    t0 = time.perf_counter()
    mats = [ops.helmholtz_workload_2d(int(s), seed=args.seed * 100003 + i)[0] for i, s in enumerate(sides)]
    dims = [(int(s), int(s), 1) for s in sides]
    bs = BatchSolver(mats, dims, cutoff=args.cutoff, precision=args.precision)
    k = int(nrhs.max())
    n = bs.n
    B = np.zeros((n, k), np.complex128, order="F")
    for p in range(args.count):
        r0, r1 = bs.seg[p], bs.seg[p + 1]
        B[r0:r1, :nrhs[p]] = ops.random_rhs(int(r1 - r0), int(nrhs[p]), seed=args.seed * 7919 + p, complex_=True)
    vals = torch.from_numpy(bs.A.values).cuda()
    Bt = torch.from_numpy(B).cuda().t().contiguous().t()
    build_s = time.perf_counter() - t0
    out = {"workload": f"{args.count} 2D Helmholtz PML problems, sides U{{{args.lo}..{args.hi}}}, "
                       f"1..{args.rhs_hi} RHS each (seeded), CFP32 fronts + FP64 refinement",
           "unknowns": int(n), "fronts": int(bs.info.num_nodes), "rhs_columns": k,
           "useful_rhs_entries": int((sides.astype(np.int64) ** 2 * nrhs).sum()),
           "factor_gflop": bs.L.FactorizationWork() / 1e9, "build_s": build_s}
    bs.run(vals, Bt, steps=args.steps, tol=1e-10)
    if not args.no_tune:
        out["autotune"] = bs.autotune(reps=2)
    X = None
    times, worst, taken = [], [], []
    for r in range(args.runs):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        X, rel, st = bs.run(vals, Bt, X=X, steps=args.steps, tol=1e-10, max_extra=args.max_extra)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
        worst.append(float(rel.max()))
        taken.append(st)
    out["fallback"] = bs.last_fallback
    out["run_ms"] = times
    out["run_kinds"] = ["direct", "recorded+replayed"] + ["replay"] * max(0, args.runs - 2)
    out["launches_per_run"] = bs.last_launches()
    out["steps_taken"] = taken
    out["worst_relres_device"] = worst
    # phases of one run, through the plan's own factor and solve entry points
    import clique_b200 as cliq
    torch.cuda.synchronize()
    with torch.cuda.stream(bs.stream):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        bs.L.set_profiling(True)
        ev[0].record()
        bs.L.Initialize(vals)
        cliq.LDL(bs.info, bs.L)
        ev[1].record()
        Xs = Bt[:, :16].t().contiguous().t()        # one 16-column sweep chunk
        cliq.Solve(bs.info, bs.L, Xs)
        ev[2].record()
        torch.cuda.synchronize()
        prof = bs.L.profile()
        bs.L.set_profiling(False)
    out["phases_ms"] = {"assemble+factor": ev[0].elapsed_time(ev[1]), "one_solve_16_columns": ev[1].elapsed_time(ev[2]),
                        "factor_breakdown": {k: v for k, v in prof.items() if k.endswith("_ms")}}
    # host check of every problem and column
    Xh = X.cpu().numpy()
    hw = 0.0
    for p in range(args.count):
        r0, r1 = bs.seg[p], bs.seg[p + 1]
        As = mats[p].to_scipy()
        R = As @ Xh[r0:r1, :nrhs[p]] - B[r0:r1, :nrhs[p]]
        hw = max(hw, float((np.linalg.norm(R, axis=0) / np.linalg.norm(B[r0:r1, :nrhs[p]], axis=0)).max()))
    out["worst_relres_host"] = hw
    prob = rel.max(axis=1)
    out["problems_above_tol"] = int((prob > 1e-10).sum())
    if args.check_worst:
        import clique_b200 as cliq
        worst_p = np.argsort(-prob)[:args.check_worst]
        rows = []
        for p in worst_p:
            A = mats[p]
            s = int(sides[p])
            r0, r1 = bs.seg[p], bs.seg[p + 1]
            Bp = B[r0:r1, :nrhs[p]].copy(order="F")
            m1, s1, i1 = cliq.NaturalNestedDissection(s, s, 1, A, args.cutoff)
            L64 = cliq.DistSymmFrontTree(A, m1, s1, i1, precision="double")
            cliq.LDL(i1, L64)
            X64 = cliq.Solve(i1, L64, Bp.copy(order="F"))
            L32 = cliq.DistSymmFrontTree(A, m1, s1, i1, precision="single")
            cliq.LDL(i1, L32)
            X32, it, rr = cliq.RefinedSolve(L32, Bp, 1e-10, 30)
            As = A.to_scipy()
            rows.append({"problem": int(p), "side": s, "nrhs": int(nrhs[p]), "batch_relres": float(prob[p]),
                         "alone_fp64_relres": float(np.linalg.norm(As @ X64 - Bp) / np.linalg.norm(Bp)),
                         "alone_fp32ir_relres": float(rr), "alone_fp32ir_solves": int(it)})
        out["worst_problems"] = rows
    out["problems_per_s"] = args.count / (min(times[1:]) / 1e3) if len(times) > 1 else None
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
