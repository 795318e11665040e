"""Parity at the full 100^3 workload (run by hand on a GPU box; pytest does not
collect this file: the oracle's FP64 factorization of the 100^3 operator takes
minutes of host CPU time).

Workload: the 100^3 complex-symmetric Helmholtz operator with a 5-cell
quadratic PML (omega for 10 points per wavelength, smoothed random velocity,
seed 0), natural nested dissection with cutoff 128, 4 complex N(0,1)
right-hand sides (seed 1) -- the configuration bench.py measures.

Reported (one JSON line):
  * the plain FP64 GPU factor + solve: per-column relative residual
    ||b - A x||_2 / ||b||_2 and normwise backward error
    ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf);
  * the oracle's FP64 factor + solve on the same ordering (OpenBLAS, all host
    cores): the same figures, its factor / solve seconds, and the GPU
    solution's normwise relative difference from it;
  * the oracle's solve run on the GPU's fronts (the GPU factorization copied
    into the oracle): separates the factorization's rounding from the solve's;
  * the FP32 + FP64-refinement GPU solution: the same figures.

Usage: python tests/headline_parity.py [--grid 100] [--no-oracle]
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


def norms(As, X, B):
    """(per-column relative residual, per-column normwise backward error)."""
    R = As @ X - B
    anorm = np.abs(As).sum(axis=1).max()
    rr = np.linalg.norm(R, axis=0) / np.linalg.norm(B, axis=0)
    be = np.abs(R).max(axis=0) / (anorm * np.abs(X).max(axis=0) + np.abs(B).max(axis=0))
    return rr.tolist(), be.tolist()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", type=int, default=100)
    ap.add_argument("--cutoff", type=int, default=128)
    ap.add_argument("--nrhs", type=int, default=4)
    ap.add_argument("--no-oracle", action="store_true")
    args = ap.parse_args()
    import torch
    import clique_b200 as cliq
    from clique_b200 import operators as ops
    n = args.grid
    A, omega, _ = ops.helmholtz_workload_3d(n, seed=0)
    B = ops.random_rhs(A.n, args.nrhs, seed=1, complex_=True)
    As = A.to_scipy()
    out = {"workload": f"{n}^3 complex Helmholtz PML (omega={omega:.2f}), {args.nrhs} RHS, cutoff {args.cutoff}"}

    map_, sep, info = cliq.NaturalNestedDissection(n, n, n, A, args.cutoff)
    L = cliq.DistSymmFrontTree(A, map_, sep, info, precision="double")
    cliq.LDL(info, L)
    X64 = cliq.Solve(info, L, B.copy(order="F"))
    out["gpu_fp64_relres"], out["gpu_fp64_backward_error"] = norms(As, X64, B)

    L32 = cliq.DistSymmFrontTree(A, map_, sep, info, precision="single")
    cliq.LDL(info, L32)
    X32, it, rr = cliq.RefinedSolve(L32, B, 1e-10, 30)
    out["gpu_fp32ir_solves"] = it
    out["gpu_fp32ir_relres"], out["gpu_fp32ir_backward_error"] = norms(As, X32, B)
    del L32
    torch.cuda.synchronize()

    if not args.no_oracle:
        from oracle import oracle as O
        O.enable_blas(os.cpu_count() or 1)
        S = O.Symbolic(n, n, n, A.rowptr, A.colind, cutoff=args.cutoff)
        # the oracle's solve with the GPU's factors
        F = O.Fronts(S, A.values, is_complex=True)
        for s in range(S.num_nodes):
            Lf, d = L.front(s)
            F.set_factored(s, Lf, d)
        Xg = F.solve(B.copy(order="F"))
        out["oracle_solve_on_gpu_factors_relres"], _ = norms(As, Xg, B)
        del F
        del L
        t0 = time.perf_counter()
        F = O.Fronts(S, A.values, is_complex=True)
        assert F.ldl(96) == 0
        t1 = time.perf_counter()
        Xo = F.solve(B.copy(order="F"))
        t2 = time.perf_counter()
        out["oracle_factor_s"], out["oracle_solve_s"], out["oracle_threads"] = t1 - t0, t2 - t1, os.cpu_count()
        out["oracle_relres"], out["oracle_backward_error"] = norms(As, Xo, B)
        out["gpu_fp64_vs_oracle"] = float(np.linalg.norm(X64 - Xo) / np.linalg.norm(Xo))
        out["gpu_fp32ir_vs_oracle"] = float(np.linalg.norm(X32 - Xo) / np.linalg.norm(Xo))
        out["gpu_factors_oracle_solve_vs_oracle"] = float(np.linalg.norm(Xg - Xo) / np.linalg.norm(Xo))
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
