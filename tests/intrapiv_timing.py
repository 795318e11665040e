"""Factor and solve timings of the LDL_2D and LDL_INTRAPIV_2D front types on
one workload.

Factors the complex Helmholtz operator (the benchmark's n^3 workload,
natural nested dissection with the given cutoff) with and without
intra-front pivoting, and times each factorization, one solve over nrhs
columns, and the refined solve to 1e-10.  Run on one GPU:

    python tests/intrapiv_timing.py --n 100 --precision single --nrhs 4
"""
import argparse
import json
import os
import sys
import time

import numpy as np
import torch

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import clique_b200 as cliq  # noqa: E402
from clique_b200 import operators as ops  # noqa: E402


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--n", type=int, default=100)
    p.add_argument("--cutoff", type=int, default=128)
    p.add_argument("--precision", default="single")
    p.add_argument("--nrhs", type=int, default=4)
    p.add_argument("--types", default="LDL_2D,LDL_INTRAPIV_2D", help="front types to time, comma-separated")
    p.add_argument("--reps", type=int, default=2, help="factorizations per type (the last one is reported)")
    a = p.parse_args()
    n = a.n
    A, _, _ = ops.helmholtz_workload_3d(n, seed=0)
    map_, sep, info = cliq.NaturalNestedDissection(n, n, n, A, a.cutoff)
    B = ops.random_rhs(A.n, a.nrhs, seed=1, complex_=True)
    out = {"n": n, "precision": a.precision, "nrhs": a.nrhs}
    for name in a.types.split(","):
        ft = getattr(cliq.SymmFrontType, name)
        L = cliq.DistSymmFrontTree(A, map_, sep, info, precision=a.precision, keep_matrix=True)
        r = {}
        for rep in range(a.reps):   # later runs reuse the plan (new values, same pattern)
            if rep:
                L.Initialize(A.values)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            cliq.LDL(info, L, ft)
            torch.cuda.synchronize()
            r["factor_s"] = round(time.perf_counter() - t0, 4)
        t0 = time.perf_counter()
        cliq.Solve(info, L, B.copy(order="F"))
        torch.cuda.synchronize()
        r["solve_s"] = round(time.perf_counter() - t0, 4)
        t0 = time.perf_counter()
        X, it, rr = cliq.RefinedSolve(L, B, 1e-10, 40)
        r["refined"] = {"s": round(time.perf_counter() - t0, 4), "iterations": it, "relres": rr}
        r["residual"] = float(np.linalg.norm(A.to_scipy() @ X - B) / np.linalg.norm(B))
        if ft in cliq.SymmFrontType.PIVOTED:
            swaps = blocks = 0
            for s in range(info.num_nodes):
                sub, piv = L.front_pivots(s)
                swaps += int((piv != np.arange(len(piv))).sum())
                blocks += int((sub != 0).sum())
            r["interchanged_rows"], r["pivot_blocks_2x2"] = swaps, blocks
        out[name] = r
        del L
    print(json.dumps(out))


if __name__ == "__main__":
    main()
