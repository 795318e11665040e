"""Solve timings of the LDL_2D and BLOCK_LDL_2D front types on one workload.

Factors the complex Helmholtz operator (the benchmark's n^3 workload,
natural nested dissection with the given cutoff) once, times the
triangular sweeps (forward, diagonal, backward) over nrhs device columns,
converts the fronts to the block form (inv(A11) over A21), times the
product-only block sweeps on the same columns, and the refined solve to
1e-10 in both forms.  Run on one GPU:

    python tests/block_solve_timing.py --n 100 --precision single --nrhs 4
"""
import argparse
import ctypes as C
import json
import os
import sys
import time

import numpy as np
import torch

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import clique_b200 as cliq  # noqa: E402
from clique_b200 import _capi  # noqa: E402
from clique_b200 import operators as ops  # noqa: E402


def timed(fn, reps):
    fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--n", type=int, default=100)
    p.add_argument("--cutoff", type=int, default=128)
    p.add_argument("--precision", default="single")
    p.add_argument("--nrhs", type=int, default=4)
    p.add_argument("--reps", type=int, default=5)
    a = p.parse_args()
    lib = _capi.load()
    n = a.n
    A, _, _ = ops.helmholtz_workload_3d(n, seed=0)
    map_, sep, info = cliq.NaturalNestedDissection(n, n, n, A, a.cutoff)
    L = cliq.DistSymmFrontTree(A, map_, sep, info, precision=a.precision)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    cliq.LDL(info, L)
    torch.cuda.synchronize()
    t_factor = time.perf_counter() - t0
    B = ops.random_rhs(A.n, a.nrhs, seed=1, complex_=True)
    Xd = torch.zeros((a.nrhs, A.n), dtype=torch.complex128, device="cuda")
    Bd = torch.from_numpy(np.ascontiguousarray(B.T)).cuda()

    def solve():
        Xd.copy_(Bd)
        st = lib.cliqgpu_solve(L._h, C.c_void_p(Xd.data_ptr()), A.n, a.nrhs, 1, 1)
        assert st == 0, st

    out = {"n": n, "precision": a.precision, "nrhs": a.nrhs, "factor_s": round(t_factor, 4)}
    out["ldl_solve_ms"] = round(timed(solve, a.reps), 3)
    _, it, rr = cliq.RefinedSolve(L, B, 1e-10, 40)
    out["ldl_refined"] = {"iterations": it, "relres": rr}
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    assert lib.cliqgpu_block_ldl(L._h) == 0
    out["convert_s"] = round(time.perf_counter() - t0, 4)
    out["block_solve_ms"] = round(timed(solve, a.reps), 3)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    X, it, rr = cliq.RefinedSolve(L, B, 1e-10, 40)
    out["block_refined"] = {"iterations": it, "relres": rr, "s": round(time.perf_counter() - t0, 4)}
    out["block_residual"] = float(np.linalg.norm(A.to_scipy() @ X - B) / np.linalg.norm(B))
    print(json.dumps(out))


if __name__ == "__main__":
    main()
