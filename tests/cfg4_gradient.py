"""Gradient workload at 64^3 (run by hand on a GPU box; pytest does not
collect this file).

3D complex Helmholtz-PML operator on a 64^3 grid (omega for 10 points per
wavelength, smoothed random velocity, seed 0), parametrised by the per-cell
squared slowness m = 1 / c^2 on the diagonal.  Loss L = 0.5 ||P x - d||^2,
P = 256 random receiver cells (seeded), x = A(m)^{-1} b for one complex
N(0,1) source, d = P x(m_true) for a perturbed velocity c_true = c (1 + 0.05 g)
(g a second smoothed field).  For the plain FP64 and the FP32 + FP64
refinement forms: time of forward + backward (factor, solve, adjoint solve,
pattern gradient), and central finite differences of L along 32 random
directions against <dL/dm, dm>.  Prints one JSON line.

Usage: python tests/cfg4_gradient.py [--grid 64] [--dirs 32]
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", type=int, default=64)
    ap.add_argument("--dirs", type=int, default=32)
    ap.add_argument("--cutoff", type=int, default=128)
    args = ap.parse_args()
    import torch
    from clique_b200 import operators as ops
    from clique_b200.autograd import SparseLDLSolver, sparse_solve
    n = args.grid
    c = ops.smooth_velocity((n, n, n), 0)
    omega = ops.omega_for_ppw(n, float(c.min()), 10.0)
    base, dpos, coef = ops.helmholtz_slowness_parts(n, n, n, omega)
    N = base.n
    g = ops.smooth_velocity((n, n, n), 1) - 1.0
    c_true = c * (1.0 + 0.05 * g / np.abs(g).max())
    dev = "cuda"
    vb = torch.from_numpy(base.values).to(dev)
    dp = torch.from_numpy(dpos).to(dev)
    cf = torch.from_numpy(coef).to(dev)

    def values(m):
        return vb.clone().index_put((dp,), cf * m.to(torch.complex128), accumulate=True)
    rng = np.random.default_rng(2)
    rec = torch.from_numpy(rng.choice(N, 256, replace=False)).to(dev)
    b = torch.from_numpy(ops.random_rhs(N, 1, seed=3, complex_=True)[:, 0]).to(dev)
    m0 = torch.from_numpy(1.0 / c ** 2).to(dev)
    mt = torch.from_numpy(1.0 / c_true ** 2).to(dev)
    out = {"workload": f"{n}^3 complex Helmholtz PML (omega={omega:.2f}), 256 receivers, 1 source",
           "dirs": args.dirs}
    for prec in ("double", "single"):
        solver = SparseLDLSolver(base, (n, n, n), cutoff=args.cutoff, precision=prec, tol=1e-12)
        with torch.no_grad():
            d = sparse_solve(values(mt), b, solver)[rec]

        def loss_of(m, bb=b):
            x = sparse_solve(values(m), bb, solver)
            return 0.5 * (x[rec] - d).abs().pow(2).sum()
        m = m0.clone().requires_grad_(True)
        bb = b.clone().requires_grad_(True)
        for _ in range(2):   # warm-up
            m.grad = bb.grad = None
            loss_of(m, bb).backward()
        torch.cuda.synchronize()
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        m.grad = bb.grad = None
        e0.record()
        L = loss_of(m, bb)
        e1.record()
        L.backward()
        e2.record()
        torch.cuda.synchronize()
        gm = m.grad.detach()
        rel_err = []
        with torch.no_grad():
            for k in range(args.dirs):
                dm = torch.from_numpy(rng.standard_normal(N)).to(dev) * m0
                h = 1e-6
                fd = (loss_of(m0 + h * dm) - loss_of(m0 - h * dm)) / (2 * h)
                ad = torch.dot(gm, dm)
                rel_err.append(abs(float(fd - ad)) / abs(float(ad)))
        out[prec] = {"loss": float(L.detach()), "forward_ms": e0.elapsed_time(e1), "backward_ms": e1.elapsed_time(e2),
                     "fd_max_rel_err": max(rel_err), "fd_median_rel_err": float(np.median(rel_err)),
                     "grad_b_norm": float(bb.grad.norm()), "grad_m_norm": float(gm.norm()),
                     "refine_solves": solver.last_iters[-4:] if solver.last_iters else None}
        del solver
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
