"""One dense front through cliqgpu_front_ldl on cuda:0, for kernel profiles
(run by hand; pytest does not collect this file).

FrontLDL of an m x n front (complex symmetric or real, FP64 or FP32) with a
diagonally dominant random matrix: the 64-column steps of the n pivots, then
the Schur-complement update of the (m - n)^2 block -- with FP64 storage the
largest launch of the FP64 tensor-core (DMMA) update kernel.  The call is
repeated --reps times; the result is checked against numpy's dense LDL^T
residual once.

Usage: python tests/profile_front.py [--m 4096] [--n 2048] [--complex] [--single] [--reps 2]
"""
from __future__ import annotations

import argparse
import ctypes as C
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--m", type=int, default=4096)
    ap.add_argument("--n", type=int, default=2048)
    ap.add_argument("--complex", action="store_true")
    ap.add_argument("--single", action="store_true")
    ap.add_argument("--reps", type=int, default=2)
    args = ap.parse_args()
    import torch
    from clique_b200 import _capi
    m, n = args.m, args.n
    rng = np.random.default_rng(0)
    k = 32
    G = rng.standard_normal((m, k)) + (1j * rng.standard_normal((m, k)) if args.complex else 0)
    G /= np.sqrt(k)
    dt = {(False, False): torch.float64, (False, True): torch.float32, (True, False): torch.complex128,
          (True, True): torch.complex64}[(args.complex, args.single)]
    AL = torch.from_numpy(G @ G[:n].T).to(dt).cuda()
    AL[:n] = torch.tril(AL[:n])
    AL[torch.arange(n), torch.arange(n)] += 4.0
    ABR = torch.from_numpy(np.tril(G[n:] @ G[n:].T)).to(dt).cuda()
    ABR[torch.arange(m - n), torch.arange(m - n)] += 4.0
    AL0, ABR0 = AL.clone(), ABR.clone()
    AL = AL.t().contiguous().t()      # column-major
    ABR = ABR.t().contiguous().t()
    lib = _capi.load()
    for r in range(args.reps):
        AL.copy_(AL0)
        ABR.copy_(ABR0)
        st = lib.cliqgpu_front_ldl(int(args.complex), int(args.single), 0, m, n, C.c_void_p(AL.data_ptr()), m,
                                   C.c_void_p(ABR.data_ptr()), m - n, None)
        torch.cuda.synchronize()
        assert st == 0, lib.cliqgpu_last_error()
    # check: A11 = L D L^T on the pivots
    Lf = AL[:n].cpu().numpy().astype(np.complex128 if args.complex else np.float64)
    d = np.diag(Lf).copy()
    Lu = np.tril(Lf, -1) + np.eye(n)
    A11 = AL0[:n].cpu().numpy().astype(Lf.dtype)
    A11 = A11 + np.tril(A11, -1).T
    err = np.linalg.norm(Lu @ np.diag(d) @ Lu.T - A11) / np.linalg.norm(A11)
    print(f"front {m} x {n}: ||L D L^T - A11|| / ||A11|| = {err:.2e}")
    assert err < (1e-4 if args.single else 1e-12)


if __name__ == "__main__":
    main()
