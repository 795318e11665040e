"""Many independent grid problems in one device plan (no reference
counterpart: Clique factors one matrix at a time).

``BatchSolver(problems, cutoff, precision)`` takes a list of CSR matrices
with their grid dimensions, builds the block-diagonal matrix, the forest of
their natural nested dissections (``cliq_batch_nested_dissection``) and one
plan over it, so that every factor and sweep launch covers the fronts of all
problems at one tree depth.  ``run(values, B)`` assembles, factors and
refines all problems with ``cliqgpu_batch_run`` (captured as one CUDA graph
from the second call on) and returns the solutions and every problem's
relative residuals; a problem still above the tolerance (an unpivoted FP32
factorization spoilt by pivot growth, or slow classical refinement) is
solved again on its own plans with FGMRES refinement and, if needed, FP64
fronts.  ``autotune()`` picks, launch by launch, the faster of
the tensor-core and CUDA-core update kernels (``cliqgpu_autotune``).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from ._capi import check
from .operators import CSR


def block_diagonal(mats):
    """CSR of the block-diagonal matrix of the given CSR matrices (same field)."""
    rowptr, colind, vals = [np.zeros(1, np.int64)], [], []
    r0, e0 = 0, 0
    for A in mats:
        rowptr.append(A.rowptr[1:] + e0)
        colind.append(A.colind.astype(np.int64) + r0)
        vals.append(A.values)
        r0 += A.n
        e0 += A.nnz
    return CSR(r0, np.concatenate(rowptr), np.concatenate(colind).astype(np.int32), np.concatenate(vals))


class BatchSolver:
    """One plan over a forest of independent problems (see module docstring)."""

    def __init__(self, mats, dims, cutoff=64, precision="single", stream=None):
        """stream: a torch.cuda.Stream for the plan (default: a new side stream)."""
        import torch
        from . import DistMap, DistSeparatorTree, DistSymmFrontTree, DistSymmInfo
        self.count = len(mats)
        self.mats = list(mats)
        self.dims = [tuple(t) for t in dims]
        self.cutoff = cutoff
        self.precision = precision
        self._alone = {}          # problem -> its own plans (fallback), built on first use
        self.A = block_diagonal(mats)
        self.sizes = np.array([A.n for A in mats], np.int64)
        self.seg = np.concatenate([[0], np.cumsum(self.sizes)]).astype(np.int64)
        d = np.ascontiguousarray(np.array([list(t) + [1] * (3 - len(t)) for t in dims], np.int32).reshape(-1))
        lib = _capi.load()
        h = C.c_void_p()
        check(lib.cliq_batch_nested_dissection(self.count, d.ctypes.data_as(C.c_void_p), self.A.n,
                                               self.A.rowptr.ctypes.data_as(C.c_void_p),
                                               self.A.colind.ctypes.data_as(C.c_void_p), cutoff, C.byref(h)),
              "BatchSolver")
        self.info = DistSymmInfo(h.value, self.A.n)
        m = np.zeros(self.A.n, np.int32)
        check(lib.cliq_symbolic_map(h.value, m.ctypes.data_as(C.c_void_p), None))
        self.map = DistMap(m)
        # a torch side stream of its own: the run is captured as a CUDA graph,
        # which the legacy default stream does not allow
        self.stream = torch.cuda.Stream() if stream is None else stream
        self.L = DistSymmFrontTree(self.A, self.map, DistSeparatorTree(self.info), self.info, precision=precision,
                                   keep_matrix=True, stream=int(self.stream.cuda_stream))
        self.is_complex = np.iscomplexobj(self.A.values)

    @property
    def n(self):
        return self.A.n

    def autotune(self, reps=2):
        """Per-launch choice of the update kernel; returns the report of cliqgpu_autotune."""
        out = np.zeros(5)
        check(_capi.load().cliqgpu_autotune(self.L._h, reps, out.ctypes.data_as(C.c_void_p)), "autotune")
        return {"tensor_ms": out[0], "cuda_core_ms": out[1], "chosen_ms": out[2], "moved_to_cuda_cores": int(out[3]),
                "switchable": int(out[4])}

    def _solve_alone(self, p, values, Bc, X, tol):
        """Problem p on its own plans: FP32 fronts + FGMRES refinement, then, if
        that stalls (an unpivoted FP32 factorization spoilt by pivot growth),
        FP64 fronts + FP64 refinement.  Writes X's rows of p; returns
        (relative residual, precision used)."""
        import torch
        from . import LDL, DistSymmFrontTree, NaturalNestedDissection, RefinedSolve
        r0, r1 = int(self.seg[p]), int(self.seg[p + 1])
        e0, e1 = int(self.A.rowptr[r0]), int(self.A.rowptr[r1])
        vals = values[e0:e1].contiguous()
        Bp = Bc[r0:r1]
        nz = Bp.abs().amax(dim=0) > 0
        if not bool(nz.any()):
            X[r0:r1] = 0
            return 0.0, "none"
        if p not in self._alone:
            A = self.mats[p]
            m, sp, info = NaturalNestedDissection(*self.dims[p], A, self.cutoff)
            self._alone[p] = {"A": A, "map": m, "sep": sp, "info": info, "plans": {}}
        ent = self._alone[p]
        best = (np.inf, None, None)
        for prec in (["single", "double"] if self.precision == "single" else ["double"]):
            if prec not in ent["plans"]:
                ent["plans"][prec] = DistSymmFrontTree(ent["A"], ent["map"], ent["sep"], ent["info"], precision=prec,
                                                       keep_matrix=True, stream=int(self.stream.cuda_stream))
            L = ent["plans"][prec]
            L.Initialize(vals)
            LDL(ent["info"], L)
            Xp, it, rr = RefinedSolve(L, Bp.t().contiguous().t(), tol, 30)
            if rr < best[0]:
                best = (rr, prec, Xp)
            if rr <= tol:
                break
        X[r0:r1] = best[2]
        return float(best[0]), best[1]

    def run(self, values, B, X=None, steps=6, tol=1e-10, max_extra=2, fallback=True):
        """Assemble values (device, the block-diagonal CSR order), factor, refine
        B (device, n x nrhs column-major).  Returns (X, relres[count, nrhs], steps).
        Problems still above tol after the batch run are solved again on their
        own plans (fallback=True; see _solve_alone): self.last_fallback lists
        them with the residual and precision they reached."""
        import torch
        Bc = B if B.dim() == 2 else B.reshape(-1, 1)
        nrhs = Bc.shape[1]
        if Bc.stride(0) != 1 or (nrhs > 1 and Bc.stride(1) != self.n):
            Bc = Bc.t().contiguous().t()          # column-major, leading dimension n
        ld = self.n
        if X is None:
            X = torch.empty((nrhs, self.n), dtype=Bc.dtype, device=Bc.device).t()
        elif X.stride(0) != 1 or (nrhs > 1 and X.stride(1) != self.n):
            raise ValueError("X must be column-major with leading dimension n")
        values = values.resolve_conj().contiguous()
        Bc = Bc.resolve_conj()
        rel = np.zeros(self.count * nrhs)
        taken = C.c_int32()
        self.stream.wait_stream(torch.cuda.current_stream())   # inputs produced on the caller's stream
        st = _capi.load().cliqgpu_batch_run(self.L._h, self.count, self.seg.ctypes.data_as(C.c_void_p),
                                            C.c_void_p(values.data_ptr()), C.c_void_p(Bc.data_ptr()),
                                            C.c_void_p(X.data_ptr()), ld, nrhs, steps, tol, max_extra,
                                            rel.ctypes.data_as(C.c_void_p), C.byref(taken))
        torch.cuda.current_stream().wait_stream(self.stream)
        if st not in (_capi.CLIQ_OK, _capi.CLIQ_ERR_NOCONV):
            check(st, "BatchSolver.run")
        rel = rel.reshape(nrhs, self.count).T.copy()
        self.last_fallback = []
        if fallback and st == _capi.CLIQ_ERR_NOCONV:
            with torch.cuda.stream(self.stream):
                for p in np.nonzero(rel.max(axis=1) > tol)[0]:
                    rr, prec = self._solve_alone(int(p), values, Bc, X, tol)
                    rel[p, :] = np.minimum(rel[p, :], rr) if prec == "none" else rr
                    self.last_fallback.append({"problem": int(p), "relres": rr, "precision": prec})
            torch.cuda.current_stream().wait_stream(self.stream)
        return X, rel, taken.value

    def last_launches(self):
        return self.L.last_launches()
