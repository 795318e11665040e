"""Differentiation through the sparse LDL^T solve (no reference counterpart:
Clique has no adjoint; the backward pass composes its own Solve with the
stored factors, include/clique/numeric/solve.hpp:41-65).

``SparseLDLSolver`` keeps one device front tree for a fixed sparsity pattern
on an nx x ny x nz grid (natural nested dissection).  ``sparse_solve(values,
B, solver)`` is a ``torch.autograd.Function``: the forward pass assembles A
from ``values`` (A's CSR entries, both triangles, on the device), factors it
and solves A X = B; the backward pass reuses the stored factors for the
adjoint solve and forms the gradient with respect to A's entries with the
pattern-restricted kernel ``cliqgpu_grad_A_pattern``:

    dL/dB = A^{-H} dL/dX,     dL/dA[e] = -(dL/dB)[i] conj(X[j])   for e = (i, j),

the conjugate-linear convention of torch's complex autograd (as
``torch.linalg.solve``).  A^{-H} needs no second factorization: A^H = A for
real symmetric and Hermitian matrices, and A^H = conj(A) for complex-symmetric
ones, so A^{-H} G = conj(A^{-1} conj(G)).

``values`` must describe a symmetric (complex-symmetric, or Hermitian with
``conjugate=True``) matrix: the factorization reads the lower triangle.  The
gradient is the one of the general matrix restricted to its stored entries;
a parametrisation that writes the same parameter into A[i, j] and A[j, i]
receives the sum of both entries from autograd.

Precision: ``"double"`` factors and solves in FP64; ``"single"`` factors in
FP32 and solves (forward and adjoint) by FP64 iterative refinement to
``tol``.  If another forward ran on the same solver before a backward, the
backward refactors from the values it saved.  The solver's kernels run on the
torch stream that was current when it was constructed.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _capi
from ._capi import LogicError, check


class SparseLDLSolver:
    """One reusable factorization for a fixed pattern (see module docstring)."""

    def __init__(self, A, dims, cutoff=128, precision="double", conjugate=False, tol=1e-10, max_iter=30):
        from . import DistSymmFrontTree, NaturalNestedDissection, _as_csr
        csr = _as_csr(A)
        self.n = csr.n
        self.is_complex = np.iscomplexobj(csr.values)
        self.conjugate = bool(conjugate)
        self.precision = precision
        self.tol, self.max_iter = tol, max_iter
        self.map, self.sep, self.info = NaturalNestedDissection(*dims, csr, cutoff)
        # the plan runs on the torch stream current at construction, so that
        # its kernels are ordered with the torch ops that produce and consume
        # values, right-hand sides and gradients
        self.stream = torch.cuda.current_stream()
        self.L = DistSymmFrontTree(csr, self.map, self.sep, self.info, conjugate, precision=precision, keep_matrix=True,
                                   stream=int(self.stream.cuda_stream))
        self.nnz = csr.nnz
        self.epoch = 0            # bumped by every factorization
        self.last_iters = []      # refinement steps of the last solves (single precision)

    @property
    def dtype(self):
        return torch.complex128 if self.is_complex else torch.float64

    def factor(self, values):
        from . import LDL
        v = values.detach()
        if not v.is_cuda or v.dtype != self.dtype or v.numel() != self.nnz:
            raise LogicError(_capi.CLIQ_ERR_ARG, f"values must be a CUDA {self.dtype} vector of {self.nnz} entries")
        self.L.Initialize(v.resolve_conj().contiguous())
        LDL(self.info, self.L)
        self.epoch += 1

    def solve(self, B):
        """A^{-1} B with the stored factors (B: n or n x k CUDA tensor)."""
        from . import RefinedSolve, Solve
        B2 = B.detach().resolve_conj().reshape(self.n, -1).to(self.dtype)
        if self.precision == "double":
            X = B2.t().contiguous().t().clone() if B2.shape[1] > 1 else B2.clone()
            Solve(self.info, self.L, X)
        else:
            X, it, _ = RefinedSolve(self.L, B2, self.tol, self.max_iter)
            self.last_iters.append(it)
        return X.reshape(B.shape)

    def adjoint_solve(self, G):
        """A^{-H} G with the same factors."""
        if self.is_complex and not self.conjugate:
            return self.solve(G.conj()).conj()
        return self.solve(G)

    def grad_pattern(self, Gb, X):
        """dL/dA on the pattern: out[e] = -sum_k Gb[i, k] conj(X[j, k])."""
        # data pointers go to the C ABI: conjugate views must be materialised
        G2 = Gb.detach().resolve_conj().reshape(self.n, -1).to(self.dtype).t().contiguous().t()
        X2 = X.detach().resolve_conj().reshape(self.n, -1).to(self.dtype).t().contiguous().t()
        out = torch.empty(self.nnz, dtype=self.dtype, device=G2.device)
        k = G2.shape[1]
        ld = G2.stride(1) if k > 1 else self.n
        if k > 1 and X2.stride(1) != ld:
            X2 = X2.t().contiguous().t()
        check(_capi.load().cliqgpu_grad_A_pattern(self.L._h, C.c_void_p(G2.data_ptr()), C.c_void_p(X2.data_ptr()), ld, k,
                                                  int(self.is_complex), C.c_void_p(out.data_ptr())), "grad_A_pattern")
        return out


class _SparseSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, values, B, solver):
        solver.factor(values)
        X = solver.solve(B)
        ctx.solver = solver
        ctx.epoch = solver.epoch
        ctx.save_for_backward(values.detach(), X)
        return X

    @staticmethod
    def backward(ctx, gX):
        values, X = ctx.saved_tensors
        s = ctx.solver
        if s.epoch != ctx.epoch:   # the solver was refactored since this forward
            s.factor(values)
            ctx.epoch = s.epoch
        gB = s.adjoint_solve(gX)
        gV = s.grad_pattern(gB, X) if ctx.needs_input_grad[0] else None
        return gV, (gB if ctx.needs_input_grad[1] else None), None


def sparse_solve(values, B, solver: SparseLDLSolver):
    """X = A(values)^{-1} B, differentiable in values and B."""
    return _SparseSolve.apply(values, B, solver)
