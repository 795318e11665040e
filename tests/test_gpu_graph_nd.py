"""Factorizations over general-graph nested dissection (cliq.NestedDissection)
on the GPU: irregular k-nearest-neighbour graphs, disconnected graphs with
isolated vertices, and the Helmholtz grid ordered as a general graph.
Tolerances: FP64 solutions within 1e-10 of scipy's sparse direct solve with
relative residual <= 1e-12 (1e-11 for the indefinite operator); FP32 fronts
with FP64 refinement reach 1e-10."""
import numpy as np
import pytest

import clique_b200 as cliq
from clique_b200 import operators as ops
from test_graph_nd import knn_graph

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def residual(A, X, B):
    return np.linalg.norm(A.to_scipy() @ X - B) / np.linalg.norm(B)


def _solve(A, cutoff, precision="double", front=cliq.SymmFrontType.LDL_2D, nrhs=3, seps=1):
    map_, sep, info = cliq.NestedDissection(A, cutoff, numSeqSeps=seps)
    L = cliq.DistSymmFrontTree(A, map_, sep, info, precision=precision, keep_matrix=precision != "double")
    cliq.LDL(info, L, front)
    B = ops.random_rhs(A.n, nrhs, seed=5, complex_=np.iscomplexobj(A.values))
    if precision == "double":
        return B, cliq.Solve(info, L, B.copy(order="F"))
    X, it, rr = cliq.RefinedSolve(L, B, 1e-10, 40)
    assert rr <= 1e-10, (it, rr)
    return B, X


@pytest.mark.parametrize("npts,k,dim,cutoff", [(3000, 8, 2, 64), (2500, 10, 3, 96)])
def test_graph_nd_knn_solve(npts, k, dim, cutoff):
    import scipy.sparse.linalg as spla
    A = knn_graph(npts, k, seed=npts, dim=dim)
    B, X = _solve(A, cutoff)
    assert residual(A, X, B) <= 1e-12
    assert rel(X, spla.spsolve(A.to_scipy().tocsc(), B)) <= 1e-10


def test_graph_nd_indefinite_pivoted():
    """Shifted below zero (indefinite): the pivoted fronts over the graph ordering."""
    A0 = knn_graph(3000, 8, seed=11, dim=2, shift=-1.7)
    B, X = _solve(A0, 64, front=cliq.SymmFrontType.LDL_INTRAPIV_2D)
    assert residual(A0, X, B) <= 1e-11


def test_graph_nd_disconnected_single():
    A = knn_graph(600, 6, seed=5, components=3, isolated=500)
    B, X = _solve(A, 48, precision="single")
    assert residual(A, X, B) <= 1e-10


def test_graph_nd_helmholtz_grid_matches_natural():
    """The Helmholtz grid ordered as a general graph: the same solution as
    with natural nested dissection."""
    n = 24
    A, _, _ = ops.helmholtz_workload_3d(n, seed=2)
    B, X = _solve(A, 128, nrhs=2, seps=2)
    map_, sep, info = cliq.NaturalNestedDissection(n, n, n, A, 128)
    L = cliq.DistSymmFrontTree(A, map_, sep, info, precision="double")
    cliq.LDL(info, L)
    Xn = cliq.Solve(info, L, B.copy(order="F"))
    assert rel(X, Xn) <= 1e-10
    assert residual(A, X, B) <= 1e-12


def test_symmetric_solve_orders_the_graph():
    """SymmetricSolve without grid dimensions orders A's graph, as the
    reference's does (solve.hpp:95-116)."""
    A = knn_graph(2000, 8, seed=21, dim=2, shift=-0.9)
    B = ops.random_rhs(A.n, 2, seed=3)
    X = cliq.SymmetricSolve(A, B, cutoff=64)
    assert residual(A, X, B) <= 1e-11


def test_hermitian_solve_black_box():
    """HermitianSolve (solve.hpp:132-140): SymmetricSolve with LDL^H, on an
    indefinite magnetic Laplacian ordered as a general graph."""
    dims = (9, 8, 7)
    A0 = ops.laplacian_3d(*dims, 0.5)
    vals = A0.values.astype(np.complex128)
    rows = np.repeat(np.arange(A0.n), np.diff(A0.rowptr))
    off = A0.colind != rows
    vals[off] = vals[off] * np.exp(1j * 0.4 * np.sign(A0.colind - rows))[off]
    A = ops.CSR(A0.n, A0.rowptr, A0.colind, vals)
    B = ops.random_rhs(A.n, 2, seed=4, complex_=True)
    X = cliq.HermitianSolve(A, B, cutoff=40)
    assert residual(A, X, B) <= 1e-11


def test_intrapiv_reports_a_singular_row():
    """A vertex with no couplings and a zero diagonal: its pivot column is
    zero in any order, and the pivoted factorization reports its ND index."""
    A0 = knn_graph(500, 6, seed=9, isolated=1)
    vals = A0.values.copy()
    v = A0.n - 1
    rows = np.repeat(np.arange(A0.n), np.diff(A0.rowptr))
    vals[(rows == v) & (A0.colind == v)] = 0.0
    A = ops.CSR(A0.n, A0.rowptr, A0.colind, vals)
    map_, sep, info = cliq.NestedDissection(A, 32)
    L = cliq.DistSymmFrontTree(A, map_, sep, info, precision="double")
    with pytest.raises(cliq.CliqueError) as e:
        cliq.LDL(info, L, cliq.SymmFrontType.LDL_INTRAPIV_2D)
    assert e.value.status == 3
    assert L.zero_pivot == int(np.asarray(map_.array)[v])
