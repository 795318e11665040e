"""Intra-front pivoting on the GPU (LDL_INTRAPIV_1D / LDL_INTRAPIV_2D,
through cliqgpu_factor_intrapiv) against the CPU oracle's FrontLDLIntraPiv.

Tolerances: FP64 -- the same pivot order and 2x2 blocks as the oracle in
every front, L, D and the 2x2 off-diagonals within 1e-10 of the oracle's
(relative to the front's largest entry), solutions within 1e-10 of the
oracle's with relative residual <= 1e-12; FP32 fronts with FP64 refinement
reach relative residual <= 1e-10.  The operators are indefinite, with their
couplings scaled by a deterministic pseudo-random symmetric factor so that
no two pivot candidates tie exactly.
"""
import numpy as np
import pytest

import clique_b200 as cliq
from clique_b200 import operators as ops

pytestmark = pytest.mark.gpu


def _perturbed(A, vals, seed=0):
    rows = np.repeat(np.arange(A.n), np.diff(A.rowptr))
    lo = np.minimum(rows, A.colind).astype(np.int64)
    hi = np.maximum(rows, A.colind).astype(np.int64)
    h = ((lo * 1000003 + hi * 7919 + seed) % 1009) / 1009.0
    return ops.CSR(A.n, A.rowptr, A.colind, vals * (1.0 + 0.4 * (h - 0.5)))


def _indefinite(kind, dims):
    """Shifted Laplacian (real symmetric), PML Helmholtz (complex symmetric),
    shifted magnetic Laplacian (Hermitian); all indefinite."""
    if kind == "complex":
        A = ops.helmholtz_pml_3d(*dims, omega=18.0, velocity=ops.smooth_velocity(dims, 3), b=2)
        return _perturbed(A, A.values), False
    A = ops.laplacian_3d(*dims, 0.5)
    vals = A.values
    if kind == "hermitian":
        vals = vals.astype(np.complex128)
        rows = np.repeat(np.arange(A.n), np.diff(A.rowptr))
        off = A.colind != rows
        vals[off] = vals[off] * np.exp(1j * 0.4 * np.sign(A.colind - rows))[off]
    return _perturbed(A, vals), kind == "hermitian"


def _tree(A, dims, cutoff, precision, conj, front_type=cliq.SymmFrontType.LDL_INTRAPIV_2D, keep=False):
    map_, sep, info = cliq.NaturalNestedDissection(*dims, A, cutoff)
    L = cliq.DistSymmFrontTree(A, map_, sep, info, conj, precision=precision, keep_matrix=keep)
    cliq.LDL(info, L, front_type)
    return map_, info, L


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def residual(A, X, B):
    return np.linalg.norm(A.to_scipy() @ X - B) / np.linalg.norm(B)


# (24, 12, 6) / 100: fronts of 66-72 pivots with rows below (two panels);
# (16, 16, 10) / 200: a 160-pivot root and 80-160-pivot fronts below it
CASES = [((9, 8, 7), 24), ((24, 12, 6), 100), ((16, 16, 10), 200)]


@pytest.mark.parametrize("kind", ["real", "complex", "hermitian"])
@pytest.mark.parametrize("dims,cutoff", CASES)
def test_intrapiv_fronts_match_oracle(oracle, kind, dims, cutoff):
    A, conj = _indefinite(kind, dims)
    cplx = kind != "real"
    _, _, L = _tree(A, dims, cutoff, "double", conj)
    S = oracle.Symbolic(*dims, A.rowptr, A.colind, cutoff=cutoff)
    F = oracle.Fronts(S, A.values, is_complex=cplx, conjugate=conj)
    assert F.ldl(96, pivot=True) == 0
    swaps = blocks = 0
    for s in range(S.num_nodes):
        Lo, do = F.front(s)
        so, po = F.pivots(s)
        Lg, dg = L.front(s)
        sg, pg = L.front_pivots(s)
        assert np.array_equal(pg, po), s
        scale = max(np.abs(Lo).max(), np.abs(do).max(), 1e-300)
        assert np.abs(Lg - Lo).max() <= 1e-10 * scale, s
        assert np.abs(dg - do).max() <= 1e-10 * scale, s
        assert np.abs(sg - so).max() <= 1e-10 * scale, s
        swaps += int((po != np.arange(len(po))).sum())
        blocks += int((so != 0).sum())
    assert swaps > 0
    if kind != "complex":   # (the PML Helmholtz fronts may interchange rows without 2x2 blocks)
        assert blocks > 0


@pytest.mark.parametrize("kind", ["real", "complex", "hermitian"])
@pytest.mark.parametrize("nrhs", [1, 5, 20])
def test_intrapiv_solve_matches_oracle(oracle, kind, nrhs):
    dims, cutoff = (24, 12, 6), 100
    A, conj = _indefinite(kind, dims)
    cplx = kind != "real"
    _, info, L = _tree(A, dims, cutoff, "double", conj)
    B = ops.random_rhs(A.n, nrhs, seed=nrhs, complex_=cplx)
    X = cliq.Solve(info, L, B.copy(order="F"))
    S = oracle.Symbolic(*dims, A.rowptr, A.colind, cutoff=cutoff)
    F = oracle.Fronts(S, A.values, is_complex=cplx, conjugate=conj)
    assert F.ldl(96, pivot=True) == 0
    assert rel(X, F.solve(B.copy(order="F"))) <= 1e-10
    assert residual(A, X, B) <= 1e-12


@pytest.mark.parametrize("kind", ["real", "complex", "hermitian"])
def test_intrapiv_single_refined(kind):
    dims, cutoff = (16, 16, 10), 200
    A, conj = _indefinite(kind, dims)
    _, _, L = _tree(A, dims, cutoff, "single", conj, keep=True)
    B = ops.random_rhs(A.n, 3, seed=2, complex_=kind != "real")
    X, it, rr = cliq.RefinedSolve(L, B, 1e-10, 40)
    assert rr <= 1e-10, (it, rr)
    assert residual(A, X, B) <= 1e-10


def test_intrapiv_zero_diagonal():
    """An exactly zero first pivot: the unpivoted factorization reports it,
    the pivoted one factors and solves to FP64 accuracy."""
    dims = (6, 5, 4)
    A0 = ops.laplacian_3d(*dims, 6.1)
    map_, sep, info = cliq.NaturalNestedDissection(*dims, A0, 30)
    g = int(np.asarray(map_.FormInverse().array)[0])   # natural index of ND position 0
    vals = A0.values.copy()
    rows = np.repeat(np.arange(A0.n), np.diff(A0.rowptr))
    vals[(rows == g) & (A0.colind == g)] = 0.0
    A = ops.CSR(A0.n, A0.rowptr, A0.colind, vals)
    L = cliq.DistSymmFrontTree(A, map_, sep, info, precision="double")
    with pytest.raises(cliq.CliqueError) as e:
        cliq.LDL(info, L)
    assert e.value.status == 3 and L.zero_pivot == 0
    L = cliq.DistSymmFrontTree(A, map_, sep, info, precision="double")
    cliq.LDL(info, L, cliq.SymmFrontType.LDL_INTRAPIV_1D)
    B = ops.random_rhs(A.n, 2, seed=3)
    X = cliq.Solve(info, L, B.copy(order="F"))
    assert residual(A, X, B) <= 1e-12


def test_intrapiv_nodal_and_refactor():
    """ND-order (nodal) solves keep the ND order with pivoted fronts; the same
    plan refactored unpivoted (new values) solves with its maps restored."""
    dims, cutoff = (14, 12, 10), 80
    A, _ = _indefinite("real", dims)
    map_, info, L = _tree(A, dims, cutoff, "double", False)
    B = ops.random_rhs(A.n, 2, seed=3)
    inv = map_.FormInverse()
    Xn = cliq.DistNodalMultiVec(inv, info, B)
    cliq.Solve(info, L, Xn)
    X1 = np.zeros_like(B, order="F")
    Xn.Push(inv, info, X1)
    X2 = cliq.Solve(info, L, B.copy(order="F"))
    assert rel(X1, X2) <= 1e-14
    assert residual(A, X2, B) <= 1e-11   # indefinite shifted Laplacian: measured 1.5e-12
    Apd = ops.laplacian_3d(*dims, 6.1)
    L.Initialize(Apd.values)
    cliq.LDL(info, L, cliq.SymmFrontType.LDL_2D)
    X3 = cliq.Solve(info, L, B.copy(order="F"))
    assert residual(Apd, X3, B) <= 1e-12
    L.Initialize(A.values)
    cliq.LDL(info, L, cliq.SymmFrontType.LDL_INTRAPIV_2D)
    X4 = cliq.Solve(info, L, B.copy(order="F"))
    assert rel(X4, X2) <= 1e-13


def test_symmetric_solve_pivots_by_default():
    """SymmetricSolve factors with LDL_INTRAPIV_1D, as solve.hpp:110 does."""
    dims = (10, 9, 8)
    A, _ = _indefinite("complex", dims)
    B = ops.random_rhs(A.n, 2, seed=6, complex_=True)
    X = cliq.SymmetricSolve(A, B, *dims, cutoff=40)
    assert residual(A, X, B) <= 1e-12


@pytest.mark.parametrize("kind", ["real", "complex", "hermitian"])
def test_block_intrapiv_matches_oracle(oracle, kind):
    """BLOCK_LDL_INTRAPIV_2D: the GPU fronts hold inv(P A11 P^T) over A21 P^T
    (the pivoted order its solves use); the oracle's hold inv(A11) over A21 in
    the assembled order (FrontBlockLDL's intraPiv branch).  Same pivots, the
    same blocks once permuted, the same solutions; FP32 fronts refine."""
    dims, cutoff = (24, 12, 6), 100
    A, conj = _indefinite(kind, dims)
    cplx = kind != "real"
    bt = cliq.SymmFrontType.BLOCK_LDL_INTRAPIV_2D
    _, info, L = _tree(A, dims, cutoff, "double", conj, front_type=bt)
    S = oracle.Symbolic(*dims, A.rowptr, A.colind, cutoff=cutoff)
    F = oracle.Fronts(S, A.values, is_complex=cplx, conjugate=conj)
    assert F.ldl(96, block=True, pivot=True) == 0
    for s in range(S.num_nodes):
        Lo, _ = F.front(s)
        _, po = F.pivots(s)
        Lg, _ = L.front(s)
        _, pg = L.front_pivots(s)
        assert np.array_equal(pg, po), s
        n = Lg.shape[1]
        top = Lo[:n][np.ix_(po, po)]
        assert np.abs(Lg[:n] - top).max() <= 1e-9 * np.abs(top).max(), s
        if Lg.shape[0] > n:
            low = Lo[n:][:, po]
            assert np.abs(Lg[n:] - low).max() <= 1e-10 * max(np.abs(low).max(), 1.0), s
    B = ops.random_rhs(A.n, 4, seed=8, complex_=cplx)
    X = cliq.Solve(info, L, B.copy(order="F"))
    assert rel(X, F.solve(B.copy(order="F"))) <= 1e-9
    assert residual(A, X, B) <= 1e-10   # explicit inverses of the pivot blocks: measured up to 1.5e-11
    _, _, L32 = _tree(A, dims, cutoff, "single", conj, front_type=bt, keep=True)
    X32, it, rr = cliq.RefinedSolve(L32, B, 1e-10, 40)
    assert rr <= 1e-10, (it, rr)


@pytest.mark.parametrize("kind", ["real", "complex", "hermitian"])
def test_intrapiv_fp32_tensor_core_schur(kind, monkeypatch):
    """FP32 pivoted fronts with the Schur complements on the tensor cores
    (2xFP16 split, D's 2x2 blocks packed into the S operand) are about as
    accurate as with the CUDA-core Schur update, measured against the FP64
    pivoted fronts on the fronts whose pivot order all three share."""
    dims, cutoff = (16, 16, 10), 200
    A, conj = _indefinite(kind, dims)
    runs = {}
    for name, prec, tc in (("fp64", "double", "1"), ("tc", "single", "1"), ("cc", "single", "0")):
        monkeypatch.setenv("CLIQGPU_TENSOR_CORES", tc)
        _, info, L = _tree(A, dims, cutoff, prec, conj)
        runs[name] = [(L.front(s), L.front_pivots(s)) for s in range(info.num_nodes)]
    err = {"tc": 0.0, "cc": 0.0}
    same = 0
    for s in range(len(runs["fp64"])):
        (L64, d64), (_, p64) = runs["fp64"][s]
        if not all(np.array_equal(runs[k][s][1][1], p64) for k in ("tc", "cc")):
            continue
        same += 1
        scale = max(np.abs(L64).max(), np.abs(d64).max(), 1e-300)
        for k in ("tc", "cc"):
            (Lk, dk), _ = runs[k][s]
            err[k] = max(err[k], np.abs(Lk - L64).max() / scale, np.abs(dk - d64).max() / scale)
    print(f"{same} of {len(runs['fp64'])} fronts with the FP64 pivot order; worst error vs FP64: "
          f"tensor-core Schur {err['tc']:.2e}, CUDA-core Schur {err['cc']:.2e}")
    assert same >= len(runs["fp64"]) // 2
    # measured: 5.6e-3 / 1.5e-3 (real), 1.8e-6 / 1.8e-6 (complex), 2.8e-3 / 3.2e-3
    # (Hermitian); a wrong 2x2 term in the packed operand gives O(1)
    assert err["tc"] <= 6.0 * err["cc"] + 1e-6, err


@pytest.mark.parametrize("dims,cutoff", [((1, 1, 1), 1), ((5, 1, 1), 1), ((2, 2, 2), 100), ((17, 3, 1), 4),
                                         ((7, 5, 3), 6), ((65, 2, 1), 16), ((3, 70, 1), 100)])
def test_intrapiv_edge_grids(oracle, dims, cutoff):
    """Degenerate trees (one node, empty leaves, thin grids, one front of
    210 pivots) with pivoting: the oracle's pivoted solution."""
    A0 = ops.laplacian_3d(*dims, 0.5)
    A = _perturbed(A0, A0.values)
    B = ops.random_rhs(A.n, 2, seed=4)
    _, info, L = _tree(A, dims, cutoff, "double", False)
    X = cliq.Solve(info, L, B.copy(order="F"))
    S = oracle.Symbolic(*dims, A.rowptr, A.colind, cutoff=cutoff)
    F = oracle.Fronts(S, A.values)
    assert F.ldl(96, pivot=True) == 0
    assert rel(X, F.solve(B.copy(order="F"))) <= 1e-10


@pytest.mark.parametrize("front", ["LDL_2D", "LDL_INTRAPIV_2D"])
def test_many_right_hand_sides(oracle, front):
    """A SolveRange-sized solve (tests/SolveRange.cpp solves 100-1000
    right-hand sides): 130 columns, several 16-column chunks and a ragged
    tail, against the oracle's solve."""
    dims, cutoff = (14, 12, 10), 80
    A, conj = _indefinite("complex", dims)
    _, info, L = _tree(A, dims, cutoff, "double", conj, front_type=getattr(cliq.SymmFrontType, front))
    B = ops.random_rhs(A.n, 130, seed=13, complex_=True)
    X = cliq.Solve(info, L, B.copy(order="F"))
    S = oracle.Symbolic(*dims, A.rowptr, A.colind, cutoff=cutoff)
    F = oracle.Fronts(S, A.values, is_complex=True, conjugate=conj)
    assert F.ldl(96, pivot=front != "LDL_2D") == 0
    assert rel(X, F.solve(B.copy(order="F"))) <= 1e-10
    assert residual(A, X, B) <= 1e-12


@pytest.mark.parametrize("kind", ["real", "complex"])
def test_intrapiv_clustered_panels(oracle, kind):
    """A root front of 528 pivots (26 x 24 x 22 grid, cutoff 256): the top
    levels' panels run on clusters of CTAs; pivots and fronts as the
    oracle's, and the oracle's solution."""
    dims, cutoff = (26, 24, 22), 256
    A, conj = _indefinite(kind, dims)
    cplx = kind != "real"
    _, info, L = _tree(A, dims, cutoff, "double", conj)
    S = oracle.Symbolic(*dims, A.rowptr, A.colind, cutoff=cutoff)
    F = oracle.Fronts(S, A.values, is_complex=cplx, conjugate=conj)
    assert F.ldl(96, pivot=True) == 0
    assert max(L.front(s)[0].shape[1] for s in range(S.num_nodes)) >= 512
    for s in range(S.num_nodes):
        Lo, do = F.front(s)
        so, po = F.pivots(s)
        Lg, dg = L.front(s)
        sg, pg = L.front_pivots(s)
        assert np.array_equal(pg, po), s
        scale = max(np.abs(Lo).max(), np.abs(do).max(), 1e-300)
        assert np.abs(Lg - Lo).max() <= 1e-10 * scale, s
        assert np.abs(dg - do).max() <= 1e-10 * scale, s
        assert np.abs(sg - so).max() <= 1e-10 * scale, s
    B = ops.random_rhs(A.n, 3, seed=5, complex_=cplx)
    X = cliq.Solve(info, L, B.copy(order="F"))
    assert rel(X, F.solve(B.copy(order="F"))) <= 1e-10


@pytest.mark.parametrize("kind", ["real", "complex", "hermitian"])
@pytest.mark.parametrize("dims,cutoff", [((16, 16, 10), 200), ((26, 24, 22), 256)])
def test_intrapiv_fp32_in_front_update_kernels(kind, dims, cutoff, monkeypatch):
    """The FP32 in-front updates on the 128 x 64 tile kernel are as accurate
    as on the 64 x 64 one (CLIQGPU_PIV_UPDATE=tile64), measured against the
    FP64 pivoted fronts on the fronts whose pivot order all three share, and
    the refined solve reaches 1e-10.  The 26 x 24 x 22 grid's top fronts
    (528 and 264 pivots, trailing blocks of several 128-row tiles and odd
    numbers of 64-column blocks) exercise the tile map."""
    A, conj = _indefinite(kind, dims)
    runs = {}
    for name, prec, upd in (("fp64", "double", ""), ("wide", "single", ""), ("tile64", "single", "tile64")):
        monkeypatch.setenv("CLIQGPU_PIV_UPDATE", upd)
        _, info, L = _tree(A, dims, cutoff, prec, conj, keep=name == "wide")
        runs[name] = [(L.front(s), L.front_pivots(s)) for s in range(info.num_nodes)]
        if name == "wide":
            B = ops.random_rhs(A.n, 2, seed=9, complex_=kind != "real")
            X, it, rr = cliq.RefinedSolve(L, B, 1e-10, 40)
            assert rr <= 1e-10, (it, rr)
            assert residual(A, X, B) <= 1e-9
    err = {"wide": 0.0, "tile64": 0.0}
    same = 0
    for s in range(len(runs["fp64"])):
        (L64, d64), (_, p64) = runs["fp64"][s]
        if not all(np.array_equal(runs[k][s][1][1], p64) for k in err):
            continue
        same += 1
        scale = max(np.abs(L64).max(), np.abs(d64).max(), 1e-300)
        for k in err:
            (Lk, dk), _ = runs[k][s]
            err[k] = max(err[k], np.abs(Lk - L64).max() / scale, np.abs(dk - d64).max() / scale)
    print(f"{same} of {len(runs['fp64'])} fronts with the FP64 pivot order; worst error vs FP64: "
          f"128 x 64 tiles {err['wide']:.2e}, 64 x 64 tiles {err['tile64']:.2e}")
    assert same >= len(runs["fp64"]) // 2
    # both sum the same products in different orders; a wrong tile or a lost
    # 2x2 term gives O(1)
    assert err["wide"] <= 4.0 * err["tile64"] + 1e-6, err


@pytest.mark.parametrize("kind", ["real", "complex", "hermitian"])
def test_intrapiv_fp64_in_front_update_on_dmma(kind, monkeypatch):
    """FP64 pivoted fronts with the in-front updates on DMMA (the default)
    and on the CUDA cores (CLIQGPU_PIV_UPDATE=tile64) agree to FP64
    rounding, with the same pivots, and give the same solution.  (The
    shifted Laplacian here is ill-conditioned -- solutions of size ~500 for
    right-hand sides of size 1 -- so its residual is ~1e-11, not 1e-12.)"""
    dims, cutoff = (26, 24, 22), 256
    A, conj = _indefinite(kind, dims)
    B = ops.random_rhs(A.n, 2, seed=6, complex_=kind != "real")
    runs, sols = {}, {}
    for name, upd in (("dmma", ""), ("cuda", "tile64")):
        monkeypatch.setenv("CLIQGPU_PIV_UPDATE", upd)
        _, info, L = _tree(A, dims, cutoff, "double", conj)
        runs[name] = [(L.front(s), L.front_pivots(s)) for s in range(info.num_nodes)]
        sols[name] = cliq.Solve(info, L, B.copy(order="F"))
        assert residual(A, sols[name], B) <= 1e-10, name
    assert rel(sols["dmma"], sols["cuda"]) <= 1e-10
    same = 0
    worst = 0.0
    for (Fd, Pd), (Fc, Pc) in zip(runs["dmma"], runs["cuda"]):
        if not np.array_equal(Pd[1], Pc[1]):
            continue
        same += 1
        scale = max(np.abs(Fc[0]).max(), np.abs(Fc[1]).max(), 1e-300)
        worst = max(worst, np.abs(Fd[0] - Fc[0]).max() / scale, np.abs(Fd[1] - Fc[1]).max() / scale,
                    np.abs(Pd[0] - Pc[0]).max() / scale)
    print(f"{same} of {len(runs['dmma'])} fronts with the same pivots; worst difference {worst:.2e}")
    assert same == len(runs["dmma"])
    # measured: 0 (real: both kernels sum each entry's products as fused
    # multiply-adds in k order), 7.0e-16 (complex), 6.1e-12 (Hermitian)
    assert worst <= 1e-10
