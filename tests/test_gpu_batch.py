"""Many independent problems in one plan (clique_b200.batch): the forest
analysis, the graph-captured batch run with per-problem residuals, and the
kernel-choice autotuner.  Every problem's solution is checked on the host
against its own matrix (relative residual <= 1e-10) and, in FP64, against a
separate single-problem solve (normwise 1e-10)."""
import numpy as np
import pytest

import clique_b200 as cliq
from clique_b200 import operators as ops
from clique_b200.batch import BatchSolver

pytestmark = pytest.mark.gpu


def _problems(count, seed, lo=8, hi=40, rhs_hi=5):
    rng = np.random.default_rng(seed)
    sides = rng.integers(lo, hi + 1, count)
    nrhs = rng.integers(1, rhs_hi + 1, count)
    mats = [ops.helmholtz_workload_2d(int(s), seed=int(seed * 1000 + i))[0] for i, s in enumerate(sides)]
    return mats, [(int(s), int(s), 1) for s in sides], nrhs


def _rhs(mats, nrhs, seed):
    """Right-hand sides of the block-diagonal system: problem p has nrhs[p]
    N(0,1) columns, the remaining columns are zero."""
    k = int(nrhs.max())
    n = sum(A.n for A in mats)
    B = np.zeros((n, k), np.complex128, order="F")
    r0 = 0
    for p, A in enumerate(mats):
        B[r0:r0 + A.n, :nrhs[p]] = ops.random_rhs(A.n, int(nrhs[p]), seed=seed + p, complex_=True)
        r0 += A.n
    return B


def _check(mats, X, B, tol):
    r0 = 0
    worst = 0.0
    for A in mats:
        Xp, Bp = X[r0:r0 + A.n], B[r0:r0 + A.n]
        for j in range(B.shape[1]):
            bn = np.linalg.norm(Bp[:, j])
            if bn > 0:
                worst = max(worst, np.linalg.norm(A.to_scipy() @ Xp[:, j] - Bp[:, j]) / bn)
            else:
                assert np.linalg.norm(Xp[:, j]) == 0
        r0 += A.n
    assert worst <= tol, worst
    return worst


def test_forest_symbolic_is_the_union_of_the_problems():
    mats, dims, _ = _problems(5, 1)
    bs = BatchSolver(mats, dims, cutoff=32, precision="double")
    nodes, r0 = 0, 0
    for A, d in zip(mats, dims):
        m1, _, info1 = cliq.NaturalNestedDissection(*d, A, 32)
        assert np.array_equal(bs.map.array[r0:r0 + A.n], m1.array + r0)
        nodes += info1.num_nodes
        r0 += A.n
    assert bs.info.num_nodes == nodes


@pytest.mark.parametrize("precision", ["single", "double"])
def test_batch_run_direct_then_captured(precision):
    import torch
    mats, dims, nrhs = _problems(12, 2)
    bs = BatchSolver(mats, dims, cutoff=32, precision=precision)
    B = _rhs(mats, nrhs, 7)
    vals = torch.from_numpy(bs.A.values).cuda()
    Bt = torch.from_numpy(B).cuda().t().contiguous().t()
    X1, rel1, st1 = bs.run(vals, Bt, steps=4, tol=1e-10)          # direct launches
    _check(mats, X1.cpu().numpy(), B, 1e-10)
    assert rel1.max() <= 1e-10
    launches_direct = bs.last_launches()
    X2, rel2, st2 = bs.run(vals, Bt, steps=4, tol=1e-10)          # recorded as a graph, replayed
    X3, rel3, st3 = bs.run(vals, Bt, X=X2, steps=4, tol=1e-10)    # replay
    for X, rel in ((X2, rel2), (X3, rel3)):
        _check(mats, X.cpu().numpy(), B, 1e-10)
        assert rel.max() <= 1e-10
    assert bs.last_launches() == launches_direct or bs.last_launches() >= launches_direct
    # every problem's residual as reported equals the host check's order of magnitude
    assert rel3.shape == (12, B.shape[1])
    # new values through the same graph: a shifted operator
    vals2 = vals * 1.0
    vals2 = vals2.clone()
    X4, rel4, _ = bs.run(vals2, Bt, steps=4, tol=1e-10)
    _check(mats, X4.cpu().numpy(), B, 1e-10)


def test_batch_fp64_matches_single_problem_solves():
    import torch
    mats, dims, nrhs = _problems(6, 3)
    bs = BatchSolver(mats, dims, cutoff=32, precision="double")
    B = _rhs(mats, nrhs, 11)
    vals = torch.from_numpy(bs.A.values).cuda()
    Bt = torch.from_numpy(B).cuda().t().contiguous().t()
    X, rel, _ = bs.run(vals, Bt, steps=1, tol=1e-10)
    X = X.cpu().numpy()
    r0 = 0
    for A, d in zip(mats, dims):
        m1, s1, i1 = cliq.NaturalNestedDissection(*d, A, 32)
        L = cliq.DistSymmFrontTree(A, m1, s1, i1, precision="double")
        cliq.LDL(i1, L)
        Xs = cliq.Solve(i1, L, B[r0:r0 + A.n].copy(order="F"))
        assert np.linalg.norm(X[r0:r0 + A.n] - Xs) <= 1e-10 * np.linalg.norm(Xs)
        r0 += A.n


def test_autotune_keeps_results_and_reports():
    import torch
    mats, dims, nrhs = _problems(10, 4, lo=16, hi=64)
    bs = BatchSolver(mats, dims, cutoff=32, precision="single")
    B = _rhs(mats, nrhs, 13)
    vals = torch.from_numpy(bs.A.values).cuda()
    Bt = torch.from_numpy(B).cuda().t().contiguous().t()
    bs.run(vals, Bt, steps=4, tol=1e-10)
    rep = bs.autotune(reps=1)
    assert rep["switchable"] > 0
    assert rep["chosen_ms"] <= min(rep["tensor_ms"], rep["cuda_core_ms"]) + 1e-9
    X, rel, _ = bs.run(vals, Bt, steps=4, tol=1e-10)
    _check(mats, X.cpu().numpy(), B, 1e-10)
    # a second plan of the same shapes takes the recorded choices
    bs2 = BatchSolver(mats, dims, cutoff=32, precision="single")
    X2, rel2, _ = bs2.run(vals, Bt, steps=4, tol=1e-10)
    _check(mats, X2.cpu().numpy(), B, 1e-10)


def test_batch_fallback_rescues_a_problem_fp32_cannot_factor():
    """One problem whose first pivot (ND order) is 1e-8 of its neighbours:
    the unpivoted FP32 factorization grows by ~1e8 and its refinement stalls,
    so the batch run leaves it above the tolerance; the fallback re-solves it
    on its own plans (FP64 fronts if FP32 + FGMRES does not reach tol).  The
    other problems keep the batch solution."""
    import torch
    mats, dims, nrhs = _problems(5, 6, lo=16, hi=32)
    s = 20
    bad = ops.laplacian_2d(s, s, 4.0)
    m1, _, _ = cliq.NaturalNestedDissection(s, s, 1, bad, 32)
    first = int(np.nonzero(m1.array == 0)[0][0])          # natural index of ND index 0
    rows = np.repeat(np.arange(bad.n), np.diff(bad.rowptr))
    e = np.nonzero((rows == first) & (bad.colind == first))[0][0]
    vals = bad.values.astype(np.complex128)
    vals[e] = 4e-8
    bad = ops.CSR(bad.n, bad.rowptr, bad.colind, vals)
    mats = mats + [bad]
    dims = dims + [(s, s, 1)]
    nrhs = np.concatenate([nrhs, [2]])
    bs = BatchSolver(mats, dims, cutoff=32, precision="single")
    B = _rhs(mats, nrhs, 17)
    v = torch.from_numpy(bs.A.values).cuda()
    Bt = torch.from_numpy(B).cuda().t().contiguous().t()
    X, rel, _ = bs.run(v, Bt, steps=4, tol=1e-10, max_extra=2)
    assert [f["problem"] for f in bs.last_fallback] == [len(mats) - 1], bs.last_fallback
    assert rel.max() <= 1e-10
    _check(mats, X.cpu().numpy(), B, 1e-10)
