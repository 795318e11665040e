"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle and
the dense golden factors, on the same orderings.

Tolerances: FP64 factor entries within 1e-12 of the dense LDL^T (relative to
the largest entry); FP64 solutions within 1e-10 normwise relative error of
the oracle's with relative residual <= 1e-12; the mixed form (FP32 fronts,
FP64 refinement) reaches relative residual <= 1e-10.
"""
import os

import numpy as np
import pytest

import clique_b200 as cliq
from clique_b200 import operators as ops

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def build(A, dims, cutoff, precision="double", conjugate=False):
    map_, sep, info = cliq.NaturalNestedDissection(*dims, A, cutoff)
    L = cliq.DistSymmFrontTree(A, map_, sep, info, conjugate, precision=precision)
    cliq.LDL(info, L)
    return map_, info, L


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def residual(A, X, B):
    return np.linalg.norm(A.to_scipy() @ X - B) / np.linalg.norm(B)


@pytest.mark.parametrize("fx", ["ldl_lap_3x3x1.npz", "ldl_helm_3x3x1.npz", "ldl_lap_6x5x4_c8.npz", "ldl_helm_6x5x4_c8.npz"])
def test_fronts_match_dense_golden(fx):
    z = np.load(os.path.join(GOLD, fx))
    A = ops.CSR(len(z["map"]), z["rowptr"], z["colind"], z["values"])
    dims = [int(t) for t in fx[:-4].split("_")[2].split("x")]
    cutoff = 8 if "c8" in fx else 2
    map_, info, L = build(A, dims, cutoff)
    assert np.array_equal(map_.array, z["map"])
    Ld, Dd = z["L"], z["D"]
    scale = np.abs(Ld).max()
    for s, nd in enumerate(info.localNodes):
        Lf, d = L.front(s)
        rows = np.concatenate([np.arange(nd.off, nd.off + nd.size), nd.lowerStruct]).astype(int)
        np.testing.assert_allclose(Lf, Ld[np.ix_(rows, np.arange(nd.off, nd.off + nd.size))], atol=1e-12 * scale, rtol=0)
        np.testing.assert_allclose(d, Dd[nd.off:nd.off + nd.size], rtol=1e-12)
    x = cliq.Solve(info, L, np.asfortranarray(z["b"].reshape(-1, 1)))[:, 0]
    assert rel(x, z["x"]) <= 1e-12


@pytest.mark.parametrize("complex_", [False, True])
def test_fronts_match_oracle(oracle, complex_):
    dims, cutoff = (12, 10, 9), 30
    if complex_:
        A = ops.helmholtz_pml_3d(*dims, omega=20.0, velocity=ops.smooth_velocity(dims, 4), b=3)
    else:
        A = ops.laplacian_3d(*dims, 6.1)
    map_, info, L = build(A, dims, cutoff)
    S = oracle.Symbolic(*dims, A.rowptr, A.colind, cutoff=cutoff)
    F = oracle.Fronts(S, A.values, is_complex=complex_)
    assert F.ldl(96) == 0
    for s in range(S.num_nodes):
        Lg, dg = L.front(s)
        Lo, do = F.front(s)
        assert Lg.shape == Lo.shape
        assert rel(Lg, Lo) <= 1e-11, s
        assert rel(dg, do) <= 1e-11, s


def test_cfg1_plain_fp64_30cubed(oracle):
    """The 30^3 7-point operator (diag 6.1, cutoff 128, 1 N(0,1) RHS): GPU vs oracle on the same ordering."""
    n = 30
    A = ops.laplacian_3d(n, n, n, 6.1)
    b = ops.random_rhs(A.n, 1, seed=0)
    map_, info, L = build(A, (n, n, n), 128)
    x = cliq.Solve(info, L, b.copy(order="F"))
    oracle.enable_blas(0)
    try:
        S = oracle.Symbolic(n, n, n, A.rowptr, A.colind, cutoff=128)
        F = oracle.Fronts(S, A.values)
        assert F.ldl(96) == 0
        xo = F.solve(b.copy(order="F"))
    finally:
        oracle.disable_blas()
    assert rel(x, xo) <= 1e-10
    assert residual(A, x, b) <= 1e-12


@pytest.mark.parametrize("nrhs", [1, 4, 20])
def test_helmholtz_fp64_solve(oracle, nrhs):
    n = 16
    A, omega, c = ops.helmholtz_workload_3d(n, seed=3)
    B = ops.random_rhs(A.n, nrhs, seed=1, complex_=True)
    map_, info, L = build(A, (n, n, n), 64)
    X = cliq.Solve(info, L, B.copy(order="F"))
    S = oracle.Symbolic(n, n, n, A.rowptr, A.colind, cutoff=64)
    F = oracle.Fronts(S, A.values, is_complex=True)
    assert F.ldl(96) == 0
    Xo = F.solve(B.copy(order="F"))
    assert rel(X, Xo) <= 1e-10
    assert residual(A, X, B) <= 1e-12


@pytest.mark.parametrize("complex_", [False, True])
def test_mixed_fp32_refinement(complex_):
    n = 20
    if complex_:
        A, _, _ = ops.helmholtz_workload_3d(n, seed=5)
    else:
        A = ops.laplacian_3d(n, n, n, 6.1)
    B = ops.random_rhs(A.n, 3, seed=2, complex_=complex_)
    map_, info, L = build(A, (n, n, n), 64, precision="single")
    X, iters, rr = cliq.RefinedSolve(L, B, tol=1e-10, max_iter=30)
    assert rr <= 1e-10, (iters, rr)
    assert residual(A, X, B) <= 1e-10
    Xd = np.linalg.solve(A.to_scipy().toarray(), B) if A.n <= 9000 else None
    if Xd is not None:
        assert rel(X, Xd) <= 1e-8


@pytest.mark.parametrize("complex_", [False, True])
def test_refinement_fgmres_vs_classical(complex_, monkeypatch):
    """FGMRES refinement (default) reaches the tolerance in no more solves
    than classical refinement over the same FP32 factors, and both converge
    to the same solution."""
    n = 24
    if complex_:
        A, _, _ = ops.helmholtz_workload_3d(n, seed=7)
    else:
        A = ops.laplacian_3d(n, n, n, 6.1)
    B = ops.random_rhs(A.n, 4, seed=3, complex_=complex_)
    out = {}
    for mode in ("gmres", "ir"):
        monkeypatch.setenv("CLIQGPU_REFINE", mode)
        map_, info, L = build(A, (n, n, n), 64, precision="single")
        out[mode] = cliq.RefinedSolve(L, B, tol=1e-11, max_iter=30)
        del L
    (Xg, itg, rrg), (Xi, iti, rri) = out["gmres"], out["ir"]
    print(f"solves: FGMRES {itg} (relres {rrg:.1e}), classical {iti} (relres {rri:.1e})")
    assert rrg <= 1e-11 and rri <= 1e-11
    assert residual(A, Xg, B) <= 1e-11
    assert itg <= iti
    assert rel(Xg, Xi) <= 1e-8


def test_refined_solve_into_pinned_host_buffer():
    """RefinedSolve with host buffers writes into a caller-provided
    Fortran-ordered X (pinned memory, as the end-to-end benchmark passes it)
    the same solution it returns in a fresh array."""
    import torch
    n = 20
    A, _, _ = ops.helmholtz_workload_3d(n, seed=5)
    B = np.asfortranarray(ops.random_rhs(A.n, 3, seed=2, complex_=True))
    map_, info, L = build(A, (n, n, n), 64, precision="single")
    X0, it0, rr0 = cliq.RefinedSolve(L, B, tol=1e-11, max_iter=30)
    Xp = torch.empty((3, A.n), dtype=torch.complex128, pin_memory=True).numpy().T
    Bp = torch.empty((3, A.n), dtype=torch.complex128, pin_memory=True).numpy().T
    Bp[...] = B
    X1, it1, rr1 = cliq.RefinedSolve(L, Bp, tol=1e-11, max_iter=30, X=Xp)
    assert X1 is Xp
    assert rr1 <= 1e-11 and residual(A, X1, B) <= 1e-11
    assert rel(X1, X0) <= 1e-9
    with pytest.raises(Exception):
        cliq.RefinedSolve(L, Bp, tol=1e-11, max_iter=30, X=np.zeros((A.n, 3), np.complex128))   # C-ordered: rejected


def test_factor_graph_replay_matches_direct(monkeypatch):
    """CLIQGPU_GRAPH=1: the second and later factorizations replay a captured
    graph of the launch sequence; the factors and the refined solution match
    the direct launches."""
    n = 24
    A, _, _ = ops.helmholtz_workload_3d(n, seed=11)
    B = ops.random_rhs(A.n, 2, seed=4, complex_=True)
    out = {}
    for mode in ("0", "1"):
        monkeypatch.setenv("CLIQGPU_GRAPH", mode)
        map_, info, L = build(A, (n, n, n), 64, precision="single")
        for _ in range(3):   # the first run launches directly, the second captures, the third replays
            L.Initialize(A.values)
            cliq.LDL(info, L)
        out[mode] = cliq.RefinedSolve(L, B, tol=1e-11, max_iter=30)
        del L
    (X0, it0, rr0), (X1, it1, rr1) = out["0"], out["1"]
    assert rr0 <= 1e-11 and rr1 <= 1e-11
    assert residual(A, X1, B) <= 1e-11
    assert rel(X1, X0) <= 1e-8


def test_schur_chunks_match_single_update(monkeypatch):
    """CLIQGPU_SCHUR_CHUNK: the Schur complement applied in K chunks on the
    third stream gives the same refined solution as the single update."""
    n = 28
    A, _, _ = ops.helmholtz_workload_3d(n, seed=13)
    B = ops.random_rhs(A.n, 2, seed=6, complex_=True)
    out = {}
    for chunk in ("0", "128"):
        monkeypatch.setenv("CLIQGPU_SCHUR_CHUNK", chunk)
        monkeypatch.setenv("CLIQGPU_OUTER_BLOCK", "64")
        map_, info, L = build(A, (n, n, n), 64, precision="single")
        L.Initialize(A.values)
        cliq.LDL(info, L)
        out[chunk] = cliq.RefinedSolve(L, B, tol=1e-11, max_iter=30)
        del L
    (X0, it0, rr0), (X1, it1, rr1) = out["0"], out["128"]
    assert rr0 <= 1e-11 and rr1 <= 1e-11
    assert residual(A, X1, B) <= 1e-11
    assert rel(X1, X0) <= 1e-8


def test_bounded_wait_times_out_and_plan_stays_usable():
    """A device-side wait on a flag that nothing sets gives up after its
    limit: the call reports CLIQ_ERR_TIMEOUT with the wait site, and the same
    plan then refactors and solves correctly (no GPU fault, no hang)."""
    import time
    from clique_b200 import _capi
    n = 16
    A, _, _ = ops.helmholtz_workload_3d(n, seed=9)
    B = ops.random_rhs(A.n, 1, seed=1, complex_=True)
    map_, info, L = build(A, (n, n, n), 64, precision="single")
    X0, _, rr0 = cliq.RefinedSolve(L, B, tol=1e-11, max_iter=30)
    lib = _capi.load()
    t0 = time.perf_counter()
    st = lib.cliqgpu_wait_selftest(L._h, 50_000_000)   # 50 ms
    dt = time.perf_counter() - t0
    assert st == _capi.CLIQ_ERR_TIMEOUT
    assert "solve: block flag" in lib.cliqgpu_last_error().decode()
    assert 0.04 <= dt < 5.0
    assert lib.cliqgpu_wait_selftest(L._h, 0) == _capi.CLIQ_ERR_ARG
    L.Initialize(A.values)
    cliq.LDL(info, L)
    X1, _, rr1 = cliq.RefinedSolve(L, B, tol=1e-11, max_iter=30)
    assert rr1 <= 1e-11 and residual(A, X1, B) <= 1e-11
    assert rel(X1, X0) <= 1e-8


def _magnetic(dims, shift=6.5, theta=0.3):
    A = ops.laplacian_3d(*dims, shift)
    vals = A.values.astype(np.complex128)
    rows = np.repeat(np.arange(A.n), np.diff(A.rowptr))
    off = A.colind != rows
    vals[off] = vals[off] * np.exp(1j * theta * np.sign(A.colind - rows))[off]
    return ops.CSR(A.n, A.rowptr, A.colind, vals)


@pytest.mark.parametrize("precision", ["double", "single"])
def test_hermitian_ldlh(oracle, precision):
    dims = (11, 9, 8)
    A = _magnetic(dims)
    B = ops.random_rhs(A.n, 2, seed=9, complex_=True)
    map_, info, L = build(A, dims, 40, precision=precision, conjugate=True)
    if precision == "double":
        X = cliq.Solve(info, L, B.copy(order="F"))
        S = oracle.Symbolic(*dims, A.rowptr, A.colind, cutoff=40)
        F = oracle.Fronts(S, A.values, is_complex=True, conjugate=True)
        assert F.ldl(96) == 0
        assert rel(X, F.solve(B.copy(order="F"))) <= 1e-10
        assert residual(A, X, B) <= 1e-12
    else:
        X, it, rr = cliq.RefinedSolve(L, B, 1e-11, 20)
        assert rr <= 1e-11


def test_nodal_solve_equals_natural():
    n = 14
    A = ops.laplacian_3d(n, n, n, 6.1)
    B = ops.random_rhs(A.n, 2, seed=3)
    map_, info, L = build(A, (n, n, n), 50)
    inv = map_.FormInverse()
    Xn = cliq.DistNodalMultiVec(inv, info, B)
    cliq.Solve(info, L, Xn)
    X1 = np.zeros_like(B, order="F")
    Xn.Push(inv, info, X1)
    X2 = cliq.Solve(info, L, B.copy(order="F"))
    assert rel(X1, X2) <= 1e-14
    assert sum(x.shape[0] for x in Xn.localNodes) == A.n


@pytest.mark.parametrize("dims,cutoff", [((1, 1, 1), 1), ((5, 1, 1), 1), ((2, 2, 2), 100), ((17, 3, 1), 4),
                                         ((7, 5, 3), 6), ((65, 2, 1), 16), ((3, 70, 1), 100)])
def test_edge_grids(oracle, dims, cutoff):
    A = ops.laplacian_3d(*dims, 6.1)
    B = ops.random_rhs(A.n, 2, seed=4)
    map_, info, L = build(A, dims, cutoff)
    X = cliq.Solve(info, L, B.copy(order="F"))
    S = oracle.Symbolic(*dims, A.rowptr, A.colind, cutoff=cutoff)
    F = oracle.Fronts(S, A.values)
    F.ldl(96)
    assert rel(X, F.solve(B.copy(order="F"))) <= 1e-12


def test_zero_pivot_is_reported():
    A = ops.laplacian_3d(3, 1, 1, 6.1)
    vals = A.values.copy()
    rows = np.repeat(np.arange(A.n), np.diff(A.rowptr))
    vals[(rows == 0) & (A.colind == 0)] = 0.0
    A0 = ops.CSR(A.n, A.rowptr, A.colind, vals)
    map_, sep, info = cliq.NaturalNestedDissection(3, 1, 1, A0, 1)
    L = cliq.DistSymmFrontTree(A0, map_, sep, info)
    with pytest.raises(cliq.CliqueError) as e:
        cliq.LDL(info, L)
    assert e.value.status == 3
    assert L.zero_pivot == 0


def test_ldl_twice_is_a_logic_error():
    A = ops.laplacian_3d(4, 4, 4, 6.1)
    map_, info, L = build(A, (4, 4, 4), 8)
    with pytest.raises(cliq.LogicError):
        cliq.LDL(info, L)


def test_refactor_with_new_values_reuses_plan(oracle):
    """tests/Refactor.cpp pattern: reassemble new values into the same front tree and factor again."""
    n = 12
    A = ops.laplacian_3d(n, n, n, 6.1)
    map_, info, L = build(A, (n, n, n), 32)
    A2 = ops.laplacian_3d(n, n, n, 7.3)
    L.Initialize(A2.values)
    cliq.LDL(info, L)
    B = ops.random_rhs(A.n, 1, seed=8)
    X = cliq.Solve(info, L, B.copy(order="F"))
    assert residual(A2, X, B) <= 1e-12


def test_device_resident_inputs():
    import torch
    n = 16
    A, _, _ = ops.helmholtz_workload_3d(n, seed=1)
    map_, sep, info = cliq.NaturalNestedDissection(n, n, n, A, 64)
    L = cliq.DistSymmFrontTree(A, map_, sep, info, precision="single")
    L.Initialize(torch.from_numpy(A.values).cuda())
    cliq.LDL(info, L)
    B = ops.random_rhs(A.n, 2, seed=3, complex_=True)
    Bt = torch.from_numpy(B).cuda().t().contiguous().t()
    X, it, rr = cliq.RefinedSolve(L, Bt, 1e-10, 30)
    assert rr <= 1e-10
    Xh = X.cpu().numpy()
    assert residual(A, Xh, B) <= 1e-10
    Y = torch.zeros_like(Bt)
    cliq.Multiply(1.0, L, X, 0.0, Y)
    assert rel(Y.cpu().numpy(), B) <= 1e-10


@pytest.mark.parametrize("complex_", [False, True])
@pytest.mark.parametrize("precision", ["double", "single"])
def test_single_front_ldl(oracle, complex_, precision):
    """cliqgpu_front_ldl (FrontLDL on one dense front) against the oracle's FrontLDL."""
    import ctypes as C
    import torch
    from clique_b200 import _capi
    m, n = 300, 150
    rng = np.random.default_rng(7)
    G = rng.standard_normal((m, m)) + (1j * rng.standard_normal((m, m)) if complex_ else 0)
    S = G @ G.T / m + 8 * np.eye(m)      # symmetric (complex-symmetric when complex)
    AL = np.asfortranarray(np.tril(S)[:, :n])
    ABR = np.asfortranarray(np.tril(S[n:, n:]))
    ALo, ABRo = AL.copy(order="F"), ABR.copy(order="F")
    assert oracle.front_ldl(ALo, ABRo, nb=96) == 0
    tdt = {("double", False): torch.float64, ("double", True): torch.complex128,
           ("single", False): torch.float32, ("single", True): torch.complex64}[(precision, complex_)]
    tAL = torch.from_numpy(AL).to(tdt).cuda().t().contiguous().t()
    tABR = torch.from_numpy(ABR).to(tdt).cuda().t().contiguous().t()
    st = _capi.load().cliqgpu_front_ldl(int(complex_), 0 if precision == "double" else 1, 0, m, n,
                                        C.c_void_p(tAL.data_ptr()), m, C.c_void_p(tABR.data_ptr()), m - n, None)
    assert st == 0
    torch.cuda.synchronize()
    tol = 1e-12 if precision == "double" else 1e-4
    assert rel(tAL.cpu().numpy().astype(ALo.dtype), ALo) <= tol
    g = np.tril(tABR.cpu().numpy().astype(ABRo.dtype))
    assert rel(g, np.tril(ABRo)) <= tol


@pytest.mark.parametrize("split", ["f16", "tf32"])
@pytest.mark.parametrize("complex_", [False, True])
def test_fp32_tensor_core_fronts(oracle, complex_, split, monkeypatch):
    """FP32 fronts from the tcgen05 update kernel (2xFP16 split with per-row
    scales, or 3xTF32) agree with the FP64 oracle to FP32-level accuracy, and
    with the CUDA-core FP32 kernel."""
    monkeypatch.setenv("CLIQGPU_SPLIT", split)
    dims, cutoff = (14, 13, 12), 40
    if complex_:
        A = ops.helmholtz_pml_3d(*dims, omega=25.0, velocity=ops.smooth_velocity(dims, 6), b=3)
    else:
        A = ops.laplacian_3d(*dims, 6.1)
    S = oracle.Symbolic(*dims, A.rowptr, A.colind, cutoff=cutoff)
    F = oracle.Fronts(S, A.values, is_complex=complex_)
    assert F.ldl(96) == 0
    fronts = {}
    for tc in ("1", "0"):
        monkeypatch.setenv("CLIQGPU_TENSOR_CORES", tc)
        map_, info, L = build(A, dims, cutoff, precision="single")
        fronts[tc] = [L.front(s) for s in range(S.num_nodes)]
    worst_tc = worst_cc = 0.0
    for s in range(S.num_nodes):
        Lo, do = F.front(s)
        Lt, dt = fronts["1"][s]
        Ls, ds = fronts["0"][s]
        worst_tc = max(worst_tc, rel(Lt, Lo), rel(dt, do))
        worst_cc = max(worst_cc, rel(Ls, Lo), rel(ds, do))
    # the split products are about as accurate as FP32 CUDA-core arithmetic
    # (measured: 1.1-1.6x its error on the Laplacian, 1.0x on the Helmholtz
    # operator, whose absolute level reflects unpivoted FP32 LDL^T of an
    # indefinite operator)
    print(f"worst front error: tensor cores {worst_tc:.2e}, CUDA cores {worst_cc:.2e}")
    assert worst_tc <= 2.5 * worst_cc, (worst_tc, worst_cc)
    assert worst_tc <= (2e-3 if complex_ else 1e-6), worst_tc


@pytest.mark.parametrize("complex_", [False, True])
def test_gpu_multiply_matches_oracle(oracle, complex_):
    """Y := alpha A X + beta Y on the device (the plan's copy of A, and the
    plan-free cliqgpu_sparse_multiply with device and host buffers) against
    the oracle's Multiply (multiply.hpp:28-166)."""
    import ctypes as C
    import torch
    from clique_b200 import _capi
    n = 11
    if complex_:
        A, _, _ = ops.helmholtz_workload_3d(n, seed=2)
    else:
        A = ops.laplacian_3d(n, n, n, 6.1)
    rng = np.random.default_rng(4)
    dt = np.complex128 if complex_ else np.float64
    X = np.asfortranarray(ops.random_rhs(A.n, 3, seed=5, complex_=complex_))
    Y0 = np.asfortranarray(ops.random_rhs(A.n, 3, seed=6, complex_=complex_))
    alpha, beta = (dt(1.5 - 0.5j), dt(-0.25 + 2j)) if complex_ else (1.5, -0.25)
    Yo = oracle.multiply(A.rowptr, A.colind, A.values, alpha, X, beta, Y0.copy(order="F"))
    # plan-held matrix
    map_, sep, info = cliq.NaturalNestedDissection(n, n, n, A, 32)
    L = cliq.DistSymmFrontTree(A, map_, sep, info, precision="double")
    Xt = torch.from_numpy(X).cuda().t().contiguous().t()
    Yt = torch.from_numpy(Y0).cuda().t().contiguous().t()
    cliq.Multiply(alpha, L, Xt, beta, Yt)
    assert rel(Yt.cpu().numpy(), Yo) <= 1e-14
    # plan-free product, device buffers
    lib = _capi.load()
    a = np.array([alpha], dt).view(np.float64)
    b = np.array([beta], dt).view(np.float64)
    rp = torch.from_numpy(A.rowptr).cuda()
    ci = torch.from_numpy(A.colind).cuda()
    va = torch.from_numpy(A.values).cuda()
    Yt = torch.from_numpy(Y0).cuda().t().contiguous().t()
    st = lib.cliqgpu_sparse_multiply(int(complex_), A.n, C.c_void_p(rp.data_ptr()), C.c_void_p(ci.data_ptr()),
                                     C.c_void_p(va.data_ptr()), a.ctypes.data_as(C.c_void_p), C.c_void_p(Xt.data_ptr()),
                                     b.ctypes.data_as(C.c_void_p), C.c_void_p(Yt.data_ptr()), A.n, 3, 1, None)
    assert st == 0
    torch.cuda.synchronize()
    assert rel(Yt.cpu().numpy(), Yo) <= 1e-14
    # plan-free product, host buffers (the C++ drop-in's Multiply)
    Yh = Y0.copy(order="F")
    st = lib.cliqgpu_sparse_multiply(int(complex_), A.n, A.rowptr.ctypes.data_as(C.c_void_p),
                                     A.colind.ctypes.data_as(C.c_void_p), A.values.ctypes.data_as(C.c_void_p),
                                     a.ctypes.data_as(C.c_void_p), X.ctypes.data_as(C.c_void_p),
                                     b.ctypes.data_as(C.c_void_p), Yh.ctypes.data_as(C.c_void_p), A.n, 3, 0, None)
    assert st == 0
    assert rel(Yh, Yo) <= 1e-14


@pytest.mark.parametrize("complex_", [False, True])
def test_nodal_pull_push_on_device(complex_):
    """DistNodalMultiVec.Pull / Push on device tensors run the pull / push
    kernels and match the host permutation exactly."""
    import torch
    n = 9
    A = ops.laplacian_3d(n, n, n, 6.1)
    map_, sep, info = cliq.NaturalNestedDissection(n, n, n, A, 16)
    inv = map_.FormInverse()
    X = ops.random_rhs(A.n, 2, seed=3, complex_=complex_)
    Xt = torch.from_numpy(X).cuda().t().contiguous().t()
    nod = cliq.DistNodalMultiVec(inv, info, Xt)
    assert np.array_equal(nod.X.cpu().numpy(), X[inv.array])
    Yt = torch.zeros_like(Xt)
    nod.Push(inv, info, Yt)
    assert np.array_equal(Yt.cpu().numpy(), X)


def test_helmholtz48_fp64_vs_oracle(oracle):
    """The largest complex FP64 case the oracle factors in seconds: 48^3
    Helmholtz-PML workload, cutoff 128, 4 right-hand sides."""
    n = 48
    A, _, _ = ops.helmholtz_workload_3d(n, seed=0)
    B = ops.random_rhs(A.n, 4, seed=1, complex_=True)
    map_, info, L = build(A, (n, n, n), 128)
    X = cliq.Solve(info, L, B.copy(order="F"))
    oracle.enable_blas(0)
    try:
        S = oracle.Symbolic(n, n, n, A.rowptr, A.colind, cutoff=128)
        F = oracle.Fronts(S, A.values, is_complex=True)
        assert F.ldl(96) == 0
        Xo = F.solve(B.copy(order="F"))
    finally:
        oracle.disable_blas()
    err = rel(X, Xo)
    res = residual(A, X, B)
    print(f"48^3 FP64: vs oracle {err:.2e}, residual {res:.2e} (oracle {residual(A, Xo, B):.2e})")
    assert err <= 1e-10
    assert res <= 1e-12


@pytest.mark.parametrize("complex_,conjugate", [(False, False), (True, False), (True, True)])
def test_fp64_dmma_updates_match_cuda_cores(oracle, complex_, conjugate, monkeypatch):
    """The FP64 updates on the FP64 tensor cores (DMMA, the default) and on the
    CUDA cores give the same fronts to FP64 rounding, and both match the oracle."""
    dims, cutoff = (17, 15, 14), 48
    if complex_:
        A = _magnetic(dims) if conjugate else \
            ops.helmholtz_pml_3d(*dims, omega=22.0, velocity=ops.smooth_velocity(dims, 2), b=3)
    else:
        A = ops.laplacian_3d(*dims, 6.1)
    S = oracle.Symbolic(*dims, A.rowptr, A.colind, cutoff=cutoff)
    F = oracle.Fronts(S, A.values, is_complex=complex_, conjugate=conjugate)
    assert F.ldl(96) == 0
    fronts = {}
    for v in ("1", "0"):
        monkeypatch.setenv("CLIQGPU_FP64_DMMA", v)
        map_, info, L = build(A, dims, cutoff, conjugate=conjugate)
        fronts[v] = [L.front(s) for s in range(S.num_nodes)]
    for s in range(S.num_nodes):
        Lo, do = F.front(s)
        for v in ("1", "0"):
            Lg, dg = fronts[v][s]
            assert rel(Lg, Lo) <= 1e-11, (v, s)
            assert rel(dg, do) <= 1e-11, (v, s)
        assert rel(fronts["1"][s][0], fronts["0"][s][0]) <= 1e-12


def test_selinv_front_types_factor_and_solve_as_ldl():
    """LDL_SELINV_1D / LDL_SELINV_2D at one process: the reference inverts only
    distributed fronts (change_front_type.hpp:86-98), so the factorization and
    the solve are the LDL_2D ones; likewise LDL_INTRAPIV_SELINV_* and
    LDL_INTRAPIV_*; the unfactored types are refused."""
    n = 12
    A, _, _ = ops.helmholtz_workload_3d(n, seed=4)
    B = ops.random_rhs(A.n, 2, seed=5, complex_=True)
    map_, sep, info = cliq.NaturalNestedDissection(n, n, n, A, 64)
    X = {}
    for ft in (cliq.SymmFrontType.LDL_2D, cliq.SymmFrontType.LDL_SELINV_2D, cliq.SymmFrontType.LDL_SELINV_1D):
        L = cliq.DistSymmFrontTree(A, map_, sep, info, precision="double")
        cliq.LDL(info, L, ft)
        assert L.frontType == ft
        X[ft] = cliq.Solve(info, L, B.copy(order="F"))
    assert rel(X[cliq.SymmFrontType.LDL_SELINV_2D], X[cliq.SymmFrontType.LDL_2D]) <= 1e-14
    assert residual(A, X[cliq.SymmFrontType.LDL_SELINV_1D], B) <= 1e-12
    Xp = {}
    for ft in (cliq.SymmFrontType.LDL_INTRAPIV_2D, cliq.SymmFrontType.LDL_INTRAPIV_SELINV_2D,
               cliq.SymmFrontType.LDL_INTRAPIV_SELINV_1D):
        L = cliq.DistSymmFrontTree(A, map_, sep, info, precision="double")
        cliq.LDL(info, L, ft)
        Xp[ft] = cliq.Solve(info, L, B.copy(order="F"))
    assert rel(Xp[cliq.SymmFrontType.LDL_INTRAPIV_SELINV_2D], Xp[cliq.SymmFrontType.LDL_INTRAPIV_2D]) <= 1e-14
    assert residual(A, Xp[cliq.SymmFrontType.LDL_INTRAPIV_SELINV_1D], B) <= 1e-12
    for ft in (cliq.SymmFrontType.SYMM_1D, cliq.SymmFrontType.SYMM_2D):
        L = cliq.DistSymmFrontTree(A, map_, sep, info, precision="double")
        with pytest.raises(cliq.LogicError):
            cliq.LDL(info, L, ft)


@pytest.mark.parametrize("kind,precision", [("real", "double"), ("complex", "double"), ("hermitian", "double"),
                                            ("complex", "single")])
def test_block_ldl_matches_oracle(oracle, kind, precision):
    """BLOCK_LDL_2D (FrontBlockLDL, ldl/local_front_block.hpp:27-71): every
    front holds inv(A11) over A21 as in the oracle, the product-only block
    sweeps (20 right-hand sides: a 16-column chunk and a 4-column one) give
    the oracle's solution, and a refactorization in the LDL_2D form goes back
    to the triangular sweeps."""
    dims, cutoff = (17, 15, 14), 48
    conj = kind == "hermitian"
    if kind == "real":
        A = ops.laplacian_3d(*dims, 6.1)
    elif kind == "complex":
        A = ops.helmholtz_pml_3d(*dims, omega=22.0, velocity=ops.smooth_velocity(dims, 2), b=3)
    else:
        A = _magnetic(dims)
    cplx = kind != "real"
    map_, sep, info = cliq.NaturalNestedDissection(*dims, A, cutoff)
    L = cliq.DistSymmFrontTree(A, map_, sep, info, conj, precision=precision)
    cliq.LDL(info, L, cliq.SymmFrontType.BLOCK_LDL_2D)
    assert L.frontType == cliq.SymmFrontType.BLOCK_LDL_2D
    B = ops.random_rhs(A.n, 20, seed=11, complex_=cplx)
    if precision == "double":
        S = oracle.Symbolic(*dims, A.rowptr, A.colind, cutoff=cutoff)
        F = oracle.Fronts(S, A.values, is_complex=cplx, conjugate=conj)
        assert F.ldl(96, block=True) == 0
        for s in range(S.num_nodes):
            Lg, _ = L.front(s)
            Lo, _ = F.front(s)
            assert rel(Lg, Lo) <= 1e-10, s
        X = cliq.Solve(info, L, B.copy(order="F"))
        assert rel(X, F.solve(B.copy(order="F"))) <= 1e-10
        assert residual(A, X, B) <= 1e-11
    else:
        X, it, rr = cliq.RefinedSolve(L, B, 1e-10, 40)
        assert rr <= 1e-10, (it, rr)
        assert residual(A, X, B) <= 1e-10
    L.Initialize(A.values)
    cliq.LDL(info, L, cliq.SymmFrontType.LDL_2D)
    if precision == "double":
        X2 = cliq.Solve(info, L, B.copy(order="F"))
        assert residual(A, X2, B) <= 1e-12
        assert rel(X2, X) <= 1e-10


@pytest.mark.parametrize("kind", ["real", "complex"])
def test_block_ldl_split_products_64cubed(kind):
    """At 64^3 the block sweeps split the long products over several CTAs
    (the root's 4096 x 4096 inv(A11) and the 4096-row A21 of its children)
    and add the partial sums in a second launch: the block solution matches
    the LDL_2D one on the same matrix."""
    n = 64
    if kind == "real":
        A = ops.laplacian_3d(n, n, n, 6.1)
        precision = "double"
    else:
        A, _, _ = ops.helmholtz_workload_3d(n, seed=2)
        precision = "single"
    B = ops.random_rhs(A.n, 5, seed=4, complex_=kind == "complex")
    map_, sep, info = cliq.NaturalNestedDissection(n, n, n, A, 128)
    L = cliq.DistSymmFrontTree(A, map_, sep, info, precision=precision)
    cliq.LDL(info, L, cliq.SymmFrontType.LDL_2D)
    if precision == "double":
        X0 = cliq.Solve(info, L, B.copy(order="F"))
    else:
        X0, _, rr0 = cliq.RefinedSolve(L, B, 1e-10, 40)
        assert rr0 <= 1e-10
    L.Initialize(A.values)
    cliq.LDL(info, L, cliq.SymmFrontType.BLOCK_LDL_2D)
    if precision == "double":
        X = cliq.Solve(info, L, B.copy(order="F"))
        assert residual(A, X, B) <= 1e-11
        assert rel(X, X0) <= 1e-10
    else:
        X, it, rr = cliq.RefinedSolve(L, B, 1e-10, 40)
        assert rr <= 1e-10, (it, rr)
        assert rel(X, X0) <= 1e-8


@pytest.mark.parametrize("form,precision", [("exact", "single"), ("tiles", "double"), ("exact", "double")])
def test_solve_form_override(oracle, form, precision, monkeypatch):
    """CLIQGPU_SOLVE_FORM: the plan and its sweeps use the chosen chain form
    (product form with chain tiles, or substitution form without them) in
    either precision."""
    monkeypatch.setenv("CLIQGPU_SOLVE_FORM", form)
    n = 14
    A, _, _ = ops.helmholtz_workload_3d(n, seed=6)
    B = ops.random_rhs(A.n, 3, seed=8, complex_=True)
    map_, info, L = build(A, (n, n, n), 64, precision=precision)
    if precision == "double":
        X = cliq.Solve(info, L, B.copy(order="F"))
        assert residual(A, X, B) <= 1e-12
    else:
        X, it, rr = cliq.RefinedSolve(L, B, 1e-10, 30)
        assert rr <= 1e-10, (it, rr)


def test_refined_solve_fp64_fallback():
    """RefinedSolve(fallback=True): when the FP32 factors cannot bring the
    residual to tol within max_iter steps, the matrix is factored again with
    FP64 fronts (kept with the tree for the same values) and the solve
    reaches tol; without fallback the FP32 attempt reports its residual."""
    n = 14
    A, _, _ = ops.helmholtz_workload_3d(n, seed=7)
    B = ops.random_rhs(A.n, 2, seed=9, complex_=True)
    map_, sep, info = cliq.NaturalNestedDissection(n, n, n, A, 64)
    L = cliq.DistSymmFrontTree(A, map_, sep, info, precision="single")
    cliq.LDL(info, L)
    _, it0, rr0 = cliq.RefinedSolve(L, B, 1e-13, 1)
    assert rr0 > 1e-13 and not L.last_fallback
    X, it, rr = cliq.RefinedSolve(L, B, 1e-13, 1, fallback=True)
    assert L.last_fallback and rr <= 1e-13, (it, rr)
    assert residual(A, X, B) <= 1e-12
    twin = L._fp64_tree()
    X2, _, rr2 = cliq.RefinedSolve(L, B, 1e-13, 1, fallback=True)
    assert L._fp64_tree() is twin and rr2 <= 1e-13
    L.Initialize(A.values)
    cliq.LDL(info, L)
    _, _, rr3 = cliq.RefinedSolve(L, B, 1e-10, 30, fallback=True)
    assert rr3 <= 1e-10 and not L.last_fallback


@pytest.mark.parametrize("kind", ["real", "complex", "hermitian"])
@pytest.mark.parametrize("nrhs", [3, 9, 20])
def test_tiny_front_sweeps_match_oracle(oracle, kind, nrhs):
    """A 2D grid whose leaves have one pivot block and at most 64 rows below
    (the one-warp-per-front sweeps) solved in FP64 for 3, 9 and 20
    right-hand sides (the 4-, 16- and 16 + 4-column sweep instantiations),
    against the oracle's solve on the same ordering."""
    n1, n2, cutoff = 41, 37, 32
    conj = kind == "hermitian"
    if kind == "real":
        A = ops.laplacian_2d(n1, n2, 4.1)
    elif kind == "complex":
        A = ops.helmholtz_pml_2d(n1, n2, omega=18.0, b=4)
    else:
        L0 = ops.laplacian_2d(n1, n2, 4.5)
        vals = L0.values.astype(np.complex128)
        rows = np.repeat(np.arange(L0.n), np.diff(L0.rowptr))
        off = L0.colind != rows
        vals[off] = vals[off] * np.exp(1j * 0.3 * np.sign(L0.colind - rows))[off]
        A = ops.CSR(L0.n, L0.rowptr, L0.colind, vals)
    cplx = kind != "real"
    map_, info, L = build(A, (n1, n2, 1), cutoff, conjugate=conj)
    sizes = [(nd.size, len(nd.lowerStruct)) for nd in info.localNodes]
    assert any(0 < s <= 64 and u <= 64 for s, u in sizes)
    B = ops.random_rhs(A.n, nrhs, seed=nrhs, complex_=cplx)
    X = cliq.Solve(info, L, B.copy(order="F"))
    S = oracle.Symbolic(n1, n2, 1, A.rowptr, A.colind, cutoff=cutoff)
    F = oracle.Fronts(S, A.values, is_complex=cplx, conjugate=conj)
    assert F.ldl(96) == 0
    assert rel(X, F.solve(B.copy(order="F"))) <= 1e-10
    assert residual(A, X, B) <= 1e-11
