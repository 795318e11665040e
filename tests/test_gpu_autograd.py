"""Differentiation through the sparse solve (clique_b200.autograd): the
reused-factor adjoint solve and the pattern-restricted gradient kernel,
checked against a dense FP64 torch reference and central finite
differences, in the plain FP64 and the FP32 + FP64-refinement forms.

Tolerances: dense reference -- gradients within 1e-9 (FP64) / 1e-8 (FP32 +
refinement to 1e-12) relative to their norm; finite differences (step 1e-6
relative to m) -- directional derivatives within 1e-5 relative.
"""
import numpy as np
import pytest

from clique_b200 import operators as ops

pytestmark = pytest.mark.gpu


def _problem(n, seed, complex_=True):
    import torch
    if complex_:
        c = ops.smooth_velocity((n, n, n), seed)
        omega = ops.omega_for_ppw(n, float(c.min()), 10.0)
        base, dpos, coef = ops.helmholtz_slowness_parts(n, n, n, omega, b=max(2, n // 8))
        m = 1.0 / c ** 2
    else:
        base = ops.laplacian_3d(n, n, n, 0.0)
        rows = np.repeat(np.arange(base.n), np.diff(base.rowptr))
        dpos = np.nonzero(base.colind == rows)[0]
        coef = np.ones(base.n)
        m = 6.1 + 0.3 * np.random.default_rng(seed).random(base.n)
    dev = "cuda"
    dt = torch.complex128 if complex_ else torch.float64
    t = dict(base=torch.from_numpy(base.values).to(dev, dt), dpos=torch.from_numpy(dpos).to(dev),
             coef=torch.from_numpy(np.asarray(coef)).to(dev, dt), m=torch.from_numpy(m).to(dev, torch.float64))
    return base, t


def _values(t, m):
    import torch
    v = t["base"].clone()
    return v.index_put((t["dpos"],), t["coef"] * m.to(v.dtype), accumulate=True)


def _loss_setup(N, nrec, seed, complex_):
    import torch
    rng = np.random.default_rng(seed)
    rec = torch.from_numpy(rng.choice(N, nrec, replace=False)).cuda()
    b = ops.random_rhs(N, 1, seed=seed + 7, complex_=complex_)[:, 0]
    d = 0.1 * ops.random_rhs(nrec, 1, seed=seed + 8, complex_=complex_)[:, 0]
    dt = torch.complex128 if complex_ else torch.float64
    return rec, torch.from_numpy(b).cuda().to(dt), torch.from_numpy(d).cuda().to(dt)


@pytest.mark.parametrize("complex_", [True, False])
@pytest.mark.parametrize("precision", ["double", "single"])
def test_gradients_match_dense_reference(complex_, precision):
    """L = 0.5 ||P x - d||^2 with A(m) x = b: dL/dm, dL/db and dL/dvalues
    against torch.linalg.solve on the dense matrix (16^3 = 4096 unknowns)."""
    import torch
    from clique_b200.autograd import SparseLDLSolver, sparse_solve
    n = 16
    base, t = _problem(n, 3, complex_)
    N = base.n
    rec, b, d = _loss_setup(N, 256, 5, complex_)
    solver = SparseLDLSolver(base, (n, n, n), cutoff=64, precision=precision, tol=1e-12)

    m = t["m"].clone().requires_grad_(True)
    bb = b.clone().requires_grad_(True)
    vals = _values(t, m)
    vals.retain_grad()
    x = sparse_solve(vals, bb, solver)
    loss = 0.5 * (x[rec] - d).abs().pow(2).sum()
    loss.backward()

    m2 = t["m"].clone().requires_grad_(True)
    b2 = b.clone().requires_grad_(True)
    vals2 = _values(t, m2)
    vals2.retain_grad()
    rows = torch.repeat_interleave(torch.arange(N, device="cuda"), torch.from_numpy(np.diff(base.rowptr)).cuda())
    cols = torch.from_numpy(base.colind.astype(np.int64)).cuda()
    Ad = torch.zeros(N, N, dtype=vals2.dtype, device="cuda").index_put((rows, cols), vals2)
    x2 = torch.linalg.solve(Ad, b2)
    loss2 = 0.5 * (x2[rec] - d).abs().pow(2).sum()
    loss2.backward()

    tol = 1e-9 if precision == "double" else 1e-8

    def rel(a, r):
        return float((a - r).norm() / r.norm())
    assert rel(x.detach(), x2.detach()) <= tol
    assert rel(bb.grad, b2.grad) <= tol
    assert rel(vals.grad, vals2.grad) <= tol
    assert rel(m.grad, m2.grad) <= tol


@pytest.mark.parametrize("precision", ["double", "single"])
def test_gradient_matches_central_differences(precision):
    """Directional derivatives of L(m) along 8 random directions (24^3
    complex Helmholtz): <dL/dm, dm> against (L(m + h dm) - L(m - h dm)) / 2h."""
    import torch
    from clique_b200.autograd import SparseLDLSolver, sparse_solve
    n = 24
    base, t = _problem(n, 9, True)
    N = base.n
    rec, b, d = _loss_setup(N, 256, 11, True)
    solver = SparseLDLSolver(base, (n, n, n), cutoff=128, precision=precision, tol=1e-12)

    def loss_of(m):
        x = sparse_solve(_values(t, m), b, solver)
        return 0.5 * (x[rec] - d).abs().pow(2).sum()
    m = t["m"].clone().requires_grad_(True)
    loss_of(m).backward()
    g = m.grad.detach()
    rng = np.random.default_rng(13)
    with torch.no_grad():
        for k in range(8):
            dm = torch.from_numpy(rng.standard_normal(N)).cuda() * t["m"]
            h = 1e-6
            fd = (loss_of(t["m"] + h * dm) - loss_of(t["m"] - h * dm)) / (2 * h)
            ad = torch.dot(g, dm)
            assert abs(float(fd - ad)) <= 1e-5 * abs(float(ad)) + 1e-12, (k, float(fd), float(ad))


def test_backward_after_another_forward_refactors():
    """A second forward on the same solver before the first backward: the first
    backward still uses its own matrix (it refactors from the saved values)."""
    import torch
    from clique_b200.autograd import SparseLDLSolver, sparse_solve
    n = 10
    base, t = _problem(n, 1, True)
    solver = SparseLDLSolver(base, (n, n, n), cutoff=64)
    b = torch.from_numpy(ops.random_rhs(base.n, 2, seed=2, complex_=True)).cuda()
    m1 = t["m"].clone().requires_grad_(True)
    x1 = sparse_solve(_values(t, m1), b, solver)
    m2 = (1.1 * t["m"]).requires_grad_(True)
    x2 = sparse_solve(_values(t, m2), b, solver)
    x1.abs().pow(2).sum().backward()
    g_late = m1.grad.clone()
    m1.grad = None
    x1b = sparse_solve(_values(t, m1), b, solver)
    x1b.abs().pow(2).sum().backward()
    assert float((g_late - m1.grad).norm() / m1.grad.norm()) <= 1e-12
    del x2
