"""Synthetic operators with the shapes and formulas of the reference drivers.

* ``laplacian_3d``  -- 7-point negative Laplacian, tests/Solve.cpp:59-82
  (diagonal 6 by default; the benchmark workloads add a shift of 0.1).
* ``helmholtz_pml_3d`` / ``helmholtz_pml_2d`` -- complex-symmetric Helmholtz
  with a PML, examples/HelmholtzPML3D.cpp:14-149 and
  examples/HelmholtzPML2D.cpp (``sInv``/``PML`` stretching, the
  ``(xTempL+xTempM)/(2 h^2)`` face averages), with a heterogeneous velocity
  ``c(x)`` entering the mass term as ``-(omega/c)^2 s1 s2 s3``.

All matrices are returned in CSR form, rows in natural order
``x + y*n1 + z*n1*n2``, columns sorted within each row and duplicates summed,
which is what ``DistSparseMatrix::StopAssembly`` produces
(core/dist_sparse_matrix/impl.hpp:209-257).  Data is synthetic and seeded;
there is no dataset involved.
"""
from __future__ import annotations

import math

import numpy as np


class CSR:
    """Sorted, duplicate-free CSR matrix (both triangles stored)."""

    def __init__(self, n, rowptr, colind, values):
        self.n = int(n)
        self.rowptr = np.ascontiguousarray(rowptr, np.int64)
        self.colind = np.ascontiguousarray(colind, np.int32)
        self.values = np.ascontiguousarray(values)

    @property
    def nnz(self):
        return int(self.rowptr[-1])

    @property
    def is_complex(self):
        return np.iscomplexobj(self.values)

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.values, self.colind, self.rowptr), shape=(self.n, self.n))

    def matvec(self, x):
        return self.to_scipy() @ x


def from_triplets(n, rows, cols, vals):
    """Sort by (row, col) and sum duplicates, as StopAssembly does."""
    rows = np.asarray(rows, np.int64)
    cols = np.asarray(cols, np.int64)
    key = rows * n + cols
    order = np.argsort(key, kind="stable")
    key = key[order]
    vals = np.asarray(vals)[order]
    uniq, start = np.unique(key, return_index=True)
    summed = np.add.reduceat(vals, start) if len(vals) else vals
    r = uniq // n
    c = uniq % n
    rowptr = np.zeros(n + 1, np.int64)
    np.add.at(rowptr, r + 1, 1)
    rowptr = np.cumsum(rowptr)
    return CSR(n, rowptr, c.astype(np.int32), summed)


def _stencil(dims, center, offdiag):
    """Assemble a (2d+1)-point stencil.  ``center`` has one value per grid
    point; ``offdiag[axis] = (minus, plus)`` are per-point couplings to the
    neighbour at -1 / +1 along that axis (only where it exists)."""
    n = int(np.prod(dims))
    idx = np.arange(n, dtype=np.int64)
    coords = []
    rem = idx.copy()
    for d in dims:
        coords.append(rem % d)
        rem //= d
    rows = [idx]
    cols = [idx]
    vals = [np.asarray(center).reshape(-1)]
    stride = 1
    for axis, d in enumerate(dims):
        c = coords[axis]
        mi, pl = offdiag[axis]
        m = c != 0
        rows.append(idx[m]); cols.append(idx[m] - stride); vals.append(np.asarray(mi).reshape(-1)[m])
        p = c != d - 1
        rows.append(idx[p]); cols.append(idx[p] + stride); vals.append(np.asarray(pl).reshape(-1)[p])
        stride *= d
    return from_triplets(n, np.concatenate(rows), np.concatenate(cols), np.concatenate(vals))


def laplacian_3d(n1, n2, n3, diag=6.0):
    """tests/Solve.cpp:59-82 with a configurable diagonal (6 + shift)."""
    n = n1 * n2 * n3
    one = -np.ones(n)
    return _stencil((n1, n2, n3), np.full(n, float(diag)), [(one, one)] * 3)


def laplacian_2d(n1, n2, diag=4.0):
    n = n1 * n2
    one = -np.ones(n)
    return _stencil((n1, n2), np.full(n, float(diag)), [(one, one)] * 2)


def _pml(x, w, p, sigma, k):
    """PML() of examples/HelmholtzPML3D.cpp:14-24."""
    return 1.0 + 1j * (sigma / w) * (x / w) ** p / k


def _s_inv(j, n, b, h, p, sigma, k):
    """sInv() of examples/HelmholtzPML3D.cpp:26-35, vectorised over j."""
    j = np.asarray(j, np.float64)
    out = np.ones(j.shape, np.complex128)
    lo = j < b - 1
    hi = j > n - b
    out[lo] = _pml((b - 1 - j[lo]) * h, b * h, p, sigma, k)
    out[hi] = _pml((j[hi] - (n - b)) * h, b * h, p, sigma, k)
    return out


def smooth_velocity(dims, seed, amplitude=0.3, corr_cells=None):
    """c = 1 + amplitude * (Gaussian-smoothed N(0,1) field, scaled to max |.| = 1)."""
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(seed)
    f = rng.standard_normal(tuple(reversed(dims)))   # z, y, x so that ravel() is natural order
    if corr_cells is None:
        corr_cells = max(1.0, min(dims) / 10.0)
    f = gaussian_filter(f, sigma=corr_cells, mode="wrap")
    f /= np.max(np.abs(f))
    return (1.0 + amplitude * f).reshape(-1)


def omega_for_ppw(n, c_min, ppw=10.0, L=1.0):
    """Angular frequency giving ``ppw`` grid points per wavelength at speed c_min."""
    h = L / (n + 1)
    return 2.0 * math.pi * c_min / (ppw * h)


def helmholtz_pml_3d(n1, n2, n3, omega, velocity=None, b=5, sigma=1.5, p=2.0, L=(1.0, 1.0, 1.0)):
    """Complex-symmetric 3D Helmholtz operator, examples/HelmholtzPML3D.cpp:73-149."""
    n = n1 * n2 * n3
    k = omega / (2 * math.pi)
    hs = [L[0] / (n1 + 1), L[1] / (n2 + 1), L[2] / (n3 + 1)]
    idx = np.arange(n, dtype=np.int64)
    x = idx % n1
    y = (idx // n1) % n2
    z = idx // (n1 * n2)
    dims = (n1, n2, n3)
    co = (x, y, z)
    s = []
    for a in range(3):
        s.append((_s_inv(co[a] - 1, dims[a], b, hs[a], p, sigma, k),
                  _s_inv(co[a], dims[a], b, hs[a], p, sigma, k),
                  _s_inv(co[a] + 1, dims[a], b, hs[a], p, sigma, k)))
    terms = []
    for a in range(3):
        others = [s[o][1] for o in range(3) if o != a]
        top = others[0] * others[1]
        tl, tm, tr = top / s[a][0], top / s[a][1], top / s[a][2]
        h2 = hs[a] ** 2
        terms.append(((tl + tm) / (2 * h2), (tm + tr) / (2 * h2)))
    vel = np.ones(n) if velocity is None else np.asarray(velocity).reshape(-1)
    main = sum(t[0] + t[1] for t in terms) - (omega / vel) ** 2 * s[0][1] * s[1][1] * s[2][1]
    return _stencil(dims, main, [(-t[0], -t[1]) for t in terms])


def helmholtz_pml_2d(n1, n2, omega, velocity=None, b=5, sigma=1.5, p=2.0, L=(1.0, 1.0)):
    """Complex-symmetric 2D Helmholtz operator in the form of examples/HelmholtzPML2D.cpp."""
    n = n1 * n2
    k = omega / (2 * math.pi)
    hs = [L[0] / (n1 + 1), L[1] / (n2 + 1)]
    idx = np.arange(n, dtype=np.int64)
    co = (idx % n1, idx // n1)
    dims = (n1, n2)
    s = []
    for a in range(2):
        s.append((_s_inv(co[a] - 1, dims[a], b, hs[a], p, sigma, k),
                  _s_inv(co[a], dims[a], b, hs[a], p, sigma, k),
                  _s_inv(co[a] + 1, dims[a], b, hs[a], p, sigma, k)))
    terms = []
    for a in range(2):
        top = s[1 - a][1]
        tl, tm, tr = top / s[a][0], top / s[a][1], top / s[a][2]
        h2 = hs[a] ** 2
        terms.append(((tl + tm) / (2 * h2), (tm + tr) / (2 * h2)))
    vel = np.ones(n) if velocity is None else np.asarray(velocity).reshape(-1)
    main = sum(t[0] + t[1] for t in terms) - (omega / vel) ** 2 * s[0][1] * s[1][1]
    return _stencil(dims, main, [(-t[0], -t[1]) for t in terms])


def helmholtz_workload_3d(n, seed=0, ppw=10.0, b=5, sigma=1.5, p=2.0):
    """The 100^3-style workload: smoothed random velocity, omega at ``ppw`` points
    per wavelength at the slowest speed, quadratic 5-cell PML."""
    c = smooth_velocity((n, n, n), seed)
    omega = omega_for_ppw(n, float(c.min()), ppw)
    return helmholtz_pml_3d(n, n, n, omega, c, b=b, sigma=sigma, p=p), omega, c


def helmholtz_workload_2d(n, seed=0, ppw=10.0, b=5, sigma=1.5, p=2.0):
    c = smooth_velocity((n, n), seed)
    omega = omega_for_ppw(n, float(c.min()), ppw)
    return helmholtz_pml_2d(n, n, omega, c, b=b, sigma=sigma, p=p), omega, c


def helmholtz_slowness_parts(n1, n2, n3, omega, b=5, sigma=1.5, p=2.0):
    """The 3D Helmholtz-PML operator as an affine function of the per-cell
    squared slowness m = 1 / c^2: A(m).values = base + (diag_pos -> coef * m),
    with coef = -omega^2 s1 s2 s3 (the PML-stretched mass term of
    examples/HelmholtzPML3D.cpp).  Returns (pattern CSR holding the base
    values, diag_pos: CSR index of each diagonal entry, coef)."""
    n = n1 * n2 * n3
    base = helmholtz_pml_3d(n1, n2, n3, omega, np.full(n, np.inf), b=b, sigma=sigma, p=p)
    unit = helmholtz_pml_3d(n1, n2, n3, omega, np.ones(n), b=b, sigma=sigma, p=p)
    rows = np.repeat(np.arange(n), np.diff(base.rowptr))
    diag_pos = np.nonzero(base.colind == rows)[0]
    assert len(diag_pos) == n
    coef = unit.values[diag_pos] - base.values[diag_pos]
    return base, diag_pos, coef


def random_rhs(n, nrhs, seed=0, complex_=False):
    rng = np.random.default_rng(seed)
    if complex_:
        return np.asfortranarray(rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs)))
    return np.asfortranarray(rng.standard_normal((n, nrhs)))
