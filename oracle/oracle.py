"""ctypes wrapper around the C oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline /
reference arm import this module.  The product package ``clique_b200`` never
does.  See ``cliq_oracle.c`` for what is restated from which reference file.
"""
from __future__ import annotations

import ctypes as C
import glob
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "libcliq_oracle.so")
_lib = None

i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_SO):
        build()
    L = C.CDLL(_SO)
    L.orc_natural_nd.restype = C.c_void_p
    L.orc_natural_nd.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int64, i64p, i32p, C.c_int]
    L.orc_symb_free.argtypes = [C.c_void_p]
    L.orc_num_nodes.argtypes = [C.c_void_p]
    L.orc_node_info.argtypes = [C.c_void_p, C.c_int, i32p]
    L.orc_node_array.restype = C.c_int64
    L.orc_node_array.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p]
    L.orc_map.argtypes = [C.c_void_p, i32p, i32p]
    L.orc_set_blas.argtypes = [C.c_char_p, C.c_int]
    L.orc_fronts_create.restype = C.c_void_p
    L.orc_fronts_create.argtypes = [C.c_void_p, i64p, i32p, C.c_void_p, C.c_int, C.c_int]
    L.orc_fronts_free.argtypes = [C.c_void_p]
    L.orc_ldl.restype = C.c_int64
    L.orc_ldl.argtypes = [C.c_void_p, C.c_int]
    L.orc_ldl_ex.restype = C.c_int64
    L.orc_ldl_ex.argtypes = [C.c_void_p, C.c_int, C.c_int]
    L.orc_front_pivots.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    L.orc_front_ldl_intrapiv.restype = C.c_int64
    L.orc_front_ldl_intrapiv.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64,
                                         C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
    L.orc_front_get.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    L.orc_front_dims.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.orc_front_set.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
    L.orc_front_set_factored.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    L.orc_solve.restype = C.c_int64
    L.orc_solve.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
    L.orc_front_ldl.restype = C.c_int64
    L.orc_front_ldl.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int, C.c_int]
    L.orc_multiply.argtypes = [C.c_int, C.c_int64, i64p, i32p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
    L.orc_pull.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int]
    L.orc_push.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int]
    _lib = L
    return L


def openblas_path():
    import numpy
    d = os.path.join(os.path.dirname(os.path.dirname(numpy.__file__)), "numpy.libs")
    c = sorted(glob.glob(os.path.join(d, "libscipy_openblas64_*.so")))
    return c[0] if c else None


def enable_blas(nthreads: int = 0) -> bool:
    """Route the oracle's dense kernels through numpy's bundled OpenBLAS."""
    p = openblas_path()
    if p is None:
        return False
    return lib().orc_set_blas(p.encode(), int(nthreads)) == 0


def disable_blas():
    lib().orc_set_blas(None, 0)


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


class Symbolic:
    """Natural nested dissection + symbolic analysis (P=1)."""

    def __init__(self, nx, ny, nz, rowptr, colind, cutoff=128):
        self.N = nx * ny * nz
        self._rowptr = np.ascontiguousarray(rowptr, np.int64)
        self._colind = np.ascontiguousarray(colind, np.int32)
        h = lib().orc_natural_nd(nx, ny, nz, self.N, self._rowptr, self._colind, cutoff)
        if not h:
            raise ValueError("grid dimensions do not match the matrix")
        self.h = h
        self.num_nodes = lib().orc_num_nodes(h)
        info = np.zeros(10, np.int32)
        names = ["size", "off", "my_off", "parent", "child0", "child1", "on_left", "n_lower", "n_orig", "sep_parent"]
        cols = {k: np.zeros(self.num_nodes, np.int32) for k in names}
        for s in range(self.num_nodes):
            lib().orc_node_info(h, s, info)
            for k, v in zip(names, info):
                cols[k][s] = v
        self.__dict__.update(cols)
        self.map = np.zeros(self.N, np.int32)
        self.inv_map = np.zeros(self.N, np.int32)
        lib().orc_map(h, self.map, self.inv_map)

    def array(self, s, which):
        """which: lower, orig, orig_rel, left_rel, right_rel, inds"""
        w = ["lower", "orig", "orig_rel", "left_rel", "right_rel", "inds"].index(which)
        n = lib().orc_node_array(self.h, s, w, None)
        out = np.zeros(max(n, 0), np.int32)
        if n > 0:
            lib().orc_node_array(self.h, s, w, _ptr(out))
        return out

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_symb_free(self.h)
            self.h = None


def _as_f64_view(x, is_complex):
    x = np.asfortranarray(x, np.complex128 if is_complex else np.float64)
    return x


class Fronts:
    """DistSymmFrontTree restated on the CPU (front assembly, LocalLDL, Solve)."""

    def __init__(self, symb: Symbolic, values, is_complex=False, conjugate=False):
        self.symb = symb
        self.is_complex = bool(is_complex)
        self._vals = np.ascontiguousarray(values, np.complex128 if is_complex else np.float64)
        self.h = lib().orc_fronts_create(symb.h, symb._rowptr, symb._colind, _ptr(self._vals),
                                         int(self.is_complex), int(conjugate))

    def ldl(self, nb=96, block=False, pivot=False):
        """LocalLDL; block=True for the BLOCK_LDL_2D front type (FrontBlockLDL),
        pivot=True for LDL_INTRAPIV_2D (FrontLDLIntraPiv, Bunch-Kaufman), both
        for BLOCK_LDL_INTRAPIV_2D."""
        kind = (3 if pivot else 1) if block else (2 if pivot else 0)
        return int(lib().orc_ldl_ex(self.h, nb, kind))

    def pivots(self, s):
        """Pivoted fronts: (sub, piv) of node s -- D[k+1, k] of each 2x2 block
        starting at k (0 elsewhere) and the assembled row of each pivoted row."""
        _, n = self.dims(s)
        sub = np.zeros(n, np.complex128 if self.is_complex else np.float64)
        piv = np.zeros(n, np.int32)
        lib().orc_front_pivots(self.h, s, _ptr(sub), piv.ctypes.data_as(C.c_void_p))
        return sub, piv

    def dims(self, s):
        m, n = C.c_int(), C.c_int()
        lib().orc_front_dims(self.h, s, C.byref(m), C.byref(n))
        return m.value, n.value

    def front(self, s):
        m, n = self.dims(s)
        dt = np.complex128 if self.is_complex else np.float64
        L = np.zeros((m, n), dt, order="F")
        d = np.zeros(n, dt)
        lib().orc_front_get(self.h, s, _ptr(L), _ptr(d))
        return L, d

    def set_factored(self, s, L, d):
        """Install a front factored elsewhere (unit-lower L, m x n, and D)."""
        dt = np.complex128 if self.is_complex else np.float64
        Lf = np.asfortranarray(L, dt)
        df = np.ascontiguousarray(d, dt)
        assert Lf.shape == self.dims(s) and df.shape == (Lf.shape[1],)
        lib().orc_front_set_factored(self.h, s, _ptr(Lf), _ptr(df))

    def solve_nodal(self, Xn):
        """In-place solve on an ND-ordered (N x nrhs) multivector; returns status."""
        assert Xn.flags.f_contiguous
        nrhs = 1 if Xn.ndim == 1 else Xn.shape[1]
        return int(lib().orc_solve(self.h, _ptr(Xn), nrhs))

    def solve(self, B):
        """Pull -> Solve -> Push on a natural-order right-hand side."""
        B2 = B.reshape(B.shape[0], -1)
        dt = np.complex128 if self.is_complex else np.float64
        Bn = np.asfortranarray(B2, dt)
        Xn = np.zeros_like(Bn, order="F")
        lib().orc_pull(self.symb.h, int(self.is_complex), _ptr(Bn), _ptr(Xn), Bn.shape[1])
        st = self.solve_nodal(Xn)
        X = np.zeros_like(Bn, order="F")
        lib().orc_push(self.symb.h, int(self.is_complex), _ptr(Xn), _ptr(X), Bn.shape[1])
        if st:
            raise ZeroDivisionError(f"singular diagonal at ND index {st - 1}")
        return X.reshape(B.shape)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_fronts_free(self.h)
            self.h = None


def front_ldl(AL, ABR, conjugate=False, nb=96):
    """FrontLDL on one dense front, in place (AL m x n, ABR (m-n)^2, Fortran order)."""
    is_complex = np.iscomplexobj(AL)
    m, n = AL.shape
    assert AL.flags.f_contiguous and ABR.flags.f_contiguous
    return int(lib().orc_front_ldl(int(is_complex), m, n, _ptr(AL), m, _ptr(ABR), max(m - n, 1), int(conjugate), nb))


def front_ldl_intrapiv(AL, ABR, conjugate=False):
    """FrontLDLIntraPiv on one dense front, in place (AL m x n, ABR (m-n)^2,
    Fortran order).  Returns (status, diag, sub, piv); AL's diagonal keeps D."""
    is_complex = np.iscomplexobj(AL)
    m, n = AL.shape
    assert AL.flags.f_contiguous and ABR.flags.f_contiguous
    dt = np.complex128 if is_complex else np.float64
    diag, sub = np.zeros(n, dt), np.zeros(n, dt)
    piv = np.zeros(n, np.int32)
    st = int(lib().orc_front_ldl_intrapiv(int(is_complex), m, n, _ptr(AL), m, _ptr(ABR), max(m - n, 1), _ptr(diag),
                                          _ptr(sub), piv.ctypes.data_as(C.c_void_p), int(conjugate)))
    return st, diag, sub, piv


def multiply(rowptr, colind, vals, alpha, X, beta, Y):
    is_complex = np.iscomplexobj(vals)
    dt = np.complex128 if is_complex else np.float64
    a = np.array([alpha], dt)
    b = np.array([beta], dt)
    assert Y.flags.f_contiguous
    Xf = np.asfortranarray(X, dt)
    nrhs = 1 if Y.ndim == 1 else Y.shape[1]
    lib().orc_multiply(int(is_complex), len(rowptr) - 1, np.ascontiguousarray(rowptr, np.int64),
                       np.ascontiguousarray(colind, np.int32), _ptr(np.ascontiguousarray(vals, dt)),
                       _ptr(a), _ptr(Xf), _ptr(b), _ptr(Y), nrhs)
    return Y
