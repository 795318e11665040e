"""clique_b200 -- B200-native multifrontal LDL^T (Clique's numeric hot path).

Python mirror of the reference's ``cliq::`` API for a single process, built on
the C ABI in include/cliqgpu.h (``libcliqgpu.so``, hand-written sm_100a CUDA).
Names and argument meaning follow the reference:

* ``NaturalNestedDissection(nx, ny, nz, A, cutoff)`` -> ``(map, sepTree, info)``
  (include/clique/symbolic/natural_nested_dissection.hpp:17-26)
* ``DistSymmFrontTree(A, map, sepTree, info, conjugate)``
  (include/clique/numeric/dist_symm_front_tree/decl.hpp:216-221)
* ``LDL(info, L, frontType)`` (include/clique/numeric/ldl.hpp:23-26)
* ``Solve(info, L, X)`` on a ``DistNodalMultiVec`` (include/clique/numeric/solve.hpp:17-20)
* ``DistNodalMultiVec(inverseMap, info, X)`` / ``.Pull`` / ``.Push``
  (include/clique/numeric/dist_nodal_multi_vec/decl.hpp:26-39)
* ``Multiply(alpha, A, X, beta, Y)`` (include/clique/numeric/multiply.hpp:18-21)

Extensions with no reference counterpart: the FP32 factor precision
(``precision="single"`` on a double-valued matrix) and ``RefinedSolve``
(mixed-precision iterative refinement with FP64 residuals).

Errors: ``LogicError`` (a ValueError) for what the reference reports with
``El::LogicError``; ``CliqueError`` (a RuntimeError) for runtime failures.
There is no CPU fallback: without the built library every numeric call raises.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from ._capi import CliqueError, LogicError, check
from .operators import CSR, from_triplets

__all__ = [
    "CSR", "DistSparseMatrix", "DistMap", "DistSeparatorTree", "DistSymmInfo", "SymmNodeInfo",
    "NaturalNestedDissection", "NestedDissection", "DistSymmFrontTree", "LDL", "ChangeFrontType", "Solve",
    "DistNodalMultiVec", "DistNodalMatrix", "Multiply", "RefinedSolve", "SymmetricSolve", "HermitianSolve",
    "SymmFrontType", "Unfactored", "FrontsAre1d", "BlockFactorization", "SelInvFactorization",
    "PivotedFactorization", "ConvertTo2d", "ConvertTo1d", "AppendSelInv", "RemoveSelInv", "LogicError",
    "CliqueError",
]


class SymmFrontType:
    """The reference's SymmFrontType enum (dist_symm_front_tree/decl.hpp:17-26), same values."""
    SYMM_1D, SYMM_2D, LDL_1D, LDL_2D = 0, 1, 2, 3
    LDL_SELINV_1D, LDL_SELINV_2D, LDL_INTRAPIV_1D, LDL_INTRAPIV_2D = 4, 5, 6, 7
    LDL_INTRAPIV_SELINV_1D, LDL_INTRAPIV_SELINV_2D, BLOCK_LDL_1D, BLOCK_LDL_2D = 8, 9, 10, 11
    BLOCK_LDL_INTRAPIV_1D, BLOCK_LDL_INTRAPIV_2D = 12, 13
    # Every factored type is provided.  The selective-inversion forms invert
    # no local front at one process (change_front_type.hpp:86-98 inverts
    # distributed nodes 1 ..), so they factor and solve as their LDL /
    # pivoted LDL base types; the block-LDL forms keep inv(A11) and A21 in
    # every front (ldl/local.hpp:30-33, ldl/local_front_block.hpp:27-71); the
    # INTRAPIV forms pivot within each front (ldl/local.hpp:31-33,104-111)
    PIVOTED = (LDL_INTRAPIV_1D, LDL_INTRAPIV_2D, LDL_INTRAPIV_SELINV_1D, LDL_INTRAPIV_SELINV_2D,
               BLOCK_LDL_INTRAPIV_1D, BLOCK_LDL_INTRAPIV_2D)
    SUPPORTED = (LDL_1D, LDL_2D, LDL_SELINV_1D, LDL_SELINV_2D, BLOCK_LDL_1D, BLOCK_LDL_2D) + PIVOTED
    BLOCK = (BLOCK_LDL_1D, BLOCK_LDL_2D, BLOCK_LDL_INTRAPIV_1D, BLOCK_LDL_INTRAPIV_2D)


# front-type helpers (dist_symm_front_tree/decl.hpp:27-165): the 1D / 2D
# members of each family are adjacent (1D even, 2D odd)
def Unfactored(t):
    return t in (SymmFrontType.SYMM_1D, SymmFrontType.SYMM_2D)


def FrontsAre1d(t):
    return t % 2 == 0


def BlockFactorization(t):
    return t in SymmFrontType.BLOCK


def SelInvFactorization(t):
    T = SymmFrontType
    return t in (T.LDL_SELINV_1D, T.LDL_SELINV_2D, T.LDL_INTRAPIV_SELINV_1D, T.LDL_INTRAPIV_SELINV_2D)


def PivotedFactorization(t):
    return t in SymmFrontType.PIVOTED


def ConvertTo2d(t):
    if not 0 <= t <= 13:
        raise LogicError(_capi.CLIQ_ERR_ARG, "Invalid front type")
    return t | 1


def ConvertTo1d(t):
    if not 0 <= t <= 13:
        raise LogicError(_capi.CLIQ_ERR_ARG, "Invalid front type")
    return t & ~1


def AppendSelInv(t):
    T = SymmFrontType
    m = {T.LDL_1D: T.LDL_SELINV_1D, T.LDL_2D: T.LDL_SELINV_2D,
         T.LDL_INTRAPIV_1D: T.LDL_INTRAPIV_SELINV_1D, T.LDL_INTRAPIV_2D: T.LDL_INTRAPIV_SELINV_2D}
    if t not in m:
        raise LogicError(_capi.CLIQ_ERR_ARG, "Sel-inv does not make sense for this type")
    return m[t]


def RemoveSelInv(t):
    T = SymmFrontType
    m = {T.LDL_SELINV_1D: T.LDL_1D, T.LDL_SELINV_2D: T.LDL_2D,
         T.LDL_INTRAPIV_SELINV_1D: T.LDL_INTRAPIV_1D, T.LDL_INTRAPIV_SELINV_2D: T.LDL_INTRAPIV_2D}
    if t not in m:
        raise LogicError(_capi.CLIQ_ERR_ARG, "This type did not involve selective inversion")
    return m[t]


# ---------------------------------------------------------------------------
# host containers
# ---------------------------------------------------------------------------
class DistSparseMatrix:
    """Single-process sparse matrix with the reference's assembly semantics:
    Update() appends (i, j, value); StopAssembly() sorts and sums duplicates
    (core/dist_sparse_matrix/impl.hpp:209-257)."""

    def __init__(self, n, dtype=np.float64):
        self.n = int(n)
        self.dtype = np.dtype(dtype)
        self._rows, self._cols, self._vals = [], [], []
        self.csr = None

    @classmethod
    def from_csr(cls, csr: CSR):
        A = cls(csr.n, csr.values.dtype)
        A.csr = csr
        return A

    def StartAssembly(self):
        self._rows, self._cols, self._vals = [], [], []
        self.csr = None

    def Update(self, i, j, value):
        self._rows.append(i); self._cols.append(j); self._vals.append(value)

    def StopAssembly(self):
        self.csr = from_triplets(self.n, np.array(self._rows, np.int64), np.array(self._cols, np.int64),
                                 np.array(self._vals, self.dtype))
        self._rows, self._cols, self._vals = [], [], []

    def Height(self):
        return self.n

    @property
    def is_complex(self):
        return np.iscomplexobj(self.csr.values)


def _as_csr(A):
    if isinstance(A, DistSparseMatrix):
        if A.csr is None:
            raise LogicError(_capi.CLIQ_ERR_STATE, "matrix is still being assembled")
        return A.csr
    return A


class DistMap:
    """Natural -> nested-dissection index map (DistMap at P=1)."""

    def __init__(self, array):
        self.array = np.ascontiguousarray(array, np.int32)

    def FormInverse(self):
        inv = np.empty_like(self.array)
        inv[self.array] = np.arange(len(self.array), dtype=np.int32)
        return DistMap(inv)

    def __len__(self):
        return len(self.array)


class SymmNodeInfo:
    """One entry of DistSymmInfo::localNodes (symbolic/dist_symm_info.hpp:17-36)."""

    def __init__(self, h, s):
        lib = _capi.load()
        out = (C.c_int32 * 10)()
        check(lib.cliq_symbolic_node(h, s, out), "cliq_symbolic_node")
        (self.size, self.off, self.myOff, self.parent, l, r, onl, _nl, _no, self.sepParent) = list(out)
        self.children = [l, r] if l >= 0 else []
        self.onLeft = bool(onl)
        self._h, self._s = h, s

    def _arr(self, which):
        lib = _capi.load()
        n = C.c_int64()
        check(lib.cliq_symbolic_node_array(self._h, self._s, which, None, C.byref(n)))
        out = np.zeros(n.value, np.int32)
        if n.value:
            check(lib.cliq_symbolic_node_array(self._h, self._s, which, out.ctypes.data_as(C.c_void_p), C.byref(n)))
        return out

    lowerStruct = property(lambda self: self._arr(0))
    origLowerStruct = property(lambda self: self._arr(1))
    origLowerRelInds = property(lambda self: self._arr(2))
    leftRelInds = property(lambda self: self._arr(3))
    rightRelInds = property(lambda self: self._arr(4))


class DistSymmInfo:
    """Symbolic analysis result (owns the host symbolic handle)."""

    def __init__(self, handle, n):
        self._h = handle
        self.n = n
        lib = _capi.load()
        self._view = _capi.SymmInfo()
        check(lib.cliq_symbolic_info(handle, C.byref(self._view)))
        self.num_nodes = self._view.num_nodes
        self._nodes = None

    @property
    def localNodes(self):
        if self._nodes is None:
            self._nodes = [SymmNodeInfo(self._h, s) for s in range(self.num_nodes)]
        return self._nodes

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                _capi.load().cliq_symbolic_destroy(h)
            except Exception:
                pass
            self._h = None


class DistSeparatorTree:
    """Separator / leaf index sets (symbolic/dist_separator_tree.hpp), natural indices."""

    def __init__(self, info: DistSymmInfo):
        self._info = info

    def inds(self, s):
        return self._info.localNodes[s]._arr(5)


def NaturalNestedDissection(nx, ny, nz, A, cutoff=128):
    """Returns (map, sepTree, info) like the reference's output parameters."""
    csr = _as_csr(A)
    lib = _capi.load()
    h = C.c_void_p()
    check(lib.cliq_natural_nested_dissection(nx, ny, nz, csr.n, csr.rowptr.ctypes.data_as(C.c_void_p),
                                             csr.colind.ctypes.data_as(C.c_void_p), cutoff, C.byref(h)),
          "NaturalNestedDissection")
    info = DistSymmInfo(h.value, csr.n)
    m = np.zeros(csr.n, np.int32)
    check(lib.cliq_symbolic_map(h.value, m.ctypes.data_as(C.c_void_p), None))
    return DistMap(m), DistSeparatorTree(info), info


def NestedDissection(A, cutoff=128, numSeqSeps=1):
    """Nested dissection of A's graph (any structurally symmetric pattern),
    nested_dissection.hpp:35-44,115-230 at one process; returns (map,
    sepTree, info).  The separators come from the library's own bisection
    (breadth-first level structures), not METIS."""
    csr = _as_csr(A)
    lib = _capi.load()
    h = C.c_void_p()
    check(lib.cliq_nested_dissection(csr.n, csr.rowptr.ctypes.data_as(C.c_void_p), csr.colind.ctypes.data_as(C.c_void_p),
                                     cutoff, numSeqSeps, C.byref(h)), "NestedDissection")
    info = DistSymmInfo(h.value, csr.n)
    m = np.zeros(csr.n, np.int32)
    check(lib.cliq_symbolic_map(h.value, m.ctypes.data_as(C.c_void_p), None))
    return DistMap(m), DistSeparatorTree(info), info


# ---------------------------------------------------------------------------
# device front tree
# ---------------------------------------------------------------------------
def _is_torch_cuda(x):
    try:
        import torch
        return isinstance(x, torch.Tensor) and x.is_cuda
    except ImportError:
        return False


class DistSymmFrontTree:
    """Device-resident front tree: factor arena, pivots and workspaces in HBM.

    ``precision``: "double" (plain) or "single" (mixed: FP32 fronts, FP64
    pivots; use ``RefinedSolve`` for FP64 accuracy).  ``keep_matrix`` keeps
    A in FP64 on the device for ``Multiply`` / ``RefinedSolve``.
    """

    def __init__(self, A, map: DistMap, sepTree: DistSeparatorTree, info: DistSymmInfo, conjugate=False,
                 precision="double", keep_matrix=True, stream=None):
        csr = _as_csr(A)
        self.info = info
        self.n = csr.n
        self.is_complex = np.iscomplexobj(csr.values)
        self.isHermitian = bool(conjugate)
        self.frontType = SymmFrontType.SYMM_2D
        self.precision = precision
        opt = _capi.Options(_capi.CLIQ_COMPLEX if self.is_complex else _capi.CLIQ_REAL,
                            _capi.CLIQ_FP32 if precision in ("single", "fp32", np.float32) else _capi.CLIQ_FP64,
                            int(bool(conjugate)), 0, int(bool(keep_matrix)))
        lib = _capi.load()
        h = C.c_void_p()
        self._map = np.ascontiguousarray(map.array, np.int32)
        # None: a private stream; 0 (torch's default stream): the legacy
        # default stream, passed as its CUDA handle 0x1 (a null handle would
        # ask for a private stream)
        if stream is not None and int(stream) == 0:
            stream = 1
        check(lib.cliqgpu_plan_create(C.byref(info._view), csr.n, self._map.ctypes.data_as(C.c_void_p),
                                      csr.rowptr.ctypes.data_as(C.c_void_p), csr.colind.ctypes.data_as(C.c_void_p),
                                      C.byref(opt), C.c_void_p(stream), C.byref(h)), "DistSymmFrontTree")
        self._h = h.value
        self._csr = csr
        # for RefinedSolve(fallback=True): the analysis, options and current
        # values an FP64 copy of this tree is built from
        self._twin_args = (map, sepTree, info, conjugate, keep_matrix, stream)
        self._values_version = 0
        self._fp64_twin = None
        self.last_fallback = False
        self.Initialize(csr.values)

    def Initialize(self, values):
        """(Re)assemble the fronts from A's values (same pattern)."""
        lib = _capi.load()
        self._values = values
        self._values_version = getattr(self, "_values_version", 0) + 1
        if _is_torch_cuda(values):
            values = values.resolve_conj().contiguous()
            check(lib.cliqgpu_assemble(self._h, C.c_void_p(values.data_ptr()), 1), "assemble")
        else:
            v = np.ascontiguousarray(values, np.complex128 if self.is_complex else np.float64)
            check(lib.cliqgpu_assemble(self._h, v.ctypes.data_as(C.c_void_p), 0), "assemble")
        self.frontType = SymmFrontType.SYMM_2D

    def _fp64_tree(self):
        """The same matrix, current values, factored with FP64 fronts (built
        on first use and kept until the values change)."""
        if self._fp64_twin is not None and self._fp64_twin[0] == self._values_version:
            return self._fp64_twin[1]
        self._fp64_twin = None
        map_, sep, info, conjugate, keep, stream = self._twin_args
        L64 = DistSymmFrontTree(self._csr, map_, sep, info, conjugate, precision="double", keep_matrix=keep, stream=stream)
        L64.Initialize(self._values)
        pivoted = self.frontType in SymmFrontType.PIVOTED
        LDL(info, L64, SymmFrontType.LDL_INTRAPIV_2D if pivoted else SymmFrontType.LDL_2D)
        self._fp64_twin = (self._values_version, L64)
        return L64

    def query(self, key):
        v = C.c_double()
        check(_capi.load().cliqgpu_plan_query(self._h, key, C.byref(v)))
        return v.value

    def FactorizationWork(self):
        return self.query(0)

    def SolveWork(self, numRhs=1):
        return self.query(1) * numRhs

    def last_launches(self):
        return int(self.query(4))

    def total_launches(self):
        return int(self.query(8))

    def set_profiling(self, on=True):
        check(_capi.load().cliqgpu_set_profiling(self._h, int(bool(on))))

    PROFILE_KEYS = ["extend_add_ms", "diag_ms", "panel_ms", "trail_ms", "schur_ms", "trail_flops", "schur_flops",
                    "extend_add_bytes", "trail_launches", "schur_launches", "factor_ms", "pack_ms"]

    def profile(self):
        out = np.zeros(16)
        check(_capi.load().cliqgpu_profile_read(self._h, out.ctypes.data_as(C.c_void_p), 16))
        return dict(zip(self.PROFILE_KEYS, out.tolist()))

    def front(self, s):
        """Host copies of (frontL, diag) of node s, widened to FP64."""
        lib = _capi.load()
        dims = (C.c_int32 * 2)()
        check(lib.cliqgpu_get_front(self._h, s, None, None, dims))
        m, n = dims[0], dims[1]
        dt = np.complex128 if self.is_complex else np.float64
        L = np.zeros((m, n), dt, order="F")
        d = np.zeros(n, dt)
        check(lib.cliqgpu_get_front(self._h, s, L.ctypes.data_as(C.c_void_p), d.ctypes.data_as(C.c_void_p), dims))
        return L, d

    def front_pivots(self, s):
        """(subdiag, piv) of node s after an LDL_INTRAPIV factorization:
        subdiag[k] = D[k+1, k] of the 2x2 block starting at k (0 elsewhere),
        piv[i] = the front's assembled pivot row at pivoted position i."""
        lib = _capi.load()
        dims = (C.c_int32 * 2)()
        check(lib.cliqgpu_get_front(self._h, s, None, None, dims))
        n = dims[1]
        sub = np.zeros(n, np.complex128 if self.is_complex else np.float64)
        piv = np.zeros(n, np.int32)
        check(lib.cliqgpu_get_front_pivots(self._h, s, sub.ctypes.data_as(C.c_void_p), piv.ctypes.data_as(C.c_void_p)))
        return sub, piv

    def synchronize(self):
        check(_capi.load().cliqgpu_synchronize(self._h))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                _capi.load().cliqgpu_plan_destroy(h)
            except Exception:
                pass
            self._h = None


def LDL(info, L: DistSymmFrontTree, frontType=SymmFrontType.LDL_2D):
    """Multifrontal LDL^T in place (ldl.hpp:57-75).  Returns None; raises on a zero pivot."""
    if frontType not in SymmFrontType.SUPPORTED:
        raise LogicError(_capi.CLIQ_ERR_ARG, "the symmetric (unfactored) front types are no factorization")
    if L.frontType not in (SymmFrontType.SYMM_1D, SymmFrontType.SYMM_2D):
        raise LogicError(_capi.CLIQ_ERR_STATE, "Matrix is already factored")
    zp = C.c_int64(-1)
    if frontType in SymmFrontType.PIVOTED:
        st = _capi.load().cliqgpu_factor_intrapiv(L._h, C.byref(zp))
    else:
        st = _capi.load().cliqgpu_factor(L._h, C.byref(zp))
    L.zero_pivot = zp.value
    L.frontType = frontType
    check(st, "LDL")
    if frontType in SymmFrontType.BLOCK:
        check(_capi.load().cliqgpu_block_ldl(L._h), "LDL (block form)")


def ChangeFrontType(L, frontType):
    """change_front_type.hpp:27-107 at one process: 1D <-> 2D and appending
    selective inversion (which the reference applies to distributed fronts
    1 .. only) leave the device fronts as they are and relabel the tree;
    other changes are a LogicError, as in the reference."""
    if frontType == L.frontType:
        return
    old = L.frontType
    if frontType == ConvertTo2d(old) or frontType == ConvertTo1d(old):
        L.frontType = frontType
        return
    if SelInvFactorization(frontType):
        try:
            ok = ConvertTo2d(frontType) == ConvertTo2d(AppendSelInv(old))
        except LogicError:
            ok = False
        if ok:
            L.frontType = frontType
            return
    raise LogicError(_capi.CLIQ_ERR_ARG, "Unavailable front type change")


class DistNodalMultiVec:
    """Right-hand sides in ND (nodal) order; ``localNodes[s]`` is rows
    [off_s, off_s + size_s) of ``self.X``."""

    def __init__(self, inverseMap=None, info=None, X=None):
        self.X = None
        self._info = info
        if X is not None:
            self.Pull(inverseMap, info, X)

    @staticmethod
    def _device_map(inverseMap, device):
        import torch
        cached = getattr(inverseMap, "_dev", None)
        if cached is None or cached.device != device:
            cached = torch.as_tensor(inverseMap.array, dtype=torch.int32).to(device)
            inverseMap._dev = cached
        return cached

    @staticmethod
    def _nodal_call(fn, inverseMap, src, dst):
        """One pull / push kernel on the current stream (FP64 or complex128
        device tensors, column-major n x nrhs)."""
        import torch
        if src.dtype not in (torch.float64, torch.complex128) or dst.dtype != src.dtype:
            raise LogicError(_capi.CLIQ_ERR_ARG, "device multivectors must be float64 or complex128")
        if dst.is_conj():
            raise LogicError(_capi.CLIQ_ERR_ARG, "the destination must not be a lazily conjugated view")
        src = src.resolve_conj()
        s2 = src if src.dim() == 2 else src.reshape(-1, 1)
        d2 = dst if dst.dim() == 2 else dst.reshape(-1, 1)
        if s2.stride(0) != 1 or d2.stride(0) != 1:
            raise LogicError(_capi.CLIQ_ERR_ARG, "device multivectors must be column-major")
        n, k = s2.shape
        lds = s2.stride(1) if k > 1 else n
        ldd = d2.stride(1) if k > 1 else n
        perm = DistNodalMultiVec._device_map(inverseMap, src.device)
        field = _capi.CLIQ_COMPLEX if src.is_complex() else _capi.CLIQ_REAL
        stream = torch.cuda.current_stream(src.device).cuda_stream
        check(fn(field, n, C.c_void_p(perm.data_ptr()), C.c_void_p(s2.data_ptr()), lds, C.c_void_p(d2.data_ptr()), ldd, k,
                 C.c_void_p(stream)), "DistNodalMultiVec")

    def Pull(self, inverseMap, info, X):
        self._info = info
        if _is_torch_cuda(X):
            import torch
            Xn = torch.empty_like(X if X.dim() == 2 else X.reshape(-1, 1)).t().contiguous().t() if X.dim() == 2 \
                else torch.empty_like(X)
            self._nodal_call(_capi.load().cliqgpu_nodal_pull, inverseMap, X, Xn)
            self.X = Xn
        else:
            X = np.asarray(X)
            self.X = np.asfortranarray(X[inverseMap.array])

    def Push(self, inverseMap, info, X):
        if _is_torch_cuda(X):
            self._nodal_call(_capi.load().cliqgpu_nodal_push, inverseMap, self.X, X)
        else:
            X[inverseMap.array] = self.X
        return X

    @property
    def localNodes(self):
        return [self.X[n.off:n.off + n.size] for n in self._info.localNodes]

    def Height(self):
        return self.X.shape[0]

    def Width(self):
        return 1 if self.X.ndim == 1 else self.X.shape[1]


# DistNodalMatrix (dist_nodal_matrix/decl.hpp:19-50): at one process the
# reference's [MC,MR] nodal matrix holds the same per-node blocks as the
# nodal multivector, and Solve takes either (solve.hpp:17-24)
DistNodalMatrix = DistNodalMultiVec


def _solve_array(L, X, nodal):
    lib = _capi.load()
    if _is_torch_cuda(X):
        if X.is_conj():
            raise LogicError(_capi.CLIQ_ERR_ARG, "device right-hand sides must not be lazily conjugated views")
        assert X.is_contiguous() or X.t().is_contiguous()
        Xc = X if X.dim() == 2 else X.reshape(-1, 1)
        # column-major expected: a (n, k) tensor stored with stride (1, n)
        if Xc.stride(0) != 1:
            raise LogicError(_capi.CLIQ_ERR_ARG, "device right-hand sides must be column-major (use X.t().contiguous().t())")
        ld = Xc.stride(1) if Xc.shape[1] > 1 else Xc.shape[0]
        check(lib.cliqgpu_solve(L._h, C.c_void_p(Xc.data_ptr()), ld, Xc.shape[1], 1, int(nodal)), "Solve")
        return X
    X2 = X.reshape(X.shape[0], -1, order="F")
    if not X2.flags.f_contiguous:
        raise LogicError(_capi.CLIQ_ERR_ARG, "host right-hand sides must be Fortran-ordered")
    check(lib.cliqgpu_solve(L._h, X2.ctypes.data_as(C.c_void_p), X2.shape[0], X2.shape[1], 0, int(nodal)), "Solve")
    return X


def Solve(info, L: DistSymmFrontTree, X):
    """Forward, diagonal and backward solves (solve.hpp:41-65), in place.
    X: a DistNodalMultiVec (ND order), or a natural-order array (Pull/Push done on the device)."""
    if L.frontType not in SymmFrontType.SUPPORTED:
        raise LogicError(_capi.CLIQ_ERR_STATE, "Invalid front type for solve (factor with LDL first)")
    if isinstance(X, DistNodalMultiVec):
        _solve_array(L, X.X, nodal=True)
        return X
    return _solve_array(L, X, nodal=False)


def RefinedSolve(L: DistSymmFrontTree, B, tol=1e-10, max_iter=20, X=None, fallback=False):
    """X = A^{-1} B by iterative refinement over the stored factors (FP64
    residuals and updates).  Returns (X, iterations, relative residual).
    For host right-hand sides an output array X (Fortran-ordered, B's shape
    and dtype, e.g. a view of pinned memory) may be passed and is filled.
    fallback=True on an FP32 tree: if the refinement does not reach tol in
    max_iter steps (unpivoted growth the FP32 factors cannot absorb), the
    matrix is factored again with FP64 fronts -- once per set of values; the
    FP64 tree is kept with L -- and refined from there; L.last_fallback says
    whether that happened, the iterations count both attempts."""
    lib = _capi.load()
    it = C.c_int32()
    rr = C.c_double()
    if _is_torch_cuda(B):
        import torch
        B = B.resolve_conj()
        Bc = B if B.dim() == 2 else B.reshape(-1, 1)
        X = torch.zeros_like(Bc).t().contiguous().t()
        Bc = Bc.t().contiguous().t()
        st = lib.cliqgpu_refine(L._h, C.c_void_p(Bc.data_ptr()), C.c_void_p(X.data_ptr()), Bc.shape[0], Bc.shape[1], 1,
                                tol, max_iter, C.byref(it), C.byref(rr))
    else:
        B2 = np.asfortranarray(np.asarray(B).reshape(B.shape[0], -1), np.complex128 if L.is_complex else np.float64)
        if X is None:
            Xo = np.zeros_like(B2, order="F")
        else:
            Xo = X.reshape(B2.shape[0], -1, order="A")
            if Xo.dtype != B2.dtype or Xo.shape != B2.shape or not Xo.flags.f_contiguous or not Xo.flags.writeable:
                raise LogicError(_capi.CLIQ_ERR_ARG, "X must be a writable Fortran-ordered array of B's shape and dtype")
        st = lib.cliqgpu_refine(L._h, B2.ctypes.data_as(C.c_void_p), Xo.ctypes.data_as(C.c_void_p), B2.shape[0],
                                B2.shape[1], 0, tol, max_iter, C.byref(it), C.byref(rr))
        X = X if X is not None else Xo.reshape(np.asarray(B).shape)
    if st not in (_capi.CLIQ_OK, _capi.CLIQ_ERR_NOCONV):
        check(st, "RefinedSolve")
    L.last_fallback = False
    if st == _capi.CLIQ_ERR_NOCONV and fallback and L.precision not in ("double", "fp64", np.float64):
        # the FP32 factors did not bring the residual to tol (pivot growth
        # beyond what refinement absorbs): solve with FP64 fronts instead
        X64, it64, rr64 = RefinedSolve(L._fp64_tree(), B, tol, max_iter, X=X)
        L.last_fallback = True
        return X64, it.value + it64, rr64
    return X, it.value, rr.value


def Multiply(alpha, L: DistSymmFrontTree, X, beta, Y):
    """Y := alpha A X + beta Y with the FP64 copy of A held by the front tree
    (device arrays, column-major)."""
    lib = _capi.load()
    dt = np.complex128 if L.is_complex else np.float64
    a = np.array([alpha], dt).view(np.float64)
    b = np.array([beta], dt).view(np.float64)
    if Y.is_conj():
        raise LogicError(_capi.CLIQ_ERR_ARG, "Y must not be a lazily conjugated view")
    X = X.resolve_conj()
    Xc = X if X.dim() == 2 else X.reshape(-1, 1)
    Yc = Y if Y.dim() == 2 else Y.reshape(-1, 1)
    check(lib.cliqgpu_multiply(L._h, a.ctypes.data_as(C.c_void_p), C.c_void_p(Xc.data_ptr()), b.ctypes.data_as(C.c_void_p),
                               C.c_void_p(Yc.data_ptr()), Yc.shape[0], Yc.shape[1]), "Multiply")
    return Y


def SymmetricSolve(A, X, nx=None, ny=None, nz=None, conjugate=False, cutoff=128, precision="double", tol=1e-10,
                   max_iter=20, frontType=SymmFrontType.LDL_INTRAPIV_1D, numSeqSeps=1):
    """Black-box solve (solve.hpp:95-116): nested dissection of A's graph, as
    the reference orders it (or natural nested dissection when the grid
    dimensions nx, ny, nz are given), intra-front pivoted fronts as in the
    reference (LDL_2D etc. on request).  Returns the solution (natural order)."""
    if nx is None or ny is None or nz is None:
        map_, sepTree, info = NestedDissection(A, cutoff, numSeqSeps)
    else:
        map_, sepTree, info = NaturalNestedDissection(nx, ny, nz, A, cutoff)
    L = DistSymmFrontTree(A, map_, sepTree, info, conjugate, precision=precision, keep_matrix=True)
    LDL(info, L, frontType)
    if precision == "double":
        Y = np.array(X, copy=True, order="F")
        return Solve(info, L, Y)
    Y, _, _ = RefinedSolve(L, X, tol, max_iter)
    return Y


def HermitianSolve(A, X, nx=None, ny=None, nz=None, cutoff=128, precision="double", tol=1e-10, max_iter=20,
                   frontType=SymmFrontType.LDL_INTRAPIV_1D, numSeqSeps=1):
    """SymmetricSolve with conjugate=True (LDL^H of a Hermitian A), solve.hpp:132-140."""
    return SymmetricSolve(A, X, nx, ny, nz, True, cutoff, precision, tol, max_iter, frontType, numSeqSeps)