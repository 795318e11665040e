"""cliqgpu_front_ldl_noalloc: the single-front LDL^T for callers that may not
allocate device memory (a caller with its own memory pool that bans
cudaMalloc/cudaFree while it runs).  Checked through the C ABI against the
allocating cliqgpu_front_ldl and against the oracle's FrontLDL, on two calls
in a row (the fixed scratch array keeps the previous call's contents, which
must not leak into the next), up to the largest front the array admits.

Kept in a file of its own that pytest collects last."""
import ctypes as C

import numpy as np
import pytest

from clique_b200 import _capi

pytestmark = pytest.mark.gpu


def _front(m, n, complex_, seed, hermitian=False):
    rng = np.random.default_rng(seed)
    G = rng.standard_normal((m, m)) + (1j * rng.standard_normal((m, m)) if complex_ else 0)
    S = (G @ G.conj().T if hermitian else G @ G.T) / m + 8 * np.eye(m)
    return np.asfortranarray(np.tril(S)[:, :n]), np.asfortranarray(np.tril(S[n:, n:]))


def _dev(a, dtype):
    import torch
    return torch.from_numpy(a).to(dtype).cuda().t().contiguous().t()


def _run(fn, field, prec, AL, ABR, dtype, conj=0):
    import torch
    m, n = AL.shape
    tAL, tABR = _dev(AL, dtype), _dev(ABR, dtype)
    st = fn(field, prec, conj, m, n, C.c_void_p(tAL.data_ptr()), m, C.c_void_p(tABR.data_ptr()), max(m - n, 1), None)
    torch.cuda.synchronize()
    return st, tAL.cpu().numpy(), np.tril(tABR.cpu().numpy())


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _dtype(precision, complex_):
    import torch
    return {("double", False): torch.float64, ("double", True): torch.complex128,
            ("single", False): torch.float32, ("single", True): torch.complex64}[(precision, complex_)]


@pytest.mark.parametrize("complex_,precision,conj,tol", [(False, "double", 0, 1e-12), (True, "double", 0, 1e-12),
                                                         (True, "double", 1, 1e-12), (False, "single", 0, 1e-4),
                                                         (True, "single", 0, 1e-4), (True, "single", 1, 1e-4)])
def test_noalloc_matches_allocating_entry_point(complex_, precision, conj, tol):
    lib = _capi.load()
    dtype = _dtype(precision, complex_)
    field = int(complex_)
    prec = 0 if precision == "double" else 1
    # two calls in a row with different fronts: the second must not see the first's scratch
    for (m, n, seed) in [(300, 150, 1), (197, 70, 2)]:
        AL, ABR = _front(m, n, complex_, seed, hermitian=bool(conj))
        st_ref, AL_ref, ABR_ref = _run(lib.cliqgpu_front_ldl, field, prec, AL, ABR, dtype, conj)
        st_new, AL_new, ABR_new = _run(lib.cliqgpu_front_ldl_noalloc, field, prec, AL, ABR, dtype, conj)
        assert st_ref == 0 and st_new == 0, lib.cliqgpu_last_error()
        assert _rel(AL_new, AL_ref) <= tol
        assert _rel(ABR_new, ABR_ref) <= tol


@pytest.mark.parametrize("complex_,conj", [(False, 0), (True, 1)])
def test_noalloc_matches_oracle(oracle, complex_, conj):
    """Checked directly against the oracle's FrontLDL (ldl/local_front.hpp:30-71),
    not only against the allocating entry point that shares its kernels."""
    lib = _capi.load()
    for (m, n, seed) in [(260, 130, 3), (129, 65, 4)]:
        AL, ABR = _front(m, n, complex_, seed, hermitian=bool(conj))
        ALo, ABRo = AL.copy(order="F"), ABR.copy(order="F")
        assert oracle.front_ldl(ALo, ABRo, conjugate=bool(conj), nb=96) == 0
        st, ALg, ABRg = _run(lib.cliqgpu_front_ldl_noalloc, int(complex_), 0, AL, ABR, _dtype("double", complex_), conj)
        assert st == 0, lib.cliqgpu_last_error()
        assert _rel(ALg, ALo) <= 1e-12
        assert _rel(ABRg, np.tril(ABRo)) <= 1e-12


def test_noalloc_at_its_limits_allocates_nothing(oracle):
    """The largest front the fixed scratch admits (n = 1024, m = 16384, real
    FP64), twice in a row, against the oracle; the device's free memory is the
    same before and after each call (kernels are loaded by a first small call)."""
    import torch
    lib = _capi.load()
    AL0, ABR0 = _front(70, 20, False, 9)
    _run(lib.cliqgpu_front_ldl_noalloc, 0, 0, AL0, ABR0, torch.float64)
    m, n = 16384, 1024
    rng = np.random.default_rng(11)
    # a diagonally dominant symmetric front built without an m x m dense product
    G = rng.standard_normal((m, 48)) / np.sqrt(48)
    AL = np.asfortranarray(G @ G[:n].T)
    AL[:n] = np.tril(AL[:n])
    AL[np.arange(n), np.arange(n)] += 4.0
    ABR = np.asfortranarray(np.tril(G[n:] @ G[n:].T))
    ABR[np.arange(m - n), np.arange(m - n)] += 4.0
    ALo, ABRo = AL.copy(order="F"), ABR.copy(order="F")
    oracle.enable_blas(0)
    try:
        assert oracle.front_ldl(ALo, ABRo, nb=96) == 0
    finally:
        oracle.disable_blas()
    ABRo = np.tril(ABRo)
    tAL, tABR = _dev(AL, torch.float64), _dev(ABR, torch.float64)
    for call in range(2):
        tAL.copy_(_dev(AL, torch.float64))
        tABR.copy_(_dev(ABR, torch.float64))
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        st = lib.cliqgpu_front_ldl_noalloc(0, 0, 0, m, n, C.c_void_p(tAL.data_ptr()), m, C.c_void_p(tABR.data_ptr()),
                                           m - n, None)
        torch.cuda.synchronize()
        free1 = torch.cuda.mem_get_info()[0]
        assert st == 0, lib.cliqgpu_last_error()
        assert free1 == free0, (call, free0, free1)
        assert _rel(tAL.cpu().numpy(), ALo) <= 1e-12
        assert _rel(np.tril(tABR.cpu().numpy()), ABRo) <= 1e-12


def test_noalloc_reports_zero_pivot_column():
    lib = _capi.load()
    AL, ABR = _front(40, 20, False, 5)
    AL[:, 7] = 0.0
    AL[7, :] = 0.0                                   # row 7 of the lower part: column 7 gets a zero pivot
    st, _, _ = _run(lib.cliqgpu_front_ldl_noalloc, 0, 0, np.asfortranarray(AL), ABR, _dtype("double", False))
    assert st == _capi.CLIQ_ERR_ZERO_PIVOT
    assert b"zero pivot at column 7" in lib.cliqgpu_last_error()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    lib = _capi.load()
    t = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = C.c_void_p(t.data_ptr())
    assert lib.cliqgpu_front_ldl_noalloc(0, 0, 0, 2048, 1025, p, 2048, p, 1023, None) == _capi.CLIQ_ERR_ARG
    assert b"too large" in lib.cliqgpu_last_error()
    assert lib.cliqgpu_front_ldl_noalloc(0, 0, 0, 20000, 100, p, 20000, p, 19900, None) == _capi.CLIQ_ERR_ARG
    assert lib.cliqgpu_front_ldl_noalloc(0, 0, 0, 4, 2, p, 5, p, 2, None) == _capi.CLIQ_ERR_ARG   # lda != m
    assert lib.cliqgpu_front_ldl_noalloc(0, 0, 0, 4, 2, p, 4, p, 2**31, None) == _capi.CLIQ_ERR_ARG   # ldabr > INT_MAX
    assert b"INT_MAX" in lib.cliqgpu_last_error()
