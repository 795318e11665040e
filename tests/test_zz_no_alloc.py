"""cliqgpu_front_ldl_noalloc: the single-front LDL^T for callers that may not
allocate device memory (a caller with its own memory pool that bans
cudaMalloc/cudaFree while it runs).  Checked through the C ABI against the
allocating cliqgpu_front_ldl, on two calls in a row (the fixed scratch array
keeps the previous call's contents, which must not leak into the next).

Kept in a file of its own that pytest collects last."""
import ctypes as C

import numpy as np
import pytest

from clique_b200 import _capi

pytestmark = pytest.mark.gpu


def _front(m, n, complex_, seed):
    rng = np.random.default_rng(seed)
    G = rng.standard_normal((m, m)) + (1j * rng.standard_normal((m, m)) if complex_ else 0)
    S = G @ G.T / m + 8 * np.eye(m)
    return np.asfortranarray(np.tril(S)[:, :n]), np.asfortranarray(np.tril(S[n:, n:]))


def _dev(a, dtype):
    import torch
    return torch.from_numpy(a).to(dtype).cuda().t().contiguous().t()


def _run(fn, field, prec, AL, ABR, dtype):
    import torch
    m, n = AL.shape
    tAL, tABR = _dev(AL, dtype), _dev(ABR, dtype)
    st = fn(field, prec, 0, m, n, C.c_void_p(tAL.data_ptr()), m, C.c_void_p(tABR.data_ptr()), max(m - n, 1), None)
    torch.cuda.synchronize()
    return st, tAL.cpu().numpy(), np.tril(tABR.cpu().numpy())


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("complex_,precision,tol", [(False, "double", 1e-12), (True, "double", 1e-12),
                                                    (True, "single", 1e-4)])
def test_noalloc_matches_allocating_entry_point(complex_, precision, tol):
    import torch
    lib = _capi.load()
    dtype = {("double", False): torch.float64, ("double", True): torch.complex128,
             ("single", False): torch.float32, ("single", True): torch.complex64}[(precision, complex_)]
    field = int(complex_)
    prec = 0 if precision == "double" else 1
    # two calls in a row with different fronts: the second must not see the first's scratch
    for (m, n, seed) in [(300, 150, 1), (197, 70, 2)]:
        AL, ABR = _front(m, n, complex_, seed)
        st_ref, AL_ref, ABR_ref = _run(lib.cliqgpu_front_ldl, field, prec, AL, ABR, dtype)
        st_new, AL_new, ABR_new = _run(lib.cliqgpu_front_ldl_noalloc, field, prec, AL, ABR, dtype)
        assert st_ref == 0 and st_new == 0, lib.cliqgpu_last_error()
        assert _rel(AL_new, AL_ref) <= tol
        assert _rel(ABR_new, ABR_ref) <= tol


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    lib = _capi.load()
    t = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = C.c_void_p(t.data_ptr())
    assert lib.cliqgpu_front_ldl_noalloc(0, 0, 0, 2048, 1025, p, 2048, p, 1023, None) == _capi.CLIQ_ERR_ARG
    assert b"too large" in lib.cliqgpu_last_error()
    assert lib.cliqgpu_front_ldl_noalloc(0, 0, 0, 20000, 100, p, 20000, p, 19900, None) == _capi.CLIQ_ERR_ARG
    assert lib.cliqgpu_front_ldl_noalloc(0, 0, 0, 4, 2, p, 5, p, 2, None) == _capi.CLIQ_ERR_ARG   # lda != m
