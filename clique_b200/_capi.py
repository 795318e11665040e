"""ctypes binding of ``libcliqgpu.so`` (declared in include/cliqgpu.h).

The library is loaded from the package tree (``clique_b200/_lib``).  There is
no fallback: if the library is missing, importing the numeric API raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libcliqgpu.so")

CLIQ_OK = 0
CLIQ_ERR_ARG = 1
CLIQ_ERR_OOM = 2
CLIQ_ERR_ZERO_PIVOT = 3
CLIQ_ERR_CUDA = 4
CLIQ_ERR_TIMEOUT = 5
CLIQ_ERR_STATE = 6
CLIQ_ERR_NOCONV = 7
CLIQ_REAL, CLIQ_COMPLEX = 0, 1
CLIQ_FP64, CLIQ_FP32 = 0, 1


class SymmInfo(C.Structure):
    _fields_ = [("num_nodes", C.c_int32), ("size", C.c_void_p), ("off", C.c_void_p), ("parent", C.c_void_p),
                ("children", C.c_void_p), ("lower_ptr", C.c_void_p), ("lower", C.c_void_p),
                ("orig_lower_ptr", C.c_void_p), ("orig_lower", C.c_void_p)]


class Options(C.Structure):
    _fields_ = [("field", C.c_int32), ("precision", C.c_int32), ("conjugate", C.c_int32),
                ("block_size", C.c_int32), ("keep_matrix", C.c_int32)]


# every symbol include/cliqgpu.h declares, with (restype, argtypes)
_SIGS = {
    "cliq_natural_nested_dissection": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_int64, C.c_void_p, C.c_void_p,
                                                 C.c_int32, C.POINTER(C.c_void_p)]),
    "cliq_symbolic_info": (C.c_int, [C.c_void_p, C.POINTER(SymmInfo)]),
    "cliq_symbolic_node": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p]),
    "cliq_symbolic_node_array": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.POINTER(C.c_int64)]),
    "cliq_symbolic_map": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "cliq_symbolic_destroy": (None, [C.c_void_p]),
    "cliqgpu_plan_create": (C.c_int, [C.POINTER(SymmInfo), C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.POINTER(Options), C.c_void_p, C.POINTER(C.c_void_p)]),
    "cliqgpu_assemble": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32]),
    "cliqgpu_factor": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "cliqgpu_block_ldl": (C.c_int, [C.c_void_p]),
    "cliqgpu_factor_intrapiv": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "cliqgpu_get_front_pivots": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
    "cliqgpu_solve": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_int32, C.c_int32, C.c_int32]),
    "cliqgpu_multiply": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int32]),
    "cliqgpu_sparse_multiply": (C.c_int, [C.c_int32, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int32, C.c_int32,
                                          C.c_void_p]),
    "cliqgpu_nodal_pull": (C.c_int, [C.c_int32, C.c_int64, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64,
                                     C.c_int32, C.c_void_p]),
    "cliqgpu_nodal_push": (C.c_int, [C.c_int32, C.c_int64, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64,
                                     C.c_int32, C.c_void_p]),
    "cliqgpu_grad_A_pattern": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int32, C.c_int32,
                                         C.c_void_p]),
    "cliq_nested_dissection": (C.c_int, [C.c_int64, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p]),
    "cliq_batch_nested_dissection": (C.c_int, [C.c_int32, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_int32,
                                               C.POINTER(C.c_void_p)]),
    "cliqgpu_batch_run": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                    C.c_int32, C.c_int32, C.c_double, C.c_int32, C.c_void_p, C.POINTER(C.c_int32)]),
    "cliqgpu_autotune": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p]),
    "cliqgpu_refine": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int32, C.c_int32, C.c_double,
                                 C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_double)]),
    "cliqgpu_get_front": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "cliqgpu_plan_query": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double)]),
    "cliqgpu_synchronize": (C.c_int, [C.c_void_p]),
    "cliqgpu_wait_selftest": (C.c_int, [C.c_void_p, C.c_int64]),
    "cliqgpu_set_profiling": (C.c_int, [C.c_void_p, C.c_int32]),
    "cliqgpu_profile_read": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32]),
    "cliqgpu_plan_destroy": (None, [C.c_void_p]),
    "cliqgpu_status_string": (C.c_char_p, [C.c_int32]),
    "cliqgpu_last_error": (C.c_char_p, []),
    "cliqgpu_front_ldl": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_int64,
                                    C.c_void_p, C.c_int64, C.c_void_p]),
    "cliqgpu_front_ldl_noalloc": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_void_p,
                                            C.c_int64, C.c_void_p, C.c_int64, C.c_void_p]),
}

_lib = None


def load():
    """Load the library (no fallback: raises OSError if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(f"{LIB_PATH} is missing; run `python -m clique_b200.build`")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def exported_symbols():
    return list(_SIGS)


class CliqueError(RuntimeError):
    def __init__(self, status, where=""):
        lib = load()
        msg = lib.cliqgpu_status_string(status).decode()
        detail = lib.cliqgpu_last_error().decode()
        super().__init__(f"{where}: {msg}" + (f" ({detail})" if detail else ""))
        self.status = status


class LogicError(CliqueError, ValueError):
    """El::LogicError counterpart (bad arguments, calls out of order)."""


def check(status, where=""):
    if status == CLIQ_OK:
        return
    if status in (CLIQ_ERR_ARG, CLIQ_ERR_STATE):
        raise LogicError(status, where)
    raise CliqueError(status, where)
