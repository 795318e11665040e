"""The C-ABI library loads and exports every symbol include/cliqgpu.h declares
(no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

from clique_b200 import _capi

HDR = os.path.join(os.path.dirname(os.path.dirname(__file__)), "include", "cliqgpu.h")


def declared_symbols():
    src = open(HDR).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b((?:cliq|cliqgpu)_[A-Za-z_0-9]+)\s*\(", src)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "cliqgpu_factor" in syms and "cliqgpu_solve" in syms and "cliq_natural_nested_dissection" in syms


def test_library_exports_every_declared_symbol():
    lib = _capi.load()
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(declared_symbols()) == set(_capi.exported_symbols())


def test_status_strings():
    lib = _capi.load()
    for code in range(8):
        assert lib.cliqgpu_status_string(code)
    assert lib.cliqgpu_status_string(_capi.CLIQ_ERR_ZERO_PIVOT) == b"zero pivot"


def test_null_arguments_are_rejected_without_gpu():
    lib = _capi.load()
    assert lib.cliqgpu_factor(None, None) == _capi.CLIQ_ERR_ARG
    assert lib.cliqgpu_solve(None, None, 0, 0, 0, 0) == _capi.CLIQ_ERR_ARG
    out = ctypes.c_void_p()
    assert lib.cliq_natural_nested_dissection(2, 2, 2, 7, None, None, 4, ctypes.byref(out)) == _capi.CLIQ_ERR_ARG
