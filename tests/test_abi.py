"""The C ABI library: it loads, exports every entry point include/few_b200.h
declares, and rejects bad arguments on the host (no GPU work is launched)."""
import ctypes
import os
import re

import pytest

from fastemriwaveforms_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            names.update(re.findall(r"^FEW_API\s+[\w\s\*]*?\b(few_\w+)\s*\(", text, flags=re.M))
    return names


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_symbols()
    assert "few_get_waveform" in names and "few_interpolate_arrays" in names
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) <= set(_lib.SIGNATURES), "ctypes signatures missing for some entry points"


def test_abi_version_and_error_text():
    lib = _lib.load()
    assert lib.few_abi_version() == 4
    rc = lib.few_spline_build(None, 0, None, 1, 1, 1, 0, 1, 10, None, 0, None)
    assert rc == _lib.FEW_ERR_ARG
    assert "null" in _lib.last_error()


def test_host_validation_without_gpu():
    lib = _lib.load()
    dummy = ctypes.c_void_p(16)  # never dereferenced: the sizes are rejected first
    assert lib.few_spline_build(dummy, 0, dummy, 1, 1, 1, 0, 1, 3, dummy, 0, None) == _lib.FEW_ERR_SIZE
    assert "4 knots" in _lib.last_error()
    assert lib.few_interpolate_arrays(dummy, dummy, 2, 2, None, None, None, None, None) == _lib.FEW_ERR_SIZE
    assert lib.few_spline_eval(dummy, 0, dummy, 1, 10, dummy, 0, 5, 7, dummy, dummy, None) == _lib.FEW_ERR_ARG
    assert lib.few_sum_folded(dummy, dummy, dummy, 10, dummy, dummy, 1, dummy, dummy, 300, 0, 1, 10.0, 0, 0,
                              None) == _lib.FEW_ERR_SIZE
    assert lib.few_sum_folded(dummy, dummy, dummy, 10, dummy, dummy, 1, dummy, dummy, 3, 0, 1, 10.0, 5, 0,
                              None) == _lib.FEW_ERR_ARG
    assert lib.few_get_waveform(None, dummy, dummy, dummy, dummy, dummy, dummy, 10, 10, 1, dummy, 10.0, dummy, 0,
                                None) == _lib.FEW_ERR_ARG


def test_call_maps_status_to_exceptions():
    with pytest.raises(ValueError):
        _lib.call("few_spline_build", None, 0, None, 1, 1, 1, 0, 1, 10, None, 0, None)
