"""ctypes binding of libfew_b200.so (the C ABI declared in include/few_b200.h).

This is the whole Python <-> native boundary: tensors are passed as raw device
addresses (``tensor.data_ptr()``) with their sizes, exactly as the reference's
Cython shim passes ``size_t`` addresses (src/few/cutils/pyinterp.pyx:25-61).
The library is built in-tree on first use if it is missing or stale; there is
no CPU fallback, and a failed build or load raises.
"""
from __future__ import annotations

import ctypes
import threading

from . import build as _build

FEW_OK = 0
FEW_ERR_ARG = -1
FEW_ERR_SIZE = -2
FEW_ERR_CUDA = -3
FEW_ERR_KNOTS = -4
FEW_ERR_NOMEM = -5

FEW_SUM_FAITHFUL = 0
FEW_SUM_EXACT = 1
FEW_LAYOUT_KNOT_MAJOR = 0
FEW_LAYOUT_INTERP_MAJOR = 1
FEW_FAC_WIDTH = 16

_c_int, _c_ll, _c_dbl, _vp = ctypes.c_int, ctypes.c_longlong, ctypes.c_double, ctypes.c_void_p

# name -> argtypes (all return int unless listed in _RESTYPE)
SIGNATURES = {
    "few_last_error": [],
    "few_abi_version": [],
    "few_interpolate_arrays": [_vp, _vp, _c_int, _c_int, _vp, _vp, _vp, _vp, _vp],
    "few_get_waveform": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _c_int, _c_int, _c_int, _vp, _c_dbl, _vp, _c_int, _vp],
    "few_spline_build": [_vp, _c_ll, _vp, _c_ll, _c_ll, _c_int, _c_ll, _c_int, _c_int, _vp, _c_int, _vp],
    "few_spline_eval": [_vp, _c_ll, _vp, _c_int, _c_int, _vp, _c_ll, _c_int, _c_int, _vp, _vp, _vp],
    "few_spline_factor": [_vp, _c_int, _vp],
    "few_spline_build_factored": [_vp, _vp, _c_ll, _c_ll, _c_int, _c_ll, _c_int, _c_int, _vp, _c_int, _vp],
    "few_fold_plan": [_vp, _vp, _vp, _c_int, _c_int, _c_int, _vp, _vp, _vp, _vp, _vp],
    "few_segment_plan": [_vp, _vp, _c_int, _c_int, _c_dbl, _c_int, _c_int, _vp, _vp, _vp, _vp],
    "few_fold_coeffs": [_vp, _vp, _vp, _vp, _c_int, _c_int, _c_int, _c_int, _c_int, _vp, _vp],
    "few_sum_folded": [_vp, _vp, _vp, _c_int, _vp, _vp, _c_int, _vp, _vp, _c_int, _c_int, _c_int, _c_dbl, _c_int,
                       _c_int, _vp],
    "few_probe_fp64_fma": [_vp, _c_int, _c_int, _vp],
    "few_adjoint_phase": [_vp, _vp, _vp, _c_int, _vp, _vp, _c_int, _vp, _vp, _c_int, _c_int, _c_int, _c_dbl, _c_int,
                          _vp, _vp],
    "few_adjoint_phase_reduce": [_vp, _vp, _c_int, _vp, _vp],
    "few_adjoint_G": [_vp, _vp, _c_int, _vp, _vp, _c_int, _vp, _vp, _c_int, _c_int, _c_int, _c_dbl, _c_int, _vp, _vp],
    "few_adjoint_joint_scratch": [_c_int, _c_int, _c_int],
    "few_adjoint_joint": [_vp, _vp, _vp, _c_int, _vp, _vp, _c_int, _vp, _c_int, _vp, _vp, _c_int, _c_int, _c_int,
                          _c_dbl, _c_int, _vp, _vp, _vp, _vp],
    "few_unfold": [_vp, _vp, _vp, _vp, _c_int, _c_int, _c_int, _c_int, _vp, _vp],
    "few_spline_adjoint_factored": [_vp, _vp, _vp, _c_ll, _c_ll, _c_int, _c_ll, _c_int, _c_int, _c_int, _vp],
    "few_spline_adjoint": [_vp, _c_ll, _vp, _vp, _c_ll, _c_ll, _c_int, _c_ll, _c_int, _c_int, _c_int, _vp],
    "few_mixed_operand_bytes": [_c_int, _c_int, _c_int],
    "few_fold_mixed": [_vp, _vp, _c_int, _c_int, _c_int, _vp, _vp],
    "few_sum_mixed": [_vp, _vp, _vp, _c_int, _vp, _vp, _vp, _c_int, _vp, _vp, _c_int, _c_int, _c_int, _c_dbl, _c_int,
                      _vp, _vp],
    "few_sum_batched": [_vp, _c_int, _vp, _c_int, _c_int, _c_int, _c_int, _vp, _vp],
    "few_sum_mixed_batched": [_vp, _c_int, _vp, _c_int, _c_int, _c_int, _c_int, _c_int, _vp, _vp, _vp],
    "few_stamp": [_vp, _vp],
    "few_adjoint_G_mixed": [_vp, _vp, _c_int, _vp, _vp, _vp, _c_int, _vp, _vp, _c_int, _c_int, _c_int, _c_dbl, _c_int,
                            _vp, _vp, _vp],
    "few_mixed_adjoint_operand_bytes": [_c_int, _c_int, _c_int],
    "few_fold_mixed_adjoint": [_vp, _vp, _c_int, _c_int, _c_int, _c_int, _vp, _vp],
    "few_adjoint_phase_mixed": [_vp, _vp, _vp, _c_int, _vp, _vp, _vp, _c_int, _vp, _vp, _c_int, _c_int, _c_int, _c_dbl,
                                _c_int, _vp, _vp, _vp],
    "few_interp2d": [_vp, _vp, _c_int, _vp, _c_int, _vp, _c_int, _c_int, _vp, _c_int, _vp, _c_int, _c_int, _c_int, _vp],
    "few_amp_interp2d": [_vp, _vp, _c_int, _vp, _c_int, _vp, _c_int, _c_int, _vp, _vp, _c_int, _vp, _c_int, _c_int,
                         _vp],
    "few_get_waveform_noalloc": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _c_int, _c_int, _c_int, _vp, _c_dbl, _vp,
                                 _c_int, _vp],
    "few_fundamental_frequencies": [_vp, _c_int, _vp, _vp, _vp, _c_int, _c_dbl, _c_int, _vp, _vp, _vp, _vp, _vp],
    "few_fd_turn_bytes": [],
    "few_fd_plan_extrema": [_vp, _c_int, _c_dbl, _c_dbl, _c_dbl, _vp, _c_int, _vp, _vp, _vp, _vp, _c_int, _vp, _vp,
                            _vp],
    "few_fd_plan_bins": [_vp, _vp, _vp, _vp, _c_int, _c_int, _vp, _vp, _c_dbl, _c_dbl, _c_int, _c_dbl, _c_int, _c_int,
                         _vp, _vp, _vp, _vp, _vp],
    "few_fd_scan": [_vp, _c_ll, _vp, _vp, _vp],
    "few_fd_frequency_grid": [_vp, _c_int, _c_dbl, _vp],
    "few_fd_sum": [_vp, _c_int, _vp, _c_int, _c_int, _vp, _c_ll, _c_ll, _c_ll, _vp, _c_ll, _c_ll, _c_ll, _vp, _c_ll,
                   _c_ll, _c_ll, _vp, _vp, _c_int, _vp, _vp, _vp, _c_int, _vp, _vp, _vp, _c_int, _c_int, _vp],
    "few_fd_finalize": [_vp, _c_int, _c_int, _c_int, _vp, _vp],
    "few_ylm": [_vp, _vp, _c_int, _c_int, _c_dbl, _c_dbl, _vp, _vp, _vp],
    "few_mode_snr2": [_vp, _c_int, _c_int, _vp, _vp, _vp, _vp, _vp, _vp],
    "few_mode_keep": [_vp, _c_int, _c_dbl, _vp, _vp],
    "few_direct_sum": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _c_int, _c_int, _vp, _vp],
    "few_aak_sum": [_vp, _vp, _c_int, _vp, _vp, _c_int, _c_int, _c_dbl, _c_dbl, _c_dbl, _c_dbl, _c_dbl, _c_dbl,
                    _c_dbl, _c_dbl, _c_int, _c_int, _c_dbl, _vp],
    "few_aak_waveform": [_vp, _vp, _c_dbl, _c_dbl, _c_dbl, _c_dbl, _c_dbl, _c_dbl, _c_dbl, _c_dbl, _c_int, _c_int,
                         _c_int, _c_int, _c_dbl, _vp, _vp],
    "few_dopr853_dense": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _c_int, _c_int, _c_int,
                          _vp],
    "few_dopr853_eval": [_vp, _c_int, _vp, _c_int, _vp, _c_int, _c_int, _vp, _vp],
    "few_get_waveform_fd": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _c_int, _c_dbl, _vp, _c_int, _c_int, _vp, _vp, _vp,
                            _c_int, _vp, _c_int, _c_int, _c_int, _vp],
}
_RESTYPE = {"few_last_error": ctypes.c_char_p, "few_mixed_operand_bytes": ctypes.c_longlong,
            "few_mixed_adjoint_operand_bytes": ctypes.c_longlong, "few_adjoint_joint_scratch": ctypes.c_longlong}

_lock = threading.Lock()
_lib = None


class FewError(RuntimeError):
    """A libfew_b200 call returned a non-zero status."""

    def __init__(self, func: str, code: int, message: str):
        super().__init__(f"{func} failed with status {code}: {message}")
        self.code = code


def library_path() -> str:
    return _build.LIBPATH


def load(build_if_missing: bool = True):
    """Load (building first if needed) and return the ctypes library."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if build_if_missing:
            _build.build()
        lib = ctypes.CDLL(_build.LIBPATH)
        for name, argtypes in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = argtypes
            fn.restype = _RESTYPE.get(name, ctypes.c_int)
        _lib = lib
        return _lib


def last_error() -> str:
    return load().few_last_error().decode(errors="replace")


def call(name: str, *args) -> int:
    """Call an entry point; raise ValueError for argument/size/knot errors and
    FewError for CUDA failures."""
    lib = load()
    rc = getattr(lib, name)(*args)
    if rc != FEW_OK:
        msg = last_error()
        if rc in (FEW_ERR_ARG, FEW_ERR_SIZE, FEW_ERR_KNOTS):
            raise ValueError(f"{name}: {msg}")
        raise FewError(name, rc, msg)
    return rc
