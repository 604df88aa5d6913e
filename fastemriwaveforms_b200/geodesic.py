"""Kerr geodesic fundamental frequencies on the GPU.

Drop-in for ``few.utils.geodesic.get_fundamental_frequencies``
(``src/few/utils/geodesic.py:470-535``): the same arguments and branches
(Schwarzschild, circular, eccentric equatorial and generic Kerr orbits), the
same ValueError for an elliptic modulus outside [0, 1].  The frequencies are
computed by ``k_fundamental_frequencies`` (``csrc/geodesic.cu``); array
results are torch CUDA tensors, all-scalar arguments give Python floats.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .summation import _device, _ptr, _stream, _to_device

MTSUN_SI = 4.9254909491978065e-06  # one solar mass in seconds (src/few/cutils/global.h:24)


def _as_device(x, n, dev):
    if isinstance(x, torch.Tensor):
        t = x.to(device=dev, dtype=torch.float64).reshape(-1).contiguous()
    else:
        t = _to_device(np.atleast_1d(np.asarray(x, dtype=np.float64)), torch.float64, dev)
    if t.numel() != n:
        raise AssertionError("a, p, e and x must have the same length")
    return t


def fundamental_frequencies_into(a, p, e, x, out_phi, out_theta, out_r, denom=1.0, abs_phi=False, status=None):
    """Device-level form: writes the three frequencies (each divided by
    ``denom``) into the given float64 CUDA tensors of p's length.  ``a`` is a
    float or a tensor of p's length.  No synchronisation."""
    n = int(p.numel())
    if isinstance(a, torch.Tensor):
        a_t, a_stride = a.to(device=p.device, dtype=torch.float64).reshape(-1).contiguous(), 1
        if a_t.numel() == 1:
            a_stride = 0
        elif a_t.numel() != n:
            raise AssertionError("a, p, e and x must have the same length")
    else:
        a_t, a_stride = torch.full((1,), float(a), dtype=torch.float64, device=p.device), 0
    _lib.call("few_fundamental_frequencies", _ptr(a_t), a_stride, _ptr(p), _ptr(e), _ptr(x), n, float(denom),
              int(bool(abs_phi)), _ptr(out_phi), _ptr(out_theta), _ptr(out_r),
              _ptr(status) if status is not None else None, _stream(p.device))
    return a_t  # keep alive until the caller's stream has consumed it


def check_status(status: torch.Tensor) -> None:
    """Raise the reference's ValueError if the kernel saw an elliptic modulus
    outside [0, 1] (``src/few/utils/elliptic.py:220-300``)."""
    if int(status.item()) & 1:
        raise ValueError("Elliptic integral K(k) valid only for k in [0, 1].")


def get_fundamental_frequencies(a, p, e, x, use_gpu: bool = True, device=None):
    """(OmegaPhi, OmegaTheta, OmegaR) in units of 1/M for spin a, semi-latus
    rectum p, eccentricity e and x = cos(inclination).  ``use_gpu`` is
    accepted for signature compatibility; there is only the GPU path."""
    scalar = not any(hasattr(v, "__len__") or (isinstance(v, torch.Tensor) and v.ndim > 0) for v in (a, p, e, x))
    dev = _device(device)
    p_d = _to_device(np.atleast_1d(np.asarray(p, dtype=np.float64)), torch.float64, dev) \
        if not isinstance(p, torch.Tensor) else p.to(device=dev, dtype=torch.float64).reshape(-1).contiguous()
    n = int(p_d.numel())
    e_d = _as_device(e, n, dev)
    x_d = _as_device(x, n, dev)
    a_arg = a if not hasattr(a, "__len__") and not (isinstance(a, torch.Tensor) and a.ndim > 0) else _as_device(a, n, dev)
    if isinstance(a_arg, torch.Tensor) and a_arg.ndim == 0:
        a_arg = float(a_arg.item())
    out = torch.empty((3, n), dtype=torch.float64, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    fundamental_frequencies_into(a_arg, p_d, e_d, x_d, out[0], out[1], out[2], status=status)
    check_status(status)
    if scalar:
        vals = out[:, 0].tolist()
        return vals[0], vals[1], vals[2]
    return out[0], out[1], out[2]
