"""-2 spin-weighted spherical harmonics on the GPU.

Drop-in for ``few.utils.ylm.GetYlms`` (``src/few/utils/ylm.py:278-365``): the
same constructor and call, the same (+m, then -m) doubling when
``include_minus_m`` (m = 0 duplicated, as the reference does).  The values come
from ``k_ylm`` (``csrc/ylm.cu``), one closed-form sum for every (l, m) instead
of the reference's table of l <= 10 expressions; l up to 64 is accepted.
Array arguments give a complex128 CUDA tensor, integer arguments a Python
complex (or a pair with ``include_minus_m``).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .summation import _device, _ptr, _stream, _to_device


def ylm_into(l_d: torch.Tensor, m_d: torch.Tensor, theta: float, phi: float, out: torch.Tensor,
             include_minus_m: bool = False, status: torch.Tensor | None = None) -> None:
    """Device-level form: int32 CUDA tensors l, m (n,) -> out (n or 2n,) complex128."""
    _lib.call("few_ylm", _ptr(l_d), _ptr(m_d), int(l_d.numel()), int(bool(include_minus_m)), float(theta),
              float(phi), _ptr(out), _ptr(status) if status is not None else None, _stream(out.device))


class GetYlms:
    """(-2) spin-weighted spherical harmonics Y_lm(theta, phi)."""

    def __init__(self, include_minus_m: bool = False, force_backend=None, device=None, **kwargs):
        self.include_minus_m = include_minus_m
        self._device_arg = device

    @property
    def device(self) -> torch.device:
        return _device(self._device_arg)

    def __call__(self, l_in, m_in, theta: float, phi: float, include_minus_m: bool | None = None):
        if include_minus_m is None:
            include_minus_m = self.include_minus_m
        dev = self.device
        scalar = isinstance(l_in, (int, np.integer)) or isinstance(m_in, (int, np.integer))
        if scalar:
            assert isinstance(l_in, (int, np.integer)) and isinstance(m_in, (int, np.integer))
            l_arr, m_arr = np.array([l_in], np.int32), np.array([m_in], np.int32)
        else:
            l_arr = l_in.detach().cpu().numpy() if isinstance(l_in, torch.Tensor) else np.asarray(l_in)
            m_arr = m_in.detach().cpu().numpy() if isinstance(m_in, torch.Tensor) else np.asarray(m_in)
            l_arr, m_arr = l_arr.astype(np.int32).reshape(-1), m_arr.astype(np.int32).reshape(-1)
        if l_arr.shape != m_arr.shape:
            raise ValueError("l and m must have the same length.")
        n = len(l_arr)
        out = torch.empty(2 * n if include_minus_m else n, dtype=torch.complex128, device=dev)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        if n:
            ylm_into(_to_device(l_arr, torch.int32, dev), _to_device(m_arr, torch.int32, dev), theta, phi, out,
                     include_minus_m, status)
        if int(status.item()):
            raise ValueError("(l, m) out of range: need 2 <= l <= 64 and |m| <= l.")
        if scalar:
            vals = out.cpu().numpy()
            return (complex(vals[0]), complex(vals[1])) if include_minus_m else complex(vals[0])
        return out
