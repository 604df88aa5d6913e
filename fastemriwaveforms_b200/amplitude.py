"""Teukolsky amplitudes from bicubic B-spline grids on B200: drop-in for
``few.amplitude.ampinterp2d.AmpInterp2D`` (src/few/amplitude/ampinterp2d.py:29-189)
and its backend function ``interp2D`` (src/few/cutils/pyampinterp2D.pyx:16-27).

``AmpInterp2D(w_knots, u_knots, coefficients, l_arr, m_arr, k_arr, n_arr)``
holds one pair of coefficient grids (real, imaginary) per mode;
``__call__(w, u, mode_indexes=None)`` evaluates them at the points (w, u) and
returns the complex amplitudes as an (m points, modes) torch complex128 tensor
on the GPU, which is the ``teuk_modes`` layout ``InterpolatedModeSum`` reads.
The evaluation (``few_amp_interp2d``) computes each point's B-spline basis once
for all modes and writes that layout directly; the values equal the
reference's CPU path bit for bit.  The reference loads the grids from its data
files; here they are passed in (loading files is outside this package).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .summation import _device, _ptr, _stream


def _dev_f64(x, dev) -> torch.Tensor:
    if isinstance(x, torch.Tensor):
        return x.to(device=dev, dtype=torch.float64).contiguous()
    return torch.from_numpy(np.ascontiguousarray(np.asarray(x, dtype=np.float64))).to(dev)


class AmpInterp2D:
    """Bicubic spline amplitudes (reference: ``ampinterp2d.py:29-189``).

    args:
        w_knots, u_knots: knots of the two interpolation coordinates.
        coefficients: (num_teuk_modes, 2, len_indiv_c) spline coefficients,
            real then imaginary part of each mode.
        l_arr, m_arr, k_arr, n_arr: mode indices.
        force_backend: accepted for signature compatibility; the GPU is used.
    """

    degree = 3

    def __init__(self, w_knots, u_knots, coefficients, l_arr, m_arr, k_arr, n_arr, force_backend=None, device=None):
        self.device = _device(device)
        self.l_arr, self.m_arr, self.k_arr, self.n_arr = l_arr, m_arr, k_arr, n_arr
        coeff = _dev_f64(coefficients, self.device)
        if coeff.ndim != 3 or coeff.shape[1] != 2:
            raise ValueError("coefficients must have shape (num_teuk_modes, 2, len_indiv_c).")
        self.num_teuk_modes = int(coeff.shape[0])
        self.knots = [_dev_f64(w_knots, self.device), _dev_f64(u_knots, self.device)]
        nw, nu = (int(k.shape[0]) for k in self.knots)
        self.coeff = coeff
        self.len_indiv_c = int(coeff.shape[2])
        if (nw - self.degree - 1) * (nu - self.degree - 1) != self.len_indiv_c:
            raise ValueError("len_indiv_c must equal (len(w_knots) - 4) * (len(u_knots) - 4).")

    def __call__(self, w, u, *args, mode_indexes=None, **kwargs) -> torch.Tensor:
        """Amplitudes (m points, modes) at the points (w, u) (broadcast together)."""
        dev = self.device
        w_h = w.detach().cpu().numpy() if isinstance(w, torch.Tensor) else np.asarray(w, dtype=np.float64)
        u_h = u.detach().cpu().numpy() if isinstance(u, torch.Tensor) else np.asarray(u, dtype=np.float64)
        if w_h.shape != u_h.shape:
            w_h, u_h = np.broadcast_arrays(w_h, u_h)
        w_d = _dev_f64(np.ravel(w_h), dev)
        u_d = _dev_f64(np.ravel(u_h), dev)
        m = int(w_d.shape[0])
        if mode_indexes is None:
            idx = None
            nmodes = self.num_teuk_modes
        else:
            idx = _dev_f64(mode_indexes, dev).to(torch.int32) if not isinstance(mode_indexes, torch.Tensor) \
                else mode_indexes.to(device=dev, dtype=torch.int32).contiguous()
            nmodes = int(idx.shape[0])
            if nmodes and (int(idx.min()) < 0 or int(idx.max()) >= self.num_teuk_modes):
                raise ValueError("mode_indexes out of range.")
        out = torch.zeros((m, nmodes), dtype=torch.complex128, device=dev)
        if m == 0 or nmodes == 0:
            return out
        tw, tu = self.knots
        _lib.call("few_amp_interp2d", _ptr(out), _ptr(tw), int(tw.shape[0]), _ptr(tu), int(tu.shape[0]),
                  _ptr(self.coeff), self.degree, self.degree, _ptr(w_d), _ptr(u_d), m,
                  _ptr(idx) if idx is not None else None, nmodes, self.len_indiv_c, _stream(dev))
        return out


def interp2D(z, tx, nx, ty, ny, c, kx, ky, x, mx, y, my, num_indiv_c, len_indiv_c):
    """The backend function's argument list (``pyampinterp2D.pyx:16-27``) on
    CUDA tensors: z (num_indiv_c * mx,) receives every grid of c at the points."""
    for a in (z, tx, ty, c, x, y):
        if not (isinstance(a, torch.Tensor) and a.is_cuda and a.dtype == torch.float64 and a.is_contiguous()):
            raise ValueError("interp2D takes contiguous float64 CUDA tensors.")
    _lib.call("few_interp2d", _ptr(z), _ptr(tx), int(nx), _ptr(ty), int(ny), _ptr(c), int(kx), int(ky), _ptr(x),
              int(mx), _ptr(y), int(my), int(num_indiv_c), int(len_indiv_c), _stream(z.device))
