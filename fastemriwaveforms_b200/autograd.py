"""Differentiable pieces around the mode sum.

* ``spline_coefficients(t, y)`` -- not-a-knot cubic spline coefficients
  (4, N, ninterps) of y (ninterps, N) over shared knots t, differentiable in y
  (backward: ``few_spline_adjoint``, the transposed solve).
* ``phase_coeffs_from_knots(t, phase_knots)`` -- (N-1, 3, 8) phase coefficients
  in the 8-term basis of the sum kernel (``src/few/cutils/interpolate.cu:642-644``)
  from phase values at the knots (3, N) = (Phi_phi, Phi_theta, Phi_r), through
  not-a-knot cubics: a cubic y0 + A1 s + A2 s^2 + A3 s^3 in s = (t - t_j)/h is
  exactly (y0, A1+A2+A3, -A2-A3, -A3, 0, 0, 0, 0).
* ``interpolated_mode_sum(...)`` -- functional form of ``InterpolatedModeSum``;
  gradients flow to ``teuk_modes`` and ``phase_interp_coeffs`` (and so, through
  the helpers above, to amplitude and phase knots).

The reference has no gradients; everything here is new.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .summation import InterpolatedModeSum, _device, _ptr, _stream, _to_device, spline_factor_table


class _SplineFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, y, fac):
        ni, N = y.shape
        dev = y.device
        coeffs = torch.empty((4, N, ni), dtype=torch.float64, device=dev)
        yc = y.detach().contiguous()
        _lib.call("few_spline_build_factored", _ptr(fac), _ptr(yc), 1, N, ni, 0, ni, N, _ptr(coeffs),
                  _lib.FEW_LAYOUT_KNOT_MAJOR, _stream(dev))
        ctx.save_for_backward(fac)
        ctx.shape = (ni, N)
        return coeffs

    @staticmethod
    def backward(ctx, grad):
        (fac,) = ctx.saved_tensors
        ni, N = ctx.shape
        gc = grad.to(torch.float64).contiguous().clone()  # consumed by the adjoint kernel
        gy = torch.empty((ni, N), dtype=torch.float64, device=grad.device)
        _lib.call("few_spline_adjoint_factored", _ptr(fac), _ptr(gc), _ptr(gy), 1, N, ni, 0, ni, N, 0,
                  _stream(grad.device))
        return gy, None


def spline_coefficients(t, y: torch.Tensor) -> torch.Tensor:
    """Coefficients (4, N, ninterps): y, c1, c2, c3 at every knot (the last knot
    holds the derivative-extrapolated coefficients, as the reference does)."""
    dev = y.device if isinstance(y, torch.Tensor) else _device()
    y = y if isinstance(y, torch.Tensor) else _to_device(y, torch.float64, dev)
    if y.ndim == 1:
        y = y[None, :]
    t_h = t.detach().cpu().numpy() if isinstance(t, torch.Tensor) else np.asarray(t, dtype=np.float64)
    if t_h.ndim != 1 or t_h.shape[0] != y.shape[1] or y.shape[1] < 4:
        raise ValueError("t must be (N,) with N >= 4 matching y's last axis.")
    return _SplineFunction.apply(y.to(torch.float64), spline_factor_table(t_h, y.device))


def phase_coeffs_from_knots(t, phase_knots: torch.Tensor) -> torch.Tensor:
    """(N-1, 3, 8) phase coefficients from (3, N) knot values, differentiable."""
    coeffs = spline_coefficients(t, phase_knots)  # (4, N, 3)
    dev = coeffs.device
    t_dev = _to_device(t, torch.float64, dev)
    h = (t_dev[1:] - t_dev[:-1])[:, None]  # (N-1, 1)
    y0, c1, c2, c3 = (coeffs[c, :-1, :] for c in range(4))  # (N-1, 3)
    A1, A2, A3 = c1 * h, c2 * h * h, c3 * h * h * h
    zeros = torch.zeros_like(y0)
    return torch.stack([y0, A1 + A2 + A3, -A2 - A3, -A3, zeros, zeros, zeros, zeros], dim=-1)


def interpolated_mode_sum(t, teuk_modes, ylms, phase_interp_t, phase_interp_coeffs, l_arr, m_arr, k_arr, n_arr,
                          T: float = 1.0, dt: float = 10.0, precision: str = "faithful", **kwargs) -> torch.Tensor:
    """``InterpolatedModeSum(precision=...)(...)`` as a function."""
    return InterpolatedModeSum(precision=precision, **kwargs)(t, teuk_modes, ylms, phase_interp_t,
                                                              phase_interp_coeffs, l_arr, m_arr, k_arr, n_arr,
                                                              T=T, dt=dt)
