"""Dense output of the DOPR853 trajectory integrator on the GPU.

Mirrors the dense-output half of ``few.trajectory.dopr853.DOPR853``
(``src/few/trajectory/dopr853.py:606-875``): ``prep_evaluate`` turns the
stages a step stored into the 8-term interpolation basis of the step (for a
trajectory, components 3..5 of that basis are ``InterpolatedModeSum``'s
``phase_interp_coeffs``), ``eval`` and ``eval_derivative`` evaluate it.  The
stepper itself (``take_step``) belongs to the trajectory integration and is
not part of this package.

The basis arithmetic runs in ``k_dense_output`` / ``k_dense_eval``
(csrc/dopr853.cu) through the C ABI, batched over any number of steps (the
reference's ``numSys`` axis).  The four right-hand-side evaluations that
``prep_evaluate`` needs -- the derivative at each step's end and three extra
stages -- call the ``ode`` given to the constructor with the reference's
signature ``ode(x, y, dydx, additionalArgs)``, here on device tensors
(x (nsys,), y and dydx (node, nsys)), for all steps at once.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .summation import _device, _ptr, _stream

__all__ = ["DOPR853"]


def _dev64(x, device) -> torch.Tensor:
    if isinstance(x, torch.Tensor):
        return x.to(device=device, dtype=torch.float64).contiguous()
    return torch.as_tensor(np.ascontiguousarray(x, dtype=np.float64), device=device)


class DOPR853:
    """GPU dense output of the Dormand-Prince 8(5,3) stepper.

    Args:
        ode: ``ode(x, y, dydx, additionalArgs)`` writing f(x, y) into dydx; it
            is called with device tensors, batched over steps.
        device: CUDA device (default: the current one).

    ``k_coefficient_storage`` holds the ten stage slots of the steps to be
    prepared, each (node, nsys), as the reference's ``take_step`` leaves them
    (slots 1 and 2 hold stages 11 and 12).  Unlike the reference,
    ``prep_evaluate`` does not overwrite slots 1, 2 and 9 with the extra stages.
    """

    def __init__(self, ode, device=None):
        self.ode = ode
        self.device = _device(device)
        self.fix_step = False
        self.k_coefficient_storage = None

    @property
    def xp(self):
        return torch

    def prep_evaluate_single(self, x0, y0, h0, x1, y1, additionalArgs):
        """One step: y0, y1 (node,); returns its basis (node, 8)."""
        d = self.device
        y0 = _dev64(y0, d)[:, None]
        y1 = _dev64(y1, d)[:, None]
        out = self.prep_evaluate(_dev64([x0], d), y0, _dev64([h0], d), _dev64([x1], d), y1, additionalArgs)
        return out[0]

    def prep_evaluate(self, x0, y0, h0, x1, y1, additionalArgs):
        """Basis of every step (dopr853.py:621-758): x0, h0, x1 (nsys,),
        y0, y1 (node, nsys); returns rcont (nsys, node, 8) on the device."""
        assert not self.fix_step
        if self.k_coefficient_storage is None:
            raise ValueError("prep_evaluate needs the steps' stages in k_coefficient_storage")
        d = self.device
        y0, y1 = _dev64(y0, d), _dev64(y1, d)
        if y0.dim() != 2 or y1.shape != y0.shape:
            raise ValueError("y0 and y1 must both be (node, nsys)")
        node, nsys = y0.shape
        x0, h0, x1 = _dev64(x0, d).reshape(-1), _dev64(h0, d).reshape(-1), _dev64(x1, d).reshape(-1)
        if not (x0.numel() == h0.numel() == x1.numel() == nsys):
            raise ValueError("x0, h0 and x1 must have one entry per system")
        if len(self.k_coefficient_storage) != 10:
            raise ValueError("k_coefficient_storage must hold the ten stage slots")
        stages = torch.stack([_dev64(k, d).reshape(node, nsys) for k in self.k_coefficient_storage]).contiguous()
        st = _stream(d)
        rcont = torch.empty((nsys, node, 8), dtype=torch.float64, device=d)
        if nsys == 0:
            return rcont
        f1 = torch.zeros_like(y0)
        self.ode(x1, y1, f1, additionalArgs)
        arg = torch.empty_like(y0)
        xarg = torch.empty_like(x0)
        ks = [torch.zeros_like(y0) for _ in range(3)]
        for phase in range(4):
            k14 = ks[0] if phase >= 1 else None
            k15 = ks[1] if phase >= 2 else None
            k16 = ks[2] if phase >= 3 else None
            _lib.call("few_dopr853_dense", _ptr(x0), _ptr(h0), _ptr(x1), _ptr(y0), _ptr(y1), _ptr(f1),
                      _ptr(stages), _ptr(k14) if k14 is not None else None,
                      _ptr(k15) if k15 is not None else None, _ptr(k16) if k16 is not None else None,
                      _ptr(arg), _ptr(xarg), _ptr(rcont), node, nsys, phase, st)
            if phase < 3:
                self.ode(xarg, arg, ks[phase], additionalArgs)
        return rcont

    def _eval(self, t_new, t_old, spline_coeffs, order):
        d = self.device
        t_new = _dev64(t_new, d).reshape(-1)
        t_old = _dev64(t_old, d).reshape(-1)
        c = _dev64(spline_coeffs, d)
        assert c.dim() == 3 and c.shape[-1] == 8
        if c.shape[0] != t_old.numel() - 1:
            raise ValueError("spline_coeffs must hold one basis per interval of t_old")
        t_min, t_max = float(t_old.min()), float(t_old.max())
        if t_new.numel() and not bool(((t_min <= t_new) & (t_new <= t_max)).all()):
            raise ValueError(f"All t_new values must be between t_min ({t_min}) and t_max ({t_max}).")
        node = c.shape[1]
        out = torch.empty((t_new.numel(), node), dtype=torch.float64, device=d)
        _lib.call("few_dopr853_eval", _ptr(t_new), t_new.numel(), _ptr(t_old), t_old.numel(), _ptr(c), node, order,
                  _ptr(out), _stream(d))
        return out

    def eval(self, t_new, t_old, spline_coeffs):
        """The basis at t_new (dopr853.py:760-803): (npts, node)."""
        assert not self.fix_step
        return self._eval(t_new, t_old, spline_coeffs, 0)

    def eval_derivative(self, t_new, t_old, spline_coeffs, order: int = 1):
        """d^order/dt^order of the basis at t_new (dopr853.py:805-875), order
        0..3: (npts, node)."""
        if order not in (0, 1, 2, 3):
            raise ValueError("order must be 0, 1, 2 or 3")
        return self._eval(t_new, t_old, spline_coeffs, order)
