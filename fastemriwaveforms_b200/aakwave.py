"""AAK waveform summation on the GPU.

Drop-in for ``few.summation.aakwave.AAKSummation``
(``src/few/summation/aakwave.py:12-196``): the same ``sum`` arguments (tvec,
m1, a, dist, m2, qS, phiS, qK, phiK, nmodes, interp_t, interp_coeffs; mich,
dt, integrate_backwards), the same pole shift of qS and qK, the same
equatorial substitution Phi_theta := Phi_phi when |Y| == 1, and the waveform
hI - i hII in ``self.waveform``.  The kernel is ``k_aak`` (``csrc/aak.cu``),
reached through ``few_aak_sum`` on device tables (asynchronous);
``few_aak_waveform`` is the reference-shaped entry (its ``get_waveform`` of
``gpuAAK.hh``).  The caller's ``interp_coeffs`` is not modified (the
reference writes the substitution into it).
"""
from __future__ import annotations

import logging

import numpy as np
import torch

from . import _lib
from .summation import SummationBase, _ptr, _stream, _to_host, _upload

logger = logging.getLogger("fastemriwaveforms_b200")


class AAKSummation(SummationBase):
    """Augmented analytic kludge waveform from an input trajectory."""

    def __init__(self, force_backend=None, device=None, **kwargs):
        kw = {k: v for k, v in kwargs.items() if k in ("output_type", "pad_output", "odd_len")}
        SummationBase.__init__(self, device=device, **kw)

    def sum(self, tvec, m1, a, dist, m2, qS, phiS, qK, phiK, nmodes, interp_t, interp_coeffs, *args, mich=False,
            dt=10.0, integrate_backwards=False, **kwargs):
        fill = 1e-6
        if qK < fill or qK > np.pi - fill:
            logger.warning("qK is within 1e-6 of the poles. We shift this value automatically away from poles by 1e-6.")
            qK = fill if qK < fill else np.pi - fill
        if qS < fill or qS > np.pi - fill:
            logger.warning("qS is within 1e-6 of the poles. We shift this value automatically away from poles by 1e-6.")
            qS = fill if qS < fill else np.pi - fill
        it = _to_host(interp_t, np.float64)
        init_len = len(it)
        if integrate_backwards:
            tv = _to_host(tvec, np.float64)
            offset = tv[-1] - int(tv[-1] / dt) * dt
            it = it - offset
        dev = self.device
        if isinstance(interp_coeffs, torch.Tensor):
            c = interp_coeffs.to(device=dev, dtype=torch.float64)
        else:
            c = torch.as_tensor(np.asarray(interp_coeffs, dtype=np.float64), device=dev)
        if c.ndim != 3 or tuple(c.shape[1:]) != (6, 8) or c.shape[0] != init_len - 1:
            raise ValueError("interp_coeffs must have shape (len(interp_t) - 1, 6, 8).")
        if abs(float(c[0, 2, 0])) == 1.0:  # equatorial: Phi_theta follows Phi_phi (aakwave.py:170-171)
            c = c.clone()
            c[:, 4] = c[:, 3]
        coeffs = c.permute(2, 0, 1).contiguous()  # (8, N-1, 6), the kernel's layout
        first = aak_segments(it, int(self.num_pts), float(dt))
        nseg = len(first) - 1
        if nseg < 1:
            return
        t_d = _upload(np.ascontiguousarray(it), dev)
        first_d = _upload(first, dev)
        _lib.call("few_aak_sum", _ptr(self.waveform), _ptr(coeffs), init_len - 1, _ptr(t_d), _ptr(first_d), nseg,
                  int(first[-1]), float(m1), float(a), float(m2), float(qS), float(phiS), float(qK), float(phiK),
                  float(dist), int(nmodes), int(bool(mich)), float(dt), _stream(dev))


def aak_segments(h_t: np.ndarray, out_len: int, dt: float) -> np.ndarray:
    """First sample of each trajectory segment (gpuAAK.cu:495-519): ceil(t_j / dt)
    while t_j < T = (out_len - 1) dt; the first knot at or past T closes the
    list with out_len.  (nseg + 1,) int32."""
    T = (out_len - 1) * dt
    tail = np.asarray(h_t[1:], dtype=np.float64)
    past = np.nonzero(tail >= T)[0]
    if len(past):
        k = int(past[0])
        first = np.concatenate([[0], np.ceil(tail[:k] / dt), [out_len]])
    else:
        first = np.concatenate([[0], np.ceil(tail / dt)])
    return first.astype(np.int32)
