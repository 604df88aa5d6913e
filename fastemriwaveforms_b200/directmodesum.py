"""Direct mode sum on the GPU.

Drop-in for ``few.summation.directmodesum.DirectModeSum``
(``src/few/summation/directmodesum.py:11-131``): amplitudes (len(t), K) and
phases (3, len(t)) given at every output sample, summed over modes with the
-m images of the m > 0 modes; ``self.waveform`` holds len(t) samples, as the
reference's does.  The kernel is ``k_direct_sum`` (``csrc/directsum.cu``).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .summation import SummationBase, _input, _ptr, _stream, _to_device, _to_host


class DirectModeSum(SummationBase):
    """Sums the amplitude and phase information as received."""

    def __init__(self, *args, force_backend=None, device=None, **kwargs):
        kw = {k: v for k, v in kwargs.items() if k in ("output_type", "pad_output", "odd_len")}
        SummationBase.__init__(self, device=device, **kw)

    def sum(self, t, teuk_modes, ylms, phase_interp_t, phases_in, l_arr, m_arr, k_arr, n_arr, *args, dt=10.0,
            integrate_backwards=False, **kwargs):
        if integrate_backwards:
            raise NotImplementedError
        dev = self.device
        teuk = _input(teuk_modes, torch.complex128, dev).contiguous()
        if teuk.ndim != 2:
            raise ValueError("teuk_modes must have shape (len(t), num_teuk_modes).")
        N, K = (int(v) for v in teuk.shape)
        y = _input(ylms, torch.complex128, dev).reshape(-1).contiguous()
        if y.numel() != 2 * K:
            raise ValueError("ylms must hold 2 * num_teuk_modes values (+m, then -m).")
        if isinstance(phases_in, torch.Tensor):
            ph = phases_in.to(device=dev, dtype=torch.float64).contiguous()
        else:
            ph = torch.stack([_input(p, torch.float64, dev).reshape(-1) for p in phases_in]).contiguous()
        if tuple(ph.shape) != (3, N):
            raise ValueError("phases_in must hold (Phi_phi, Phi_theta, Phi_r), each of len(t) values.")
        l_d, m_d, k_d, n_d = (_to_device(_to_host(v, np.int32), torch.int32, dev) for v in (l_arr, m_arr, k_arr, n_arr))
        out = torch.empty(N, dtype=torch.complex128, device=dev)
        _lib.call("few_direct_sum", _ptr(teuk), _ptr(y), _ptr(ph), _ptr(l_d), _ptr(m_d), _ptr(k_d), _ptr(n_d), N, K,
                  _ptr(out), _stream(dev))
        self.waveform = out
