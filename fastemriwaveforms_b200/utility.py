"""Overlap and mismatch of two waveforms (``src/few/utils/utility.py:16-95``).

Both are computed in the frequency domain as the reference does:
overlap = Re <a, b> / sqrt(<a, a> <b, b>) over FFTs of the common prefix.
Accepts numpy arrays or torch tensors (evaluated with torch on their device).
"""
from __future__ import annotations

import logging

import numpy as np
import torch

logger = logging.getLogger("few")


def _as_tensor(x):
    if isinstance(x, torch.Tensor):
        return x
    return torch.from_numpy(np.ascontiguousarray(np.asarray(x, dtype=np.complex128)))


def get_overlap(time_series_1, time_series_2, use_gpu: bool = False) -> float:
    a = _as_tensor(time_series_1).to(torch.complex128)
    b = _as_tensor(time_series_2).to(torch.complex128)
    if use_gpu and a.device.type == "cpu":
        a = a.cuda()
    b = b.to(a.device)
    min_len = int(min(a.shape[0], b.shape[0]))
    if a.shape[0] != b.shape[0]:
        logger.warning("The two time series are not the same length (%d vs %d). The calculation will run with "
                       "length %d starting at index 0 for both arrays.", a.shape[0], b.shape[0], min_len)
    fa = torch.fft.fft(a[:min_len])
    fb = torch.fft.fft(b[:min_len])
    ac = torch.vdot(fa, fb) / torch.sqrt(torch.vdot(fa, fa) * torch.vdot(fb, fb))
    return float(ac.real.item())


def get_mismatch(time_series_1, time_series_2, use_gpu: bool = False) -> float:
    """1 - overlap."""
    return 1.0 - get_overlap(time_series_1, time_series_2, use_gpu=use_gpu)
