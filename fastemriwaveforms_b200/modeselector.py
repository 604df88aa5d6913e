"""Mode selection on the GPU.

Drop-in for ``few.utils.modeselector.ModeSelector``
(``src/few/utils/modeselector.py:14-490``): built on an amplitude generator
that exposes the reference's mode attributes (``l_arr_no_mask``,
``m_arr_no_mask``, ``k_arr_no_mask``, ``n_arr_no_mask``, ``unique_l``,
``unique_m``, ``inverse_lm``, ``index_map_arr``) and is called as
``amplitude_generator(a, p, e, xI, specific_modes=None)``; the same three
selection forms ("all", a list of (l, m, k, n), the power threshold) and the
same outputs (teuk_modes, ylms, l, m, k, n).

The threshold form runs on the device: ``k_mode_snr2`` (``csrc/modeselect.cu``)
fuses the per-mode power |A Y|^2 (+ |conj(A) Y^-|^2 for m != 0), the optional
sensitivity weights and the knot-interval sum; torch sorts the K estimates;
``k_mode_keep`` applies the cumulative rule in sorted order.  ``GetYlms`` from
``fastemriwaveforms_b200.ylm`` is the default harmonic generator.

Deliberate difference: with ``include_minus_mkn=False`` outside the list form
the reference warns that it overrides the flag to True but then indexes a
missing mode list; here the override is applied.
"""
from __future__ import annotations

import logging

import numpy as np
import torch

from . import _lib
from .summation import _device, _ptr, _stream
from .ylm import GetYlms

logger = logging.getLogger("fastemriwaveforms_b200")


def get_mode_frequencies(f_phi, f_theta, f_r, m, k, n):
    """Mode frequencies (N, K) along the trajectory (modeselector.py:8-11)."""
    return f_phi[:, None] * m[None, :] + f_theta[:, None] * k[None, :] + f_r[:, None] * n[None, :]


def _t(x, dtype, dev):
    if isinstance(x, torch.Tensor):
        return x.to(device=dev, dtype=dtype)
    return torch.as_tensor(np.asarray(x), dtype=dtype, device=dev)


class ModeSelector:
    """Filters the Teukolsky modes of a trajectory by estimated power, or by
    a requested list (reference: ``modeselector.py:14-490``)."""

    def __init__(self, amplitude_generator, ylm_generator=None, mode_selection=None, include_minus_mkn=True,
                 mode_selection_threshold: float = 1e-5, sensitivity_fn=None, modeinds_map=None, force_backend=None,
                 device=None, **kwargs):
        self._device_arg = device
        dev = self.device
        self.amplitude_generator = amplitude_generator
        self.ylm_generator = GetYlms(device=device) if ylm_generator is None else ylm_generator
        g = amplitude_generator
        self.l_arr, self.m_arr, self.k_arr, self.n_arr = (
            _t(v, torch.int64, dev) for v in (g.l_arr_no_mask, g.m_arr_no_mask, g.k_arr_no_mask, g.n_arr_no_mask))
        self.unique_l, self.unique_m = _t(g.unique_l, torch.int64, dev), _t(g.unique_m, torch.int64, dev)
        self.inverse_lm = _t(g.inverse_lm, torch.int64, dev)
        if bool((self.m_arr < 0).any()):
            raise AssertionError("ModeSelector only supports m >= 0.")
        self.m0mask = self.m_arr != 0
        self.num_m_zero_up = int(self.m0mask.numel())
        self.num_m_1_up = int(self.m0mask.sum())
        self.num_m0 = self.num_m_zero_up - self.num_m_1_up
        self.sensitivity_fn = sensitivity_fn
        self.include_minus_mkn = include_minus_mkn
        self.mode_selection = mode_selection
        self.negative_m_flag = False
        if isinstance(mode_selection, str) and mode_selection not in ("all", "threshold"):
            raise ValueError("If mode_selection is a string, it must be either 'all', 'threshold', or None.")
        if isinstance(mode_selection, list):
            self.mode_arr = self._check_list(mode_selection, include_minus_mkn, warn_only=True)
        else:
            self.mode_arr = None
        self.mode_selection_threshold = mode_selection_threshold
        self.modeinds_map = _t(g.index_map_arr if modeinds_map is None else modeinds_map, torch.int64, dev)
        if self.modeinds_map.ndim != 4:
            raise AssertionError("Modeinds map must be a 4D array.")

    @property
    def device(self) -> torch.device:
        return _device(self._device_arg)

    def _check_list(self, sel, include_minus_mkn, warn_only=False):
        if len(sel) == 0:
            raise ValueError("If mode selection is a list, cannot be empty.")
        arr = np.asarray(sel, dtype=np.int64).reshape(len(sel), -1)
        if len(np.unique(arr, axis=0)) != len(arr):
            raise ValueError("Mode selection has duplicate modes.")
        if np.any(arr[:, 1] < 0):
            if warn_only:
                logger.warning("(ModeSelector) Warning: Only supports mode_selection with m < 0 if "
                               "include_minus_mkn = False. May lead to error during evaluation.")
                self.negative_m_flag = True
            elif include_minus_mkn:
                raise ValueError("Only supports mode_selection with m >= 0 when include_minus_mkn = True.")
        if np.any(np.abs(arr[:, 1]) > arr[:, 0]):
            raise ValueError("Mode selection has unphysical |m| > l mode(s).")
        if np.any(arr[:, 0] < 2):
            raise ValueError("Mode selection has unphysical l < 2 mode(s).")
        return torch.as_tensor(arr, device=self.device)

    def _ylms_of_list(self, theta, phi):
        y = self.ylm_generator(self.unique_l, self.unique_m, theta, phi)
        return y[self.inverse_lm]

    def _minus_index(self):
        """ylms index of each mode's -m harmonic (the m != 0 modes in order after
        the K +m values), -1 for m = 0 (modeselector.py:400-405)."""
        K = self.num_m_zero_up
        idx = torch.full((K,), -1, dtype=torch.int32, device=self.device)
        nz = torch.nonzero(self.m0mask).reshape(-1)
        idx[nz] = (K + torch.arange(nz.numel(), device=self.device)).to(torch.int32)
        return idx

    def __call__(self, t, a, p, e, xI, theta, phi, online_mode_selection_args=None, mode_selection=None,
                 include_minus_mkn=None, mode_selection_threshold=None, return_sort_inds=False):
        dev = self.device
        if include_minus_mkn is None:
            include_minus_mkn = self.include_minus_mkn
        if mode_selection is None:
            mode_selection, mode_arr = self.mode_selection, self.mode_arr
            if self.negative_m_flag and include_minus_mkn:
                raise ValueError("Only supports mode_selection with m >= 0 when include_minus_mkn = True.")
        elif isinstance(mode_selection, str) and mode_selection not in ("all", "threshold"):
            raise ValueError("If mode_selection is a string, it must be either 'all', 'threshold', or None.")
        elif isinstance(mode_selection, list):
            mode_arr = self._check_list(mode_selection, include_minus_mkn)
        else:
            mode_arr = None
        if mode_selection_threshold is None:
            mode_selection_threshold = self.mode_selection_threshold
        if not include_minus_mkn and not isinstance(mode_selection, list):
            logger.warning("(ModeSelector) Warning: Overriding include_minus_mkn to True as mode_selection is not "
                           "a list.")
            include_minus_mkn = True

        def idx_of_ylm_minus(keep):
            return keep * (keep < self.num_m0) + (keep + self.num_m_1_up) * (keep >= self.num_m0)

        if mode_selection == "all":
            teuk = _t(self.amplitude_generator(a, p, e, xI), torch.complex128, dev)
            ylms = self._ylms_of_list(theta, phi)
            keep = torch.arange(teuk.shape[1], device=dev)
            ylms_out = ylms[torch.cat([keep, idx_of_ylm_minus(keep)])]
            return teuk, ylms_out, self.l_arr, self.m_arr, self.k_arr, self.n_arr
        if isinstance(mode_selection, list):
            try:
                keep = self.modeinds_map[mode_arr[:, 0], mode_arr[:, 1], mode_arr[:, 2], mode_arr[:, 3]]
            except IndexError:
                raise ValueError("Mode selection indices are out of bounds.")
            teuk = _t(self.amplitude_generator(a, p, e, xI, specific_modes=keep), torch.complex128, dev)
            ylms_out = self.ylm_generator(mode_arr[:, 0], mode_arr[:, 1], theta, phi, include_minus_m=True)
            if not include_minus_mkn:
                ylms_out[teuk.shape[1]:] = 0.0
            return teuk, ylms_out, mode_arr[:, 0], mode_arr[:, 1], mode_arr[:, 2], mode_arr[:, 3]

        # threshold form (modeselector.py:393-486)
        teuk = _t(self.amplitude_generator(a, p, e, xI), torch.complex128, dev).contiguous()
        ylms = self._ylms_of_list(theta, phi).contiguous()
        N, K = teuk.shape
        t_d = _t(t, torch.float64, dev).contiguous()
        psd = None
        if self.sensitivity_fn is not None:
            f = online_mode_selection_args
            freqs = get_mode_frequencies(_t(f["f_phi"], torch.float64, dev), _t(f["f_theta"], torch.float64, dev),
                                         _t(f["f_r"], torch.float64, dev), self.m_arr.double(), self.k_arr.double(),
                                         self.n_arr.double()).abs()
            psd = _t(self.sensitivity_fn(freqs.flatten()), torch.float64, dev).reshape(freqs.shape).contiguous()
        snr2 = torch.empty(K, dtype=torch.float64, device=dev)
        minus = self._minus_index()
        st = _stream(dev)
        _lib.call("few_mode_snr2", _ptr(teuk), N, K, _ptr(ylms), _ptr(minus), _ptr(psd) if psd is not None else None,
                  _ptr(t_d), _ptr(snr2), st)
        vals, inds_sort = torch.sort(snr2, descending=True, stable=True)
        keep_flag = torch.empty(K, dtype=torch.int32, device=dev)
        _lib.call("few_mode_keep", _ptr(vals), K, float(mode_selection_threshold), _ptr(keep_flag), st)
        keep_tmp = inds_sort[keep_flag.bool()]
        keep_tmp = keep_tmp * (keep_tmp < self.num_m_zero_up) + (keep_tmp - self.num_m_1_up) * (
            keep_tmp >= self.num_m_zero_up)
        keep, inv = torch.unique(keep_tmp, sorted=True, return_inverse=True)
        ylms_out = ylms[torch.cat([keep, idx_of_ylm_minus(keep)])]
        out = (teuk[:, keep], ylms_out, self.l_arr[keep], self.m_arr[keep], self.k_arr[keep], self.n_arr[keep])
        if return_sort_inds:
            out += (inv,)
        return out
