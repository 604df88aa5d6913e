"""Frequency-domain interpolated mode sum on the GPU.

Drop-in for ``few.summation.fdinterp.FDInterpolatedModeSum``
(``src/few/summation/fdinterp.py:92-542``): the same constructor options
(``output_type="fd"`` is implied), ``sum`` arguments, attributes
(``waveform`` of shape (2, L) with rows h+ and hx, ``frequency``) and errors.

Every stage runs on the device, on the caller's stream:

1. the trajectory's fundamental frequencies in Hz (``few_fundamental_frequencies``),
2. not-a-knot splines of the amplitudes and of the three frequencies,
3. the turnover search on the 5000-point dense grid (``few_fd_plan_extrema``),
4. each (mode, segment)'s frequency-bin range (``few_fd_plan_bins``) and the
   prefix of the bin counts (``few_fd_scan``),
5. the stationary-phase sum (``few_fd_sum``) and the (h+, hx) assembly
   (``few_fd_finalize``).

The call synchronises once at the end to raise the reference's errors
(a turnover segment holding two roots, a negative discriminant below -1e10,
an elliptic modulus out of range).  ``separate_modes=True`` is refused: the
reference kernel writes mode_i * data_length + i into a buffer of data_length
elements (``interpolate.cu:1512``).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .geodesic import MTSUN_SI, fundamental_frequencies_into
from .summation import SummationBase, _device, _input, _ptr, _stream, _to_device, _to_host, spline_factor_table

DENSE_POINTS = 5000  # dense grid of the turnover search (fdinterp.py:266)


def _linspace_params(t0: float, t1: float, num: int):
    """numpy.linspace(t0, t1, num): y_j = j*step + t0 (j < num-1), y_{num-1} = t1."""
    step = (t1 - t0) / (num - 1)
    return t0, step, t1


class FDInterpolatedModeSum(SummationBase):
    """Frequency-domain waveform from a sparse trajectory by the stationary
    phase approximation (reference: ``fdinterp.py:92-542``)."""

    def __init__(self, force_backend=None, device=None, **kwargs):
        kw = {k: v for k, v in kwargs.items() if k in ("pad_output", "odd_len")}
        SummationBase.__init__(self, output_type="fd", device=device, **kw)
        self.frequency = None
        # optional (start, end) torch.cuda.Events recorded around the sum kernel
        self.sum_events = None
        # launch shape of the sum kernel (few_fd_sum): grid CTAs (0: 16 per SM) and
        # the register budget (resident CTAs per SM, 0: the default)
        self.sum_blocks = 0
        self.sum_ctas_per_sm = 0

    def sum(self, t, teuk_modes, ylms, phase_interp_t, phase_interp_coeffs, l_arr, m_arr, k_arr, n_arr, M, a, p, e,
            xI, *args, include_minus_m=True, separate_modes=False, dt=10.0, f_arr=None, mask_positive=False,
            integrate_backwards=False, host_out=None, **kwargs):
        dev = self.device
        N = len(t)
        p_d, e_d, x_d = (_to_device(np.atleast_1d(_to_host(v, np.float64)), torch.float64, dev) for v in (p, e, xI))
        for v in (p_d, e_d, x_d):
            if v.numel() != N:
                raise AssertionError("p, e and xI must hold one value per knot.")
        # frequencies in Hz at the knots (fdinterp.py:224-242)
        fk = torch.empty((3, N), dtype=torch.float64, device=dev)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        a_arg = a if not hasattr(a, "__len__") else _to_device(_to_host(a, np.float64), torch.float64, dev)
        fundamental_frequencies_into(a_arg, p_d, e_d, x_d, fk[0], fk[1], fk[2], denom=2 * np.pi * M * MTSUN_SI,
                                     abs_phi=True, status=status)
        self.sum_with_frequencies(t, teuk_modes, ylms, phase_interp_t, phase_interp_coeffs, l_arr, m_arr, k_arr,
                                  n_arr, fk, include_minus_m=include_minus_m, separate_modes=separate_modes, dt=dt,
                                  f_arr=f_arr, mask_positive=mask_positive, host_out=host_out,
                                  _geodesic_status=status)

    def sum_with_frequencies(self, t, teuk_modes, ylms, phase_interp_t, phase_interp_coeffs, l_arr, m_arr, k_arr,
                             n_arr, frequencies, include_minus_m=True, separate_modes=False, dt=10.0, f_arr=None,
                             mask_positive=False, host_out=None, _geodesic_status=None):
        """``sum`` with the trajectory's frequencies given instead of (M, a, p,
        e, xI): ``frequencies`` (3, len(t)) = (|f_phi|, f_theta, f_r) in Hz at
        the knots (an extension for callers whose trajectory already carries
        them).  Needs ``self.num_pts`` / ``self.num_pts_pad`` (set by
        ``__call__``) unless f_arr is given.  ``host_out`` (extension): a
        pinned complex128 CPU tensor of the output's shape that receives the
        (h+, hx) result as well."""
        if separate_modes:
            raise ValueError("separate_modes=True is not supported: the reference kernel writes each mode at "
                             "mode_i * data_length + i of a data_length buffer (interpolate.cu:1512).")
        dev = self.device
        st = _stream(dev)
        t_h = _to_host(t, np.float64)
        N = len(t_h)
        teuk = _input(teuk_modes, torch.complex128, dev)
        if teuk.ndim != 2 or teuk.shape[0] != N:
            raise ValueError("teuk_modes must have shape (len(t), num_teuk_modes).")
        K = int(teuk.shape[1])
        l_h, m_h, k_h, n_h = (_to_host(v, np.int32) for v in (l_arr, m_arr, k_arr, n_arr))
        m_d, k_d, n_d = (_to_device(v, torch.int32, dev) for v in (m_h, k_h, n_h))
        y_d = _input(ylms, torch.complex128, dev).reshape(-1)
        if y_d.numel() != 2 * K:
            raise ValueError("ylms must hold 2 * num_teuk_modes values (+m, then -m).")
        # (-1)^l on the -m half (fdinterp.py:486-487)
        sgn = torch.from_numpy(np.where(l_h % 2 == 0, 1.0, -1.0)).to(dev, non_blocking=True)
        y_d = torch.cat([y_d[:K], y_d[K:] * sgn])
        pt = _to_device(_to_host(phase_interp_t, np.float64), torch.float64, dev)
        pc = _input(phase_interp_coeffs, torch.float64, dev)
        if tuple(pc.shape) != (N - 1, 3, 8):
            raise ValueError("phase_interp_coeffs must have shape (len(t) - 1, 3, 8).")
        t_d = _to_device(t_h, torch.float64, dev)
        fk = _to_device(frequencies, torch.float64, dev)
        if tuple(fk.shape) != (3, N):
            raise ValueError("frequencies must have shape (3, len(t)).")
        status = torch.zeros(2, dtype=torch.int32, device=dev)  # planning flags, turnover count

        # 2. splines: amplitudes (4, N, 2K) knot-major, frequencies (4, N, 3)
        amp = torch.empty((4, N, 2 * K), dtype=torch.float64, device=dev)
        fac = spline_factor_table(t_h, dev)
        tv = torch.view_as_real(teuk)
        _lib.call("few_spline_build_factored", _ptr(fac), _ptr(tv), 2 * K, 2, K, 1, 2 * K, N, _ptr(amp),
                  _lib.FEW_LAYOUT_KNOT_MAJOR, st)
        fco = torch.empty((4, N, 3), dtype=torch.float64, device=dev)
        _lib.call("few_spline_build", _ptr(t_d), 0, _ptr(fk), 1, N, 3, 0, 3, N, _ptr(fco), _lib.FEW_LAYOUT_KNOT_MAJOR,
                  st)

        # 3. turnover search (fdinterp.py:262-376)
        t0, step, t1 = _linspace_params(float(t_h.min()), float(t_h.max()), DENSE_POINTS)
        tn = _to_device(np.linspace(t_h.min(), t_h.max(), DENSE_POINTS), torch.float64, dev)
        fdense = torch.empty((3, DENSE_POINTS), dtype=torch.float64, device=dev)
        eflags = torch.zeros(2, dtype=torch.int32, device=dev)
        _lib.call("few_spline_eval", _ptr(t_d), 0, _ptr(fco), 3, N, _ptr(tn), 0, DENSE_POINTS, 0, _ptr(fdense),
                  _ptr(eflags), st)
        turns = torch.empty(2 * K * _lib.load().few_fd_turn_bytes(), dtype=torch.uint8, device=dev)
        _lib.call("few_fd_plan_extrema", _ptr(fdense), DENSE_POINTS, t0, step, t1, _ptr(t_d), N, _ptr(fco), _ptr(m_d),
                  _ptr(k_d), _ptr(n_d), K, _ptr(turns), _ptr(status), st)

        # 4. frequency grid and bin ranges (fdinterp.py:378-430)
        if f_arr is not None:
            freq_h = _to_host(f_arr, np.float64)
            if len(freq_h) == 0:
                raise ValueError("Input f_arr kwarg has zero length.")
            self.frequency = _to_device(freq_h, torch.float64, dev)
            L = len(freq_h)
            if np.sum(freq_h == 0.0) != 1:
                raise AssertionError("the frequency array must hold exactly one zero")
            zero_index = int(np.where(freq_h == 0.0)[0][0])
            if zero_index != int(L / 2):
                raise AssertionError("the zero frequency must sit at index len(frequency) // 2")
            f0, df = float(freq_h[0]), float(freq_h[1] - freq_h[0])
            fpos1 = float(freq_h[zero_index + 1]) if zero_index + 1 < L else 0.0
            has_farr = 1
            first_pos = int(np.argmax(freq_h >= 0.0))
            npos = int(np.sum(freq_h >= 0.0))
        else:
            L = self.num_pts + self.num_pts_pad
            Ldt = L * dt
            self.frequency = torch.empty(L, dtype=torch.float64, device=dev)
            _lib.call("few_fd_frequency_grid", _ptr(self.frequency), L, float(Ldt), st)
            zero_index = L // 2
            f0 = float(np.float64(-(L // 2)) / Ldt)
            df = float(np.float64(1 - L // 2) / Ldt - f0) if L > 1 else 0.0
            fpos1 = 0.0
            has_farr = 0
            first_pos, npos = zero_index, L - zero_index
        E = K * (N - 1)
        start32 = torch.empty(E, dtype=torch.int32, device=dev)
        end32 = torch.empty(E, dtype=torch.int32, device=dev)
        lo = torch.empty(E, dtype=torch.int32, device=dev)
        count = torch.empty(E, dtype=torch.int64, device=dev)
        _lib.call("few_fd_plan_bins", _ptr(fk), _ptr(m_d), _ptr(k_d), _ptr(n_d), K, N, _ptr(turns), _ptr(status),
                  f0, df, has_farr, fpos1, zero_index, L, _ptr(start32), _ptr(end32), _ptr(lo), _ptr(count), st)
        prefix = torch.empty(E + 1 + 1024, dtype=torch.int64, device=dev)  # prefix, then the scan's scratch
        _lib.call("few_fd_scan", _ptr(count), E, _ptr(prefix), _ptr(prefix[E + 1:]), st)
        self.seg_start_inds, self.seg_end_inds = start32.view(K, N - 1), end32.view(K, N - 1)

        # 5. the sum and (h+, hx)
        wf = torch.zeros(L, dtype=torch.complex128, device=dev)
        if self.sum_events is not None:
            self.sum_events[0].record()
        _lib.call("few_fd_sum", _ptr(wf), L, _ptr(self.frequency), zero_index, int(bool(include_minus_m)), _ptr(amp),
                  N * 2 * K, 1, 2 * K, _ptr(fco), 3 * N, 1, 3, _ptr(pc), 1, 8, 24, _ptr(pt), _ptr(t_d), N, _ptr(m_d),
                  _ptr(k_d), _ptr(n_d), K, _ptr(y_d), _ptr(lo), _ptr(prefix), self.sum_blocks, self.sum_ctas_per_sm, st)
        if self.sum_events is not None:
            self.sum_events[1].record()
        self.total_bins = prefix[E]  # device scalar: bins the sum visited
        first, cnt = (first_pos, npos) if mask_positive else (0, L)
        out = torch.empty((2, cnt), dtype=torch.complex128, device=dev)
        _lib.call("few_fd_finalize", _ptr(wf), L, first, cnt, _ptr(out), st)
        self.waveform = out
        if host_out is not None:
            if (not isinstance(host_out, torch.Tensor) or host_out.device.type != "cpu" or not host_out.is_pinned()
                    or host_out.dtype != torch.complex128 or tuple(host_out.shape) != tuple(out.shape)):
                raise ValueError(f"host_out must be a pinned complex128 CPU tensor of shape {tuple(out.shape)}")
            host_out.copy_(out, non_blocking=True)

        # the one synchronisation: the reference's errors
        if _geodesic_status is not None and int(_geodesic_status.item()) & 1:
            raise ValueError("Elliptic integral K(k) valid only for k in [0, 1].")
        flags = int(status[0].item())
        if flags & 2:
            raise ValueError("a turnover segment holds both roots of the frequency derivative "
                             "(the reference stops at a breakpoint(), fdinterp.py:353-354)")
        if flags & 4:
            raise ValueError("turnover discriminant below -1e10 (the reference stops at a breakpoint(), "
                             "fdinterp.py:335-336)")
