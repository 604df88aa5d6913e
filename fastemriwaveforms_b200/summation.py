"""Drop-in ``CubicSplineInterpolant`` and ``InterpolatedModeSum`` on B200.

Mirrors ``few.summation.interpolatedmodesum`` (src/few/summation/interpolatedmodesum.py)
and ``few.summation.base.SummationBase`` (src/few/summation/base.py): same
class names, call signatures, attribute names, output layout and ValueErrors.
Arrays may be numpy arrays or torch tensors; results are torch tensors on the
CUDA device (the reference returns cupy arrays on its GPU backend), e.g.
``waveform.cpu().numpy()`` in place of cupy's ``.get()``.

All arithmetic runs in the CUDA kernels of libfew_b200.so; there is no CPU
path.  Extra keyword ``precision`` of ``InterpolatedModeSum``:

* ``"faithful"`` (default) -- FP64, replays the reference's rounding of each
  mode phase, so results match the reference CPU path to ~1e-15 relative L2;
* ``"exact"`` -- FP64, mode phasors by recurrence with no rounding of the
  combined phase (more accurate than the reference, ~2x less FP64 work);
* ``"mixed"`` -- FP64 phases and anchors, FP32 phasor recurrence, the
  per-segment contraction on the tcgen05 tensor cores in split BF16 with FP32
  accumulation (waveform mismatch ~1e-10 against FP64).

Keyword ``backward`` chooses the adjoint used when gradients are requested:
``"fp64"`` (the default for the FP64 forms) or ``"mixed"`` (the default for
``precision="mixed"``): the amplitude gradient's per-segment contraction over
samples and the phase gradient's per-sample sums on the tensor cores, with the
precision plan of the mixed forward.
"""
from __future__ import annotations

import logging
from collections import OrderedDict

import numpy as np
import torch

from . import _lib
from .synthetic import YRSID_SI, output_length

logger = logging.getLogger("few")

_PRECISIONS = {"faithful": _lib.FEW_SUM_FAITHFUL, "exact": _lib.FEW_SUM_EXACT, "mixed": -1}
DEFAULT_CHUNK = 1024  # output samples per work unit of the sum kernel


def _device(device=None) -> torch.device:
    if device is not None:
        return torch.device(device)
    if not torch.cuda.is_available():
        raise RuntimeError("fastemriwaveforms_b200 needs a CUDA device (B200); no CPU path exists")
    return torch.device("cuda", torch.cuda.current_device())


def _stream(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def _to_device(x, dtype, device) -> torch.Tensor:
    if isinstance(x, torch.Tensor):
        return x.to(device=device, dtype=dtype).contiguous()
    a = np.asarray(x)
    if dtype.is_complex:
        a = a.astype(np.complex128, copy=False)
    elif dtype == torch.float64:
        a = a.astype(np.float64, copy=False)
    elif dtype == torch.int32:
        a = a.astype(np.int32, copy=False)
    return _upload(a, device)


def _upload(a: np.ndarray, device) -> torch.Tensor:
    """Host array -> device through pinned staging, without blocking the host:
    a copy from pageable memory would wait for the kernels already queued on
    the stream, leaving the GPU idle while the next call is planned.  torch's
    pinned-block cache keeps the staging buffer alive until the copy is done."""
    t = torch.from_numpy(np.ascontiguousarray(a))
    if torch.device(device).type != "cuda":
        return t.to(device)
    return t.pin_memory().to(device, non_blocking=True)


_COPY_STREAMS: dict = {}


def _copy_stream(device) -> torch.cuda.Stream:
    d = torch.device(device)
    key = d.index if d.index is not None else torch.cuda.current_device()
    if key not in _COPY_STREAMS:
        _COPY_STREAMS[key] = torch.cuda.Stream(torch.device("cuda", key))
    return _COPY_STREAMS[key]


_D2H_STREAMS: dict = {}


def _download_stream(device) -> torch.cuda.Stream:
    d = torch.device(device)
    key = d.index if d.index is not None else torch.cuda.current_device()
    if key not in _D2H_STREAMS:
        _D2H_STREAMS[key] = torch.cuda.Stream(torch.device("cuda", key))
    return _D2H_STREAMS[key]


_SIDE_STREAMS: dict = {}


def _side_stream(device) -> torch.cuda.Stream:
    """A second compute stream per device (the phase branch of a backward)."""
    d = torch.device(device)
    key = d.index if d.index is not None else torch.cuda.current_device()
    if key not in _SIDE_STREAMS:
        _SIDE_STREAMS[key] = torch.cuda.Stream(torch.device("cuda", key))
    return _SIDE_STREAMS[key]


def _input(x, dtype, device) -> torch.Tensor:
    """A user input on the device.  Device tensors (and host tensors that
    require grad) go through torch's ``.to``; host data is copied on a separate
    copy stream, so the copy does not queue behind kernels already on the
    caller's stream (the next call's inputs arrive while the previous call's
    kernels run).  The caller's stream waits for the copy, and the call returns
    only once the copy has read the caller's buffer, as a blocking copy would."""
    if isinstance(x, torch.Tensor) and (x.is_cuda or x.requires_grad or torch.device(device).type != "cuda"):
        return x.to(device=device, dtype=dtype).contiguous()
    if isinstance(x, torch.Tensor):
        src = x.detach().to(dtype).contiguous()
    else:
        a = np.asarray(x)
        a = a.astype(np.complex128 if dtype.is_complex else np.float64, copy=False)
        src = torch.from_numpy(np.ascontiguousarray(a))
    pinned = src if src.is_pinned() else src.pin_memory()
    cs = _copy_stream(device)
    with torch.cuda.stream(cs):
        dst = torch.empty(pinned.shape, dtype=pinned.dtype, device=device)
        dst.copy_(pinned, non_blocking=True)
    main = torch.cuda.current_stream(device)
    main.wait_stream(cs)
    dst.record_stream(main)
    if pinned is src and (isinstance(x, torch.Tensor) and pinned.data_ptr() == x.data_ptr()):
        cs.synchronize()  # the copy reads the caller's own pinned buffer
    return dst


def _to_host(x, dtype) -> np.ndarray:
    if isinstance(x, torch.Tensor):
        x = x.detach().cpu().numpy()
    return np.ascontiguousarray(np.asarray(x), dtype=dtype)


def _ptr(t: torch.Tensor) -> int:
    return t.data_ptr()


def spline_factor_table(h_t: np.ndarray, device) -> torch.Tensor:
    """Device copy of the not-a-knot factorization for knots h_t (few_spline_factor)."""
    h_t = np.ascontiguousarray(h_t, dtype=np.float64)
    N = len(h_t)
    fac = np.zeros(_lib.FEW_FAC_WIDTH * (N + 1), np.float64)
    _lib.call("few_spline_factor", h_t.ctypes.data, N, fac.ctypes.data)
    return torch.from_numpy(fac).pin_memory().to(device, non_blocking=True)


class CubicSplineInterpolant:
    """Multiple not-a-knot cubic splines on the GPU
    (reference: ``interpolatedmodesum.py:12-257``).

    args:
        t: knots, shape (length,) shared by all interpolants or (ninterps, length).
        y_all: values, shape (length,) or (ninterps, length).
        device: CUDA device (default: the current one).
    """

    def __init__(self, t, y_all, device=None, **kwargs):
        dev = _device(device)
        self.device = dev
        y = _to_device(y_all, torch.float64, dev)
        if y.ndim == 1:
            y = y[None, :]
        if y.ndim != 2:
            raise ValueError("y_all must be 1 or 2 dimensions.")
        self.degree = 3
        ninterps, length = y.shape
        self.ninterps = int(ninterps)
        self.length = int(length)
        t_arr = t if isinstance(t, torch.Tensor) else np.asarray(t)
        if t_arr.ndim == 1:
            if len(t_arr) < 2:
                raise ValueError("t must have length greater than 2.")
            t_dev = _to_device(t_arr, torch.float64, dev)
            t_rs = 0
        elif t_arr.ndim == 2:
            if t_arr.shape[1] < 2:
                raise ValueError("t must have length greater than 2 along time axis.")
            t_dev = _to_device(t_arr, torch.float64, dev)
            if tuple(t_dev.shape) != (self.ninterps, self.length):
                raise ValueError("2D t must have shape (ninterps, length).")
            t_rs = self.length
        else:
            raise ValueError("t must be 1 or 2 dimensions.")
        if t_dev.shape[-1] != self.length:
            raise ValueError("t and y_all must have the same length along the time axis.")
        if self.length < 4:
            raise ValueError("not-a-knot cubic splines need at least 4 knots.")
        if not bool((t_dev[..., 1:] > t_dev[..., :-1]).all()):
            raise ValueError("t must increase strictly along the time axis.")
        self._t_knots = t_dev
        self._t_rs = t_rs
        coeffs = torch.empty((4, self.length, self.ninterps), dtype=torch.float64, device=dev)
        if t_rs == 0:
            # shared knots: factor once on the host, sweep per series on the device
            fac = spline_factor_table(t_dev.cpu().numpy(), dev)
            _lib.call("few_spline_build_factored", _ptr(fac), _ptr(y), 1, self.length, self.ninterps, 0,
                      self.ninterps, self.length, _ptr(coeffs), _lib.FEW_LAYOUT_KNOT_MAJOR, _stream(dev))
        else:
            _lib.call("few_spline_build", _ptr(t_dev), t_rs, _ptr(y), 1, self.length, self.ninterps, 0,
                      self.ninterps, self.length, _ptr(coeffs), _lib.FEW_LAYOUT_KNOT_MAJOR, _stream(dev))
        self.interp_array = coeffs.reshape(-1)
        """Flattened array containing all spline coefficients, (4, length, ninterps)."""
        self.reshape_shape = (self.degree + 1, self.length, self.ninterps)

    @property
    def t(self) -> torch.Tensor:
        """Knots, shape (ninterps, length)."""
        if self._t_rs == 0:
            return self._t_knots[None, :].expand(self.ninterps, self.length)
        return self._t_knots

    @property
    def y(self):
        return self.interp_array.reshape(self.reshape_shape)[0].T

    @property
    def c1(self):
        return self.interp_array.reshape(self.reshape_shape)[1].T

    @property
    def c2(self):
        return self.interp_array.reshape(self.reshape_shape)[2].T

    @property
    def c3(self):
        return self.interp_array.reshape(self.reshape_shape)[3].T

    def __call__(self, tnew, deriv_order: int = 0):
        """Evaluate every interpolant (or its derivative of order 1..3) at tnew.
        Points outside the knots take the edge values (deriv_order 0) or raise
        ValueError (derivatives), as ``interpolatedmodesum.py:161-257`` does."""
        if deriv_order not in (0, 1, 2, 3):
            raise ValueError("deriv_order must be within 0 <= deriv_order <= 3.")
        dev = self.device
        tn = _to_device(tnew, torch.float64, dev)
        if tn.ndim == 0:
            tn = tn[None]
        if tn.ndim == 2:
            if tn.shape[0] != self.ninterps:
                raise ValueError("If providing a 2D tnew array, must have same number of interpolants as was "
                                 "entered during initialization.")
            tn_rs = tn.shape[1]
        elif tn.ndim == 1:
            tn_rs = 0
        else:
            raise ValueError("tnew must be 1 or 2 dimensions.")
        M = int(tn.shape[-1])
        out = torch.empty((self.ninterps, M), dtype=torch.float64, device=dev)
        flags = torch.zeros(2, dtype=torch.int32, device=dev)
        _lib.call("few_spline_eval", _ptr(self._t_knots), self._t_rs, _ptr(self.interp_array), self.ninterps,
                  self.length, _ptr(tn), tn_rs, M, int(deriv_order), _ptr(out), _ptr(flags), _stream(dev))
        left, right = (bool(v) for v in flags.cpu().tolist())
        if left or right:
            if deriv_order != 0:
                raise ValueError("x points outside of the domain of the spline are not supported when taking "
                                 "derivatives.")
            logger.warning("(CubicSplineInterpolant) Warning: New t array outside bounds of input t array. "
                           "These points are filled with edge values.")
        return out.squeeze()


class SummationBase:
    """Output-length contract of ``src/few/summation/base.py:8-144``."""

    def __init__(self, output_type: str = "td", pad_output: bool = False, odd_len: bool = False,
                 force_backend=None, device=None):
        self.pad_output = pad_output
        self.odd_len = odd_len
        if output_type not in ["td", "fd"]:
            raise ValueError("{} waveform domain not available. Choices are 'td' (time domain) or 'fd' (frequency "
                             "domain).".format(output_type))
        self.output_type = output_type
        if self.output_type == "fd":
            self.odd_len = True
        self.num_pts = None
        self.num_pts_pad = None
        self.waveform = None
        self._device_arg = device

    @property
    def device(self) -> torch.device:
        return _device(self._device_arg)

    def sum(self, *args, **kwargs):
        raise NotImplementedError

    def __call__(self, t, *args, T: float = 1.0, dt: float = 10.0, **kwargs):
        t_last = float(t[-1].item() if hasattr(t[-1], "item") else t[-1])
        t_first = float(t[0].item() if hasattr(t[0], "item") else t[0])
        if not t_last > t_first:
            raise ValueError("t must increase: t[-1] <= t[0].")
        num_pts, num_pts_pad = output_length(np.array([t_first, t_last]), T, dt, self.pad_output, self.odd_len)
        if num_pts < 1:
            raise ValueError("the observation window holds no output sample.")
        self.num_pts = num_pts
        self.num_pts_pad = num_pts_pad
        self.dt = dt
        dev = self.device
        if self.output_type == "fd" and "f_arr" in kwargs:
            frequency = _to_host(kwargs["f_arr"], np.float64)
            if not np.all(frequency == np.sort(frequency)):
                raise ValueError("Frequency array must be sorted in ascending order.")
            if not np.allclose(np.diff(frequency), np.diff(frequency)[0], 1e-10):
                raise ValueError("Frequency array must be equally spaced.")
            if len(frequency) < num_pts:
                raise ValueError("f_arr is shorter than the time-domain output of this summation.")
            self.waveform = torch.zeros(len(frequency), dtype=torch.complex128, device=dev)
        else:
            self.waveform = torch.zeros(num_pts + num_pts_pad, dtype=torch.complex128, device=dev)
        self.sum(t, *args, dt=dt, **kwargs)
        return self.waveform


class _FoldPlan:
    """Device tables of the mode fold map (few_fold_plan)."""

    def __init__(self, m, k, n, device):
        K = len(m)
        max_rows = 256
        nmax = int(max(np.abs(n).max(), 0))
        max_keys = max_rows * (2 * nmax + 1)
        row_m = np.zeros(max_rows, np.int32)
        row_k = np.zeros(max_rows, np.int32)
        dims = np.zeros(3, np.int32)
        key_ptr = np.zeros(max_keys + 1, np.int32)
        key_list = np.zeros(2 * K, np.int32)
        _lib.call("few_fold_plan", m.ctypes.data, k.ctypes.data, n.ctypes.data, K, max_rows, max_keys,
                  row_m.ctypes.data, row_k.ctypes.data, dims.ctypes.data, key_ptr.ctypes.data, key_list.ctypes.data)
        self.R, self.nlo, self.NN = (int(v) for v in dims)
        nkeys = self.R * self.NN
        self.row_m = row_m[: self.R].copy()
        self.row_k = row_k[: self.R].copy()
        self.use_theta = int(np.any(self.row_k != 0))
        self.key_ptr = key_ptr[: nkeys + 1].copy()
        self.key_list = key_list[: int(self.key_ptr[-1])].copy()
        self.K = K
        # key of each mode's + term and - term (-1: m = 0 has no - term)
        self.key_plus = np.full(K, -1, np.int32)
        self.key_minus = np.full(K, -1, np.int32)
        for q in range(nkeys):
            for code in self.key_list[self.key_ptr[q]:self.key_ptr[q + 1]]:
                if code & 1:
                    self.key_minus[code >> 1] = q
                else:
                    self.key_plus[code >> 1] = q
        host = np.concatenate([self.row_m, self.row_k, self.key_ptr, self.key_list, self.key_plus,
                               self.key_minus]).astype(np.int32)
        self.table = _upload(host, device)
        o = 0
        self.d_row_m = self.table[o:o + self.R]; o += self.R
        self.d_row_k = self.table[o:o + self.R]; o += self.R
        self.d_key_ptr = self.table[o:o + nkeys + 1]; o += nkeys + 1
        self.d_key_list = self.table[o:o + len(self.key_list)]; o += len(self.key_list)
        self.d_key_plus = self.table[o:o + K]; o += K
        self.d_key_minus = self.table[o:o + K]


class _SegmentPlan:
    """Host segment/unit tables (few_segment_plan) and their device copies."""

    def __init__(self, h_t, phase_t, out_len, dt, chunk, device):
        N = len(h_t)
        max_units = N + out_len // chunk + 1
        seg_start = np.zeros(N, np.int32)
        seg_info = np.zeros(3 * (N - 1), np.float64)
        units = np.zeros(3 * max_units, np.int32)
        counts = np.zeros(2, np.int32)
        _lib.call("few_segment_plan", h_t.ctypes.data, phase_t.ctypes.data, N, int(out_len), float(dt), int(chunk),
                  max_units, seg_start.ctypes.data, seg_info.ctypes.data, units.ctypes.data, counts.ctypes.data)
        self.nseg, self.nunits = int(counts[0]), int(counts[1])
        self.seg_start = seg_start[: self.nseg + 1]
        self.units_host = units[: 3 * self.nunits]
        self.seg_info_host = seg_info[: 3 * max(self.nseg, 1)]
        self.d_seg_info = _upload(self.seg_info_host, device)
        self.d_units = _upload(self.units_host if self.nunits else np.zeros(3, np.int32), device)
        self._device = device

    def backward_tables(self):
        """Device (seg_start, seg_units), each (nseg+1,) int32, for the adjoint kernels."""
        if not hasattr(self, "_bwd"):
            seg_units = np.zeros(self.nseg + 1, np.int32)
            useg = self.units_host.reshape(-1, 3)[:, 0] if self.nunits else np.zeros(0, np.int32)
            seg_units[1:] = np.cumsum(np.bincount(useg, minlength=self.nseg)[: self.nseg])
            host = np.concatenate([self.seg_start.astype(np.int32), seg_units])
            t = _upload(host, self._device)
            self._bwd = (t[: self.nseg + 1], t[self.nseg + 1:])
        return self._bwd

    def balanced_units(self, chunk: int = 1024):
        """Device (units (n, 3), seg_units (nseg+1,)) int32 for the joint adjoint:
        each segment's samples cut into ceil(len / chunk) parts of equal length
        (within one sample), so no work unit is a short remainder."""
        if not hasattr(self, "_bal"):
            lo = self.seg_start[: self.nseg].astype(np.int64)
            hi = self.seg_start[1: self.nseg + 1].astype(np.int64)
            n = np.maximum(hi - lo, 0)
            parts = (n + chunk - 1) // chunk
            seg_units = np.zeros(self.nseg + 1, np.int32)
            seg_units[1:] = np.cumsum(parts)
            total = int(seg_units[-1])
            seg = np.repeat(np.arange(self.nseg), parts)
            k = np.arange(total) - np.repeat(seg_units[:-1], parts)
            P = np.repeat(parts, parts)
            a = np.repeat(lo, parts) + (k * np.repeat(n, parts)) // np.maximum(P, 1)
            b = np.repeat(lo, parts) + ((k + 1) * np.repeat(n, parts)) // np.maximum(P, 1)
            units = np.stack([seg, a, b], axis=1).astype(np.int32).reshape(-1)
            host = np.concatenate([units, seg_units])
            t = _upload(host, self._device)
            self._bal = (t[: 3 * total], t[3 * total:], total)
        return self._bal


class _Prepared:
    """Inputs, plans and device tensors of one call (kept for the backward)."""


class _ModeSumFunction(torch.autograd.Function):
    """h = InterpolatedModeSum(teuk_modes, phase_interp_coeffs; fixed t, ylms, modes).

    Backward: the adjoint kernels (phasors recomputed from the phase
    polynomials, not stored; the folded coefficients W of the forward are kept)."""

    @staticmethod
    def forward(ctx, teuk, pc, module, prep, total):
        out = torch.zeros(total, dtype=torch.complex128, device=prep.dev)
        module._launch(prep, out)
        prep.teuk_in = prep.pc_in = None  # do not keep the autograd inputs alive through ctx
        ctx.prep = prep
        ctx.module = module
        return out

    @staticmethod
    def backward(ctx, grad):
        g_teuk, g_pc = ctx.module._backward_hook(ctx.prep, grad, ctx.needs_input_grad[0], ctx.needs_input_grad[1])
        return g_teuk, g_pc, None, None, None


class InterpolatedModeSum(SummationBase):
    """Create a waveform by interpolating a sparse trajectory
    (reference: ``interpolatedmodesum.py:260-375``).

    args:
        precision: "faithful" (default), "exact" or "mixed"; see the module docstring.
        backward: "fp64" or "mixed" adjoint (default: "mixed" for
            precision="mixed", else "fp64").
        chunk: output samples per work unit of the sum kernel.
        Others as ``SummationBase``.
    """

    def __init__(self, force_backend=None, precision: str = "faithful", chunk: int = DEFAULT_CHUNK,
                 backward: str | None = None, **kwargs):
        SummationBase.__init__(self, force_backend=force_backend, **kwargs)
        if precision not in _PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(_PRECISIONS)}")
        self.precision = precision
        if backward is None:
            backward = "mixed" if precision == "mixed" else "fp64"
        if backward not in ("fp64", "mixed"):
            raise ValueError("backward must be 'fp64' or 'mixed'")
        self.backward = backward
        if not 1 <= int(chunk) <= 1024:
            raise ValueError("chunk must be within 1..1024 output samples")
        self.chunk = int(chunk)
        self._fold_cache: OrderedDict = OrderedDict()
        self.record_stages = False  # set True to time the kernels of each call with CUDA events
        self._stage_events = None
        self._mixed_err = None

    def mixed_error(self) -> bool:
        """True if a tensor-core wait of a mixed-precision call timed out (the
        kernel then stopped early and its output is incomplete).  Synchronises."""
        return bool(self._mixed_err is not None and int(self._mixed_err.item()) != 0)

    def _fold_plan(self, m, k, n, device) -> _FoldPlan:
        key = (m.tobytes(), k.tobytes(), n.tobytes(), str(device))
        plan = self._fold_cache.get(key)
        if plan is None:
            plan = _FoldPlan(m, k, n, device)
            self._fold_cache[key] = plan
            while len(self._fold_cache) > 8:
                self._fold_cache.popitem(last=False)
        else:
            self._fold_cache.move_to_end(key)
        return plan

    def sum(self, t, teuk_modes, ylms, phase_interp_t, phase_interp_coeffs, l_arr, m_arr, k_arr, n_arr, *args,
            dt: float = 10.0, integrate_backwards: bool = False, host_out=None, **kwargs):
        """Interpolated summation into ``self.waveform`` (``interpolatedmodesum.py:283-375``).

        If ``teuk_modes`` or ``phase_interp_coeffs`` is a torch tensor that
        requires grad (and grad mode is on), the waveform is the output of a
        ``torch.autograd.Function`` whose backward runs the adjoint kernels."""
        needs_grad = torch.is_grad_enabled() and any(
            isinstance(x, torch.Tensor) and x.requires_grad for x in (teuk_modes, phase_interp_coeffs))
        if host_out is not None:
            if needs_grad:
                raise ValueError("host_out is for calls without gradients.")
            if not (isinstance(host_out, torch.Tensor) and host_out.device.type == "cpu" and host_out.is_pinned()
                    and host_out.dtype == torch.complex128 and host_out.is_contiguous()
                    and host_out.numel() >= self.waveform.numel()):
                raise ValueError("host_out must be a pinned, contiguous complex128 CPU tensor at least as long as "
                                 "the waveform.")
        prep = self._prepare(t, teuk_modes, ylms, phase_interp_t, phase_interp_coeffs, l_arr, m_arr, k_arr, n_arr,
                             dt, integrate_backwards, keep=needs_grad)
        if needs_grad:
            total = self.waveform.shape[0]
            self.waveform = _ModeSumFunction.apply(prep.teuk_in, prep.pc_in, self, prep, total)
        else:
            self._launch(prep, self.waveform, host_out)
        return self.waveform

    def _prepare(self, t, teuk_modes, ylms, phase_interp_t, phase_interp_coeffs, l_arr, m_arr, k_arr, n_arr, dt,
                 integrate_backwards, keep=False):
        """Validates the inputs, makes the host plans and the device tensors."""
        dev = self.device
        p = _Prepared()
        h_t = _to_host(t, np.float64)
        phase_t = _to_host(phase_interp_t, np.float64)
        if h_t.ndim != 1:
            raise ValueError("t must be 1-dimensional.")
        N = len(h_t)
        if N < 4:
            raise ValueError("not-a-knot cubic splines need at least 4 knots.")
        if not np.all(np.diff(h_t) > 0):
            raise ValueError("t must increase strictly.")
        if len(phase_t) != N:
            raise ValueError("phase_interp_t must have the same length as t.")
        teuk_in = _input(teuk_modes, torch.complex128, dev)
        teuk = teuk_in.detach().contiguous()
        if teuk.ndim != 2 or teuk.shape[0] != N:
            raise ValueError("teuk_modes must have shape (len(t), num_teuk_modes).")
        K = int(teuk.shape[1])
        l_h = _to_host(l_arr, np.int64)
        m_h = _to_host(m_arr, np.int32)
        k_h = _to_host(k_arr, np.int32)
        n_h = _to_host(n_arr, np.int32)
        if not (len(l_h) == len(m_h) == len(k_h) == len(n_h) == K):
            raise ValueError("l_arr, m_arr, k_arr, n_arr must have num_teuk_modes entries.")
        if tuple(np.shape(ylms)) != (2 * K,):
            raise ValueError("ylms must have shape (2 * num_teuk_modes,).")
        if tuple(phase_interp_coeffs.shape) != (N - 1, 3, 8):
            raise ValueError("phase_interp_coeffs must have shape (len(t) - 1, 3, 8).")
        if integrate_backwards:
            # align the knots with t=0 as the reference does (interpolatedmodesum.py:341-345)
            offset = h_t[-1] - int(h_t[-1] / dt) * dt
            h_t = h_t - offset
            phase_t = phase_t - offset
        pc_in = _input(phase_interp_coeffs, torch.float64, dev)
        p.dev, p.st, p.N, p.K, p.dt = dev, _stream(dev), N, K, float(dt)
        p.teuk, p.teuk_in, p.pc_in = teuk, (teuk_in if keep else None), (pc_in if keep else None)
        p.t_dev = _upload(h_t, dev)
        p.fac = spline_factor_table(h_t, dev)
        # ylms[K:] *= (-1)^l (interpolatedmodesum.py:357-358)
        sign = np.where(l_h % 2 == 0, 1.0, -1.0)
        ylm = _input(ylms, torch.complex128, dev).clone()
        ylm[K:] *= _upload(sign, dev)
        p.ylm = ylm
        # (N-1, 3, 8) -> (8, N-1, 3) (interpolatedmodesum.py:352-354)
        p.pc = pc_in.detach().permute(2, 0, 1).contiguous()
        p.fold = self._fold_plan(m_h, k_h, n_h, dev)
        p.bwd_mixed = self.backward == "mixed"
        if p.bwd_mixed:
            if self._mixed_err is None or self._mixed_err.device != dev:
                self._mixed_err = torch.zeros(1, dtype=torch.int32, device=dev)
            p.err = self._mixed_err
        p.seg = _SegmentPlan(h_t, phase_t, self.num_pts, dt, self.chunk, dev)
        p.out_len = int(self.num_pts)
        return p

    def _launch(self, p, out, host_out=None):
        """Spline build, fold and sum into `out` (three launches on the current stream).
        With `host_out` the sum runs in parts of consecutive work units (consecutive
        output samples) and each finished slice is copied to `host_out` on a
        download stream while the next part computes."""
        fold, seg, N, K, st = p.fold, p.seg, p.N, p.K, p.st
        coeffs = torch.empty((4, N, 2 * K), dtype=torch.float64, device=p.dev)
        W = torch.empty((max(seg.nseg, 1), fold.R, fold.NN, 4), dtype=torch.complex128, device=p.dev)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)] if self.record_stages else None
        if ev:
            ev[0].record()
        # amplitude splines straight from the (N, K) complex array: real parts are
        # interpolants 0..K-1, imaginary parts K..2K-1 (interpolatedmodesum.py:331-337)
        _lib.call("few_spline_build_factored", _ptr(p.fac), _ptr(p.teuk), 2 * K, 2, K, 1, 2 * K, N, _ptr(coeffs),
                  _lib.FEW_LAYOUT_KNOT_MAJOR, st)
        if ev:
            ev[1].record()
        _lib.call("few_fold_coeffs", _ptr(coeffs), _ptr(p.ylm), _ptr(fold.d_key_ptr), _ptr(fold.d_key_list), K, N,
                  seg.nseg, fold.R, fold.NN, _ptr(W), st)
        if ev:
            ev[2].record()
        if self.precision == "mixed":
            nbytes = int(_lib.load().few_mixed_operand_bytes(max(seg.nseg, 1), fold.R, fold.NN))
            if nbytes <= 0:
                raise ValueError("precision='mixed' supports at most 64 (m, k) rows")
            Bpk = torch.empty(nbytes, dtype=torch.uint8, device=p.dev)
            if self._mixed_err is None or self._mixed_err.device != p.dev:
                self._mixed_err = torch.zeros(1, dtype=torch.int32, device=p.dev)
            _lib.call("few_fold_mixed", _ptr(W), _ptr(p.t_dev), seg.nseg, fold.R, fold.NN, _ptr(Bpk), st)

            def run(u0, u1):
                _lib.call("few_sum_mixed", _ptr(out), _ptr(Bpk), _ptr(p.pc), N, _ptr(seg.d_seg_info),
                          _ptr(p.t_dev), _ptr(seg.d_units) + 12 * u0, u1 - u0, _ptr(fold.d_row_m),
                          _ptr(fold.d_row_k), fold.R, fold.nlo, fold.NN, p.dt, fold.use_theta,
                          _ptr(self._mixed_err), st)
        else:
            def run(u0, u1):
                _lib.call("few_sum_folded", _ptr(out), _ptr(W), _ptr(p.pc), N, _ptr(seg.d_seg_info),
                          _ptr(seg.d_units) + 12 * u0, u1 - u0, _ptr(fold.d_row_m), _ptr(fold.d_row_k), fold.R,
                          fold.nlo, fold.NN, p.dt, _PRECISIONS[self.precision], fold.use_theta, st)
        if host_out is None or seg.nunits == 0:
            run(0, seg.nunits)
            if host_out is not None:
                host_out[: out.numel()].copy_(out)
        else:
            self._sum_streamed(run, seg, out, host_out, p.dev)
        if ev:
            ev[3].record()
            self._stage_events = ev
        self._last_plan = (fold, seg)
        p.W = W
        return out

    @staticmethod
    def _sum_streamed(run, seg, out, host_out, dev, parts: int = 8):
        """The sum in `parts` launches over consecutive units; after each, the
        samples it finished go to host_out on the download stream."""
        main = torch.cuda.current_stream(dev)
        ds = _download_stream(dev)
        units = seg.units_host.reshape(-1, 3)
        n = seg.nunits
        bounds = sorted({min(n, (n * q + parts - 1) // parts) for q in range(parts + 1)})
        done = 0
        for u0, u1 in zip(bounds[:-1], bounds[1:]):
            if u1 <= u0:
                continue
            run(u0, u1)
            end = out.numel() if u1 == n else int(units[u1, 1])
            ev = torch.cuda.Event()
            ev.record(main)
            ds.wait_event(ev)
            with torch.cuda.stream(ds):
                host_out[done:end].copy_(out[done:end], non_blocking=True)
            done = end
        out.record_stream(ds)
        main.wait_stream(ds)

    def _backward_hook(self, p, grad, need_teuk, need_pc):
        """The backward of one call (overridden by the sharded summation)."""
        return InterpolatedModeSum._backward(p, grad, need_teuk, need_pc)

    @staticmethod
    def _backward(p, grad, need_teuk=True, need_pc=True, concurrent=True):
        """Adjoint kernels: (dL/d teuk_modes (N, K) complex, dL/d phase_interp_coeffs (N-1, 3, 8)).
        Both FP64 gradients come from one joint pass.  With both gradients wanted
        from the tensor-core kernels and ``concurrent``, the phase branch runs on
        a second stream beside the amplitude branch."""
        fold, seg, N, K, st, dev = p.fold, p.seg, p.N, p.K, p.st, p.dev
        grad = grad[: p.out_len].to(torch.complex128).contiguous()
        # the segment tables are uploaded on the caller's stream before the side
        # stream forks from it: the phase branch reads them there
        seg_start, _ = seg.backward_tables()
        mixed = getattr(p, "bwd_mixed", False)
        if mixed and need_pc and fold.R > 64:
            raise ValueError("backward='mixed' supports at most 64 (m, k) rows for phase gradients")
        if need_teuk and not mixed:
            return InterpolatedModeSum._joint_backward(p, grad, need_pc)
        both = need_teuk and need_pc and concurrent
        main = torch.cuda.current_stream(dev)
        side = None
        if both:
            side = _side_stream(dev)
            side.wait_stream(main)
        g_teuk = g_pc = None
        if need_teuk:
            G = torch.empty((max(seg.nseg, 1), fold.R, fold.NN, 4), dtype=torch.complex128, device=dev)
            if mixed:
                _lib.call("few_adjoint_G_mixed", _ptr(grad), _ptr(p.pc), N, _ptr(seg.d_seg_info), _ptr(p.t_dev),
                          _ptr(seg_start), seg.nseg, _ptr(fold.d_row_m), _ptr(fold.d_row_k), fold.R, fold.nlo,
                          fold.NN, p.dt, fold.use_theta, _ptr(G), _ptr(p.err), st)
            else:
                _lib.call("few_adjoint_G", _ptr(grad), _ptr(p.pc), N, _ptr(seg.d_seg_info), _ptr(seg_start),
                          seg.nseg, _ptr(fold.d_row_m), _ptr(fold.d_row_k), fold.R, fold.nlo, fold.NN, p.dt,
                          fold.use_theta, _ptr(G), st)
            g_teuk = InterpolatedModeSum._amplitude_backward(p, G)
        if need_pc:
            with torch.cuda.stream(side) if both else torch.cuda.stream(main):
                g_pc = InterpolatedModeSum._phase_backward(p, grad, mixed, side.cuda_stream if both else st)
            if both:
                main.wait_stream(side)
                if not torch.cuda.is_current_stream_capturing():
                    g_pc.record_stream(main)
        return g_teuk, g_pc

    @staticmethod
    def _amplitude_backward(p, G):
        """dL/d teuk_modes (N, K) from G (nseg, R, NN, 4): the transposes of the fold and the spline."""
        fold, seg, N, K, st, dev = p.fold, p.seg, p.N, p.K, p.st, p.dev
        gcoef = torch.empty((4, N, 2 * K), dtype=torch.float64, device=dev)
        _lib.call("few_unfold", _ptr(G), _ptr(p.ylm), _ptr(fold.d_key_plus), _ptr(fold.d_key_minus), K, N,
                  seg.nseg, fold.R * fold.NN, _ptr(gcoef), st)
        g_teuk = torch.empty((N, K), dtype=torch.complex128, device=dev)
        _lib.call("few_spline_adjoint_factored", _ptr(p.fac), _ptr(gcoef), _ptr(g_teuk), 2 * K, 2, K, 1, 2 * K, N,
                  0, st)
        return g_teuk

    @staticmethod
    def _joint_backward(p, grad, want_pc=True):
        """FP64 gradients from one pass (few_adjoint_joint): the per-key moments
        give G and, with want_pc, the phase-coefficient gradients together; G
        alone takes the kernel's five-moment form."""
        fold, seg, N, st, dev = p.fold, p.seg, p.N, p.st, p.dev
        units, seg_units, nunits = seg.balanced_units()
        G = torch.empty((max(seg.nseg, 1), fold.R, fold.NN, 4), dtype=torch.complex128, device=dev)
        g_pc = torch.zeros((N - 1, 3, 8), dtype=torch.float64, device=dev) if want_pc else None
        nscratch = int(_lib.load().few_adjoint_joint_scratch(max(nunits, 1), fold.R, fold.NN))
        scratch = torch.empty(max(nscratch, 1), dtype=torch.float64, device=dev)
        _lib.call("few_adjoint_joint", _ptr(grad), _ptr(p.W), _ptr(p.pc), N, _ptr(seg.d_seg_info), _ptr(units),
                  nunits, _ptr(seg_units), seg.nseg, _ptr(fold.d_row_m), _ptr(fold.d_row_k), fold.R, fold.nlo,
                  fold.NN, p.dt, fold.use_theta, _ptr(G), _ptr(g_pc) if want_pc else 0, _ptr(scratch), st)
        return InterpolatedModeSum._amplitude_backward(p, G), g_pc

    @staticmethod
    def _phase_backward(p, grad, mixed, st):
        """dL/d phase_interp_coeffs on stream st (tensors allocated on the current stream)."""
        fold, seg, N, dev = p.fold, p.seg, p.N, p.dev
        _, seg_units = seg.backward_tables()
        partial = torch.empty((max(seg.nunits, 1), 24), dtype=torch.float64, device=dev)
        if mixed:
            nbytes = int(_lib.load().few_mixed_adjoint_operand_bytes(max(seg.nseg, 1), fold.R, fold.NN))
            Bpk = torch.empty(nbytes, dtype=torch.uint8, device=dev)
            _lib.call("few_fold_mixed_adjoint", _ptr(p.W), _ptr(p.t_dev), seg.nseg, fold.R, fold.nlo, fold.NN,
                      _ptr(Bpk), st)
            _lib.call("few_adjoint_phase_mixed", _ptr(grad), _ptr(Bpk), _ptr(p.pc), N, _ptr(seg.d_seg_info),
                      _ptr(p.t_dev), _ptr(seg.d_units), seg.nunits, _ptr(fold.d_row_m), _ptr(fold.d_row_k),
                      fold.R, fold.nlo, fold.NN, p.dt, fold.use_theta, _ptr(partial), _ptr(p.err), st)
        else:
            _lib.call("few_adjoint_phase", _ptr(grad), _ptr(p.W), _ptr(p.pc), N, _ptr(seg.d_seg_info),
                      _ptr(seg.d_units), seg.nunits, _ptr(fold.d_row_m), _ptr(fold.d_row_k), fold.R, fold.nlo,
                      fold.NN, p.dt, fold.use_theta, _ptr(partial), st)
        g_pc = torch.zeros((N - 1, 3, 8), dtype=torch.float64, device=dev)
        _lib.call("few_adjoint_phase_reduce", _ptr(partial), _ptr(seg_units), seg.nseg, _ptr(g_pc), st)
        return g_pc

    def stage_times(self) -> dict:
        """Kernel times (ms) of the last call with ``record_stages`` set:
        spline build, fold and sum (three back-to-back launches)."""
        ev = self._stage_events
        if ev is None:
            return {}
        ev[3].synchronize()
        return {"spline": ev[0].elapsed_time(ev[1]), "fold": ev[1].elapsed_time(ev[2]),
                "sum": ev[2].elapsed_time(ev[3])}
