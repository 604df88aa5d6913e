"""Many waveforms of uneven length, knot count and mode count in one
persistent launch, optionally captured in a CUDA graph.

The reference sums one waveform at a time, one kernel launch per knot segment
(src/few/cutils/interpolate.cu:745-781).  Here every waveform of a batch gets
its spline build and fold (small launches), and then a single persistent sum
kernel (``few_sum_batched`` / ``few_sum_mixed_batched``) strides over the work
units of all waveforms, longest units first, so the SMs stay busy while short
and long waveforms finish together.  The unit length and the CTAs per SM come
from the autotuner (``fastemriwaveforms_b200.autotune``).  ``capture()``
records the whole forward (and, with ``backward=True``, the adjoint of every
waveform for fixed upstream-gradient buffers) in one CUDA graph; ``replay()``
re-runs it after new amplitudes / phase coefficients are written into the
static input buffers (``update``).

Gradients of a batched forward are each waveform's adjoint, as for
``InterpolatedModeSum``: the tensor-core adjoint for ``precision="mixed"``
(``backward="mixed"``, the default there), the FP64 one otherwise.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib, autotune
from .summation import InterpolatedModeSum, _device, _ptr, _stream, _upload
from .synthetic import output_length

# Layout of few_wave_desc (include/few_b200.h): 8 pointers, 6 ints, 1 double.
DESC_DTYPE = np.dtype([("wf", "u8"), ("W", "u8"), ("Bpk", "u8"), ("pc", "u8"), ("seg_info", "u8"),
                       ("t_knots", "u8"), ("row_m", "u8"), ("row_k", "u8"), ("N", "i4"), ("R", "i4"),
                       ("nlo", "i4"), ("NN", "i4"), ("use_theta", "i4"), ("reserved", "i4"), ("dt", "f8")])
assert DESC_DTYPE.itemsize == 96


def _args_of(w):
    """(call args, T, dt) of a waveform given as ModeSumInputs or a dict."""
    if hasattr(w, "call_args"):
        return w.call_args(), float(w.T), float(w.dt)
    keys = ("t", "teuk_modes", "ylms", "phase_interp_t", "phase_interp_coeffs", "l_arr", "m_arr", "k_arr", "n_arr")
    return tuple(w[k] for k in keys), float(w.get("T", 1.0)), float(w.get("dt", 10.0))


class BatchedInterpolatedModeSum:
    """Batched interpolated mode sum.

    args:
        precision: "mixed" (tensor cores), "exact" or "faithful" (FP64).
        autotune: choose the unit length, CTAs per SM and (tensor cores) the
            operand pipeline shape by timing (cached).
        chunk, ctas_per_sm: fixed shape (overrides the autotuner); astages,
            bstages: fixed operand pipeline (A stages per producer half, 1 or 2;
            B bulk-copy slots, 2..4; default: the tuned ones, or the library's
            choice when chunk and ctas_per_sm are given).
        backward: "mixed" or "fp64" adjoint (default: "mixed" for precision="mixed").
        streams: side streams over which the per-waveform spline builds, folds
            and adjoints are spread (they are small launches; running several
            waveforms' chains at once keeps the GPU busy).
    """

    def __init__(self, precision: str = "mixed", device=None, autotune: bool = True, chunk: int | None = None,
                 ctas_per_sm: int | None = None, backward: str | None = None, streams: int = 8,
                 astages: int | None = None, bstages: int | None = None):
        if precision not in ("mixed", "exact", "faithful"):
            raise ValueError("precision must be 'mixed', 'exact' or 'faithful'")
        self.precision = precision
        if backward is None:
            backward = "mixed" if precision == "mixed" else "fp64"
        if backward not in ("mixed", "fp64"):
            raise ValueError("backward must be 'mixed' or 'fp64'")
        self.backward_precision = backward
        if streams < 1:
            raise ValueError("streams must be >= 1")
        self.nstreams = int(streams)
        self._side = None
        self.device = _device(device)
        self.autotune = autotune
        self.chunk = chunk
        self.ctas_per_sm = ctas_per_sm
        if bstages is not None and not 2 <= bstages <= 4:
            raise ValueError("bstages must be 2, 3 or 4")
        if astages is not None and astages not in (1, 2):
            raise ValueError("astages must be 1 or 2")
        self.astages = astages
        self.bstages = bstages
        self.graph = None
        self.tuning = None

    # ------------------------------------------------------------------ set-up
    def setup(self, waveforms, requires_grad: bool = False):
        """Plans every waveform and allocates its buffers; returns self."""
        dev = self.device
        self.preps, self.mods, self.lengths = [], [], []
        for w in waveforms:
            args, T, dt = _args_of(w)
            t = args[0]
            t0 = float(t[0].item() if hasattr(t[0], "item") else t[0])
            t1 = float(t[-1].item() if hasattr(t[-1], "item") else t[-1])
            num_pts, num_pts_pad = output_length(np.array([t0, t1]), T, dt)
            mod = InterpolatedModeSum(precision="exact", device=dev, backward=self.backward_precision)
            mod.num_pts = num_pts
            prep = mod._prepare(*args, dt=dt, integrate_backwards=False)
            if requires_grad:
                prep.seg.backward_tables()
            self.mods.append(mod)
            self.preps.append(prep)
            self.lengths.append(num_pts + num_pts_pad)
        self.offsets = np.concatenate([[0], np.cumsum(self.lengths)]).astype(np.int64)
        self.out = torch.zeros(int(self.offsets[-1]), dtype=torch.complex128, device=dev)
        self.outputs = [self.out[self.offsets[i]:self.offsets[i + 1]] for i in range(len(self.preps))]
        self.max_R = max(p.fold.R for p in self.preps)
        max_NN = max(p.fold.NN for p in self.preps)
        if self.precision == "mixed" and self.max_R > 64:
            raise ValueError("precision='mixed' supports at most 64 (m, k) rows")
        # the FP64 kernels keep a segment's rows in shared memory in blocks of up to 8 rows
        self.smem_bytes = int(min(200 * 1024, max((p.fold.R + 7) // 8 * 8 * p.fold.NN * 64 for p in self.preps)))
        descs = np.zeros(len(self.preps), DESC_DTYPE)
        for i, p in enumerate(self.preps):
            p.coeffs = torch.empty((4, p.N, 2 * p.K), dtype=torch.float64, device=dev)
            p.W = torch.empty((max(p.seg.nseg, 1), p.fold.R, p.fold.NN, 4), dtype=torch.complex128, device=dev)
            p.Bpk = None
            if self.precision == "mixed":
                nbytes = int(_lib.load().few_mixed_operand_bytes(max(p.seg.nseg, 1), p.fold.R, p.fold.NN))
                p.Bpk = torch.empty(nbytes, dtype=torch.uint8, device=dev)
            d = descs[i]
            d["wf"] = self.outputs[i].data_ptr()
            d["W"] = p.W.data_ptr()
            d["Bpk"] = p.Bpk.data_ptr() if p.Bpk is not None else 0
            d["pc"] = p.pc.data_ptr()
            d["seg_info"] = p.seg.d_seg_info.data_ptr()
            d["t_knots"] = p.t_dev.data_ptr()
            d["row_m"] = p.fold.d_row_m.data_ptr()
            d["row_k"] = p.fold.d_row_k.data_ptr()
            d["N"], d["R"], d["nlo"], d["NN"] = p.N, p.fold.R, p.fold.nlo, p.fold.NN
            d["use_theta"] = p.fold.use_theta
            d["dt"] = p.dt
        self.descs = _upload(descs.view(np.uint8), dev)
        self.err = torch.zeros(1, dtype=torch.int32, device=dev)
        # time stamps (GPU global timer, ns): [0] start of the forward, [1 + w]
        # completion of waveform w's sum, [1 + n + w] completion of its backward
        self.stamps = torch.zeros(1 + 2 * len(self.preps), dtype=torch.int64, device=dev)
        self.mode_samples = sum(p.K * p.out_len for p in self.preps)
        seg_lens = [np.diff(p.seg.seg_start).mean() for p in self.preps if p.seg.nseg > 0]
        self._key = autotune.key_of(dev, self.precision, self.max_R, max_NN, float(np.mean(seg_lens)),
                                    len(self.preps))
        self.sms = torch.cuda.get_device_properties(dev).multi_processor_count
        chunk, per_sm, ast, bst = self.chunk, self.ctas_per_sm, self.astages, self.bstages
        if chunk is None or per_sm is None:
            cached = autotune.lookup(self._key) if self.autotune else None
            if cached is None and self.autotune:
                self._prepare_operands()
                cached = autotune.tune(self._key, self._runner, autotune.candidates_for(self.precision))
            if cached is None:
                cached = {"chunk": 1024, "ctas_per_sm": 2, "astages": 0, "bstages": 0}
            self.tuning = cached
            chunk = chunk or cached["chunk"]
            per_sm = per_sm or cached["ctas_per_sm"]
            ast = ast or cached.get("astages", 0)
            bst = bst or cached.get("bstages", 0)
        self.chunk, self.ctas_per_sm = int(chunk), int(per_sm)
        self.astages, self.bstages = int(ast or 0), int(bst or 0)
        self.units = self._units(self.chunk)
        return self

    def _units(self, chunk: int) -> torch.Tensor:
        """Work units {waveform, segment, first, end} of every waveform, longest
        (in key-samples) first so the persistent CTAs finish together."""
        rows = []
        for w, p in enumerate(self.preps):
            st = p.seg.seg_start
            for j in range(p.seg.nseg):
                a, b = int(st[j]), int(st[j + 1])
                for u in range(a, b, chunk):
                    rows.append((w, j, u, min(u + chunk, b), (min(u + chunk, b) - u) * p.fold.R * p.fold.NN))
        arr = np.array(rows, dtype=np.int64).reshape(-1, 5)
        order = np.argsort(-arr[:, 4], kind="stable")
        units = np.ascontiguousarray(arr[order, :4].astype(np.int32))
        return _upload(units.reshape(-1), self.device)

    # ------------------------------------------------------------ the kernels
    def _streams(self):
        if self._side is None:
            self._side = [torch.cuda.Stream(self.device) for _ in range(self.nstreams)]
        return self._side

    def _fork(self):
        main = torch.cuda.current_stream(self.device)
        side = self._streams()
        for s in side:
            s.wait_stream(main)
        return main, side

    @staticmethod
    def _join(main, side):
        for s in side:
            main.wait_stream(s)

    def _prepare_operands(self):
        """Spline builds and folds of every waveform, spread over the side streams."""
        main, side = self._fork()
        for i, p in enumerate(self.preps):
            st = side[i % len(side)].cuda_stream
            p.st = st
            _lib.call("few_spline_build_factored", _ptr(p.fac), _ptr(p.teuk), 2 * p.K, 2, p.K, 1, 2 * p.K, p.N,
                      _ptr(p.coeffs), _lib.FEW_LAYOUT_KNOT_MAJOR, st)
            _lib.call("few_fold_coeffs", _ptr(p.coeffs), _ptr(p.ylm), _ptr(p.fold.d_key_ptr), _ptr(p.fold.d_key_list),
                      p.K, p.N, p.seg.nseg, p.fold.R, p.fold.NN, _ptr(p.W), st)
            if p.Bpk is not None:
                _lib.call("few_fold_mixed", _ptr(p.W), _ptr(p.t_dev), p.seg.nseg, p.fold.R, p.fold.NN, _ptr(p.Bpk),
                          st)
        self._join(main, side)

    def _sum(self, units: torch.Tensor, ctas: int, done=None, astages: int | None = None,
             bstages: int | None = None):
        st = _stream(self.device)
        nunits = units.numel() // 4
        if self.precision == "mixed":
            ast = self.astages if astages is None else astages
            bst = self.bstages if bstages is None else bstages
            _lib.call("few_sum_mixed_batched", _ptr(self.descs), len(self.preps), _ptr(units), nunits, self.max_R,
                      ctas, int(ast or 0), int(bst or 0), _ptr(self.err), done, st)
        else:
            mode = _lib.FEW_SUM_FAITHFUL if self.precision == "faithful" else _lib.FEW_SUM_EXACT
            _lib.call("few_sum_batched", _ptr(self.descs), len(self.preps), _ptr(units), nunits, self.smem_bytes, mode,
                      ctas, done, st)

    def _runner(self, chunk: int, ctas_per_sm: int, astages: int = 0, bstages: int = 0):
        units = self._units(chunk)

        def run():
            self.out.zero_()
            self._sum(units, ctas_per_sm * self.sms, astages=astages, bstages=bstages)

        return run

    def forward(self):
        """All waveforms; returns the list of output tensors (views of one buffer).
        Time stamps: ``stamps[0]`` the start, ``stamps[1 + w]`` waveform w's
        completion inside the persistent sum (see ``latencies``)."""
        st = _stream(self.device)
        self.stamps.zero_()
        _lib.call("few_stamp", _ptr(self.stamps), st)
        self.out.zero_()
        self._prepare_operands()
        self._sum(self.units, self.ctas_per_sm * self.sms, _ptr(self.stamps) + 8)
        return self.outputs

    def backward(self, grads):
        """Adjoint of every waveform for upstream gradients grads[i] (torch's
        convention for a complex output), the waveforms spread over the side
        streams; returns a list of (dL/d teuk_modes, dL/d phase_interp_coeffs)."""
        main, side = self._fork()
        out = []
        n = len(self.preps)
        for i, (p, g) in enumerate(zip(self.preps, grads)):
            s = side[i % len(side)]
            with torch.cuda.stream(s):
                p.st = s.cuda_stream
                out.append(InterpolatedModeSum._backward(p, g, concurrent=False))
                _lib.call("few_stamp", _ptr(self.stamps) + 8 * (1 + n + i), s.cuda_stream)
        self._join(main, side)
        if not torch.cuda.is_current_stream_capturing():
            for pair in out:  # made on side streams, used on the caller's stream
                for t in pair:
                    if t is not None:
                        t.record_stream(main)
        return out

    def latencies(self):
        """Per-waveform times (ms) of the last forward (and backward) run, from
        the forward's start: (forward completion (n,), backward completion
        (n,) or None).  The forward times end when the waveform's last work
        unit of the persistent sum finished; the backward times when its
        adjoint chain finished."""
        s = self.stamps.cpu().numpy()
        n = len(self.preps)
        fwd = (s[1:1 + n] - s[0]) * 1e-6
        bwd = s[1 + n:]
        return fwd, ((bwd - s[0]) * 1e-6 if np.all(bwd > 0) else None)

    def mixed_error(self) -> bool:
        """True if a tensor-core wait of the batched sum or of a mixed adjoint timed out."""
        return bool(int(self.err.item()) != 0) or any(m.mixed_error() for m in self.mods)

    # ------------------------------------------------------------ CUDA graphs
    def update(self, i: int, teuk_modes=None, phase_interp_coeffs=None):
        """Write new inputs of waveform i into the static buffers the graph reads."""
        p = self.preps[i]
        if teuk_modes is not None:
            p.teuk.copy_(torch.as_tensor(teuk_modes, dtype=torch.complex128))
        if phase_interp_coeffs is not None:
            pc = torch.as_tensor(phase_interp_coeffs, dtype=torch.float64).to(self.device)
            p.pc.copy_(pc.permute(2, 0, 1))

    def capture(self, backward: bool = False, grads=None):
        """Records forward (+ backward for the static gradient buffers `grads`,
        zeros if None) in one CUDA graph."""
        if backward:
            self.grad_in = [torch.zeros_like(o) if grads is None else torch.as_tensor(g).to(self.device).clone()
                            for o, g in zip(self.outputs, grads or [None] * len(self.outputs))]
        # warm up outside the capture (sets kernel attributes, fills caches)
        self.forward()
        if backward:
            self.backward(self.grad_in)
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            with torch.cuda.graph(self.graph, stream=s):
                self.forward()
                self.grad_out = self.backward(self.grad_in) if backward else None
        torch.cuda.current_stream(self.device).wait_stream(s)
        return self

    def replay(self):
        if self.graph is None:
            raise RuntimeError("capture() first")
        self.graph.replay()
        return self.outputs
