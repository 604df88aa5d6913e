"""ctypes front end for the oracle (test infrastructure only).

Two CPU implementations of the reference's time-domain interpolated mode sum
(and of its amplitude grid evaluation and frequency-domain sum):

* ``impl="oracle"`` -- ``few_oracle.c``, the C restatement in this folder;
* ``impl="ref"``    -- the reference's own CPU path
  (``src/few/cutils/interpolate.cu`` compiled as C++ by ``make -C oracle ref``
  into ``oracle/_ref``; present only where the reference sources were).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module, and only as the checker.  The product package never imports it.

The host-side preprocessing mirrors ``InterpolatedModeSum.sum``
(``src/few/summation/interpolatedmodesum.py:331-375``) and
``CubicSplineInterpolant.__init__`` (``interpolatedmodesum.py:35-107``).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_ORACLE = os.path.join(HERE, "_build", "liboracle.so")
LIB_REF = os.path.join(HERE, "_ref", "libfew_ref.so")


def _reference_root() -> str:
    """The reference checkout: $FEW_REFERENCE_ROOT, else the Makefile's REF default."""
    env = os.environ.get("FEW_REFERENCE_ROOT")
    if env:
        return env
    try:
        out = subprocess.run(["make", "-s", "--no-print-directory", "-C", HERE, "print-ref"], capture_output=True,
                             text=True, timeout=30)
        return out.stdout.strip()
    except (OSError, subprocess.SubprocessError):
        return ""


REFERENCE_ROOT = _reference_root()

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_libs: dict = {}


def build(ref: bool | None = None) -> None:
    """Compile the C restatement, and the reference's CPU path when its
    sources are present (``ref=None``: only if they exist)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    if ref is None:
        ref = os.path.isfile(os.path.join(REFERENCE_ROOT, "src/few/cutils/interpolate.cu"))
    if ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={REFERENCE_ROOT}"], check=True)


def have_ref() -> bool:
    return os.path.isfile(LIB_REF)


def _lib(impl: str):
    if impl in _libs:
        return _libs[impl]
    if impl == "oracle":
        if not os.path.isfile(LIB_ORACLE):
            build(ref=False)
        lib = ctypes.CDLL(LIB_ORACLE)
        lib.oracle_interpolate_arrays.restype = ctypes.c_int
        lib.oracle_interpolate_arrays.argtypes = [_dp, _dp, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _dp]
        lib.oracle_get_waveform.restype = ctypes.c_int
        lib.oracle_get_waveform.argtypes = [_dp, _dp, _dp, _dp, _ip, _ip, _ip, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_int, _dp, ctypes.c_double, _dp, ctypes.c_int,
                                            ctypes.c_int, ctypes.c_int]
        lib.oracle_get_waveform_dphase.restype = ctypes.c_int
        lib.oracle_get_waveform_dphase.argtypes = [_dp, _dp, _dp, _dp, _dp, ctypes.c_double, _ip, _ip, _ip,
                                                   ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_double,
                                                   _dp, ctypes.c_int, ctypes.c_int]
        lib.oracle_find_start_inds.restype = ctypes.c_int
        lib.oracle_find_start_inds.argtypes = [_ip, _dp, ctypes.c_double, ctypes.c_int, ctypes.c_int]
        lib.oracle_interp2d.argtypes = [_dp, _dp, ctypes.c_int, _dp, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int,
                                        _dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        lib.oracle_interp2d.restype = None
    elif impl == "ref":
        if not os.path.isfile(LIB_REF):
            raise FileNotFoundError("reference CPU build missing: make -C oracle ref")
        lib = ctypes.CDLL(LIB_REF)
        lib.few_ref_interpolate_arrays.restype = None
        lib.few_ref_interpolate_arrays.argtypes = [_dp, _dp, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _dp]
        lib.few_ref_get_waveform.restype = None
        lib.few_ref_interp2d.argtypes = [_dp, _dp, ctypes.c_int, _dp, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int,
                                         _dp, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        lib.few_ref_interp2d.restype = None
        lib.few_ref_get_waveform.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, _ip, _ip, _ip, ctypes.c_int,
                                             ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_double,
                                             _dp, ctypes.c_int]
    else:
        raise ValueError(impl)
    _libs[impl] = lib
    return lib


def _p(a, typ=_dp):
    return a.ctypes.data_as(typ)


def interpolate_arrays(t, y_all, impl: str = "oracle") -> np.ndarray:
    """Spline coefficients in the reference's native layout (4, ninterps, N):
    ``interpolate_arrays`` applied as ``CubicSplineInterpolant.__init__`` does
    before its final transpose (``interpolatedmodesum.py:52-97``)."""
    y_all = np.atleast_2d(np.asarray(y_all, dtype=np.float64))
    ninterps, length = y_all.shape
    t = np.asarray(t, dtype=np.float64)
    if t.ndim == 1:
        t_full = np.ascontiguousarray(np.tile(t, (ninterps, 1)).reshape(-1))
    else:
        t_full = np.ascontiguousarray(t.reshape(-1))
    interp = np.zeros((4, ninterps, length))
    interp[0] = y_all
    interp = np.ascontiguousarray(interp.reshape(-1))
    B = np.zeros(ninterps * length)
    up, dg, lo = np.zeros_like(B), np.zeros_like(B), np.zeros_like(B)
    lib = _lib(impl)
    if impl == "oracle":
        st = lib.oracle_interpolate_arrays(_p(t_full), _p(interp), ninterps, length, _p(B), _p(up), _p(dg), _p(lo))
        if st != 0:
            raise ValueError(f"oracle spline build failed with status {st}")
    else:
        lib.few_ref_interpolate_arrays(_p(t_full), _p(interp), ninterps, length, _p(B), _p(up), _p(dg), _p(lo))
    return interp.reshape(4, ninterps, length)


def spline_coeffs(t, y_all, impl: str = "oracle") -> np.ndarray:
    """``CubicSplineInterpolant.interp_array`` reshaped to (4, N, ninterps)."""
    return np.ascontiguousarray(np.transpose(interpolate_arrays(t, y_all, impl), (0, 2, 1)))


def spline_eval(t, coeffs, tnew, deriv_order: int = 0) -> np.ndarray:
    """``CubicSplineInterpolant.__call__`` (``interpolatedmodesum.py:118-257``)
    for 1-D knots t and coefficients (4, N, ninterps) -> (ninterps, M)."""
    t = np.asarray(t, dtype=np.float64)
    tnew = np.atleast_1d(np.asarray(tnew, dtype=np.float64))
    inds = np.searchsorted(t, tnew, side="right") - 1
    inds[tnew == t[-1]] = len(t) - 2
    bad_l = tnew < t[0]
    bad_r = tnew > t[-1]
    inds = np.clip(inds, 0, len(t) - 1)
    x = tnew - t[inds]
    y, c1, c2, c3 = (coeffs[c][inds].T for c in range(4))
    if deriv_order == 0:
        out = y + c1 * x + c2 * (x * x) + c3 * (x * x * x)
        out[:, bad_l] = coeffs[0][0][:, None]
        out[:, bad_r] = coeffs[0][-1][:, None]
    else:
        if bad_l.any() or bad_r.any():
            raise ValueError("x points outside of the domain of the spline are not supported when taking derivatives.")
        if deriv_order == 1:
            out = c1 + 2 * c2 * x + 3 * c3 * (x * x)
        elif deriv_order == 2:
            out = 2 * c2 + 6 * c3 * x
        elif deriv_order == 3:
            out = 6 * c3 * np.ones_like(x)
        else:
            raise ValueError("deriv_order must be within 0 <= deriv_order <= 3.")
    return out


def prepare_sum(inp):
    """The preprocessing of ``InterpolatedModeSum.sum``
    (``interpolatedmodesum.py:321-358``): y_all = [Re; Im] of teuk_modes.T,
    phase coefficients (N-1,3,8) -> flat (8,N-1,3), ylms[K:] *= (-1)^l."""
    K = inp.teuk_modes.shape[1]
    y_all = np.concatenate([inp.teuk_modes.T.real, inp.teuk_modes.T.imag], axis=0)
    pc = np.ascontiguousarray(np.transpose(np.asarray(inp.phase_coeffs, dtype=np.float64), (2, 0, 1)).reshape(-1))
    ylms = np.array(inp.ylms, dtype=np.complex128, copy=True)
    ylms[K:] *= (-1.0) ** np.asarray(inp.l)
    return y_all, pc, ylms


def mode_sum(inp, impl: str = "oracle", extended: bool = False, window=None,
             coeffs: np.ndarray | None = None, out_len: int | None = None, dphase=None) -> np.ndarray:
    """The waveform of ``InterpolatedModeSum.__call__`` on the CPU.

    impl="oracle": the C restatement (``extended`` selects the long double
    form; ``window=(lo, hi)`` computes only those output samples, the rest
    stay zero).  impl="ref": the reference's own get_waveform (whole output).
    ``coeffs`` optionally supplies amplitude spline coefficients (4, N, 2K).
    ``dphase=(dcoeffs, delta)`` (long double form only) adds delta times the
    phase basis dcoeffs (N-1, 3, 8) to the phases in long double: a phase
    finite difference whose step is not rounded into the large coefficients."""
    from fastemriwaveforms_b200.synthetic import output_length

    K = inp.teuk_modes.shape[1]
    N = len(inp.t)
    if out_len is None:
        out_len = output_length(inp.t, inp.T, inp.dt)[0]
    y_all, pc, ylms = prepare_sum(inp)
    if coeffs is None:
        coeffs = spline_coeffs(inp.t, y_all, impl=impl)
    interp = np.ascontiguousarray(coeffs.reshape(-1))
    m = np.ascontiguousarray(inp.m, dtype=np.int32)
    k = np.ascontiguousarray(inp.k, dtype=np.int32)
    n = np.ascontiguousarray(inp.n, dtype=np.int32)
    h_t = np.ascontiguousarray(inp.t, dtype=np.float64)
    pt = np.ascontiguousarray(inp.phase_t, dtype=np.float64)
    ylm_flat = np.ascontiguousarray(ylms).view(np.float64)
    wf = np.zeros(out_len, dtype=np.complex128)
    lib = _lib(impl)
    if impl == "oracle" and dphase is not None:
        lo, hi = (0, out_len) if window is None else window
        dpc_in, delta = dphase
        dpc = np.ascontiguousarray(np.transpose(np.asarray(dpc_in, dtype=np.float64), (2, 0, 1)).reshape(-1))
        st = lib.oracle_get_waveform_dphase(_p(wf.view(np.float64)), _p(interp), _p(pt), _p(pc), _p(dpc),
                                            float(delta), _p(m, _ip), _p(k, _ip), _p(n, _ip), N, out_len, K,
                                            _p(ylm_flat), float(inp.dt), _p(h_t), int(lo), int(hi))
        if st != 0:
            raise ValueError(f"oracle mode sum failed with status {st}")
    elif impl == "oracle":
        lo, hi = (0, out_len) if window is None else window
        st = lib.oracle_get_waveform(_p(wf.view(np.float64)), _p(interp), _p(pt), _p(pc), _p(m, _ip), _p(k, _ip),
                                     _p(n, _ip), N, out_len, K, _p(ylm_flat), float(inp.dt), _p(h_t),
                                     int(lo), int(hi), 1 if extended else 0)
        if st != 0:
            raise ValueError(f"oracle mode sum failed with status {st}")
    else:
        if window is not None or extended:
            raise ValueError("the reference build computes the whole waveform in double precision")
        lib.few_ref_get_waveform(wf.ctypes.data, _p(interp), _p(pt), _p(pc), _p(m, _ip), _p(k, _ip), _p(n, _ip),
                                 N, out_len, K, ylm_flat.ctypes.data, float(inp.dt), _p(h_t), 0)
    return wf


def find_start_inds(t, dt: float, out_len: int):
    """Segment starts of ``find_start_inds`` (``interpolate.cu:694-723``);
    returns (start (nseg+1,), nseg)."""
    t = np.ascontiguousarray(t, dtype=np.float64)
    start = np.zeros(len(t), dtype=np.int32)
    nseg = _lib("oracle").oracle_find_start_inds(_p(start, _ip), _p(t), float(dt), len(t), int(out_len))
    if nseg < 0:
        raise ValueError("knots do not reach the end of the output")
    return start[: nseg + 1], nseg


def rel_l2(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def mismatch(a, b) -> float:
    """1 - overlap, as ``get_mismatch`` (``src/few/utils/utility.py:16-95``)."""
    fa = np.fft.fft(np.asarray(a))
    fb = np.fft.fft(np.asarray(b))
    ac = np.vdot(fa, fb) / np.sqrt(np.vdot(fa, fa) * np.vdot(fb, fb))
    return float(1.0 - ac.real)


def window_problem(inp, coeffs, j0: int, samples: int):
    """Arguments of the reference's get_waveform for `samples` output samples
    starting at the first sample of knot segment j0, as a problem of its own:
    knots from j0 on, shifted by that sample's time so that it becomes sample
    0, with the same spline and phase coefficients (sliced).  Used to spread a
    CPU baseline over processes; the values differ from the whole-waveform call
    only by the rounding of the shifted times."""
    K = inp.teuk_modes.shape[1]
    start = int(np.ceil(inp.t[j0] / inp.dt)) if j0 > 0 else 0
    shift = start * inp.dt
    t_sub = np.ascontiguousarray(inp.t[j0:] - shift)
    pt_sub = np.ascontiguousarray(inp.phase_t[j0:] - shift)
    c_sub = np.ascontiguousarray(coeffs[:, j0:, :])
    _, pc, ylms = prepare_sum(inp)
    N = len(inp.t)
    pc_sub = np.ascontiguousarray(pc.reshape(8, N - 1, 3)[:, j0:, :].reshape(-1))
    return dict(t=t_sub, phase_t=pt_sub, coeffs=c_sub, pc=pc_sub, ylms=ylms, K=K, out_len=int(samples),
                m=np.ascontiguousarray(inp.m, dtype=np.int32), k=np.ascontiguousarray(inp.k, dtype=np.int32),
                n=np.ascontiguousarray(inp.n, dtype=np.int32), dt=float(inp.dt))


def run_window(prob, impl: str = "ref") -> np.ndarray:
    """Runs a window_problem through the reference's get_waveform (or the
    restatement) and returns its output."""
    lib = _lib(impl)
    wf = np.zeros(prob["out_len"], dtype=np.complex128)
    N = len(prob["t"])
    interp = prob["coeffs"].reshape(-1)
    ylm = np.ascontiguousarray(prob["ylms"]).view(np.float64)
    args = (_p(interp), _p(prob["phase_t"]), _p(prob["pc"]), _p(prob["m"], _ip), _p(prob["k"], _ip),
            _p(prob["n"], _ip), N, prob["out_len"], prob["K"])
    if impl == "ref":
        lib.few_ref_get_waveform(wf.ctypes.data, *args, ylm.ctypes.data, prob["dt"], _p(prob["t"]), 0)
    else:
        st = lib.oracle_get_waveform(_p(wf.view(np.float64)), *args, _p(ylm), prob["dt"], _p(prob["t"]), 0,
                                     prob["out_len"], 0)
        if st != 0:
            raise ValueError(f"oracle mode sum failed with status {st}")
    return wf


def interp2d(tx, ty, c, kx: int, ky: int, x, y, impl: str = "oracle") -> np.ndarray:
    """``interp2D`` (``src/few/cutils/AmpInterp2D.cu:86-208``): every grid of c
    (ngrid, len_indiv_c) evaluated at the points (x, y) -> (ngrid, m)."""
    tx = np.ascontiguousarray(tx, dtype=np.float64)
    ty = np.ascontiguousarray(ty, dtype=np.float64)
    c = np.ascontiguousarray(c, dtype=np.float64).reshape(-1, (len(tx) - kx - 1) * (len(ty) - ky - 1))
    x = np.ascontiguousarray(np.atleast_1d(x), dtype=np.float64)
    y = np.ascontiguousarray(np.atleast_1d(y), dtype=np.float64)
    m, ngrid, nc = len(x), c.shape[0], c.shape[1]
    z = np.zeros((ngrid, m), dtype=np.float64)
    if impl == "ref":
        _lib("ref").few_ref_interp2d(_p(z), _p(tx), len(tx), _p(ty), len(ty), _p(c), kx, ky, _p(x), m, _p(y), m,
                                     ngrid, nc)
    else:
        _lib("oracle").oracle_interp2d(_p(z), _p(tx), len(tx), _p(ty), len(ty), _p(c), kx, ky, _p(x), _p(y), m,
                                       ngrid, nc)
    return z


# ---------------------------------------------------------------------------
# Frequency-domain sum (FDInterpolatedModeSum.sum, src/few/summation/fdinterp.py)
# ---------------------------------------------------------------------------

FD_DENSE_POINTS = 5000  # fdinterp.py:266


def fd_frequency_grid(L: int, dt: float) -> np.ndarray:
    """The default two-sided grid (fdinterp.py:398-403)."""
    return np.hstack((np.arange(-(L // 2), 0), np.arange(0, (L - 1) // 2 + 1))) / (L * dt)


def fd_plan(t, fknots, fcoef, m, k, n, frequency, has_farr: bool):
    """Bin ranges of every (mode, segment): restates fdinterp.py:262-430.

    fknots (3, N): |f_phi|, f_theta, f_r at the knots; fcoef (4, N, 3): their
    spline coefficients.  Returns (start, end) int32 (K, N-1) as the reference
    hands them to its kernel.  Mirrored details: numpy.argmax/argmin on the
    5000-point dense grid, the Python index -1 for a turnover found at the
    first knot, and the widening of a turnover segment only when there is
    exactly one interior turnover (the join of the (n, 2) bounds with the
    (1, n) turnover row raises the ValueError the reference swallows)."""
    t = np.asarray(t, dtype=np.float64)
    m, k, n = (np.asarray(v, dtype=np.int64) for v in (m, k, n))
    N = len(t)
    tn = np.linspace(t.min(), t.max(), FD_DENSE_POINTS)
    dense = spline_eval(t, fcoef, tn)                                   # (3, D)
    knot = m[:, None] * fknots[0][None] + k[:, None] * fknots[1][None] + n[:, None] * fknots[2][None]
    bounds = np.sort(np.stack([knot[:, :-1], knot[:, 1:]], axis=-1), axis=-1)   # (K, N-1, 2)
    per_mode = m[:, None] * dense[0][None] + k[:, None] * dense[1][None] + n[:, None] * dense[2][None]
    turns = []
    for extreme in (per_mode.argmax(axis=-1), per_mode.argmin(axis=-1)):
        t_ext = tn[extreme]
        modes = np.where((t_ext > 0.0) & (t_ext < t[-1]))[0]
        segs = np.searchsorted(t, t_ext[modes]) - 1
        turns.extend(zip(modes.tolist(), segs.tolist()))
    if turns:
        modes = np.array([q[0] for q in turns])
        segs = np.array([q[1] for q in turns])
        cf = [m[modes] * fcoef[c][segs, 0] + k[modes] * fcoef[c][segs, 1] + n[modes] * fcoef[c][segs, 2]
              for c in range(4)]
        d, c, b, a = cf
        disc = (2 * b) ** 2 - 4 * (3 * a) * c
        if np.any(disc < -1e10):
            raise ValueError("turnover discriminant below -1e10")
        disc[disc < 0.0] = 0.0
        with np.errstate(divide="ignore", invalid="ignore"):
            r1 = (-(2 * b) + np.sqrt(disc)) / (2 * (3 * a))
            r2 = (-(2 * b) - np.sqrt(disc)) / (2 * (3 * a))
        tr1, tr2 = t[segs] + r1, t[segs] + r2
        keep1 = (t[segs] < tr1) & (t[segs + 1] > tr1)
        keep2 = (t[segs] < tr2) & (t[segs + 1] > tr2)
        if np.any(keep1 & keep2):
            raise ValueError("a turnover segment holds both roots")
        if np.any(keep1 | keep2) and len(turns) == 1:
            x = tr1 * keep1 + tr2 * keep2 - t[segs]
            f_ext = a * x ** 3 + b * x ** 2 + c * x + d
            three = np.sort(np.concatenate([bounds[modes, segs], f_ext[:, None]], axis=-1), axis=-1)
            bounds[modes, segs] = three[:, [0, 2]]
    f0 = frequency[0]
    df = frequency[1] - frequency[0]
    idx = np.abs((bounds - f0) / df).astype(int)
    if has_farr:
        z = int(np.where(frequency == 0.0)[0][0])
        pos = bounds > 0.0
        idx[pos] = (np.abs((bounds - frequency[z + 1]) / df).astype(int) + z + 1)[pos]
    return (idx[..., 0] + 1).astype(np.int32), idx[..., 1].astype(np.int32)


def fd_kernel(interp, phase_t, pc_kernel, m, k, n, t, frequency, start, end, ylms_signed, zero_index: int,
              include_minus_m: bool, impl: str = "oracle") -> np.ndarray:
    """The stationary-phase kernel on the reference's kernel inputs: few_oracle.c's
    restatement (impl="oracle") or the reference's get_waveform_generic_fd
    (impl="ref").  Returns the two-sided sum (L,) complex."""
    K, N, L = len(m), len(t), len(frequency)
    wf = np.zeros(L, dtype=np.complex128)
    a = dict(interp=np.ascontiguousarray(interp, dtype=np.float64).reshape(-1),
             pt=np.ascontiguousarray(phase_t, dtype=np.float64), pc=np.ascontiguousarray(pc_kernel).reshape(-1),
             m=np.ascontiguousarray(m, dtype=np.int32), k=np.ascontiguousarray(k, dtype=np.int32),
             n=np.ascontiguousarray(n, dtype=np.int32), t=np.ascontiguousarray(t, dtype=np.float64),
             f=np.ascontiguousarray(frequency, dtype=np.float64),
             s=np.ascontiguousarray(start, dtype=np.int32).reshape(-1),
             e=np.ascontiguousarray(end, dtype=np.int32).reshape(-1),
             y=np.ascontiguousarray(ylms_signed, dtype=np.complex128))
    lib = _lib(impl)
    if impl == "oracle":
        fn = lib.oracle_fd_sum
        fn.restype = None
        fn(wf.ctypes.data_as(_dp), _p(a["interp"]), _p(a["pt"]), _p(a["pc"]), _p(a["m"], _ip), _p(a["k"], _ip),
           _p(a["n"], _ip), ctypes.c_int(K), _p(a["t"]), ctypes.c_int(N), ctypes.c_int(L), _p(a["f"]),
           _p(a["s"], _ip), _p(a["e"], _ip), a["y"].ctypes.data_as(_dp), ctypes.c_int(zero_index),
           ctypes.c_int(int(include_minus_m)))
    else:
        fn = lib.few_ref_get_waveform_fd
        fn.restype = None
        fn(wf.ctypes.data_as(ctypes.c_void_p), _p(a["interp"]), _p(a["pt"]), _p(a["pc"]), _p(a["m"], _ip),
           _p(a["k"], _ip), _p(a["n"], _ip), ctypes.c_int(K), ctypes.c_double(0.0), _p(a["t"]), ctypes.c_int(N),
           ctypes.c_int(L), _p(a["f"]), _p(a["s"], _ip), _p(a["e"], _ip), ctypes.c_int(N - 1),
           a["y"].ctypes.data_as(ctypes.c_void_p), ctypes.c_int(zero_index), ctypes.c_int(int(include_minus_m)),
           ctypes.c_int(0))
    return wf


def fd_finalize(w: np.ndarray, frequency: np.ndarray, mask_positive: bool) -> np.ndarray:
    """(h+, hx) from the two-sided sum (fdinterp.py:518-536)."""
    s = -np.flip(w)
    p = np.real(s + np.flip(s)) / 2.0 + 1j * np.imag(s - np.flip(s)) / 2.0
    c = -np.imag(s + np.flip(s)) / 2.0 + 1j * np.real(s - np.flip(s)) / 2.0
    if mask_positive:
        keep = frequency >= 0.0
        return np.vstack((p[keep], c[keep]))
    return np.vstack((p, c))


def fd_sum(inp, fknots, L: int | None = None, f_arr=None, include_minus_m: bool = True,
           mask_positive: bool = False, impl: str = "oracle"):
    """The whole FD sum on the CPU from the trajectory's knot frequencies
    (3, N) in Hz: splines (the reference's interpolate_arrays layout), bin
    plan, kernel, (h+, hx).  Returns (waveform, frequency, start, end)."""
    K = inp.teuk_modes.shape[1]
    y_all = np.concatenate([inp.teuk_modes.T.real, inp.teuk_modes.T.imag, np.asarray(fknots)], axis=0)
    interp = interpolate_arrays(inp.t, y_all, impl="oracle" if impl == "oracle" else "ref")   # (4, 2K+3, N)
    fcoef = np.ascontiguousarray(np.transpose(interp[:, 2 * K:], (0, 2, 1)))                 # (4, N, 3)
    frequency = np.asarray(f_arr, dtype=np.float64) if f_arr is not None else fd_frequency_grid(L, inp.dt)
    start, end = fd_plan(inp.t, np.asarray(fknots), fcoef, inp.m, inp.k, inp.n, frequency, f_arr is not None)
    pc_kernel = np.transpose(np.asarray(inp.phase_coeffs, dtype=np.float64), (2, 1, 0))      # (8, 3, N-1)
    ylms = np.array(inp.ylms, dtype=np.complex128, copy=True)
    ylms[K:] *= (-1) ** np.asarray(inp.l)
    zero_index = int(np.where(frequency == 0.0)[0][0])
    w = fd_kernel(interp, inp.phase_t, pc_kernel, inp.m, inp.k, inp.n, inp.t, frequency, start, end, ylms,
                  zero_index, include_minus_m, impl=impl)
    return fd_finalize(w, frequency, mask_positive), frequency, start, end


# ---------------------------------------------------------------------------
# AAK summation (AAKSummation.sum, src/few/summation/aakwave.py; kernel gpuAAK.cu)
# ---------------------------------------------------------------------------

_GPCINSEC = 1.02927125054339e+17     # global.h:26
_AUSEC = 499.00478383615643          # global.h:27
_MTSUN = 4.9254909491978065e-06      # global.h:24
_YRSID = 31558149.763545595          # global.h:23


def aak_segments(h_t, out_len: int, dt: float):
    """First sample of each trajectory segment (gpuAAK.cu:495-519): ceil(t_j/dt)
    while t_j < T = (out_len-1) dt, then out_len at the first knot past T."""
    T = (out_len - 1) * dt
    first = [0]
    for tt in h_t[1:]:
        if tt < T:
            first.append(int(np.ceil(tt / dt)))
        else:
            first.append(out_len)
            break
    return np.array(first, dtype=np.int64)


def aak_waveform(interp_t, interp_coeffs, M, S, mu, qS, phiS, qK, phiK, dist, nmodes: int, mich: bool,
                 out_len: int, dt: float, impl: str = "numpy") -> np.ndarray:
    """The AAK waveform (out_len,) complex: restated in numpy with scipy's
    Bessel functions (impl="numpy", restates gpuAAK.cu:181-482), or the
    reference's own CPU kernel (impl="ref", whose Bessel functions are the
    Numerical Recipes approximations).  interp_coeffs (N-1, 6, 8) as
    AAKSummation.sum receives them (after its |Y| == 1 substitution)."""
    interp_t = np.ascontiguousarray(interp_t, dtype=np.float64)
    N = len(interp_t)
    kernel_layout = np.ascontiguousarray(np.transpose(np.asarray(interp_coeffs, dtype=np.float64), (2, 0, 1)))
    wf = np.zeros(out_len, dtype=np.complex128)
    if impl == "ref":
        fn = _lib("ref").few_ref_aak_waveform
        fn.restype = None
        fn(wf.ctypes.data_as(ctypes.c_void_p), _p(kernel_layout.reshape(-1)), ctypes.c_double(M), ctypes.c_double(S),
           ctypes.c_double(mu), ctypes.c_double(qS), ctypes.c_double(phiS), ctypes.c_double(qK), ctypes.c_double(phiK),
           ctypes.c_double(dist), ctypes.c_int(nmodes), ctypes.c_int(int(mich)), ctypes.c_int(N),
           ctypes.c_int(out_len), ctypes.c_double(dt), _p(interp_t))
        return wf
    from scipy.special import jv

    first = aak_segments(interp_t, out_len, dt)
    nseg = len(first) - 1
    idx = np.arange(first[0], first[-1])
    seg = np.searchsorted(first, idx, side="right") - 1
    seg = np.clip(seg, 0, nseg - 1)
    c = np.asarray(interp_coeffs, dtype=np.float64)[seg]          # (ns, 6, 8)
    t = dt * idx
    h = interp_t[seg + 1] - interp_t[seg]
    s = (t - interp_t[seg]) / h
    s1 = 1.0 - s

    def nested(q):
        cc = c[:, q]
        return cc[:, 0] + s * (cc[:, 1] + s1 * (cc[:, 2] + s * (cc[:, 3] + s1 * (cc[:, 4] + s * (cc[:, 5] + s1 * (
            cc[:, 6] + s * cc[:, 7]))))))

    def deriv(q):
        cc = c[:, q]
        s2, s3, s4, s5, s6 = s * s, s ** 3, s ** 4, s ** 5, s ** 6
        return (cc[:, 1] + cc[:, 2] * (1. - 2. * s) + cc[:, 3] * (2. * s - 3. * s2)
                + cc[:, 4] * (2. * s - 6. * s2 + 4. * s3) + cc[:, 5] * (3. * s2 - 8. * s3 + 5. * s4)
                + cc[:, 6] * (3. * s2 - 12. * s3 + 15 * s4 - 6. * s5)
                + cc[:, 7] * (4. * s3 - 15. * s4 + 18. * s5 - 7. * s6)) / h

    fill = 1e-6
    qS = min(max(qS, fill), np.pi - fill)
    qK = min(max(qK, fill), np.pi - fill)
    cosqS, sinqS, cosqK, sinqK = np.cos(qS), np.sin(qS), np.cos(qK), np.sin(qK)
    cosphiK, sinphiK = np.cos(phiK), np.sin(phiK)
    halfsqrt3 = np.sqrt(3.) / 2.
    zeta = mu * _MTSUN / dist / _GPCINSEC
    e, Y = nested(1), nested(2)
    Pphi, Pth, Pr = nested(3), nested(4), nested(5)
    Ophi, Oth, Or = deriv(3), deriv(4), deriv(5)
    Phi, gim, alp = Pr, Pth - Pr, Pphi - Pth
    nu, gimdot = Or / (2. * np.pi), Oth - Or
    lam = np.arccos(Y)
    coslam, sinlam, cosalp, sinalp = np.cos(lam), np.sin(lam), np.cos(alp), np.sin(alp)
    cosqL = cosqK * coslam + sinqK * sinlam * cosalp
    sinqL = np.sqrt(1. - cosqL * cosqL)
    up = sinqK * sinphiK * coslam - cosphiK * sinlam * sinalp - cosqK * sinphiK * sinlam * cosalp
    down = sinqK * cosphiK * coslam + sinphiK * sinlam * sinalp - cosqK * cosphiK * sinlam * cosalp
    phiL = np.arctan2(up, down)
    Ldotn = cosqL * cosqS + sinqL * sinqS * np.cos(phiL - phiS)
    Ldotn2 = Ldotn * Ldotn
    Sdotn = cosqK * cosqS + sinqK * sinqS * np.cos(phiK - phiS)
    bup = -Sdotn + coslam * Ldotn
    bdown = sinqS * np.sin(phiK - phiS) * sinlam * cosalp + (cosqK * Sdotn - cosqS) / sinqK * sinlam * sinalp
    beta = np.where((S == 0.0) | (lam < 1e-10) | (lam > np.pi - 1e-10), 0.0, np.arctan2(bup, bdown))
    gam = 2. * (gim + beta)
    cos2gam, sin2gam = np.cos(gam), np.sin(gam)
    if mich:
        orb = 2. * np.pi * t / _YRSID
        cosorb, sinorb = np.cos(orb - phiS), np.sin(orb - phiS)
        cosq = .5 * cosqS - halfsqrt3 * sinqS * cosorb
        phiw = orb + np.arctan2(halfsqrt3 * cosqS + .5 * sinqS * cosorb, sinqS * sinorb)
        psiup = .5 * cosqK - halfsqrt3 * sinqK * np.cos(orb - phiK) - cosq * (cosqK * cosqS + sinqK * sinqS * np.cos(phiK - phiS))
        psidown = (.5 * sinqK * sinqS * np.sin(phiK - phiS)
                   - halfsqrt3 * np.cos(orb) * (cosqK * sinqS * np.sin(phiS) - cosqS * sinqK * np.sin(phiK))
                   - halfsqrt3 * np.sin(orb) * (cosqS * sinqK * np.cos(phiK) - cosqK * sinqS * np.cos(phiS)))
        psi = np.arctan2(psiup, psidown)
        cosq1 = .5 * (1. + cosq * cosq)
        c2phi, s2phi, c2psi, s2psi = np.cos(2. * phiw), np.sin(2. * phiw), np.cos(2. * psi), np.sin(2. * psi)
        FpI = cosq1 * c2phi * c2psi - cosq * s2phi * s2psi
        FcI = cosq1 * c2phi * s2psi + cosq * s2phi * c2psi
        FpII = cosq1 * s2phi * c2psi + cosq * c2phi * s2psi
        FcII = cosq1 * s2phi * s2psi - cosq * c2phi * c2psi
    else:
        FpI, FcI, FpII, FcII = 1.0, 0.0, 0.0, 1.0
    Amp = (np.abs(Ophi) * M * _MTSUN) ** (2. / 3.) * zeta
    # polarisation rotation (gpuAAK.cu:141-177)
    nv = np.array([np.sin(qS) * np.cos(phiS), np.sin(qS) * np.sin(phiS), np.cos(qS)])
    Sv = np.array([np.sin(qK) * np.cos(phiK), np.sin(qK) * np.sin(phiK), np.cos(qK)])
    ci, si = np.cos(lam), np.sin(lam)
    Lv = np.stack([ci * np.sin(qK) * np.cos(phiK) + si * (sinalp * np.sin(phiK) - cosalp * np.cos(qK) * np.cos(phiK)),
                   ci * np.sin(qK) * np.sin(phiK) - si * (sinalp * np.cos(phiK) + cosalp * np.cos(qK) * np.sin(phiK)),
                   ci * np.cos(qK) + si * cosalp * np.sin(qK)], axis=1)
    nxL = np.cross(np.broadcast_to(nv, Lv.shape), Lv)
    nxS = np.cross(nv, Sv)
    norm = np.linalg.norm(nxL, axis=1) * np.linalg.norm(nxS)
    norm = np.where(norm < 1e-6, 1e-6, norm)
    cosrot = (nxL @ nxS) / norm
    sinrot = (Lv @ nxS - nxL @ Sv) / norm
    rot0, rot1 = 2. * cosrot * cosrot - 1., cosrot * sinrot
    rot2, rot3 = -rot1, rot0
    hI = np.zeros_like(t)
    hII = np.zeros_like(t)
    for n in range(1, nmodes + 1):
        if mich:
            fn = n * nu + gimdot / np.pi
            nPhi = n * Phi + 2. * np.pi * fn * _AUSEC * sinqS * cosorb
        else:
            nPhi = n * Phi
        x = n * e
        J0, J1, J2, J3, J4 = (jv(n - 2 + q, x) for q in range(5))
        a = -n * Amp * (J0 - 2. * e * J1 + 2. / n * J2 + 2. * e * J3 - J4) * np.cos(nPhi)
        b = -n * Amp * np.sqrt(1 - e * e) * (J0 - 2. * J2 + J4) * np.sin(nPhi)
        cc = 2. * Amp * J2 * np.cos(nPhi)
        Ap0 = -(1. + Ldotn2) * (a * cos2gam - b * sin2gam) + cc * (1 - Ldotn2)
        Ac0 = 2. * Ldotn * (b * cos2gam + a * sin2gam)
        Ap, Ac = Ap0 * rot0 + Ac0 * rot1, Ap0 * rot2 + Ac0 * rot3
        scale = halfsqrt3 if mich else 1.0
        hI += scale * (FpI * Ap + FcI * Ac)
        hII += scale * (FpII * Ap + FcII * Ac)
    wf[idx] = hI - 1j * hII
    return wf


def direct_sum(teuk, ylms, phases, l, m, k, n) -> np.ndarray:
    """DirectModeSum.sum restated (src/few/summation/directmodesum.py:101-131):
    the +m terms of every mode and the -m images of the m > 0 modes."""
    teuk = np.asarray(teuk)
    K = teuk.shape[1]
    pp, pt, pr = (np.asarray(p, dtype=np.float64)[:, None] for p in phases)
    m, k, n, l = (np.asarray(v)[None, :] for v in (m, k, n, l))
    phase = m * pp + k * pt + n * pr
    w1 = (np.asarray(ylms)[None, :K] * teuk * np.exp(-1j * phase)).sum(axis=1)
    pos = m[0] > 0
    w2 = ((-1.0) ** l[:, pos] * np.asarray(ylms)[None, K:][:, pos] * np.conj(teuk[:, pos])
          * np.exp(1j * phase[:, pos])).sum(axis=1)
    return w1 + w2


# ---------------------------------------------------------------------------
# DOPR853 dense output (src/few/trajectory/dopr853.py)
# ---------------------------------------------------------------------------

# Dense-output weights of DOP853 (Hairer, Norsett & Wanner; dopr853.py:130-181):
# rows rcont5..8, columns k1, k6, k7, k8, k9, k10, k11, k12, f(x1), k14, k15, k16.
DOPR853_D = np.array([
    [-0.84289382761090128651353491142e01, 0.56671495351937776962531783590e00, -0.30689499459498916912797304727e01,
     0.23846676565120698287728149680e01, 0.21170345824450282767155149946e01, -0.87139158377797299206789907490e00,
     0.22404374302607882758541771650e01, 0.63157877876946881815570249290e00, -0.88990336451333310820698117400e-01,
     0.18148505520854727256656404962e02, -0.91946323924783554000451984436e01, -0.44360363875948939664310572000e01],
    [0.10427508642579134603413151009e02, 0.24228349177525818288430175319e03, 0.16520045171727028198505394887e03,
     -0.37454675472269020279518312152e03, -0.22113666853125306036270938578e02, 0.77334326684722638389603898808e01,
     -0.30674084731089398182061213626e02, -0.93321305264302278729567221706e01, 0.15697238121770843886131091075e02,
     -0.31139403219565177677282850411e02, -0.93529243588444783865713862664e01, 0.35816841486394083752465898540e02],
    [0.19985053242002433820987653617e02, -0.38703730874935176555105901742e03, -0.18917813819516756882830838328e03,
     0.52780815920542364900561016686e03, -0.11573902539959630126141871134e02, 0.68812326946963000169666922661e01,
     -0.10006050966910838403183860980e01, 0.77771377980534432092869265740e00, -0.27782057523535084065932004339e01,
     -0.60196695231264120758267380846e02, 0.84320405506677161018159903784e02, 0.11992291136182789328035130030e02],
    [-0.25693933462703749003312586129e02, -0.15418974869023643374053993627e03, -0.23152937917604549567536039109e03,
     0.35763911791061412378285349910e03, 0.93405324183624310003907691704e02, -0.37458323136451633156875139351e02,
     0.10409964950896230045147246184e03, 0.29840293426660503123344363579e02, -0.43533456590011143754432175058e02,
     0.96324553959188282948394950600e02, -0.39177261675615439165231486172e02, -0.14972683625798562581422125276e03]])
# extra stages 14..16 (dopr853.py:98-128): node, then couplings in the reference's summation order
DOPR853_EXTRA = [
    (0.1, [(0, 5.61675022830479523392909219681e-2), (6, 2.53500210216624811088794765333e-1),
           (7, -2.46239037470802489917441475441e-1), (8, -1.24191423263816360469010140626e-1),
           (9, 1.5329179827876569731206322685e-1), (1, 8.20105229563468988491666602057e-3),
           (2, 7.56789766054569976138603589584e-3), ("f", -8.298e-3)]),
    (0.2, [(0, 3.18346481635021405060768473261e-2), (5, 2.83009096723667755288322961402e-2),
           (6, 5.35419883074385676223797384372e-2), (7, -5.49237485713909884646569340306e-2),
           (1, -1.08347328697249322858509316994e-4), (2, 3.82571090835658412954920192323e-4),
           ("f", -3.40465008687404560802977114492e-4), (14, 1.41312443674632500278074618366e-1)]),
    (0.777777777777777777777777777778,
     [(0, -4.28896301583791923408573538692e-1), (5, -4.69762141536116384314449447206e0),
      (6, 7.68342119606259904184240953878e0), (7, 4.06898981839711007970213554331e0),
      (8, 3.56727187455281109270669543021e-1), ("f", -1.39902416515901462129418009734e-3),
      (14, 2.9475147891527723389556272149e0), (15, -9.15095847217987001081870187138e0)]),
]


def dopr853_prep_evaluate(x0, y0, h0, x1, y1, stages, ode, args=None):
    """DOPR853.prep_evaluate (dopr853.py:621-758) restated in numpy, batched:
    x0, h0, x1 (nsys,), y0, y1 (node, nsys), stages (10, node, nsys) as
    take_step leaves them (slots 1, 2 = stages 11, 12); ``ode(x, y, dydx,
    args)`` the right-hand side.  Every sum runs left to right as numpy
    evaluates the reference's expressions.  Returns rcont (nsys, node, 8)."""
    k = [np.asarray(s, dtype=np.float64) for s in stages]
    f1 = np.zeros_like(y0)
    ode(x1, y1, f1, args)
    diff = y1 - y0
    bspl = h0 * k[0] - diff
    rc = [y0, diff, bspl, diff - h0 * f1 - bspl]
    cols = [k[0], k[5], k[6], k[7], k[8], k[9], k[1], k[2]]
    part = []
    for q in range(4):
        s = DOPR853_D[q][0] * cols[0]
        for c in range(1, 8):
            s = s + DOPR853_D[q][c] * cols[c]
        part.append(s)
    extra = {}
    for node_c, terms in DOPR853_EXTRA:
        s = None
        for src, coef in terms:
            v = f1 if src == "f" else (extra[src] if src in (14, 15) else k[src])
            s = coef * v if s is None else s + coef * v
        arg = y0 + h0 * s
        out = np.zeros_like(y0)
        ode(x0 + node_c * h0, arg, out, args)
        extra[14 + len(extra)] = out
    for q in range(4):
        s = part[q]
        for c, v in zip(range(8, 12), (f1, extra[14], extra[15], extra[16])):
            s = s + DOPR853_D[q][c] * v
        rc.append(h0 * s)
    return np.array(rc).T
