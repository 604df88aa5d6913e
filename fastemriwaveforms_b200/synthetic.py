"""Seeded synthetic EMRI-like inputs for the interpolated mode sum.

No public dataset is involved in this path: the inputs of
``InterpolatedModeSum`` (``src/few/summation/interpolatedmodesum.py:283-375``)
are a trajectory's knot times, Teukolsky amplitudes at those knots, spherical
harmonics and DOPR853-style phase coefficients.  This module draws them from
fixed generators with the shapes and value ranges of a FastEMRIWaveforms
trajectory, seeded with ``numpy.random.default_rng``.

Workloads (sizes are part of the benchmark definition):

* ``plain_small``  -- K=200 modes (l=2..4, m=0..l, n=-10..10, truncated),
  N=100 knots on [0, 1e6] s, dt=10 s, 100,001 samples.
* ``plain_full``   -- K=3843 modes (l=2..10, m=0..l, n=-30..30), N=1000 knots
  on [0, 3.15e7] s, dt=10 s, 3,150,001 samples (one year at 10 s cadence).
* ``adjoint``      -- K=1000 (prefix of the full list), N=500 knots,
  1,000,000 samples.
* ``batch``        -- many waveforms with uneven T, N and K.
* ``fd_case``      -- inputs of the frequency-domain sum: the above plus a
  trajectory (M, a, p(t), e(t), x) whose Kerr geodesic frequencies set each
  mode's frequency track; ``fd_full`` is the one-year, 3843-mode size.

Phases are closed-form integrals of a chirping frequency
f(t) = 1e-3 (1 - t/t_c)^(-3/8) Hz:
Phi_phi = int 2 pi f dt and Phi_r = int 0.78 * 2 pi f (1 + 0.1 t/S) dt.
They are fitted with not-a-knot cubic splines and written in the 8-term
dense-output basis the sum kernel evaluates (``interpolate.cu:637-644``): a
cubic y0 + A1 s + A2 s^2 + A3 s^3 in s = (t - t_j)/h is exactly the basis
vector (y0, A1+A2+A3, -A2-A3, -A3, 0, 0, 0, 0).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

YRSID_SI = 31558149.763545595  # seconds per sidereal year (src/few/cutils/global.h:23)


@dataclass
class ModeSumInputs:
    """Arguments of ``InterpolatedModeSum.__call__`` for one waveform."""

    t: np.ndarray              # (N,) knot times, s
    teuk_modes: np.ndarray     # (N, K) complex amplitudes at the knots
    ylms: np.ndarray           # (2K,) complex: +m harmonics, then -m harmonics
    phase_t: np.ndarray        # (N,) knot times of the phase polynomials
    phase_coeffs: np.ndarray   # (N-1, 3, 8) [Phi_phi, Phi_theta, Phi_r] basis coefficients
    l: np.ndarray              # (K,) int
    m: np.ndarray
    k: np.ndarray
    n: np.ndarray
    dt: float
    T: float                   # observation time in years (SummationBase.__call__)
    phase_knots: np.ndarray = field(default=None)  # (3, N) phase values at the knots
    name: str = ""
    seed: int = 0

    @property
    def num_modes(self) -> int:
        return int(self.teuk_modes.shape[1])

    @property
    def num_knots(self) -> int:
        return int(self.t.shape[0])

    @property
    def out_len(self) -> int:
        """Output length as SummationBase.__call__ computes it (no padding)."""
        return output_length(self.t, self.T, self.dt)[0]

    def call_args(self):
        return (self.t, self.teuk_modes, self.ylms, self.phase_t, self.phase_coeffs,
                self.l, self.m, self.k, self.n)


def output_length(t, T: float, dt: float, pad_output: bool = False, odd_len: bool = False):
    """(num_pts, num_pts_pad) exactly as ``SummationBase.__call__``
    (``src/few/summation/base.py:87-124``)."""
    n_pts = int(T * YRSID_SI / dt)
    Tsec = n_pts * dt
    t0 = float(t[0])
    t1 = float(t[-1])
    if Tsec < t1:
        num_pts = int((Tsec - t0) / dt) + 1
        num_pts_pad = 0
    else:
        num_pts = int((t1 - t0) / dt) + 1
        num_pts_pad = int((Tsec - t0) / dt) + 1 - num_pts if pad_output else 0
    if odd_len and (num_pts + num_pts_pad) % 2 == 0:
        num_pts_pad += 1
    return num_pts, num_pts_pad


def mode_list(lmax: int, nmax: int, count: int | None = None):
    """(l, m, k, n) in product order l=2..lmax, m=0..l, n=-nmax..nmax, k=0."""
    ls, ms, ns = [], [], []
    for l in range(2, lmax + 1):
        for m in range(0, l + 1):
            for n in range(-nmax, nmax + 1):
                ls.append(l)
                ms.append(m)
                ns.append(n)
    ls = np.asarray(ls, dtype=np.int32)
    ms = np.asarray(ms, dtype=np.int32)
    ns = np.asarray(ns, dtype=np.int32)
    if count is not None:
        ls, ms, ns = ls[:count], ms[:count], ns[:count]
    return ls, ms, np.zeros_like(ms), ns


def knot_times(rng, N: int, span: float, min_gap: float) -> np.ndarray:
    """N sorted knots on [0, span]: endpoints fixed, N-2 uniform draws
    conditioned on every gap being >= min_gap (spacing transform of sorted
    uniforms, equal in law to redrawing until the condition holds)."""
    free = span - (N - 1) * min_gap
    if free <= 0:
        raise ValueError("min_gap too large for the span")
    u = np.sort(rng.uniform(0.0, free, N - 2))
    t = np.empty(N)
    t[0] = 0.0
    t[-1] = span
    t[1:-1] = u + min_gap * np.arange(1, N - 1)
    return t


def phase_values(t, t_c: float, scale: float, f0: float = 1e-3):
    """Closed-form Phi_phi(t), Phi_r(t) of the chirp f = f0 (1 - t/t_c)^(-3/8)."""
    w = 1.0 - np.asarray(t, dtype=np.float64) / t_c
    a = 0.1 * t_c / scale
    phi = 2.0 * np.pi * f0 * t_c * 1.6 * (1.0 - w ** 0.625)
    phr = 2.0 * np.pi * 0.78 * f0 * t_c * ((1.0 + a) * 1.6 * (1.0 - w ** 0.625)
                                           - a * (8.0 / 13.0) * (1.0 - w ** 1.625))
    return phi, phr


def cubic_to_basis(y0, c1, c2, c3, h):
    """Map cubic segments y0 + c1 x + c2 x^2 + c3 x^3 (x = t - t_j, width h)
    onto the 8-term basis y + s(b1 + s1(b2 + s(b3 + s1(...)))) of
    ``interpolate.cu:637-644`` with s = x/h, s1 = 1 - s.  Returns (..., 8)."""
    A1 = c1 * h
    A2 = c2 * h * h
    A3 = c3 * h * h * h
    out = np.zeros(np.shape(y0) + (8,))
    out[..., 0] = y0
    out[..., 1] = A1 + A2 + A3
    out[..., 2] = -A2 - A3
    out[..., 3] = -A3
    return out


def not_a_knot_coeffs(t, y):
    """Not-a-knot cubic spline coefficients (y, c1, c2, c3) per segment, each
    (..., N-1), via scipy (same boundary conditions as the reference spline)."""
    from scipy.interpolate import CubicSpline

    cs = CubicSpline(t, y, axis=-1, bc_type="not-a-knot")
    c = cs.c  # (4, N-1, ...) highest power first
    c = np.moveaxis(c, 1, -1) if c.ndim == 3 else c
    return c[3], c[2], c[1], c[0]


def phase_basis_from_knots(t, phase_knots):
    """(N-1, 3, 8) phase coefficients from (3, N) phase knot values, through
    not-a-knot cubic splines."""
    N = len(t)
    h = np.diff(t)
    out = np.zeros((N - 1, 3, 8))
    for q in range(3):
        if not np.any(phase_knots[q]):
            continue
        y0, c1, c2, c3 = not_a_knot_coeffs(t, phase_knots[q])
        out[:, q, :] = cubic_to_basis(y0, c1, c2, c3, h)
    return out


def make_inputs(K: int, N: int, span: float, t_c: float, lmax: int, nmax: int, seed: int,
                dt: float = 10.0, scale: float | None = None, name: str = "",
                min_gap: float | None = None) -> ModeSumInputs:
    rng = np.random.default_rng(seed)
    scale = span if scale is None else scale
    if min_gap is None:
        # 1e3 s at N=100 on [0, 1e6] s, rescaled with the mean gap elsewhere
        min_gap = 0.099 * span / (N - 1)
    t = knot_times(rng, N, span, min_gap)
    l, m, k, n = mode_list(lmax, nmax, K)
    K = len(l)
    phi, phr = phase_values(t, t_c, scale)
    phase_knots = np.stack([phi, np.zeros_like(phi), phr])
    phase_coeffs = phase_basis_from_knots(t, phase_knots)

    a = (rng.standard_normal(K) + 1j * rng.standard_normal(K)) / np.sqrt(2.0)
    a *= np.exp(-np.abs(n) / 4.0) / (l.astype(np.float64) ** 2)
    omega = rng.uniform(0.0, 1e-6, K)
    teuk = a[None, :] * (1.0 + 0.5 * t[:, None] / scale) * np.exp(1j * omega[None, :] * t[:, None])

    # one (+m, -m) harmonic pair per (l, m)
    lm_keys = sorted(set(zip(l.tolist(), m.tolist())))
    yp = {}
    for key in lm_keys:
        z = (rng.standard_normal(4)) / np.sqrt(2.0)
        yp[key] = (z[0] + 1j * z[1], z[2] + 1j * z[3])
    ylms = np.empty(2 * K, dtype=np.complex128)
    for j in range(K):
        p, q = yp[(int(l[j]), int(m[j]))]
        ylms[j] = p
        ylms[K + j] = q

    T = (span + dt) / YRSID_SI
    return ModeSumInputs(t=t, teuk_modes=np.ascontiguousarray(teuk), ylms=ylms, phase_t=t.copy(),
                         phase_coeffs=phase_coeffs, l=l, m=m, k=k, n=n, dt=dt, T=T,
                         phase_knots=phase_knots, name=name, seed=seed)


def plain_small(seed: int = 1) -> ModeSumInputs:
    """K=200, N=100 on [0, 1e6] s, t_c=1.2e6 s, S=1e6 s, dt=10 s, 100,001 samples."""
    return make_inputs(K=200, N=100, span=1e6, t_c=1.2e6, lmax=4, nmax=10, seed=seed,
                       scale=1e6, name="plain_small", min_gap=1e3)


def plain_full(seed: int = 2) -> ModeSumInputs:
    """K=3843, N=1000 on [0, 3.15e7] s, t_c=3.2e7 s, S=span, dt=10 s, 3,150,001 samples."""
    return make_inputs(K=3843, N=1000, span=3.15e7, t_c=3.2e7, lmax=10, nmax=30, seed=seed,
                       name="plain_full")


def adjoint_case(seed: int = 4) -> ModeSumInputs:
    """K=1000 (prefix of the full list), N=500, 1,000,000 samples (span 1e7 s)."""
    return make_inputs(K=1000, N=500, span=1e7 - 10.0, t_c=1.1e7, lmax=10, nmax=30, seed=seed,
                       name="adjoint")


def batch_cases(count: int = 256, seed: int = 5):
    """Waveforms with T ~ logU[1e5, 3.15e6] samples, N ~ U[50, 2000], K ~ U[200, 3843]
    (prefixes of the full mode list), independent seeds."""
    rng = np.random.default_rng(seed)
    out = []
    for w in range(count):
        T_samples = int(np.exp(rng.uniform(np.log(1e5), np.log(3.15e6))))
        N = int(rng.integers(50, 2001))
        K = int(rng.integers(200, 3844))
        span = (T_samples - 1) * 10.0
        out.append(make_inputs(K=K, N=N, span=span, t_c=span * 1.02, lmax=10, nmax=30,
                               seed=int(rng.integers(1 << 31)), name=f"batch{w}"))
    return out


def small_case(K: int = 10, N: int = 20, out_len: int = 4000, seed: int = 7, dt: float = 10.0,
               theta: bool = True, high_order: bool = True) -> ModeSumInputs:
    """A small case in the style of the reference's own summation test
    (tests/test_mode_summation.py:64-151): random m in [2,4], k in {0,1},
    n in [-4,3], arbitrary 8-term phase polynomials (all coefficients set,
    Phi_theta included), linear-ramp amplitudes."""
    rng = np.random.default_rng(seed)
    span = (out_len - 1) * dt
    t = knot_times(rng, N, span, 0.2 * span / (N - 1))
    l = rng.integers(2, 5, K).astype(np.int32)
    m = rng.integers(2, 5, K).astype(np.int32)
    k = (rng.integers(0, 2, K) if theta else np.zeros(K)).astype(np.int32)
    n = rng.integers(-4, 4, K).astype(np.int32)
    # phase polynomials: smooth growth plus small high-order terms
    phase_coeffs = np.zeros((N - 1, 3, 8))
    rates = np.array([2e-3, 1.3e-3, 0.9e-3]) * 2 * np.pi
    for q in range(3):
        base = rates[q] * t
        h = np.diff(t)
        phase_coeffs[:, q, 0] = base[:-1]
        phase_coeffs[:, q, 1] = rates[q] * h
        if high_order:
            phase_coeffs[:, q, 2:] = rng.normal(0, 1e-3, (N - 1, 6))
    if not theta:
        phase_coeffs[:, 1, :] = 0.0
    lo = rng.uniform(-1, 1, (2, K))
    hi = rng.uniform(-1, 1, (2, K))
    frac = (t / span)[:, None]
    teuk = (lo[0] + (hi[0] - lo[0]) * frac) + 1j * (lo[1] + (hi[1] - lo[1]) * frac)
    ylms = (rng.standard_normal(2 * K) + 1j * rng.standard_normal(2 * K)) / np.sqrt(2.0)
    T = (span + dt) / YRSID_SI
    return ModeSumInputs(t=t, teuk_modes=np.ascontiguousarray(teuk), ylms=ylms, phase_t=t.copy(),
                         phase_coeffs=phase_coeffs, l=l, m=m, k=k, n=n, dt=dt, T=T,
                         name="small", seed=seed)


def many_rows_case(seed: int = 9, N: int = 30, out_len: int = 20000, mmax: int = 10, kmax: int = 1,
                   nmax: int = 5, dt: float = 10.0) -> ModeSumInputs:
    """Every (m, k) with m in 0..mmax and |k| <= kmax, n in -nmax..nmax (l = max(2, m)):
    (2 mmax + 1) (2 kmax + 1) fold rows (63 by default, more than 32, so the
    tensor-core forms use two MMA column groups); phases as ``small_case``."""
    base = small_case(K=4, N=N, out_len=out_len, seed=seed, dt=dt, theta=True)
    rng = np.random.default_rng(seed + 1)
    modes = [(max(2, m), m, k, n) for m in range(mmax + 1) for k in range(-kmax, kmax + 1)
             for n in range(-nmax, nmax + 1)]
    l = np.array([q[0] for q in modes], np.int32)
    m = np.array([q[1] for q in modes], np.int32)
    k = np.array([q[2] for q in modes], np.int32)
    n = np.array([q[3] for q in modes], np.int32)
    K = len(modes)
    t = base.t
    frac = (t / t[-1])[:, None]
    lo = rng.uniform(-1, 1, (2, K))
    hi = rng.uniform(-1, 1, (2, K))
    teuk = (lo[0] + (hi[0] - lo[0]) * frac) + 1j * (lo[1] + (hi[1] - lo[1]) * frac)
    ylms = (rng.standard_normal(2 * K) + 1j * rng.standard_normal(2 * K)) / np.sqrt(2.0)
    return ModeSumInputs(t=t, teuk_modes=np.ascontiguousarray(teuk), ylms=ylms, phase_t=t.copy(),
                         phase_coeffs=base.phase_coeffs, l=l, m=m, k=k, n=n, dt=dt, T=base.T,
                         name="many_rows", seed=seed)


def amplitude_grids(num_modes: int, nw: int = 40, nu: int = 40, seed: int = 11, degree: int = 3):
    """Seeded B-spline amplitude grids in the shape the reference's data files
    hold: clamped knots on w in [0, 1] and u in [0, 1] (end knots repeated
    degree + 1 times, interior knots uniform), coefficients (num_modes, 2,
    (nw - degree - 1)(nu - degree - 1)) decaying with the mode index."""
    rng = np.random.default_rng(seed)
    k1 = degree + 1
    tw = np.concatenate([np.zeros(k1), np.linspace(0, 1, nw - 2 * k1 + 2)[1:-1], np.ones(k1)])
    tu = np.concatenate([np.zeros(k1), np.linspace(0, 1, nu - 2 * k1 + 2)[1:-1], np.ones(k1)])
    nc = (nw - k1) * (nu - k1)
    scale = 1.0 / (1.0 + np.arange(num_modes))[:, None, None]
    coeff = rng.standard_normal((num_modes, 2, nc)) * scale
    return tw, tu, coeff


def amplitude_points(N: int, seed: int = 12):
    """A smooth trajectory in (w, u) through the grid's domain, N points."""
    s = np.linspace(0.0, 1.0, N)
    return 0.05 + 0.9 * s ** 1.5, 0.5 + 0.4 * np.sin(2.0 * np.pi * s) * (1.0 - s)


@dataclass
class FDTrajectory:
    """The orbit arguments of ``FDInterpolatedModeSum.sum`` (fdinterp.py:138-160)."""

    M: float          # primary mass, solar masses
    a: float          # dimensionless spin
    p: np.ndarray     # (N,) semi-latus rectum at the knots
    e: np.ndarray     # (N,) eccentricity at the knots
    xI: np.ndarray    # (N,) cos of the inclination at the knots


def fd_mode_list(lmax: int, kmax: int, nmax: int, count: int | None = None):
    """(l, m, k, n) for l = 2..lmax, m = 0..l, k = -kmax..kmax, n = -nmax..nmax."""
    modes = [(l, m, k, n) for l in range(2, lmax + 1) for m in range(0, l + 1)
             for k in range(-kmax, kmax + 1) for n in range(-nmax, nmax + 1)]
    if count is not None:
        modes = modes[:count]
    arr = np.asarray(modes, dtype=np.int32).reshape(-1, 4)
    return (np.ascontiguousarray(arr[:, i]) for i in range(4))


def phase_knots_from_frequencies(t, t_dense, f_dense):
    """Phases 2 pi int_{t0}^{t} f dt at the knots t from frequencies f_dense
    (3, D) sampled on t_dense (through the antiderivative of a cubic spline)."""
    from scipy.interpolate import CubicSpline

    cs = CubicSpline(t_dense, np.asarray(f_dense), axis=1)
    anti = cs.antiderivative()
    return 2.0 * np.pi * (anti(np.asarray(t)) - anti(np.asarray(t)[0])[:, None])


def fd_case(K: int = 77, N: int = 50, span: float = 2e6, seed: int = 21, a: float = 0.0, x: float = 1.0,
            M: float = 1e6, lmax: int = 3, kmax: int = 0, nmax: int = 5, dt: float = 10.0,
            p_range=(12.0, 7.4), e_range=(0.4, 0.2), frequencies=None, name: str = "fd"):
    """Inputs of the frequency-domain sum: (ModeSumInputs, FDTrajectory).

    p falls from p_range[0] to p_range[1] as 1 - (1 - u)^0.8 (u = t/span) and
    e linearly; x is constant.  Amplitudes and harmonics are drawn as in
    ``make_inputs``.  ``frequencies`` (optional) is a callable
    (M, a, p, e, x) -> (3, D) array of (|f_phi|, f_theta, f_r) in Hz along
    the trajectory; given it, the phases are their integrals (a self-consistent
    waveform, whose stationary phase is flat at the roots), otherwise the
    closed-form chirp of ``phase_values`` (any smooth phases exercise the sum)."""
    rng = np.random.default_rng(seed)
    t = knot_times(rng, N, span, 0.099 * span / (N - 1))
    def orbit(tt):
        u = np.asarray(tt) / span
        return (p_range[0] + (p_range[1] - p_range[0]) * (1.0 - (1.0 - u) ** 0.8),
                e_range[0] + (e_range[1] - e_range[0]) * u)

    u = t / span
    p, e = orbit(t)
    xI = np.full(N, float(x))
    l, m, k, n = fd_mode_list(lmax, kmax, nmax, K)
    K = len(l)
    amp = (rng.standard_normal(K) + 1j * rng.standard_normal(K)) / np.sqrt(2.0)
    amp *= np.exp(-np.abs(n) / 4.0) / (l.astype(np.float64) ** 2)
    omega = rng.uniform(0.0, 1e-6, K)
    teuk = amp[None, :] * (1.0 + 0.5 * u[:, None]) * np.exp(1j * omega[None, :] * t[:, None])
    ylms = (rng.standard_normal(2 * K) + 1j * rng.standard_normal(2 * K)) / np.sqrt(2.0)
    if frequencies is None:
        phi, phr = phase_values(t, 1.2 * span, span)
        phase_knots = np.stack([phi, 0.6 * phi, phr])
    else:
        td = np.linspace(t[0], t[-1], 20 * N)
        pd, ed = orbit(td)
        fdense = np.asarray(frequencies(M, a, pd, ed, np.full(len(td), float(x))), dtype=np.float64)
        phase_knots = phase_knots_from_frequencies(t, td, fdense)
    phase_coeffs = phase_basis_from_knots(t, phase_knots)
    T = (span + dt) / YRSID_SI
    inp = ModeSumInputs(t=t, teuk_modes=np.ascontiguousarray(teuk), ylms=ylms, phase_t=t.copy(),
                        phase_coeffs=phase_coeffs, l=l, m=m, k=k, n=n, dt=dt, T=T,
                        phase_knots=phase_knots, name=name, seed=seed)
    return inp, FDTrajectory(M=M, a=a, p=p, e=e, xI=xI)


def fd_full(seed: int = 23, frequencies=None):
    """One year at dt = 10 s: K = 3843 modes (l = 2..10, m = 0..l, n = -30..30),
    N = 1000 knots on [0, 3.15e7] s, M = 1e6, a = 0.5, prograde equatorial,
    p 12 -> 7.4, e 0.4 -> 0.2."""
    return fd_case(K=3843, N=1000, span=3.15e7, seed=seed, a=0.5, x=1.0, lmax=10, kmax=0, nmax=30,
                   frequencies=frequencies, name="fd_full")


class FixedAmplitudes:
    """A stand-in amplitude generator for ``ModeSelector``: seeded amplitudes
    (N, K) on the mode list of the reference's amplitude modules
    (``src/few/utils/baseclasses.py:205-330``: l = 2..lmax, m = 0..l,
    k = -kmax..kmax, n = -nmax..nmax, ordered m = 0 first), with the mode
    bookkeeping attributes ModeSelector reads (``l_arr_no_mask`` ...,
    ``unique_l``, ``unique_m``, ``inverse_lm``, ``index_map_arr`` with Python's
    wrap-around for negative m, k, n).  The amplitude magnitudes fall off with
    l and |n| so that a power threshold keeps a strict subset."""

    def __init__(self, lmax: int = 4, kmax: int = 0, nmax: int = 6, N: int = 60, seed: int = 41):
        md = [(l, m, k, n) for l in range(2, lmax + 1) for m in range(0, l + 1)
              for k in range(-kmax, kmax + 1) for n in range(-nmax, nmax + 1)]
        md = np.asarray(md, dtype=np.int32)
        order = np.concatenate([np.where(md[:, 1] == 0)[0], np.where(md[:, 1] != 0)[0]])
        md = md[order]
        self.l_arr_no_mask, self.m_arr_no_mask, self.k_arr_no_mask, self.n_arr_no_mask = (
            np.ascontiguousarray(md[:, i]) for i in range(4))
        nz = self.m_arr_no_mask != 0
        self.l_arr = np.concatenate([self.l_arr_no_mask, self.l_arr_no_mask[nz]])
        self.m_arr = np.concatenate([self.m_arr_no_mask, -self.m_arr_no_mask[nz]])
        self.k_arr = np.concatenate([self.k_arr_no_mask, self.k_arr_no_mask[nz]])
        self.n_arr = np.concatenate([self.n_arr_no_mask, self.n_arr_no_mask[nz]])
        temp, self.inverse_lm = np.unique(np.asarray([self.l_arr, self.m_arr]).T, axis=0, return_inverse=True)
        self.inverse_lm = self.inverse_lm.reshape(-1)
        self.unique_l, self.unique_m = np.asarray(temp).T
        self.index_map_arr = np.full((lmax + 1, 2 * lmax + 1, 2 * kmax + 1, 2 * nmax + 1), -1, dtype=np.int32)
        for i, (l, m, k, n) in enumerate(zip(self.l_arr, self.m_arr, self.k_arr, self.n_arr)):
            self.index_map_arr[l, m, k, n] = i
        rng = np.random.default_rng(seed)
        K = len(md)
        mag = np.exp(-np.abs(self.n_arr_no_mask) / 1.5) / self.l_arr_no_mask.astype(np.float64) ** 3
        amp = (rng.standard_normal(K) + 1j * rng.standard_normal(K)) * mag
        s = np.linspace(0.0, 1.0, N)
        self.teuk = np.ascontiguousarray(amp[None, :] * (1.0 + 0.6 * s[:, None])
                                         * np.exp(1j * rng.uniform(0, 2, K)[None, :] * s[:, None]))

    def __call__(self, a, p, e, xI, specific_modes=None):
        if specific_modes is None:
            return self.teuk
        if hasattr(specific_modes, "cpu"):  # a torch tensor (the GPU ModeSelector passes device indices)
            specific_modes = specific_modes.cpu().numpy()
        return self.teuk[:, np.asarray(specific_modes)]


@dataclass
class AAKInputs:
    """Arguments of ``AAKSummation.__call__`` (aakwave.py:35-60) for one waveform."""

    t: np.ndarray              # (N,) knot times (tvec and interp_t)
    interp_coeffs: np.ndarray  # (N-1, 6, 8): (p, e, Y, Phi_phi, Phi_theta, Phi_r) in the 8-term basis
    m1: float
    a: float
    dist: float
    m2: float
    qS: float
    phiS: float
    qK: float
    phiK: float
    nmodes: int
    dt: float
    T: float

    def call_args(self):
        return (self.t, self.m1, self.a, self.dist, self.m2, self.qS, self.phiS, self.qK, self.phiK, self.nmodes,
                self.t, self.interp_coeffs)


def aak_case(N: int = 60, span: float = 1e6, seed: int = 51, e_range=(0.6, 0.35), Y: float = 0.7,
             nmodes: int | None = None, dt: float = 10.0, a: float = 0.6, f0: float = 1.5e-3) -> AAKInputs:
    """A seeded AAK trajectory: p 12 -> 8, e and Y smooth, phases from the
    closed-form chirp (Phi_theta and Phi_r slightly slower than Phi_phi, so the
    precession angles grow), all as not-a-knot cubics in the 8-term basis.
    nmodes defaults to the reference's rule int(30 e0) (src/few/waveform/base.py:596)."""
    rng = np.random.default_rng(seed)
    t = knot_times(rng, N, span, 0.099 * span / (N - 1))
    u = t / span
    p = 12.0 - 4.0 * u ** 1.2
    e = e_range[0] + (e_range[1] - e_range[0]) * u
    Yv = Y + 0.02 * np.sin(3 * u)
    w = 1.0 - t / (1.3 * span)
    phi = 2.0 * np.pi * f0 * 1.3 * span * 1.6 * (1.0 - w ** 0.625)
    knots = np.stack([p, e, Yv, phi, 0.995 * phi, 0.97 * phi])
    coeffs = np.zeros((N - 1, 6, 8))
    h = np.diff(t)
    for q in range(6):
        y0, c1, c2, c3 = not_a_knot_coeffs(t, knots[q])
        coeffs[:, q, :] = cubic_to_basis(y0, c1, c2, c3, h)
    if nmodes is None:
        nmodes = int(30 * e_range[0])
    return AAKInputs(t=t, interp_coeffs=coeffs, m1=1e6, a=a, dist=1.0, m2=10.0, qS=0.8, phiS=1.9, qK=2.1,
                     phiK=0.4, nmodes=nmodes, dt=dt, T=(span + dt) / YRSID_SI)


def direct_case(samples: int = 20001, K: int = 24, seed: int = 61):
    """Dense inputs of ``DirectModeSum`` in the style of the reference's test
    (tests/test_mode_summation.py:152-200): linearly ramping complex amplitudes
    (samples, K), linear phases reaching ~1e6 rad, random (l, m, k, n) with
    m = 0 modes among them, complex-normal harmonics.  Returns
    (t, teuk, ylms, phases (3, samples), l, m, k, n)."""
    rng = np.random.default_rng(seed)
    t = np.linspace(0, 1e5, samples)
    amp = np.linspace(rng.uniform(-1, 1, (2, K)), rng.uniform(-1, 1, (2, K)), t.size, axis=-1)
    teuk = np.ascontiguousarray((amp[0] + 1j * amp[1]).T)
    phases = np.asarray([np.pi / 3 + 12.0 * t, np.pi / 6 + 2.0 * t, np.pi / 4 + 9.0 * t])
    l = rng.integers(2, 6, K)
    m = rng.integers(0, 5, K)
    k = rng.integers(0, 2, K)
    n = rng.integers(-3, 3, K)
    ylms = (rng.standard_normal(2 * K) + 1j * rng.standard_normal(2 * K)) / np.sqrt(2.0)
    return t, teuk, ylms, phases, l, m, k, n


def toy_inspiral_ode(xp):
    """A smooth inspiral-like ODE in the reference integrator's signature
    ``ode(x, y, dydx, additionalArgs)`` (src/few/trajectory/dopr853.py:208),
    batched over systems: y (8, nsys) = (p, e, x_I, Phi_phi, Phi_theta,
    Phi_r, u, v), x (nsys,) the time in seconds; (u, v) is an oscillator of
    period ~31 ks that wobbles e (so that the stepper takes ~1000 steps over
    1e6 s).  ``xp`` is numpy (the reference's stepper) or torch (device
    arrays).  Only +, -, *, / and sqrt appear, all correctly rounded on both,
    and every division is array / array (torch turns a division by or of a
    Python number into a multiplication by a reciprocal), so the two give the
    same bits for the same inputs.

        dp/dt   = -1e-6 (1 + 7.3 e^2) (12 / p)^3
        de/dt   = -5e-8 e (12 / p)^4 + 1e-7 u
        dx/dt   = -1e-8 (1 - x^2)
        dPhi_phi/dt = w = 2 pi 1e-3 (12 / p)^(3/2)
        dPhi_theta/dt = w (1 - 0.5 / p)
        dPhi_r/dt   = w (1 - 6 / p) sqrt(1 - e^2)
        du/dt = 2e-4 v,  dv/dt = -2e-4 u
    """

    def ode(x, y, dydx, additional_args):
        p, e, xi, u, v = y[0], y[1], y[2], y[6], y[7]
        one = xp.ones_like(p)
        q = (12.0 * one) / p
        q3 = q * q * q
        w = 6.283185307179586e-3 * (q * xp.sqrt(q))
        dydx[0] = -1e-6 * (1.0 + 7.3 * (e * e)) * q3
        dydx[1] = -5e-8 * e * (q3 * q) + 1e-7 * u
        dydx[2] = -1e-8 * (1.0 - xi * xi)
        dydx[3] = w
        dydx[4] = w * (1.0 - (0.5 * one) / p)
        dydx[5] = w * (1.0 - (6.0 * one) / p) * xp.sqrt(1.0 - e * e)
        dydx[6] = 2e-4 * v
        dydx[7] = -2e-4 * u

    return ode
