"""Generates the frequency-domain golden vectors (tests/golden/fd_*.npz,
geodesic_frequencies.npz) and the spin-weighted harmonics (ylm.npz) from the
reference itself.

The reference's Python modules for this path are imported from its sources
with stand-ins for the packages this image lacks: ``numba`` (njit and
cuda.jit become plain Python functions, so the numba kernels run as the
Python they are written in), the backend and logging layers, and the
constants module (MTSUN_SI and YRSID_SI as src/few/cutils/global.h:23-24
defines them).  The rest runs unmodified:

* ``get_fundamental_frequencies`` (src/few/utils/geodesic.py:470-535) with
  the elliptic integrals of src/few/utils/elliptic.py;
* the -2 spin-weighted harmonics of ``GetYlms`` (src/few/utils/ylm.py:17-276)
  and the selections of ``ModeSelector`` (src/few/utils/modeselector.py:252-490)
  on a fixed-amplitude generator;
* ``DirectModeSum.sum`` (src/few/summation/directmodesum.py:30-131), numpy;
* ``FDInterpolatedModeSum.sum`` (src/few/summation/fdinterp.py:138-542) with
  the reference's ``CubicSplineInterpolant`` (interpolatedmodesum.py:12-257),
  whose native ``interpolate_arrays`` and ``get_waveform_generic_fd`` are the
  reference's CPU code (interpolate.cu) built by ``make -C oracle ref``.

    python tests/golden/make_fd_golden.py       (needs the reference sources)
"""
from __future__ import annotations

import ctypes
import importlib.util
import logging
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from fastemriwaveforms_b200 import synthetic as S  # noqa: E402
from oracle import oracle as O  # noqa: E402

REF = os.path.join(O.REFERENCE_ROOT, "src", "few")
MTSUN_SI = 4.9254909491978065e-06   # global.h:24
YRSID_SI = 31558149.763545595       # global.h:23


def _module(name, **attrs):
    mod = types.ModuleType(name)
    mod.__dict__.update(attrs)
    sys.modules[name] = mod
    return mod


def _package(name, path):
    mod = _module(name)
    mod.__path__ = [path]
    return mod


def _load(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def load_reference():
    """Imports the reference modules of the path (see the module docstring)."""

    def njit(*args, **kwargs):
        if args and callable(args[0]):
            return args[0]
        return lambda f: f

    _module("numba", njit=njit, cuda=types.SimpleNamespace(jit=njit, grid=lambda n: 0))
    _package("few", REF)
    _package("few.utils", os.path.join(REF, "utils"))
    _package("few.summation", os.path.join(REF, "summation"))
    _module("few.utils.constants", PI=3.141592653589793238462643383279502884, YRSID_SI=YRSID_SI,
            MTSUN_SI=MTSUN_SI)
    _module("few.utils.globals", get_logger=lambda: logging.getLogger("few"), get_first_backend=lambda *a: None)
    _module("few.utils.citations", REFERENCE=types.SimpleNamespace(), Citable=object)

    class ParallelModuleBase:
        def __init__(self, force_backend=None, **kwargs):
            self.xp = np
            self.backend = types.SimpleNamespace(interpolate_arrays_wrap=_ref_interpolate_arrays)

        @classmethod
        def GPU_RECOMMENDED(cls):
            return ["cpu"]

    _module("few.utils.baseclasses", BackendLike=object, ParallelModuleBase=ParallelModuleBase,
            SchwarzschildEccentric=type("SchwarzschildEccentric", (), {}))
    _load("few.utils.exceptions", os.path.join(REF, "utils/exceptions.py"))
    _load("few.utils.elliptic", os.path.join(REF, "utils/elliptic.py"))
    _load("few.utils.utility", os.path.join(REF, "utils/utility.py"))
    geo = _load("few.utils.geodesic", os.path.join(REF, "utils/geodesic.py"))
    _load("few.summation.base", os.path.join(REF, "summation/base.py"))
    ims = _load("few.summation.interpolatedmodesum", os.path.join(REF, "summation/interpolatedmodesum.py"))
    fdi = _load("few.summation.fdinterp", os.path.join(REF, "summation/fdinterp.py"))
    return geo, ims, fdi


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _ref_interpolate_arrays(t, interp_array, ninterps, length, B, upper, diag, lower):
    O._lib("ref").few_ref_interpolate_arrays(_dp(t), _dp(interp_array), ninterps, length, _dp(B), _dp(upper),
                                             _dp(diag), _dp(lower))


CAPTURE = {}


def _ref_get_waveform_fd(waveform, interp_array, phase_t, phase_coeffs, m, k, n, K, dt, t, init_len, data_len,
                         frequency, start_inds, end_inds, nseg, ylms, zero_index, include_minus_m, separate_modes):
    lib = O._lib("ref")
    f = lib.few_ref_get_waveform_fd
    f.restype = None
    m, k, n = (np.ascontiguousarray(q, dtype=np.int32) for q in (m, k, n))
    ns = 2 * K + 3
    fknots = interp_array.reshape(4, ns, init_len)[0, 2 * K:]
    CAPTURE.update(start_inds=start_inds.copy(), end_inds=end_inds.copy(), zero_index=int(zero_index),
                   ylms_signed=ylms.copy(), interp_array=interp_array.copy(), phase_kernel=phase_coeffs.copy(),
                   fknots=fknots.copy(), frequency=frequency.copy())
    f(waveform.ctypes.data_as(ctypes.c_void_p), _dp(interp_array), _dp(phase_t), _dp(phase_coeffs), _ip(m), _ip(k),
      _ip(n), ctypes.c_int(K), ctypes.c_double(dt), _dp(t), ctypes.c_int(init_len), ctypes.c_int(data_len),
      _dp(frequency), _ip(start_inds), _ip(end_inds), ctypes.c_int(nseg), ylms.ctypes.data_as(ctypes.c_void_p),
      ctypes.c_int(zero_index), ctypes.c_int(int(include_minus_m)), ctypes.c_int(int(separate_modes)))
    CAPTURE["raw"] = waveform.copy()


def run_reference_fd(fdi, ims, inp, tr, T, dt, f_arr=None, include_minus_m=True, mask_positive=False,
                     pad_output=True):
    """The reference's FD sum on one input set: returns (waveform (2, L'),
    frequency, the captured kernel inputs)."""
    num_pts, num_pts_pad = S.output_length(inp.t, T, dt, pad_output, odd_len=True)
    fake = types.SimpleNamespace()
    fake.xp = np
    fake.num_pts, fake.num_pts_pad = num_pts, num_pts_pad
    L = len(f_arr) if f_arr is not None else num_pts + num_pts_pad
    fake.waveform = np.zeros(L, dtype=np.complex128)
    fake.build_with_same_backend = lambda cls, args=(), kwargs=None: cls(*args, **(kwargs or {}))
    fake.get_waveform_fd = _ref_get_waveform_fd
    CAPTURE.clear()
    fdi.FDInterpolatedModeSum.sum(fake, inp.t, inp.teuk_modes, inp.ylms, inp.phase_t, inp.phase_coeffs, inp.l,
                                  inp.m, inp.k, inp.n, tr.M, tr.a, tr.p, tr.e, tr.xI, dt=dt, f_arr=f_arr,
                                  include_minus_m=include_minus_m, mask_positive=mask_positive)
    return fake.waveform, fake.frequency, dict(CAPTURE), (num_pts, num_pts_pad)


def save_fd(name, inp, tr, wf, freq, cap, lengths, **opts):
    d = dict(t=inp.t, teuk_modes=inp.teuk_modes, ylms=inp.ylms, phase_t=inp.phase_t, phase_coeffs=inp.phase_coeffs,
             l=inp.l, m=inp.m, k=inp.k, n=inp.n, dt=inp.dt, T=inp.T, M=tr.M, a=tr.a, p=tr.p, e=tr.e, xI=tr.xI,
             waveform=wf, frequency=freq, start_inds=cap["start_inds"], end_inds=cap["end_inds"],
             raw=cap["raw"], zero_index=cap["zero_index"], num_pts=lengths[0], num_pts_pad=lengths[1],
             interp_array=cap["interp_array"], phase_kernel=cap["phase_kernel"], ylms_signed=cap["ylms_signed"],
             fknots=cap["fknots"])
    d.update({k: np.asarray(v) for k, v in opts.items() if v is not None})
    np.savez_compressed(os.path.join(HERE, name), **d)


def geodesic_case(geo):
    """Fundamental frequencies on a grid of orbits covering every branch of
    get_fundamental_frequencies: Schwarzschild (a = 0), circular equatorial,
    eccentric equatorial (pro- and retrograde) and generic inclined orbits."""
    rows = []
    for a in (0.0, 0.3, 0.9):
        for x in (1.0, -1.0, 0.6, -0.4):
            if a == 0.0 and abs(x) != 1.0:
                continue
            for e in (0.0, 1e-12, 0.1, 0.45):
                for p in (9.0, 14.0, 30.0):
                    try:
                        out = geo.get_fundamental_frequencies(a, p, e, x)
                    except (ValueError, ZeroDivisionError):
                        continue
                    if np.all(np.isfinite(out)):
                        rows.append((a, p, e, x) + tuple(float(v) for v in out))
    arr = np.array(rows)
    np.savez_compressed(os.path.join(HERE, "geodesic_frequencies.npz"), a=arr[:, 0], p=arr[:, 1], e=arr[:, 2],
                        x=arr[:, 3], OmegaPhi=arr[:, 4], OmegaTheta=arr[:, 5], OmegaR=arr[:, 6])
    return len(rows)


def reference_frequencies(geo):
    """(M, a, p, e, x) -> (3, D) Hz by the reference's own geodesic code and
    conversion (fdinterp.py:224-236): the phases of the golden inputs are the
    integrals of these, so each mode's phase is stationary at its roots."""

    def freqs(M, a, p, e, x):
        Ophi, Oth, Or = geo.get_fundamental_frequencies(a, p, e, x)
        den = 2 * np.pi * M * MTSUN_SI
        return np.stack([np.abs(Ophi / den), Oth / den, Or / den])

    return freqs


def ylm_case():
    """The reference's GetYlms kernel (src/few/utils/ylm.py:17-276) for every
    (l, m), l = 2..10, at viewing angles including the poles."""
    ylm = _load("few.utils.ylm", os.path.join(REF, "utils/ylm.py"))
    ls = np.array([l for l in range(2, 11) for m in range(-l, l + 1)], dtype=np.int32)
    ms = np.array([m for l in range(2, 11) for m in range(-l, l + 1)], dtype=np.int32)
    angles = np.array([(0.0, 0.0), (np.pi / 3, np.pi / 4), (1.1, -2.3), (np.pi / 2, 0.7), (2.9, 5.5),
                       (np.pi, 1.0), (1e-3, 0.2)])
    out = np.zeros((len(angles), len(ls)), dtype=np.complex128)
    for i, (th, ph) in enumerate(angles):
        out[i] = ylm._ylm_kernel(np.zeros(len(ls), dtype=np.complex128), ls, ms, th, ph)
    np.savez_compressed(os.path.join(HERE, "ylm.npz"), l=ls, m=ms, angles=angles, ylm=out)
    return out.shape


def modeselector_case():
    """The reference's ModeSelector (src/few/utils/modeselector.py:14-490) on a
    fixed-amplitude generator: the threshold form at two thresholds, the 'all'
    form and a list of modes (its amplitude generator and trajectory imports
    stubbed; GetYlms is the reference's)."""
    _module("few.trajectory")
    _module("few.trajectory.inspiral", EMRIInspiral=object)
    _load("few.utils.ylm", os.path.join(REF, "utils/ylm.py"))
    ms_mod = _load("few.utils.modeselector", os.path.join(REF, "utils/modeselector.py"))
    gen = S.FixedAmplitudes()
    t = np.sort(np.random.default_rng(5).uniform(0, 1e6, gen.teuk.shape[0]))
    sel = ms_mod.ModeSelector(gen)
    out = {"t": t}
    for tag, thr in (("thr5", 1e-5), ("thr2", 1e-2)):
        r = sel(t, 0.5, None, None, None, 1.1, 0.7, mode_selection_threshold=thr, return_sort_inds=True)
        for name, v in zip(("teuk", "ylms", "l", "m", "k", "n", "inv"), r):
            out[f"{tag}_{name}"] = np.asarray(v)
    r = sel(t, 0.5, None, None, None, 0.4, 2.0, mode_selection="all")
    out["all_ylms"] = np.asarray(r[1])
    modes = [(2, 2, 0, 0), (3, 1, 0, -2), (4, 0, 0, 3)]
    r = sel(t, 0.5, None, None, None, 0.4, 2.0, mode_selection=modes)
    out["list_teuk"], out["list_ylms"] = np.asarray(r[0]), np.asarray(r[1])
    np.savez_compressed(os.path.join(HERE, "modeselector.npz"), **out)
    return {k: v.shape for k, v in out.items() if k.endswith("_l")}


def _subset(inp, keep):
    """The modes `keep` of a ModeSumInputs (amplitudes, both ylm halves, l m k n)."""
    K = inp.teuk_modes.shape[1]
    keep = np.asarray(keep)
    sub = S.ModeSumInputs(t=inp.t, teuk_modes=np.ascontiguousarray(inp.teuk_modes[:, keep]),
                          ylms=np.concatenate([inp.ylms[keep], inp.ylms[K + keep]]), phase_t=inp.phase_t,
                          phase_coeffs=inp.phase_coeffs, l=inp.l[keep], m=inp.m[keep], k=inp.k[keep],
                          n=inp.n[keep], dt=inp.dt, T=inp.T, name=inp.name, seed=inp.seed)
    return sub


def _turnovers(inp, fk):
    """Interior turnovers of each mode's frequency on the reference's dense grid
    (fdinterp.py:262-300), by the oracle's spline of the knot frequencies."""
    K = inp.teuk_modes.shape[1]
    fcoef = np.ascontiguousarray(np.transpose(O.interpolate_arrays(inp.t, fk, impl="ref"), (0, 2, 1)))
    tn = np.linspace(inp.t.min(), inp.t.max(), 5000)
    dense = O.spline_eval(inp.t, fcoef, tn)
    m, k, n = (np.asarray(v, dtype=np.int64) for v in (inp.m, inp.k, inp.n))
    per = m[:, None] * dense[0][None] + k[:, None] * dense[1][None] + n[:, None] * dense[2][None]
    cnt = np.zeros(K, dtype=int)
    for ext in (per.argmax(-1), per.argmin(-1)):
        te = tn[ext]
        cnt += ((te > 0.0) & (te < inp.t[-1])).astype(int)
    return cnt


def single_turnover_case(fdi, ims, freqs):
    """A mode list with exactly one interior turnover over all modes, so the
    reference's widening of that segment (fdinterp.py:318-376) takes effect:
    one turning mode plus monotone ones, on the Schwarzschild trajectory."""
    inp, tr = S.fd_case(K=77, N=50, span=1e6, seed=21, a=0.0, x=1.0, lmax=3, nmax=5, frequencies=freqs)
    fk = np.asarray(freqs(tr.M, tr.a, tr.p, tr.e, tr.xI))
    cnt = _turnovers(inp, fk)
    turning = np.where(cnt == 1)[0]
    mono = np.where(cnt == 0)[0]
    for j in turning:
        keep = np.concatenate([[j], mono[:11]])
        sub = _subset(inp, keep)
        if int(_turnovers(sub, fk).sum()) != 1:
            continue
        wf, freq, cap, lens = run_reference_fd(fdi, ims, sub, tr, sub.T, sub.dt)
        start, end = O.fd_plan(sub.t, fk, np.ascontiguousarray(np.transpose(
            O.interpolate_arrays(sub.t, fk, impl="ref"), (0, 2, 1))), sub.m, sub.k, sub.n, freq, False)
        save_fd("fd_single_turnover.npz", sub, tr, wf, freq, cap, lens)
        return int(j), len(keep)
    raise RuntimeError("no mode list with a single interior turnover found")


def direct_sum_case():
    """The reference's DirectModeSum (src/few/summation/directmodesum.py:30-131),
    numpy all the way, on synthetic.direct_case() (the reference test's dummy
    case with random harmonics, m = 0 modes and phases of ~1e6 rad).  The
    inputs are regenerated from their seed; the file keeps the output and a
    digest of the inputs."""
    import hashlib

    dms = _load("few.summation.directmodesum", os.path.join(REF, "summation/directmodesum.py"))
    t, teuk, ylms, phases, l, m, k, n = S.direct_case()
    fake = types.SimpleNamespace(xp=np)
    dms.DirectModeSum.sum(fake, t, teuk, ylms, t, phases, l, m, k, n)
    h = hashlib.sha256()
    for a in (t, teuk, ylms, phases, l, m, k, n):
        h.update(np.ascontiguousarray(a).tobytes())
    np.savez_compressed(os.path.join(HERE, "direct_sum.npz"), waveform=fake.waveform, digest=h.hexdigest())
    return fake.waveform.shape


def main():
    O.build(ref=True)
    geo, ims, fdi = load_reference()
    print("geodesic rows:", geodesic_case(geo))
    print("ylm:", ylm_case())
    print("modeselector:", modeselector_case())
    print("direct sum:", direct_sum_case())
    freqs = reference_frequencies(geo)

    # 1. Schwarzschild, eccentric, default frequency grid, +/- m
    inp, tr = S.fd_case(K=77, N=50, span=1e6, seed=21, a=0.0, x=1.0, lmax=3, nmax=5, frequencies=freqs)
    wf, freq, cap, lens = run_reference_fd(fdi, ims, inp, tr, inp.T, inp.dt)
    save_fd("fd_schwarzschild.npz", inp, tr, wf, freq, cap, lens)
    print("fd_schwarzschild", wf.shape, float(np.abs(wf).max()))

    # 1b. exactly one interior turnover: the widening of its segment applies
    print("fd_single_turnover (mode, modes):", single_turnover_case(fdi, ims, freqs))

    # 2. Kerr prograde equatorial, user frequency grid (positive-side index rule)
    inp, tr = S.fd_case(K=66, N=40, span=8e5, seed=22, a=0.6, x=1.0, lmax=3, nmax=4, p_range=(11.0, 6.6),
                        frequencies=freqs)
    L = 2 * 40001 + 1
    f_arr = np.hstack((np.arange(-(L // 2), 0), np.arange(0, (L - 1) // 2 + 1))) * (1.0 / (L * 11.0))
    wf, freq, cap, lens = run_reference_fd(fdi, ims, inp, tr, inp.T, inp.dt, f_arr=f_arr)
    save_fd("fd_kerr_farr.npz", inp, tr, wf, freq, cap, lens, f_arr=f_arr)
    print("fd_kerr_farr", wf.shape, float(np.abs(wf).max()))

    # 3. generic inclined orbit (k != 0 modes), +m only, positive frequencies only
    inp, tr = S.fd_case(K=90, N=36, span=6e5, seed=24, a=0.7, x=0.8, lmax=2, kmax=1, nmax=4,
                        p_range=(12.0, 8.0), e_range=(0.3, 0.15), frequencies=freqs)
    wf, freq, cap, lens = run_reference_fd(fdi, ims, inp, tr, inp.T, inp.dt, include_minus_m=False,
                                           mask_positive=True)
    save_fd("fd_generic_pos.npz", inp, tr, wf, freq, cap, lens, include_minus_m=0, mask_positive=1)
    print("fd_generic_pos", wf.shape, float(np.abs(wf).max()))


if __name__ == "__main__":
    main()
