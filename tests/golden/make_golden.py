"""Generates the golden vectors in tests/golden from the reference itself.

The reference's CPU path (src/few/cutils/interpolate.cu, built as C++ from the
reference sources by ``make -C oracle ref`` into oracle/_ref) is run on small
seeded inputs and its outputs are stored next to those inputs.  The reference
ships no golden files of its own; its tests pin the spline against
scipy.interpolate.CubicSpline (tests/test_mode_summation.py:23-52) and the sum
against a direct numpy sum (tests/test_mode_summation.py:64-151), which the
tests here restate as well.

    python tests/golden/make_golden.py                    (needs the reference sources)
    python tests/golden/make_golden.py --only amplitude   (the amplitude case alone)
    python tests/golden/make_golden.py --only aak         (the AAK case alone)
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from fastemriwaveforms_b200 import synthetic as S  # noqa: E402
from oracle import oracle as O  # noqa: E402


def inputs_digest(inp) -> str:
    h = hashlib.sha256()
    for a in (inp.t, inp.teuk_modes, inp.ylms, inp.phase_t, inp.phase_coeffs, inp.l, inp.m, inp.k, inp.n):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def save_case(name, inp, wf, extra=None):
    d = dict(t=inp.t, teuk_modes=inp.teuk_modes, ylms=inp.ylms, phase_t=inp.phase_t,
             phase_coeffs=inp.phase_coeffs, l=inp.l, m=inp.m, k=inp.k, n=inp.n, dt=inp.dt, T=inp.T,
             waveform=wf)
    if extra:
        d.update(extra)
    np.savez_compressed(os.path.join(HERE, name), **d)


def amplitude_case():
    """The reference's interp2D (AmpInterp2D.cu) on seeded clamped B-spline grids:
    bicubic, and degrees (1, 5); points inside, on knots and outside the domain."""
    rng = np.random.default_rng(77)
    out = {}
    for tag, kx, ky, nx, ny in (("k33", 3, 3, 14, 17), ("k15", 1, 5, 9, 16)):
        tx = np.concatenate([np.zeros(kx + 1), np.sort(rng.uniform(0, 1, nx - 2 * kx - 2)), np.ones(kx + 1)])
        ty = np.concatenate([-np.ones(ky + 1), np.sort(rng.uniform(-1, 2, ny - 2 * ky - 2)), 2 * np.ones(ky + 1)])
        c = rng.standard_normal((6, (nx - kx - 1) * (ny - ky - 1)))
        x = np.concatenate([rng.uniform(-0.2, 1.2, 40), tx[kx:kx + 5], [0.0, 1.0]])
        y = np.concatenate([rng.uniform(-1.3, 2.3, 40), ty[ky:ky + 5], [-1.0, 2.0]])
        out.update({f"{tag}_tx": tx, f"{tag}_ty": ty, f"{tag}_c": c, f"{tag}_x": x, f"{tag}_y": y,
                    f"{tag}_z": O.interp2d(tx, ty, c, kx, ky, x, y, impl="ref")})
    np.savez_compressed(os.path.join(HERE, "amp_interp2d.npz"), **out)


def aak_case():
    """The reference's AAK kernel (gpuAAK.cu, CPU path) on a seeded trajectory
    (synthetic.aak_case), plain and with the long-wavelength response."""
    inp = S.aak_case(N=40, span=3e5)
    L = int(inp.t[-1] / inp.dt) + 1
    out = dict(t=inp.t, interp_coeffs=inp.interp_coeffs, L=L)
    for mich in (0, 1):
        out[f"wf_mich{mich}"] = O.aak_waveform(inp.t, inp.interp_coeffs, inp.m1, inp.a, inp.m2, inp.qS, inp.phiS,
                                               inp.qK, inp.phiK, inp.dist, inp.nmodes, bool(mich), L, inp.dt,
                                               impl="ref")
    np.savez_compressed(os.path.join(HERE, "aak_ref.npz"), **out)


def main(only=None):
    O.build(ref=True)
    if only == "amplitude":
        amplitude_case()
        return
    if only == "aak":
        aak_case()
        return
    rng = np.random.default_rng(2024)

    # 1. the reference spline test's inputs: cos/sin on 1000 uniform knots
    t = np.linspace(0, 100, 1000)
    y = np.vstack((np.cos(t), np.sin(t)))
    np.savez_compressed(os.path.join(HERE, "spline_cos_sin.npz"), t=t, y=y,
                        coeffs=O.interpolate_arrays(t, y, impl="ref"))

    # 2. per-interpolant knots (2-D t), uneven spacing, 5 series of 37 knots
    t2 = np.sort(rng.uniform(0, 50, (5, 37)), axis=1)
    t2[:, 0] = 0.0
    y2 = rng.standard_normal((5, 37)).cumsum(axis=1)
    np.savez_compressed(os.path.join(HERE, "spline_rows2d.npz"), t=t2, y=y2,
                        coeffs=O.interpolate_arrays(t2, y2, impl="ref"))

    # 3. small sums in the style of the reference's summation test
    for name, kw in (("sum_small_theta.npz", dict(K=10, N=20, out_len=4000, seed=7, theta=True)),
                     ("sum_small_m0.npz", dict(K=40, N=33, out_len=6001, seed=8, theta=False))):
        inp = S.small_case(**kw)
        if name == "sum_small_m0.npz":
            inp.m[:8] = 0  # m = 0 modes: no -m term
        wf = O.mode_sum(inp, impl="ref")
        save_case(name, inp, wf)

    # 4. observation shorter than the trajectory: the knot loop stops early
    inp = S.small_case(K=12, N=25, out_len=5000, seed=9)
    inp.T = 0.6 * (4999 * inp.dt) / S.YRSID_SI
    wf = O.mode_sum(inp, impl="ref")
    save_case("sum_small_truncated.npz", inp, wf)

    # 5. the K=200, N=100, 100,001-sample workload: the reference's output on
    #    the first 3000 samples and around three knots, plus whole-output norms
    inp = S.plain_small()
    wf = O.mode_sum(inp, impl="ref")
    start, nseg = O.find_start_inds(inp.t, inp.dt, len(wf))
    picks = [np.arange(0, 3000)]
    for j in (17, 50, 98):
        picks.append(np.arange(max(start[j] - 200, 0), min(start[j] + 200, len(wf))))
    idx = np.unique(np.concatenate(picks))
    np.savez_compressed(os.path.join(HERE, "plain_small_ref.npz"), idx=idx, values=wf[idx],
                        norm=np.linalg.norm(wf), sum=wf.sum(), out_len=len(wf),
                        digest=inputs_digest(inp), seed=inp.seed)
    amplitude_case()
    aak_case()
    print("golden vectors written to", HERE)


if __name__ == "__main__":
    main(sys.argv[2] if len(sys.argv) > 2 and sys.argv[1] == "--only" else None)
