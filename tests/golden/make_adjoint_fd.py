"""Generates tests/golden/adjoint_fd.npz: central finite differences of the
oracle (the reference's CPU mode sum restated in C) at the adjoint workload,
K=1000 modes, N=500 knots, 1,000,000 samples (``synthetic.adjoint_case``).

    python tests/golden/make_adjoint_fd.py            (about 3 minutes on 8 cores)

The loss is L = Re sum_i g_i h_i with g = conj(h_ref + w): h_ref the oracle's
FP64 waveform (the reference's own operation order), w white complex Gaussian
with sigma = 0.1 rms(h_ref) from numpy's default_rng(NOISE_SEED).  torch's
upstream gradient for the same L is conj(g) = h_ref + w.

64 entries, 16 per family, drawn with default_rng(PICK_SEED):
  0: Re of amplitude knot (j, k)   step 1e-2 (h is linear in it: the central
  1: Im of amplitude knot (j, k)   difference is exact up to rounding)
  2: Phi_phi knot j                step 1e-5 rad (max(|m|,|n|) * step << 1, so
  3: Phi_r knot j                  the truncation error stays ~1e-8 relative)
Phase knots reach the 8-term basis through the not-a-knot cubic of the knots
(``synthetic.phase_basis_from_knots``).  The two waveforms of an entry are
differenced sample by sample before the weighted sum, so the difference does
not inherit the rounding of the whole loss.  Each difference is evaluated on
the samples of the +-24 knot segments around the knot: on these non-uniform
knots the phase spline's influence outside +-22 segments is below 1e-13 of
its peak for every drawn knot.  Phase differences use the oracle's long
double form with the step added in long double: the knot-to-basis map is
linear, so the perturbed phases are Phi + s dPhi with dPhi the basis of a unit
knot.  Adding s = 1e-5 to the ~5e4 rad coefficients in double, or evaluating
the phases in double, would round the step by ~1e-11 rad per coefficient and
sample, which the cancelling phase gradients turn into ~1e-5 relative noise.

The file also stores a digest of the inputs, so a test can tell that
``synthetic.adjoint_case`` still generates the same waveform.
"""
import hashlib
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

INPUT_SEED = 4
NOISE_SEED = 11
PICK_SEED = 12
PER_FAMILY = 16
HALF_WINDOW = 24
AMP_STEP = 1e-2
PHASE_STEP = 1e-5
OUT = os.path.join(HERE, "adjoint_fd.npz")


def inputs():
    from fastemriwaveforms_b200 import synthetic as S

    return S.adjoint_case(seed=INPUT_SEED)


def digest(inp) -> str:
    h = hashlib.sha256()
    for a in (inp.t, inp.teuk_modes, inp.ylms, inp.phase_knots, inp.phase_coeffs, inp.m, inp.n):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()[:32]


def upstream(h_ref: np.ndarray) -> np.ndarray:
    """g (the loss's weights); torch's upstream gradient is conj(g)."""
    rng = np.random.default_rng(NOISE_SEED)
    rms = np.sqrt(np.mean(np.abs(h_ref) ** 2))
    w = (rng.standard_normal(h_ref.shape) + 1j * rng.standard_normal(h_ref.shape)) * 0.1 * rms / np.sqrt(2.0)
    return np.conj(h_ref + w)


def picks(N: int, K: int):
    rng = np.random.default_rng(PICK_SEED)
    fam, js, ks = [], [], []
    for f in range(4):
        for _ in range(PER_FAMILY):
            fam.append(f)
            js.append(int(rng.integers(0, N)))
            ks.append(int(rng.integers(0, K)) if f < 2 else -1)
    return np.array(fam), np.array(js), np.array(ks)


_W = {}


def _init(g):
    from oracle import oracle as O

    inp = inputs()
    start, nseg = O.find_start_inds(inp.t, inp.dt, inp.out_len)
    y_all, _, _ = O.prepare_sum(inp)
    _W.update(inp=inp, g=g, start=start, nseg=nseg, coeffs=O.spline_coeffs(inp.t, y_all))


def windowed_waveform(task):
    """The waveform on the +-HALF_WINDOW segment window of knot j with one entry moved by sgn * step."""
    from fastemriwaveforms_b200 import synthetic as S
    from oracle import oracle as O

    f, j, k, sgn = task
    inp, g, start, nseg = _W["inp"], _W["g"], _W["start"], _W["nseg"]
    lo = int(start[max(j - HALF_WINDOW, 0)])
    hi = int(start[min(j + HALF_WINDOW, nseg)])
    probe = S.ModeSumInputs(**{**inp.__dict__})
    if f < 2:
        probe.teuk_modes = inp.teuk_modes.copy()
        probe.teuk_modes[j, k] += sgn * AMP_STEP * (1.0 if f == 0 else 1j)
        h = O.mode_sum(probe, window=(lo, hi), extended=False)
    else:
        # the knot map is linear: Phi(knots + s e_j) = Phi(knots) + s Phi(e_j), added in long double
        unit = np.zeros_like(inp.phase_knots)
        unit[0 if f == 2 else 2, j] = 1.0
        dpc = S.phase_basis_from_knots(inp.t, unit)
        h = O.mode_sum(inp, window=(lo, hi), extended=True, coeffs=_W["coeffs"], dphase=(dpc, sgn * PHASE_STEP))
    return lo, h[lo:hi]


def main():
    from oracle import oracle as O

    t0 = time.time()
    inp = inputs()
    h_ref = O.mode_sum(inp, extended=False)
    g = upstream(h_ref)
    N, K = inp.teuk_modes.shape
    fam, js, ks = picks(N, K)
    tasks = [(int(f), int(j), int(k), s) for f, j, k in zip(fam, js, ks) for s in (1, -1)]
    # phase tasks first: they are the long ones
    order = sorted(range(len(tasks)), key=lambda i: tasks[i][0] < 2)
    with mp.get_context("spawn").Pool(os.cpu_count() or 1, initializer=_init, initargs=(g,)) as pool:
        vals = pool.map(windowed_waveform, [tasks[i] for i in order], chunksize=1)
    wins = [None] * len(tasks)
    for i, v in zip(order, vals):
        wins[i] = v
    step = np.where(fam < 2, AMP_STEP, PHASE_STEP)
    # L(+) - L(-) = Re sum g (h+ - h-): the waveforms are differenced sample by
    # sample before the sum, which keeps the rounding of the ~3e5-sized loss
    # (~1e-10 absolute) out of the ~1e-4-sized difference
    fd = np.empty(len(fam))
    for e in range(len(fam)):
        (lo, hp), (_, hm) = wins[2 * e], wins[2 * e + 1]
        fd[e] = np.sum(np.real(g[lo:lo + len(hp)] * (hp - hm))) / (2 * step[e])
    np.savez_compressed(OUT, family=fam, j=js, k=ks, step=step, fd=fd, digest=digest(inp),
                        input_seed=INPUT_SEED, noise_seed=NOISE_SEED, half_window=HALF_WINDOW,
                        h_ref_rms=np.sqrt(np.mean(np.abs(h_ref) ** 2)))
    print(f"wrote {OUT}: {len(fd)} entries in {time.time() - t0:.0f} s")


if __name__ == "__main__":
    main()
