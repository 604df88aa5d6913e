"""Frequency-domain sum on the GPU against the reference.

Golden vectors (tests/golden/make_fd_golden.py) come from the reference
itself: its get_fundamental_frequencies and FDInterpolatedModeSum.sum run from
its Python sources, with its CPU kernels (interpolate.cu) for the splines and
the stationary-phase sum.  Checked here:

* the geodesic frequencies (relative error, printed);
* the planned bin ranges, bit for bit, given the reference's own knot
  frequencies (the planning replays numpy's roundings);
* the waveform, given the reference's frequencies and end to end from
  (M, a, p, e, x): relative L2 within the FD tolerances below.  The kernel
  uses CUDA's transcendental functions where the reference uses glibc's;
  Cardano's root formula amplifies those last-place differences in the root
  time, but on a self-consistent trajectory (the golden phases are integrals
  of the reference's frequencies) the phase is stationary at the root, so the
  waveform moves only at second order;
* the C ABI drop-in few_get_waveform_fd on the reference's own kernel inputs.
"""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from fastemriwaveforms_b200 import FDInterpolatedModeSum, _lib, get_fundamental_frequencies
from fastemriwaveforms_b200.summation import _ptr

pytestmark = pytest.mark.gpu

REL_GEODESIC = 1e-11   # fundamental frequencies vs the reference (max relative; near-circular orbits
                       # lose a few digits to cancellation in both implementations)
REL_FD = 1e-11         # FD waveform vs the reference given its knot frequencies, relative L2
REL_FD_E2E = 1e-9      # end to end from (M, a, p, e, x): the geodesic frequencies differ from the
                       # reference's in the last places, which moves the spline roots

CASES = {
    "fd_schwarzschild": dict(),
    "fd_single_turnover": dict(),  # one interior turnover: its segment is widened
    "fd_kerr_farr": dict(f_arr=True),
    "fd_generic_pos": dict(include_minus_m=False, mask_positive=True),
}


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def kwargs_of(d, opts):
    kw = {}
    if opts.get("f_arr"):
        kw["f_arr"] = d["f_arr"]
    if "include_minus_m" in opts:
        kw["include_minus_m"] = opts["include_minus_m"]
    if "mask_positive" in opts:
        kw["mask_positive"] = opts["mask_positive"]
    return kw


def run_with_frequencies(d, opts):
    fd = FDInterpolatedModeSum(pad_output=True)
    fd.num_pts, fd.num_pts_pad = int(d["num_pts"]), int(d["num_pts_pad"])
    fd.sum_with_frequencies(d["t"], d["teuk_modes"], d["ylms"], d["phase_t"], d["phase_coeffs"], d["l"], d["m"],
                            d["k"], d["n"], d["fknots"], dt=float(d["dt"]), **kwargs_of(d, opts))
    torch.cuda.synchronize()
    return fd


def test_geodesic_frequencies_match_reference(cuda):
    d = load("geodesic_frequencies")
    errs = []
    for i in range(len(d["a"])):
        got = get_fundamental_frequencies(float(d["a"][i]), float(d["p"][i]), float(d["e"][i]), float(d["x"][i]))
        ref = (d["OmegaPhi"][i], d["OmegaTheta"][i], d["OmegaR"][i])
        errs.append(max(abs(g - r) / abs(r) for g, r in zip(got, ref)))
    # the array form, one launch over every orbit of the table (per-point spins)
    arr = get_fundamental_frequencies(d["a"], d["p"], d["e"], d["x"])
    for q, key in enumerate(("OmegaPhi", "OmegaTheta", "OmegaR")):
        np.testing.assert_allclose(arr[q].cpu().numpy(), d[key], rtol=REL_GEODESIC, atol=0)
    worst = int(np.argmax(errs))
    print(f"\ngeodesic frequencies: {len(errs)} orbits, max relative error {max(errs):.3e} at "
          f"(a, p, e, x) = {tuple(float(d[q][worst]) for q in 'apex')}; median {np.median(errs):.1e}")
    assert max(errs) <= REL_GEODESIC


@pytest.mark.parametrize("name", sorted(CASES))
def test_fd_plan_matches_reference(cuda, name):
    d = load(name)
    fd = run_with_frequencies(d, CASES[name])
    assert np.array_equal(fd.seg_start_inds.cpu().numpy().reshape(-1), d["start_inds"])
    assert np.array_equal(fd.seg_end_inds.cpu().numpy().reshape(-1), d["end_inds"])
    np.testing.assert_array_equal(fd.frequency.cpu().numpy(), d["frequency"])


@pytest.mark.parametrize("name", sorted(CASES))
def test_fd_waveform_matches_reference(cuda, name):
    d = load(name)
    fd = run_with_frequencies(d, CASES[name])
    got = fd.waveform.cpu().numpy()
    assert got.shape == d["waveform"].shape
    e = rel(got, d["waveform"])
    print(f"\n{name}: FD waveform (reference frequencies) rel L2 {e:.3e}")
    assert e <= REL_FD


@pytest.mark.parametrize("name", sorted(CASES))
def test_fd_end_to_end_matches_reference(cuda, name):
    """Through __call__ from (M, a, p, e, x), as a user calls it."""
    d = load(name)
    fd = FDInterpolatedModeSum(pad_output=True)
    out = fd(d["t"], d["teuk_modes"], d["ylms"], d["phase_t"], d["phase_coeffs"], d["l"], d["m"], d["k"], d["n"],
             float(d["M"]), float(d["a"]), d["p"], d["e"], d["xI"], T=float(d["T"]), dt=float(d["dt"]),
             **kwargs_of(d, CASES[name]))
    got = out.cpu().numpy()
    assert got.shape == d["waveform"].shape
    e = rel(got, d["waveform"])
    starts = fd.seg_start_inds.cpu().numpy().reshape(-1)
    diff = int(np.count_nonzero(starts != d["start_inds"]))
    print(f"\n{name}: FD waveform end to end rel L2 {e:.3e} ({diff} bin starts differ from the reference's)")
    assert e <= REL_FD_E2E


@pytest.mark.parametrize("name", sorted(CASES))
def test_drop_in_abi_matches_reference_kernel(cuda, name):
    """few_get_waveform_fd on the reference's own kernel inputs (its spline
    coefficients, phase layout, bin ranges and signed harmonics)."""
    d = load(name)
    dev = cuda
    K = len(d["m"])
    N = len(d["t"])
    freq = torch.tensor(d["frequency"], device=dev)
    L = freq.numel()
    wf = torch.zeros(L, dtype=torch.complex128, device=dev)
    T = lambda a, dt=torch.float64: torch.tensor(np.ascontiguousarray(a), dtype=dt, device=dev)  # noqa: E731
    interp, pk, pt, t = T(d["interp_array"]), T(d["phase_kernel"]), T(d["phase_t"]), T(d["t"])
    m, k, n = (T(d[q], torch.int32) for q in ("m", "k", "n"))
    s, e = T(d["start_inds"], torch.int32), T(d["end_inds"], torch.int32)
    y = T(d["ylms_signed"], torch.complex128)
    inc = int(CASES[name].get("include_minus_m", True))
    _lib.call("few_get_waveform_fd", _ptr(wf), _ptr(interp), _ptr(pt), _ptr(pk), _ptr(m), _ptr(k), _ptr(n), K,
              float(d["dt"]), _ptr(t), N, L, _ptr(freq), _ptr(s), _ptr(e), N - 1, _ptr(y), int(d["zero_index"]),
              inc, 0, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    err = rel(wf.cpu().numpy(), d["raw"])
    print(f"\n{name}: few_get_waveform_fd vs reference kernel rel L2 {err:.3e}")
    assert err <= REL_FD
    with pytest.raises(ValueError):
        _lib.call("few_get_waveform_fd", _ptr(wf), _ptr(interp), _ptr(pt), _ptr(pk), _ptr(m), _ptr(k), _ptr(n), K,
                  float(d["dt"]), _ptr(t), N, L, _ptr(freq), _ptr(s), _ptr(e), N - 1, _ptr(y), int(d["zero_index"]),
                  inc, 1, torch.cuda.current_stream().cuda_stream)


def test_fd_repeatable_and_errors(cuda):
    d = load("fd_schwarzschild")
    a = run_with_frequencies(d, {}).waveform.cpu().numpy()
    b = run_with_frequencies(d, {}).waveform.cpu().numpy()
    # FP64 atomics: the order of additions may change the last bits only
    assert rel(a, b) < 1e-14
    fd = FDInterpolatedModeSum()
    args = (d["t"], d["teuk_modes"], d["ylms"], d["phase_t"], d["phase_coeffs"], d["l"], d["m"], d["k"], d["n"],
            float(d["M"]), float(d["a"]), d["p"], d["e"], d["xI"])
    with pytest.raises(ValueError):
        fd(*args, T=float(d["T"]), dt=float(d["dt"]), separate_modes=True)
    with pytest.raises(ValueError):
        fd(*args, T=float(d["T"]), dt=float(d["dt"]), f_arr=np.array([1.0, 0.5, 0.0]))  # not ascending
    with pytest.raises(ValueError):  # inside the separatrix: the elliptic modulus exceeds 1
        bad = list(args)
        bad[11] = np.full(len(d["t"]), 6.0)
        fd(*bad, T=float(d["T"]), dt=float(d["dt"]))


def test_fd_matches_fft_of_time_domain(cuda):
    """The reference's own check (tests/test_fd.py:92-150): on a self-consistent
    trajectory (phases = integrals of the geodesic frequencies), the FD h+ at
    positive frequencies overlaps the FFT of the real part of the time-domain
    waveform to better than 1e-2."""
    from fastemriwaveforms_b200 import InterpolatedModeSum
    from fastemriwaveforms_b200 import synthetic as S
    from fastemriwaveforms_b200.geodesic import MTSUN_SI

    def gpu_freqs(M, a, p, e, x):
        O = get_fundamental_frequencies(a, p, e, x)
        den = 2 * np.pi * M * MTSUN_SI
        return np.stack([np.abs(O[0].cpu().numpy() / den), O[1].cpu().numpy() / den, O[2].cpu().numpy() / den])

    inp, tr = S.fd_case(K=77, N=120, span=4e6, seed=31, a=0.0, x=1.0, lmax=3, nmax=5, p_range=(12.0, 9.0),
                        e_range=(0.3, 0.2), frequencies=gpu_freqs)
    td = InterpolatedModeSum(pad_output=True, odd_len=True)
    h = td(*inp.call_args(), T=inp.T, dt=inp.dt)
    fd = FDInterpolatedModeSum(pad_output=True)
    hf = fd(*inp.call_args(), tr.M, tr.a, tr.p, tr.e, tr.xI, T=inp.T, dt=inp.dt)
    assert hf.shape[1] == h.numel()
    mask = fd.frequency >= 0.0
    a = torch.fft.fftshift(torch.fft.fft(h.real))[mask]
    b = hf[0, mask]
    ov = (torch.vdot(a, b) / torch.sqrt(torch.vdot(a, a) * torch.vdot(b, b))).real.item()
    print(f"\nFD vs FFT(TD): 1 - overlap = {1 - ov:.3e}")
    assert 1 - ov < 1e-2


def test_fd_host_out(cuda):
    d = load("fd_schwarzschild")
    fd = FDInterpolatedModeSum(pad_output=True)
    args = (d["t"], d["teuk_modes"], d["ylms"], d["phase_t"], d["phase_coeffs"], d["l"], d["m"], d["k"], d["n"],
            float(d["M"]), float(d["a"]), d["p"], d["e"], d["xI"])
    ref = fd(*args, T=float(d["T"]), dt=float(d["dt"])).cpu().numpy()
    h = torch.empty(ref.shape, dtype=torch.complex128).pin_memory()
    out = fd(*args, T=float(d["T"]), dt=float(d["dt"]), host_out=h)
    torch.cuda.synchronize()
    assert rel(h.numpy(), out.cpu().numpy()) == 0.0 and rel(h.numpy(), ref) < 1e-14
    with pytest.raises(ValueError):
        fd(*args, T=float(d["T"]), dt=float(d["dt"]), host_out=torch.empty(ref.shape, dtype=torch.complex128))
