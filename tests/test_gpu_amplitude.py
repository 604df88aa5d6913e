"""Amplitude grids on the GPU (few_interp2d, few_amp_interp2d, AmpInterp2D)
against the reference's interp2D output (golden vectors from its CPU path) and
the oracle restatement: bit for bit, since every operation is rounded in the
reference's order."""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from fastemriwaveforms_b200 import AmpInterp2D, InterpolatedModeSum
from fastemriwaveforms_b200 import synthetic as S
from fastemriwaveforms_b200.amplitude import interp2D

pytestmark = pytest.mark.gpu


def dev(a, cuda):
    return torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=cuda)


@pytest.mark.parametrize("tag,kx,ky", [("k33", 3, 3), ("k15", 1, 5)])
def test_interp2d_matches_reference_golden(cuda, tag, kx, ky):
    d = np.load(os.path.join(GOLDEN, "amp_interp2d.npz"))
    tx, ty, c, x, y, zref = (d[f"{tag}_{q}"] for q in ("tx", "ty", "c", "x", "y", "z"))
    z = torch.zeros(c.shape[0] * len(x), dtype=torch.float64, device=cuda)
    interp2D(z, dev(tx, cuda), len(tx), dev(ty, cuda), len(ty), dev(c, cuda), kx, ky, dev(x, cuda), len(x),
             dev(y, cuda), len(y), c.shape[0], c.shape[1])
    torch.cuda.synchronize()
    assert np.array_equal(z.cpu().numpy().reshape(c.shape[0], len(x)), zref)


def test_amp_interp2d_matches_oracle_layout_and_subsets(cuda, oracle):
    """The fused (points, modes) complex layout of AmpInterp2D.__call__ at a
    larger size, a subset of modes in any order, and empty input."""
    K, N = 300, 1000
    tw, tu, coeff = S.amplitude_grids(K, nw=40, nu=36)
    w, u = S.amplitude_points(N)
    amp = AmpInterp2D(tw, tu, coeff, None, None, None, None)
    got = amp(w, u).cpu().numpy()
    z = oracle.interp2d(tw, tu, coeff.reshape(2 * K, -1), 3, 3, w, u)  # (2K, N)
    ref = (z[0::2] + 1j * z[1::2]).T
    assert got.shape == (N, K)
    assert np.array_equal(got, ref)
    sel = np.array([7, 0, 299, 7, 150], dtype=np.int32)
    sub = amp(w, u, mode_indexes=sel).cpu().numpy()
    assert np.array_equal(sub, ref[:, sel])
    assert amp(np.zeros(0), np.zeros(0)).shape == (0, K)
    # scalar u broadcast against an array w
    b = amp(w[:10], 0.5).cpu().numpy()
    zb = oracle.interp2d(tw, tu, coeff.reshape(2 * K, -1), 3, 3, w[:10], np.full(10, 0.5))
    assert np.array_equal(b, (zb[0::2] + 1j * zb[1::2]).T)


def test_amplitudes_feed_the_mode_sum(cuda, oracle):
    """AmpInterp2D's output is the mode sum's teuk_modes layout: summing it
    equals summing the oracle's amplitudes, bit for bit."""
    inp = S.small_case(K=40, N=30, out_len=20000, seed=5, theta=True)
    tw, tu, coeff = S.amplitude_grids(inp.num_modes, nw=20, nu=20, seed=3)
    w, u = S.amplitude_points(inp.num_knots, seed=4)
    teuk_gpu = AmpInterp2D(tw, tu, coeff, inp.l, inp.m, inp.k, inp.n)(w, u)
    z = oracle.interp2d(tw, tu, coeff.reshape(2 * inp.num_modes, -1), 3, 3, w, u)
    teuk_ref = np.ascontiguousarray((z[0::2] + 1j * z[1::2]).T)
    args = dict(T=inp.T, dt=inp.dt)
    a = InterpolatedModeSum()(inp.t, teuk_gpu, inp.ylms, inp.phase_t, inp.phase_coeffs, inp.l, inp.m, inp.k, inp.n,
                              **args).cpu().numpy()
    b = InterpolatedModeSum()(inp.t, teuk_ref, inp.ylms, inp.phase_t, inp.phase_coeffs, inp.l, inp.m, inp.k, inp.n,
                              **args).cpu().numpy()
    assert np.array_equal(a, b)


def test_amplitude_errors(cuda):
    tw, tu, coeff = S.amplitude_grids(4, nw=12, nu=12)
    with pytest.raises(ValueError):
        AmpInterp2D(tw[:-1], tu, coeff, None, None, None, None)  # len_indiv_c mismatch
    amp = AmpInterp2D(tw, tu, coeff, None, None, None, None)
    with pytest.raises(ValueError):
        amp([0.5], [0.5], mode_indexes=[4])
    z = torch.zeros(8, dtype=torch.float64, device=cuda)
    t = torch.tensor(tw, device=cuda)
    c = torch.tensor(coeff.reshape(8, -1), device=cuda)
    x = torch.full((1,), 0.5, dtype=torch.float64, device=cuda)
    with pytest.raises(ValueError):  # degree 6 is beyond FITPACK's work arrays
        interp2D(z, t, len(tw), t, len(tw), c, 6, 3, x, 1, x, 1, 8, coeff.shape[2])
    with pytest.raises(ValueError):  # mx != my
        interp2D(z, t, len(tw), t, len(tw), c, 3, 3, x, 1, x, 2, 8, coeff.shape[2])
