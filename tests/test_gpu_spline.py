"""Spline build and evaluation on the GPU against the oracle, the reference's
golden vectors and scipy (the reference's own spline test)."""
import ctypes
import os

import numpy as np
import pytest
import torch
from scipy.interpolate import CubicSpline

from conftest import GOLDEN
from fastemriwaveforms_b200 import CubicSplineInterpolant, _lib

pytestmark = pytest.mark.gpu


def coeff_err(got, ref):
    """max |got - ref| per coefficient row, relative to that row's scale."""
    got = np.asarray(got)
    ref = np.asarray(ref)
    errs = []
    for c in range(4):
        scale = np.abs(ref[c]).max() or 1.0
        errs.append(np.abs(got[c] - ref[c]).max() / scale)
    return max(errs)


def test_cubic_spline_reference_test(cuda):
    # tests/test_mode_summation.py:23-52, same inputs and rtol
    t = np.linspace(0, 100, 1000)
    f = np.vstack((np.cos(t), np.sin(t)))
    spl = CubicSplineInterpolant(t, f)
    cs = CubicSpline(t, f, axis=-1)
    np.testing.assert_allclose(spl(t).cpu().numpy(), f, rtol=1e-10)
    for nu in range(1, 4):
        np.testing.assert_allclose(spl(t, deriv_order=nu).cpu().numpy(), cs(t, nu=nu), rtol=1e-10)
    te = np.linspace(0, 100, 1852)
    for nu in range(4):
        np.testing.assert_allclose(spl(te, deriv_order=nu).cpu().numpy(), cs(te, nu=nu), rtol=1e-10)


def test_build_matches_golden(cuda):
    d = np.load(os.path.join(GOLDEN, "spline_cos_sin.npz"))
    spl = CubicSplineInterpolant(d["t"], d["y"])
    got = spl.interp_array.reshape(spl.reshape_shape).permute(0, 2, 1).cpu().numpy()  # (4, ninterps, N)
    assert coeff_err(got, d["coeffs"]) < 1e-12
    d = np.load(os.path.join(GOLDEN, "spline_rows2d.npz"))
    spl = CubicSplineInterpolant(d["t"], d["y"])
    got = spl.interp_array.reshape(spl.reshape_shape).permute(0, 2, 1).cpu().numpy()
    assert coeff_err(got, d["coeffs"]) < 1e-12
    np.testing.assert_array_equal(spl.t.cpu().numpy(), d["t"])


@pytest.mark.parametrize("N,ni,seed", [(4, 3, 0), (5, 7, 1), (100, 400, 2), (1000, 7686, 3), (2000, 65, 4)])
def test_build_matches_oracle(cuda, oracle, N, ni, seed):
    rng = np.random.default_rng(seed)
    t = np.sort(rng.uniform(0, 1e6, N))
    t[0] = 0.0
    # uneven spacing stresses the no-pivot elimination
    t = np.cumsum(np.concatenate([[0.0], rng.exponential(1.0, N - 1) + 1e-3]))
    y = rng.standard_normal((ni, N)).cumsum(axis=1)
    ref = oracle.spline_coeffs(t, y)
    spl = CubicSplineInterpolant(t, y)
    got = spl.interp_array.reshape(spl.reshape_shape).cpu().numpy()
    assert coeff_err(got, ref) < 1e-11
    np.testing.assert_array_equal(spl.y.cpu().numpy(), y)
    np.testing.assert_array_equal(spl.c1.cpu().numpy(), got[1].T)


def test_complex_strided_input_matches_real_rows(cuda, oracle):
    """The InterpolatedModeSum view: (N, K) complex amplitudes splined in place."""
    rng = np.random.default_rng(5)
    N, K = 57, 33
    t = np.sort(rng.uniform(0, 100, N))
    teuk = rng.standard_normal((N, K)) + 1j * rng.standard_normal((N, K))
    y_all = np.concatenate([teuk.T.real, teuk.T.imag])
    ref = oracle.spline_coeffs(t, y_all)
    dev = cuda
    td = torch.from_numpy(t).to(dev)
    tk = torch.from_numpy(teuk).to(dev)
    out = torch.empty((4, N, 2 * K), dtype=torch.float64, device=dev)
    _lib.call("few_spline_build", td.data_ptr(), 0, tk.data_ptr(), 2 * K, 2, K, 1, 2 * K, N, out.data_ptr(),
              _lib.FEW_LAYOUT_KNOT_MAJOR, torch.cuda.current_stream().cuda_stream)
    assert coeff_err(out.cpu().numpy(), ref) < 1e-12


@pytest.mark.parametrize("N,ni,seed", [(4, 5, 0), (7, 3, 1), (1000, 7686, 2), (2000, 100, 3), (3001, 22, 4)])
def test_factored_build_matches_generic(cuda, oracle, N, ni, seed):
    """The shared-knot path (host factorization) agrees with the per-series
    kernel and the oracle, on the complex (N, K) view InterpolatedModeSum uses."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(np.concatenate([[0.0], rng.exponential(1.0, N - 1) + 1e-2]))
    K = (ni + 1) // 2
    teuk = rng.standard_normal((N, K)) + 1j * rng.standard_normal((N, K))
    td = torch.from_numpy(t).to(cuda)
    tk = torch.from_numpy(teuk).to(cuda)
    st = torch.cuda.current_stream().cuda_stream
    generic = torch.empty((4, N, 2 * K), dtype=torch.float64, device=cuda)
    _lib.call("few_spline_build", td.data_ptr(), 0, tk.data_ptr(), 2 * K, 2, K, 1, 2 * K, N, generic.data_ptr(),
              _lib.FEW_LAYOUT_KNOT_MAJOR, st)
    from fastemriwaveforms_b200.summation import spline_factor_table

    fac = spline_factor_table(t, cuda)
    fact = torch.empty_like(generic)
    _lib.call("few_spline_build_factored", fac.data_ptr(), tk.data_ptr(), 2 * K, 2, K, 1, 2 * K, N, fact.data_ptr(),
              _lib.FEW_LAYOUT_KNOT_MAJOR, st)
    assert coeff_err(fact.cpu().numpy(), generic.cpu().numpy()) < 1e-11
    if N <= 1000:
        y_all = np.concatenate([teuk.T.real, teuk.T.imag])
        assert coeff_err(fact.cpu().numpy(), oracle.spline_coeffs(t, y_all)) < 1e-11


@pytest.mark.parametrize("N,ni", [(5, 1), (64, 13), (1000, 300)])
def test_factored_build_real_series(cuda, N, ni):
    """The shared-knot build on a plain (ninterps, length) array (no complex
    split: series in consecutive lanes) equals the per-series kernel."""
    rng = np.random.default_rng(N + ni)
    t = np.cumsum(np.concatenate([[0.0], rng.uniform(0.2, 3.0, N - 1)]))
    y = rng.standard_normal((ni, N))
    td = torch.from_numpy(t).to(cuda)
    yd = torch.from_numpy(y).to(cuda)
    st = torch.cuda.current_stream().cuda_stream
    generic = torch.empty((4, N, ni), dtype=torch.float64, device=cuda)
    _lib.call("few_spline_build", td.data_ptr(), 0, yd.data_ptr(), 1, N, ni, 0, ni, N, generic.data_ptr(),
              _lib.FEW_LAYOUT_KNOT_MAJOR, st)
    from fastemriwaveforms_b200.summation import spline_factor_table

    fac = spline_factor_table(t, cuda)
    fact = torch.empty_like(generic)
    _lib.call("few_spline_build_factored", fac.data_ptr(), yd.data_ptr(), 1, N, ni, 0, ni, N, fact.data_ptr(),
              _lib.FEW_LAYOUT_KNOT_MAJOR, st)
    assert coeff_err(fact.cpu().numpy(), generic.cpu().numpy()) < 1e-11


def test_reference_shaped_interpolate_arrays(cuda, oracle):
    rng = np.random.default_rng(6)
    ni, N = 9, 41
    t = np.sort(rng.uniform(0, 10, (ni, N)), axis=1)
    y = rng.standard_normal((ni, N))
    ref = oracle.interpolate_arrays(t, y)
    interp = np.zeros((4, ni, N))
    interp[0] = y
    d_t = torch.from_numpy(np.ascontiguousarray(t.reshape(-1))).to(cuda)
    d_i = torch.from_numpy(interp.reshape(-1).copy()).to(cuda)
    scratch = torch.zeros(ni * N, dtype=torch.float64, device=cuda)
    _lib.call("few_interpolate_arrays", d_t.data_ptr(), d_i.data_ptr(), ni, N, scratch.data_ptr(),
              scratch.data_ptr(), scratch.data_ptr(), scratch.data_ptr(), None)
    torch.cuda.synchronize()
    assert coeff_err(d_i.cpu().numpy().reshape(4, ni, N), ref) < 1e-12


def test_eval_edges_and_errors(cuda):
    t = np.linspace(0, 10, 11)
    y = np.vstack([t ** 2, np.sin(t)])
    spl = CubicSplineInterpolant(t, y)
    v = spl(np.array([-1.0, 0.0, 10.0, 11.0])).cpu().numpy()
    np.testing.assert_allclose(v[:, 0], y[:, 0])
    np.testing.assert_allclose(v[:, 3], y[:, -1])
    np.testing.assert_allclose(v[:, 2], y[:, -1], rtol=1e-12)
    with pytest.raises(ValueError):
        spl(np.array([-1.0, 5.0]), deriv_order=1)
    with pytest.raises(ValueError):
        spl(t, deriv_order=4)
    with pytest.raises(ValueError):
        spl(np.zeros((3, 5)))
    # 2-D tnew, one row per interpolant
    tn = np.vstack([np.linspace(0, 10, 7), np.linspace(1, 9, 7)])
    got = spl(tn).cpu().numpy()
    cs = CubicSpline(t, y, axis=-1)
    np.testing.assert_allclose(got[0], cs(tn[0])[0], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(got[1], cs(tn[1])[1], rtol=1e-12, atol=1e-12)


def test_build_rejects_bad_sizes(cuda):
    with pytest.raises(ValueError):
        CubicSplineInterpolant(np.array([0.0]), np.array([1.0]))
    with pytest.raises(ValueError):
        CubicSplineInterpolant(np.array([0.0, 1.0, 2.0]), np.array([1.0, 2.0, 0.0]))
    with pytest.raises(ValueError):
        CubicSplineInterpolant(np.zeros((2, 2, 2)), np.zeros((2, 2)))
