"""DOPR853 dense output on the GPU (k_dense_output, k_dense_eval) against the
reference's own DOPR853 (tests/golden/dopr853_dense.npz, made by
make_dopr853_golden.py): the 8-term basis of every step from its stored
stages, the basis and its derivatives at new times, and the time-domain mode
sum fed with the trajectory's phases."""
import os

import numpy as np
import pytest
import torch

from fastemriwaveforms_b200 import DOPR853, InterpolatedModeSum
from fastemriwaveforms_b200 import synthetic as S

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "dopr853_dense.npz")
TOL_DERIV = 1e-14   # eval_derivative: relative to the component's largest value (the reference's s**k is C pow)


@pytest.fixture(scope="module")
def golden():
    return dict(np.load(GOLDEN))


def prepared(d, cuda):
    dopr = DOPR853(S.toy_inspiral_ode(torch), device=cuda)
    dopr.k_coefficient_storage = [torch.tensor(np.ascontiguousarray(d["stages"][:, s, :].T), device=cuda)
                                  for s in range(10)]
    return dopr, dopr.prep_evaluate(d["x0"], d["y0"].T.copy(), d["h0"], d["x1"], d["y1"].T.copy(), None)


def test_right_hand_side_same_bits_on_device(cuda, golden):
    """The test ODE gives the same bits through torch on the device as
    through numpy (the reference's stepper), so the basis can be compared bit
    for bit."""
    y = golden["y1"].T.copy()
    x = golden["x1"].copy()
    ref = np.zeros_like(y)
    S.toy_inspiral_ode(np)(x, y, ref, None)
    got = torch.zeros((y.shape[0], y.shape[1]), dtype=torch.float64, device=cuda)
    S.toy_inspiral_ode(torch)(torch.tensor(x, device=cuda), torch.tensor(y, device=cuda), got, None)
    assert np.array_equal(got.cpu().numpy(), ref)


def test_prep_evaluate_bitwise_all_steps_in_one_batch(cuda, golden):
    _, rc = prepared(golden, cuda)
    got = rc.cpu().numpy()
    assert got.shape == golden["rcont"].shape
    assert np.array_equal(got, golden["rcont"]), np.abs(got - golden["rcont"]).max()


def test_prep_evaluate_single_step(cuda, golden):
    d = golden
    j = 17
    dopr = DOPR853(S.toy_inspiral_ode(torch), device=cuda)
    dopr.k_coefficient_storage = [torch.tensor(d["stages"][j, s, :, None], device=cuda) for s in range(10)]
    got = dopr.prep_evaluate_single(d["x0"][j], d["y0"][j], d["h0"][j], d["x1"][j], d["y1"][j], None)
    assert np.array_equal(got.cpu().numpy(), d["rcont"][j])


def test_eval_and_derivatives(cuda, golden):
    d = golden
    dopr = DOPR853(S.toy_inspiral_ode(torch), device=cuda)
    val = dopr.eval(d["t_new"], d["t_knots"], d["rcont"]).cpu().numpy()
    assert np.array_equal(val, d["evals"][0])
    for order in (1, 2, 3):
        got = dopr.eval_derivative(d["t_new"], d["t_knots"], d["rcont"], order=order).cpu().numpy()
        ref = d["evals"][order]
        err = np.abs(got - ref).max(axis=0) / np.maximum(np.abs(ref).max(axis=0), 1e-300)
        assert err.max() <= TOL_DERIV, (order, err)
    with pytest.raises(ValueError, match="between t_min"):
        dopr.eval(np.array([d["t_knots"][-1] * 1.01]), d["t_knots"], d["rcont"])


def test_mode_sum_fed_from_the_dense_output(cuda, golden, oracle):
    """Phases Phi_phi, Phi_theta, Phi_r of the trajectory (basis components
    3..5) drive InterpolatedModeSum; the waveform equals the oracle's fed with
    the reference's basis."""
    d = golden
    _, rc = prepared(d, cuda)
    t = d["t_knots"]
    N = len(t)
    l, m, k, n = S.mode_list(4, 5, count=60)
    K = len(l)
    rng = np.random.default_rng(8)
    base = (rng.standard_normal(K) + 1j * rng.standard_normal(K)) * np.exp(-np.abs(n) / 4.0) / l ** 2
    teuk = base[None, :] * (1.0 + 0.3 * t[:, None] / t[-1]) * np.exp(1j * 1e-6 * t[:, None])
    ylms = (rng.standard_normal(2 * K) + 1j * rng.standard_normal(2 * K)) / np.sqrt(2.0)
    dt = 10.0
    T = (t[-1] - 0.5 * dt) / S.YRSID_SI
    ref_in = S.ModeSumInputs(t=t, teuk_modes=np.ascontiguousarray(teuk), ylms=ylms, phase_t=t,
                             phase_coeffs=np.ascontiguousarray(d["rcont"][:, 3:6, :]), l=l, m=m, k=k, n=n, dt=dt,
                             T=T)
    ref = oracle.mode_sum(ref_in)
    pc = rc[:, 3:6, :].contiguous()
    h = InterpolatedModeSum(precision="faithful")(t, ref_in.teuk_modes, ylms, t, pc, l, m, k, n, T=T, dt=dt)
    got = h.cpu().numpy()
    assert len(got) == len(ref) > 40000
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    assert err <= 1e-12, err
