"""Gradients at the adjoint workload (K=1000 modes, N=500 knots, 1,000,000
samples) against central finite differences of the FP64 oracle on 64 knot
entries: 16 real and 16 imaginary amplitude-knot parts, 16 Phi_phi knots and
16 Phi_r knots (tests/golden/adjoint_fd.npz, made by make_adjoint_fd.py from
the oracle).  The loss is L = Re sum g h with g = conj(h_ref + w), w white with
sigma 0.1 rms(h_ref); torch's upstream gradient is conj(g).  The phase knots
reach the mode sum through the differentiable not-a-knot phase spline.

Both adjoints are checked: the FP64 one (precision="exact") and the
tensor-core one (precision="mixed").  Each entry's error is taken relative to
max(|fd|, 1e-2 max|gradient of its family|): entries far below their family's
scale are held to 1e-2 of it (their finite differences carry the same
absolute error as the large ones)."""
import os

import numpy as np
import pytest
import torch

from fastemriwaveforms_b200 import InterpolatedModeSum
from fastemriwaveforms_b200 import synthetic as S
from fastemriwaveforms_b200.autograd import phase_coeffs_from_knots

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "adjoint_fd.npz")
TOL_FD = 1e-6        # both adjoints: relative error per entry (floor 1e-2 of the family's largest gradient)
FAMILIES = ("amplitude re", "amplitude im", "Phi_phi knots", "Phi_r knots")


def _digest(inp):
    import hashlib

    h = hashlib.sha256()
    for a in (inp.t, inp.teuk_modes, inp.ylms, inp.phase_knots, inp.phase_coeffs, inp.m, inp.n):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()[:32]


@pytest.fixture(scope="module")
def case(cuda):
    fx = dict(np.load(FIXTURE))
    inp = S.adjoint_case(seed=int(fx["input_seed"]))
    assert _digest(inp) == str(fx["digest"]), "synthetic.adjoint_case no longer makes the fixture's inputs"
    with torch.no_grad():
        h_ref = InterpolatedModeSum(precision="faithful")(*inp.call_args(), T=inp.T, dt=inp.dt).cpu().numpy()
    rng = np.random.default_rng(int(fx["noise_seed"]))
    rms = np.sqrt(np.mean(np.abs(h_ref) ** 2))
    w = (rng.standard_normal(h_ref.shape) + 1j * rng.standard_normal(h_ref.shape)) * 0.1 * rms / np.sqrt(2.0)
    G = torch.tensor(h_ref + w, device=cuda)  # torch's upstream gradient conj(g), g = conj(h_ref + w)
    return inp, fx, G


def gradients(inp, G, precision, cuda):
    teuk = torch.tensor(inp.teuk_modes, device=cuda, requires_grad=True)
    knots = torch.tensor(inp.phase_knots, device=cuda, requires_grad=True)
    pc = phase_coeffs_from_knots(inp.t, knots)
    ims = InterpolatedModeSum(precision=precision)
    h = ims(inp.t, teuk, inp.ylms, inp.phase_t, pc, inp.l, inp.m, inp.k, inp.n, T=inp.T, dt=inp.dt)
    h.backward(G)
    torch.cuda.synchronize()
    assert not ims.mixed_error()
    return teuk.grad.cpu().numpy(), knots.grad.cpu().numpy()


def errors(g_teuk, g_knots, fx):
    """Per-family max relative error of the gradient entries vs the finite differences."""
    scale = {0: np.abs(g_teuk).max(), 1: np.abs(g_teuk).max(), 2: np.abs(g_knots[0]).max(),
             3: np.abs(g_knots[2]).max()}
    out = {f: 0.0 for f in range(4)}
    worst = {}
    for f, j, k, fd in zip(fx["family"], fx["j"], fx["k"], fx["fd"]):
        f, j, k = int(f), int(j), int(k)
        got = (g_teuk[j, k].real if f == 0 else g_teuk[j, k].imag if f == 1 else
               g_knots[0 if f == 2 else 2, j])
        e = abs(got - fd) / max(abs(fd), 1e-2 * scale[f])
        if e >= out[f]:
            out[f] = e
            worst[f] = (j, k, got, float(fd))
    return out, worst


@pytest.mark.parametrize("precision", ["exact", "mixed"])
def test_adjoint_workload_gradients_vs_finite_differences(cuda, case, precision):
    inp, fx, G = case
    g_teuk, g_knots = gradients(inp, G, precision, cuda)
    err, worst = errors(g_teuk, g_knots, fx)
    print(f"\n{precision}: max relative error vs FD per family: "
          + ", ".join(f"{FAMILIES[f]} {err[f]:.2e}" for f in range(4)))
    print(f"{precision}: worst entries (j, k, gradient, FD): "
          + "; ".join(f"{FAMILIES[f]} {worst[f]}" for f in range(4)))
    for f in range(4):
        assert err[f] <= TOL_FD, (precision, FAMILIES[f], err[f], worst[f])
