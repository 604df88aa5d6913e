"""AAK summation on the GPU (k_aak through few_aak_waveform / AAKSummation):

* against the numpy restatement with scipy's Bessel functions: relative L2
  <= 1e-12 (the kernel's own Bessel recurrence and CUDA's transcendentals);
* against the reference's AAK kernel (golden vectors from its CPU path):
  <= 3e-7, the accuracy of the Numerical Recipes Bessel approximations that
  path uses (the numpy restatement differs from it by the same amount);
* the long-wavelength response, the equatorial substitution, the pole shift,
  and a trajectory that ends before the observation (later samples stay 0)."""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from fastemriwaveforms_b200 import AAKSummation
from fastemriwaveforms_b200 import synthetic as S

pytestmark = pytest.mark.gpu

REL_ORACLE = 1e-12
REL_REF = 3e-7


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def run(inp, mich, T=None, pad=False):
    aak = AAKSummation(pad_output=pad)
    out = aak(*inp.call_args(), mich=mich, T=inp.T if T is None else T, dt=inp.dt)
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("mich", [False, True])
def test_aak_matches_oracle_and_reference(cuda, oracle, mich):
    d = np.load(os.path.join(GOLDEN, "aak_ref.npz"))
    inp = S.aak_case(N=40, span=3e5)
    got = run(inp, mich)
    L = int(d["L"])
    assert got.shape == (L,)
    want = oracle.aak_waveform(inp.t, inp.interp_coeffs, inp.m1, inp.a, inp.m2, inp.qS, inp.phiS, inp.qK, inp.phiK,
                               inp.dist, inp.nmodes, mich, L, inp.dt)
    e_o = rel(got, want)
    e_r = rel(got, d[f"wf_mich{int(mich)}"])
    print(f"\nAAK mich={mich}: vs numpy restatement {e_o:.2e}, vs reference CPU {e_r:.2e}")
    assert e_o <= REL_ORACLE
    assert e_r <= REL_REF


def test_aak_equatorial_poles_and_short_trajectory(cuda, oracle):
    inp = S.aak_case(N=30, span=2e5, seed=53, Y=1.0, e_range=(0.3, 0.2))
    inp.interp_coeffs[:, 2, :] = 0.0
    inp.interp_coeffs[:, 2, 0] = 1.0  # Y = 1 exactly: Phi_theta follows Phi_phi
    inp.qK = 0.0                      # on the pole: shifted by 1e-6
    got = run(inp, False)
    c = inp.interp_coeffs.copy()
    c[:, 4] = c[:, 3]
    want = oracle.aak_waveform(inp.t, c, inp.m1, inp.a, inp.m2, inp.qS, inp.phiS, 0.0, inp.phiK, inp.dist,
                               inp.nmodes, False, len(got), inp.dt)  # the oracle applies the same pole shift
    assert rel(got, want) <= REL_ORACLE
    assert inp.interp_coeffs[0, 4, 1] != inp.interp_coeffs[0, 3, 1]  # the caller's array is untouched
    # observation longer than the trajectory (pad_output): samples past the last knot are zero
    long = run(S.aak_case(N=30, span=2e5, seed=54), False, T=3e5 / S.YRSID_SI, pad=True)
    last = int(2e5 / 10.0) + 1  # num_pts: the samples up to the last knot
    assert len(long) > last and np.all(long[last:] == 0) and np.all(long[:last] != 0)


def test_aak_reference_shaped_entry(cuda):
    """few_aak_waveform (the reference's get_waveform argument list, host knots)
    gives the same samples as AAKSummation's asynchronous path."""
    from fastemriwaveforms_b200 import _lib
    from fastemriwaveforms_b200.summation import _ptr

    inp = S.aak_case(N=40, span=3e5)
    want = run(inp, True)
    wf = torch.zeros(len(want), dtype=torch.complex128, device=cuda)
    coef = torch.tensor(np.ascontiguousarray(np.transpose(inp.interp_coeffs, (2, 0, 1))), device=cuda)
    t = np.ascontiguousarray(inp.t)
    _lib.call("few_aak_waveform", _ptr(wf), _ptr(coef), inp.m1, inp.a, inp.m2, inp.qS, inp.phiS, inp.qK, inp.phiK,
              inp.dist, inp.nmodes, 1, len(t), len(want), inp.dt, t.ctypes.data,
              torch.cuda.current_stream().cuda_stream)
    assert np.array_equal(wf.cpu().numpy(), want)
