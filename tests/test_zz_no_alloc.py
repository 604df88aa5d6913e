"""few_get_waveform_noalloc: the mode sum for callers that cannot allocate
device memory (a host framework that owns every device allocation, a fixed
device memory budget, or a pipeline that must not let an allocation block in
the driver).  It is checked through the C ABI against few_get_waveform, the
entry point that allocates its workspace, on two calls in a row.

This file is named to be collected last."""
import numpy as np
import pytest
import torch

from fastemriwaveforms_b200 import CubicSplineInterpolant, _lib
from fastemriwaveforms_b200 import synthetic as S

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative L2, the tolerance of the other mode-sum parity tests


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def device_args(inp, dev):
    """Reference-shaped arguments (as InterpolatedModeSum.sum prepares them)."""
    K = inp.teuk_modes.shape[1]
    y_all = np.concatenate([inp.teuk_modes.T.real, inp.teuk_modes.T.imag])
    spl = CubicSplineInterpolant(inp.t, y_all)
    ylms = inp.ylms.copy()
    ylms[K:] *= (-1.0) ** inp.l
    pc = np.ascontiguousarray(np.transpose(inp.phase_coeffs, (2, 0, 1)))
    return dict(
        coeffs=spl.interp_array,
        pc=torch.from_numpy(pc).to(dev),
        m=torch.from_numpy(inp.m.astype(np.int32)).to(dev),
        k=torch.from_numpy(inp.k.astype(np.int32)).to(dev),
        n=torch.from_numpy(inp.n.astype(np.int32)).to(dev),
        ylms=torch.from_numpy(ylms).to(dev),
        h_t=np.ascontiguousarray(inp.t),
        p_t=np.ascontiguousarray(inp.phase_t),
        K=K, N=len(inp.t), out_len=inp.out_len, dt=float(inp.dt))


def call(name, a, dev):
    wf = torch.zeros(a["out_len"], dtype=torch.complex128, device=dev)
    _lib.call(name, wf.data_ptr(), a["coeffs"].data_ptr(), a["p_t"].ctypes.data, a["pc"].data_ptr(),
              a["m"].data_ptr(), a["k"].data_ptr(), a["n"].data_ptr(), a["N"], a["out_len"], a["K"],
              a["ylms"].data_ptr(), a["dt"], a["h_t"].ctypes.data, dev.index or 0,
              torch.cuda.current_stream(dev).cuda_stream)
    return wf.cpu().numpy()


@pytest.mark.parametrize("case", ["small_theta", "plain_full"])
def test_noalloc_matches_allocating_entry_point(case):
    assert torch.cuda.is_available(), "GPU test"
    dev = torch.device("cuda", 0)
    inp = S.small_case(K=16, N=40, out_len=9000, seed=21) if case == "small_theta" else S.plain_full()
    a = device_args(inp, dev)
    ref = call("few_get_waveform", a, dev)
    first = call("few_get_waveform_noalloc", a, dev)
    second = call("few_get_waveform_noalloc", a, dev)
    assert rel_l2(first, ref) < TOL
    assert rel_l2(second, ref) < TOL
    # the same kernels write every sample once from the same folded
    # coefficients, so the batches of the fixed scratch change no bit
    assert np.array_equal(first, ref)
    assert np.array_equal(second, ref)


def test_noalloc_rejects_what_does_not_fit():
    assert torch.cuda.is_available(), "GPU test"
    dev = torch.device("cuda", 0)
    inp = S.small_case(K=2, N=12, out_len=2000, seed=22, theta=False)
    inp.m[:] = [1, 2]
    inp.n[:] = [-20000, 20000]  # one segment's folded coefficients: 4 rows x 40001 columns x 64 B > 8 MiB
    a = device_args(inp, dev)
    with pytest.raises(ValueError, match="scratch"):
        call("few_get_waveform_noalloc", a, dev)
