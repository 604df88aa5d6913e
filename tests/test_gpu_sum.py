"""The interpolated mode sum on the GPU against the reference's golden vectors,
the CPU oracle (double precision in the reference's operation order, and its
long double form for the recurrence), and size-independent properties at the
full one-year, 3843-mode size."""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN, load_case
from fastemriwaveforms_b200 import InterpolatedModeSum, _lib
from fastemriwaveforms_b200 import synthetic as S

pytestmark = pytest.mark.gpu

# Tolerances (relative L2 of the complex waveform).
TOL_FAITHFUL = 1e-12   # vs the reference CPU path (the stated parity bar)
TOL_EXACT = 1e-12      # "exact" recurrence vs the long double oracle with the same Phi


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def run(inp, precision="faithful", **kw):
    ims = InterpolatedModeSum(precision=precision, **kw)
    wf = ims(*inp.call_args(), T=inp.T, dt=inp.dt)
    torch.cuda.synchronize()
    return wf.cpu().numpy(), ims


@pytest.mark.parametrize("name", ["sum_small_theta.npz", "sum_small_m0.npz", "sum_small_truncated.npz"])
def test_faithful_matches_reference_golden(cuda, name):
    inp, ref = load_case(name)
    got, _ = run(inp)
    assert got.shape == ref.shape
    assert rel_l2(got, ref) < TOL_FAITHFUL


@pytest.mark.parametrize("name", ["sum_small_theta.npz", "sum_small_m0.npz"])
def test_exact_matches_extended_oracle(cuda, oracle, name):
    inp, ref = load_case(name)
    got, _ = run(inp, precision="exact")
    ext = oracle.mode_sum(inp, extended=True)
    assert rel_l2(got, ext) < TOL_EXACT


def test_plain_small_faithful_matches_reference(cuda, oracle):
    inp = S.plain_small()
    got, ims = run(inp)
    d = np.load(os.path.join(GOLDEN, "plain_small_ref.npz"))
    idx = d["idx"]
    assert rel_l2(got[idx], d["values"]) < TOL_FAITHFUL
    ref = oracle.mode_sum(inp)
    err = rel_l2(got, ref)
    assert err < TOL_FAITHFUL, err
    assert abs(np.linalg.norm(got) - float(d["norm"])) / float(d["norm"]) < 1e-13


def test_plain_small_exact(cuda, oracle):
    inp = S.plain_small()
    got, _ = run(inp, precision="exact")
    ext = oracle.mode_sum(inp, extended=True)
    assert rel_l2(got, ext) < TOL_EXACT


def test_plain_full_windows(cuda, oracle):
    """K=3843, N=1000, 3,150,001 samples: the whole waveform on the GPU, checked
    against the oracle on windows at the start, a knot crossing in the middle
    and the end (each window is ~2e8 mode-samples of CPU work)."""
    inp = S.plain_full()
    got, ims = run(inp)
    out_len = inp.out_len
    assert got.shape == (out_len,)
    start, nseg = oracle.find_start_inds(inp.t, inp.dt, out_len)
    mid = int(start[nseg // 2])
    for lo, hi in ((0, 1500), (mid - 750, mid + 750), (out_len - 1500, out_len)):
        ref = oracle.mode_sum(inp, window=(lo, hi))[lo:hi]
        assert rel_l2(got[lo:hi], ref) < TOL_FAITHFUL, (lo, hi, rel_l2(got[lo:hi], ref))
    lo, hi = mid - 400, mid + 400
    got_e, _ = run(inp, precision="exact")
    ext = oracle.mode_sum(inp, window=(lo, hi), extended=True)[lo:hi]
    assert rel_l2(got_e[lo:hi], ext) < TOL_EXACT
    # the reference's own phase rounding separates it from the exact form
    ref = oracle.mode_sum(inp, window=(lo, hi))[lo:hi]
    floor = rel_l2(ref, ext)
    assert rel_l2(got_e[lo:hi], ref) < 2 * floor + 1e-13


def test_full_size_properties(cuda):
    """Size-independent checks at full size: deterministic (bitwise equal
    reruns) and linear (scaling the amplitudes by 2 scales the output by
    exactly 2)."""
    inp = S.plain_full()
    a, _ = run(inp)
    b, _ = run(inp)
    assert np.array_equal(a, b)
    inp2 = S.plain_full()
    inp2.teuk_modes = inp2.teuk_modes * 2.0
    c, _ = run(inp2)
    assert np.array_equal(c, 2.0 * a)


def test_reference_shaped_get_waveform(cuda, oracle):
    inp, ref = load_case("sum_small_m0.npz")
    K = inp.teuk_modes.shape[1]
    N = len(inp.t)
    y_all, pc, ylms = oracle.prepare_sum(inp)
    coeffs = oracle.spline_coeffs(inp.t, y_all)
    dev = cuda
    wf = torch.zeros(len(ref), dtype=torch.complex128, device=dev)
    d_c = torch.from_numpy(coeffs.reshape(-1).copy()).to(dev)
    d_pc = torch.from_numpy(pc).to(dev)
    d_m = torch.from_numpy(inp.m.astype(np.int32)).to(dev)
    d_k = torch.from_numpy(inp.k.astype(np.int32)).to(dev)
    d_n = torch.from_numpy(inp.n.astype(np.int32)).to(dev)
    d_y = torch.from_numpy(ylms).to(dev)
    h_t = np.ascontiguousarray(inp.t)
    p_t = np.ascontiguousarray(inp.phase_t)
    _lib.call("few_get_waveform", wf.data_ptr(), d_c.data_ptr(), p_t.ctypes.data, d_pc.data_ptr(),
              d_m.data_ptr(), d_k.data_ptr(), d_n.data_ptr(), N, len(ref), K, d_y.data_ptr(), float(inp.dt),
              h_t.ctypes.data, 0, torch.cuda.current_stream().cuda_stream)
    assert rel_l2(wf.cpu().numpy(), ref) < TOL_FAITHFUL


def test_reference_summation_test_restated(cuda):
    """tests/test_mode_summation.py:64-151 with synthetic 8-term phases: random
    m in [2,4], k in {0,1}, n in [-4,3], linear-ramp amplitudes, ylm = 1 for +m
    and 0 for -m, against a direct numpy sum at rtol 1e-8 (last sample excluded)."""
    rng = np.random.default_rng(12)
    num_modes = 10
    N = 40
    t_spl = np.linspace(0, 2e5, N)
    dt = t_spl[-1] / 10000
    t_eval = np.arange(10001) * dt
    rates = np.array([3e-3, 1e-3, 2e-3])
    coeff = np.zeros((N - 1, 3, 8))
    h = np.diff(t_spl)
    for q in range(3):
        # Phi(t) = r t + 1e-9 t^2 on each segment: y0, A1 + A2, -A2 with A2 = 1e-9 h^2
        coeff[:, q, 0] = rates[q] * t_spl[:-1] + 1e-9 * t_spl[:-1] ** 2
        coeff[:, q, 1] = rates[q] * h + 1e-9 * (t_spl[1:] ** 2 - t_spl[:-1] ** 2)
        coeff[:, q, 2] = -1e-9 * h ** 2
    # phases at the samples from the same polynomials (quadratic: exact in the basis)
    phases = np.array([rates[q] * t_eval + 1e-9 * t_eval ** 2 for q in range(3)])
    amp_lo = rng.uniform(-1, 1, (2, num_modes))
    amp_hi = rng.uniform(-1, 1, (2, num_modes))
    frac = t_eval / t_eval[-1]
    amp = (amp_lo[0] + (amp_hi[0] - amp_lo[0]) * frac[:, None]) + 1j * (amp_lo[1] + (amp_hi[1] - amp_lo[1]) * frac[:, None])
    frac_k = t_spl / t_eval[-1]
    amp_spl = (amp_lo[0] + (amp_hi[0] - amp_lo[0]) * frac_k[:, None]) + 1j * (amp_lo[1] + (amp_hi[1] - amp_lo[1]) * frac_k[:, None])
    l_arr = np.full(num_modes, 2)
    m_arr = rng.integers(2, 5, num_modes)
    k_arr = rng.integers(0, 2, num_modes)
    n_arr = rng.integers(-4, 4, num_modes)
    ylms = np.ones(2 * num_modes)
    ylms[num_modes:] = 0
    ph = phases[0][:, None] * m_arr + phases[1][:, None] * k_arr + phases[2][:, None] * n_arr
    manual = (amp * np.exp(-1j * ph)).sum(-1)
    ims = InterpolatedModeSum()
    got = ims(t_spl, amp_spl, ylms, t_spl, coeff, l_arr, m_arr, k_arr, n_arr, T=t_spl[-1] / S.YRSID_SI, dt=dt)
    got = got.cpu().numpy()
    n = min(len(got), len(manual)) - 1
    np.testing.assert_allclose(got[:n], manual[:n], rtol=1e-8)


def test_integrate_backwards_and_padding(cuda, oracle):
    inp, _ = load_case("sum_small_m0.npz")
    inp.t = inp.t.copy()
    inp.t[-1] += 3.3  # last knot off the sample grid, so the shift is not trivial
    inp.phase_t = inp.t.copy()
    ims = InterpolatedModeSum(pad_output=True)
    wf = ims(*inp.call_args(), T=inp.T * 1.5, dt=inp.dt, integrate_backwards=True)
    assert wf.shape[0] == ims.num_pts + ims.num_pts_pad and ims.num_pts_pad > 0
    got = wf.cpu().numpy()
    assert not got[ims.num_pts:].any()
    # the oracle with the same knot shift
    shifted = S.ModeSumInputs(**{**inp.__dict__})
    off = inp.t[-1] - int(inp.t[-1] / inp.dt) * inp.dt
    shifted.t = inp.t - off
    shifted.phase_t = inp.phase_t - off
    ref = oracle.mode_sum(shifted, out_len=ims.num_pts)
    assert rel_l2(got[: ims.num_pts], ref) < TOL_FAITHFUL


def test_sum_rejects_bad_inputs(cuda):
    inp, _ = load_case("sum_small_m0.npz")
    ims = InterpolatedModeSum()
    args = list(inp.call_args())
    bad = list(args)
    bad[4] = inp.phase_coeffs[:-1]
    with pytest.raises(ValueError):
        ims(*bad, T=inp.T, dt=inp.dt)
    bad = list(args)
    bad[0] = inp.t[::-1].copy()
    with pytest.raises(ValueError):
        ims(*bad, T=inp.T, dt=inp.dt)
    bad = list(args)
    bad[2] = inp.ylms[:-1]
    with pytest.raises(ValueError):
        ims(*bad, T=inp.T, dt=inp.dt)
    with pytest.raises(ValueError):
        InterpolatedModeSum(output_type="wd")
    with pytest.raises(ValueError):
        InterpolatedModeSum(precision="half")


def test_sharded_ranks_sum_to_the_whole(cuda):
    """Ranks of a split waveform (run one after another on one GPU, without
    collectives): their slices add up to the whole waveform bitwise and their
    partial gradients to the whole gradient."""
    from fastemriwaveforms_b200.distributed import ShardedInterpolatedModeSum

    inp = S.plain_small()
    whole, _ = run(inp, precision="exact")
    world = 3
    parts = []
    g_teuk, g_pc = 0, 0
    rng = np.random.default_rng(0)
    G = torch.tensor(rng.standard_normal(len(whole)) + 1j * rng.standard_normal(len(whole)), device=cuda)
    for r in range(world):
        ims = ShardedInterpolatedModeSum(rank=r, world=world, gather=False, reduce_grads=False, precision="exact")
        parts.append(ims(*inp.call_args(), T=inp.T, dt=inp.dt).cpu().numpy())
        teuk = torch.tensor(inp.teuk_modes, device=cuda, requires_grad=True)
        pc = torch.tensor(inp.phase_coeffs, device=cuda, requires_grad=True)
        ims(inp.t, teuk, inp.ylms, inp.phase_t, pc, inp.l, inp.m, inp.k, inp.n, T=inp.T, dt=inp.dt).backward(G)
        g_teuk = g_teuk + teuk.grad.cpu().numpy()
        g_pc = g_pc + pc.grad.cpu().numpy()
    assert np.array_equal(sum(parts), whole)
    teuk = torch.tensor(inp.teuk_modes, device=cuda, requires_grad=True)
    pc = torch.tensor(inp.phase_coeffs, device=cuda, requires_grad=True)
    InterpolatedModeSum(precision="exact")(inp.t, teuk, inp.ylms, inp.phase_t, pc, inp.l, inp.m, inp.k, inp.n,
                                           T=inp.T, dt=inp.dt).backward(G)
    ref_t, ref_p = teuk.grad.cpu().numpy(), pc.grad.cpu().numpy()
    assert np.abs(g_teuk - ref_t).max() <= 1e-11 * np.abs(ref_t).max()
    assert np.abs(g_pc - ref_p).max() <= 1e-11 * np.abs(ref_p).max()


@pytest.mark.parametrize("precision", ["faithful", "mixed"])
def test_host_out_streams_the_same_waveform(cuda, precision):
    """host_out: the sum in parts with each finished slice copied to pinned host
    memory while the next part runs; bitwise the device waveform, two calls in a
    row, and refused where it does not apply."""
    inp = S.plain_small()
    ims = InterpolatedModeSum(precision=precision, chunk=256)  # many units: four real parts
    ref = ims(*inp.call_args(), T=inp.T, dt=inp.dt).cpu().numpy()
    host = torch.zeros(len(ref) + 5, dtype=torch.complex128).pin_memory()
    for _ in range(2):
        host.zero_()
        wf = ims(*inp.call_args(), T=inp.T, dt=inp.dt, host_out=host)
        torch.cuda.synchronize()
        assert np.array_equal(host[: len(ref)].numpy(), ref)
        assert np.array_equal(wf.cpu().numpy(), ref)
    with pytest.raises(ValueError):
        ims(*inp.call_args(), T=inp.T, dt=inp.dt, host_out=torch.zeros(len(ref), dtype=torch.complex128))
    with pytest.raises(ValueError):
        ims(*inp.call_args(), T=inp.T, dt=inp.dt, host_out=host[:10])
