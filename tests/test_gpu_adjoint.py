"""The adjoint kernels behind torch.autograd: dL/d(amplitude knots) and
dL/d(phase coefficients / phase knots) for L = Re sum_i g_i h_i, checked
against exact linear probes and central finite differences of the FP64
oracle (the reference's CPU path restated)."""
import numpy as np
import pytest
import torch

from fastemriwaveforms_b200 import InterpolatedModeSum
from fastemriwaveforms_b200 import synthetic as S
from fastemriwaveforms_b200.autograd import phase_coeffs_from_knots, spline_coefficients

pytestmark = pytest.mark.gpu

TOL_LINEAR = 1e-10   # gradients of linear maps vs exact probes (relative to the gradient's max)
TOL_FD = 1e-6        # gradients vs central finite differences (relative, per entry)


def loss_np(h, g):
    """L = Re sum g h with torch's upstream gradient G = conj(g)."""
    return float(np.real(np.sum(g * h)))


def test_spline_adjoint_is_the_transpose(cuda, oracle):
    rng = np.random.default_rng(1)
    for N in (4, 5, 9, 40, 300):
        x = np.cumsum(np.concatenate([[0.0], rng.exponential(1.0, N - 1) + 0.05]))
        ni = 3
        y = torch.tensor(rng.standard_normal((ni, N)), device=cuda, requires_grad=True)
        c = spline_coefficients(x, y)
        gc = torch.tensor(rng.standard_normal(c.shape), device=cuda)
        (c * gc).sum().backward()
        # dense Jacobian of the oracle's spline (linear in y)
        J = np.zeros((4, N, N))
        for j in range(N):
            e = np.zeros(N)
            e[j] = 1.0
            J[:, :, j] = oracle.spline_coeffs(x, e[None, :])[:, :, 0]
        ref = np.einsum("cij,cip->pj", J, gc.cpu().numpy())
        got = y.grad.cpu().numpy()
        assert np.abs(got - ref).max() / np.abs(ref).max() < 1e-11, N


def small_inputs(seed=3, K=6, N=12, out_len=3000, theta=True):
    inp = S.small_case(K=K, N=N, out_len=out_len, seed=seed, theta=theta)
    return inp


def test_amplitude_gradient_exact(cuda, oracle):
    """h is linear in the amplitude knots: probing each real parameter with the
    oracle gives the gradient exactly."""
    inp = small_inputs()
    N, K = inp.teuk_modes.shape
    rng = np.random.default_rng(5)
    g = rng.standard_normal(inp.out_len) + 1j * rng.standard_normal(inp.out_len)
    teuk = torch.tensor(inp.teuk_modes, device=cuda, requires_grad=True)
    ims = InterpolatedModeSum(precision="exact")
    h = ims(inp.t, teuk, inp.ylms, inp.phase_t, inp.phase_coeffs, inp.l, inp.m, inp.k, inp.n, T=inp.T, dt=inp.dt)
    G = torch.tensor(np.conj(g), device=cuda)
    (h * torch.conj(G)).real.sum().backward()
    got = teuk.grad.cpu().numpy()
    ref = np.zeros((N, K), complex)
    base = inp.teuk_modes
    for i in range(N):
        for j in range(K):
            for part, unit in ((0, 1.0), (1, 1j)):
                probe = S.ModeSumInputs(**{**inp.__dict__})
                probe.teuk_modes = np.zeros_like(base)
                probe.teuk_modes[i, j] = unit
                val = loss_np(oracle.mode_sum(probe, extended=True), g)
                if part == 0:
                    ref[i, j] += val
                else:
                    ref[i, j] += 1j * val
    err = np.abs(got - ref).max() / np.abs(ref).max()
    assert err < TOL_LINEAR, err


@pytest.mark.parametrize("theta", [True, False])
def test_phase_coefficient_gradient_fd(cuda, oracle, theta):
    inp = small_inputs(seed=4, theta=theta)
    rng = np.random.default_rng(6)
    g = rng.standard_normal(inp.out_len) + 1j * rng.standard_normal(inp.out_len)
    pc = torch.tensor(inp.phase_coeffs, device=cuda, requires_grad=True)
    ims = InterpolatedModeSum(precision="exact")
    h = ims(inp.t, inp.teuk_modes, inp.ylms, inp.phase_t, pc, inp.l, inp.m, inp.k, inp.n, T=inp.T, dt=inp.dt)
    (h * torch.tensor(g, device=cuda)).real.sum().backward()
    got = pc.grad.cpu().numpy()
    start, nseg = oracle.find_start_inds(inp.t, inp.dt, inp.out_len)
    picks = [(j, f, q) for j in (0, 3, nseg - 1) for f in ((0, 1, 2) if theta else (0, 2)) for q in (0, 1, 4, 7)]
    # max over s in [0, 1] of the basis term b_q(s); the step moves Phi by ~1e-6 rad for
    # every q, so the oracle's double-precision Phi (ulp ~6e-14 rad here) stays far below it
    bmax = [1.0, 1.0, 0.25, 4 / 27, 1 / 16, 0.0346, 1 / 64, 0.00840]
    for (j, f, q) in picks:
        delta = 1e-6 / bmax[q]
        vals = []
        for sgn in (1, -1):
            probe = S.ModeSumInputs(**{**inp.__dict__})
            probe.phase_coeffs = inp.phase_coeffs.copy()
            probe.phase_coeffs[j, f, q] += sgn * delta
            w = oracle.mode_sum(probe, extended=True, window=(int(start[j]), int(start[j + 1])))
            vals.append(loss_np(w, g))
        fd = (vals[0] - vals[1]) / (2 * delta)
        scale = max(abs(fd), 1e-3 * np.abs(got).max())
        assert abs(got[j, f, q] - fd) / scale < TOL_FD, (j, f, q, got[j, f, q], fd)
    # coefficients of segments without samples get no gradient
    assert not got[nseg:].any()


def test_knot_gradients_vs_finite_differences(cuda, oracle):
    """Amplitude knots (complex) and Phi_phi / Phi_r knots through the
    differentiable phase spline, against central finite differences of the
    oracle on windows around each perturbed knot (the spline's influence decays
    by ~0.27 per knot; +-12 segments leave < 2e-7)."""
    inp = S.make_inputs(K=120, N=60, span=6e5, t_c=7e5, lmax=10, nmax=30, seed=8, name="adj")
    N, K = inp.teuk_modes.shape
    rng = np.random.default_rng(9)
    w = rng.standard_normal(inp.out_len) + 1j * rng.standard_normal(inp.out_len)
    ims = InterpolatedModeSum(precision="exact")
    h_ref = ims(*inp.call_args(), T=inp.T, dt=inp.dt).cpu().numpy()
    G = np.conj(np.conj(h_ref + 0.1 * np.sqrt(np.mean(np.abs(h_ref) ** 2)) * w))  # torch upstream = conj(g)
    g = np.conj(G)
    teuk = torch.tensor(inp.teuk_modes, device=cuda, requires_grad=True)
    knots = torch.tensor(inp.phase_knots, device=cuda, requires_grad=True)
    pc = phase_coeffs_from_knots(inp.t, knots)
    h = ims(inp.t, teuk, inp.ylms, inp.phase_t, pc, inp.l, inp.m, inp.k, inp.n, T=inp.T, dt=inp.dt)
    h.backward(torch.tensor(G, device=cuda))
    g_teuk = teuk.grad.cpu().numpy()
    g_knots = knots.grad.cpu().numpy()
    start, nseg = oracle.find_start_inds(inp.t, inp.dt, inp.out_len)

    def windowed_loss(probe, j, extended):
        lo = int(start[max(j - 12, 0)])
        hi = int(start[min(j + 12, nseg)])
        return loss_np(oracle.mode_sum(probe, window=(lo, hi), extended=extended)[lo:hi], g[lo:hi])

    for _ in range(8):  # amplitude knots, real and imaginary parts
        j = int(rng.integers(0, N))
        k = int(rng.integers(0, K))
        for unit in (1.0, 1j):
            d = 1e-2  # h is linear in the amplitudes: the central difference is exact up to rounding
            vals = []
            for sgn in (1, -1):
                probe = S.ModeSumInputs(**{**inp.__dict__})
                probe.teuk_modes = inp.teuk_modes.copy()
                probe.teuk_modes[j, k] += sgn * d * unit
                vals.append(windowed_loss(probe, j, False))
            fd = (vals[0] - vals[1]) / (2 * d)
            got = g_teuk[j, k].real if unit == 1.0 else g_teuk[j, k].imag
            assert abs(got - fd) <= TOL_FD * max(abs(fd), 1e-2 * np.abs(g_teuk).max()), (j, k, unit, got, fd)
    for f in (0, 2):  # Phi_phi and Phi_r knots
        for _ in range(4):
            j = int(rng.integers(0, N))
            d = 1e-5  # rad: max(|m|, |n|) * d << 1 keeps the central difference's truncation error small
            vals = []
            for sgn in (1, -1):
                pk = inp.phase_knots.copy()
                pk[f, j] += sgn * d
                probe = S.ModeSumInputs(**{**inp.__dict__})
                probe.phase_coeffs = S.phase_basis_from_knots(inp.t, pk)
                vals.append(windowed_loss(probe, j, True))
            fd = (vals[0] - vals[1]) / (2 * d)
            got = g_knots[f, j]
            assert abs(got - fd) <= TOL_FD * max(abs(fd), 1e-2 * np.abs(g_knots[f]).max()), (f, j, got, fd)


def test_backward_deterministic_and_consistent_with_faithful_forward(cuda):
    inp = small_inputs(seed=10, K=30, N=25, out_len=8000)
    outs = []
    for precision in ("faithful", "exact", "exact"):
        teuk = torch.tensor(inp.teuk_modes, device=cuda, requires_grad=True)
        pc = torch.tensor(inp.phase_coeffs, device=cuda, requires_grad=True)
        h = InterpolatedModeSum(precision=precision)(inp.t, teuk, inp.ylms, inp.phase_t, pc, inp.l, inp.m, inp.k,
                                                     inp.n, T=inp.T, dt=inp.dt)
        (h.abs() ** 2).sum().backward()
        outs.append((teuk.grad.cpu().numpy(), pc.grad.cpu().numpy()))
    assert np.array_equal(outs[1][0], outs[2][0]) and np.array_equal(outs[1][1], outs[2][1])
    for a, b in zip(outs[0], outs[1]):
        assert np.abs(a - b).max() <= 1e-8 * np.abs(b).max()


def test_amplitude_gradient_independent_of_row_blocking(cuda):
    """L is linear in the amplitudes and the upstream gradient is fixed, so a
    mode's amplitude gradient does not depend on which other modes are summed.
    Mode sets with 41, 29, 21 and 11 rows (m' = -20..20, -14..14, -10..10,
    -5..5) make the FP64 G kernel take its 8-, 6-, 4- and 2-row blocks; the
    gradients of the modes they share agree."""
    m_all = np.repeat(np.arange(0, 21), 3).astype(np.int32)
    n_all = np.tile(np.array([-2, 0, 1]), 21).astype(np.int32)
    K_all = len(m_all)
    base = S.small_case(K=K_all, N=16, out_len=5000, seed=21, theta=False)
    rng = np.random.default_rng(22)
    g = rng.standard_normal(base.out_len) + 1j * rng.standard_normal(base.out_len)
    G = torch.tensor(np.conj(g), device=cuda)

    def amplitude_grad(sel):
        K = len(sel)
        teuk = torch.tensor(np.ascontiguousarray(base.teuk_modes[:, sel]), device=cuda, requires_grad=True)
        ylms = np.concatenate([base.ylms[sel], base.ylms[K_all + sel]])
        h = InterpolatedModeSum(precision="exact")(base.t, teuk, ylms, base.phase_t, base.phase_coeffs,
                                                   np.full(K, 20, np.int32), m_all[sel], np.zeros(K, np.int32),
                                                   n_all[sel], T=base.T, dt=base.dt)
        (h * torch.conj(G)).real.sum().backward()
        return teuk.grad.cpu().numpy()

    full = amplitude_grad(np.arange(K_all))
    assert np.abs(full).max() > 0
    for m_max in (14, 10, 5):
        sel = np.flatnonzero(m_all <= m_max)
        sub = amplitude_grad(sel)
        err = np.abs(sub - full[:, sel]).max() / np.abs(full[:, sel]).max()
        assert err <= 1e-12, (m_max, err)


@pytest.mark.parametrize("N,K", [(4, 3), (9, 5), (1000, 3843)])
def test_factored_spline_adjoint_matches_generic(cuda, N, K):
    """Shared-knot adjoint (host factorization) vs the per-series adjoint kernel,
    on the complex (N, K) view the mode-sum backward uses."""
    from fastemriwaveforms_b200 import _lib
    from fastemriwaveforms_b200.summation import spline_factor_table

    rng = np.random.default_rng(N)
    t = np.cumsum(np.concatenate([[0.0], rng.exponential(1.0, N - 1) + 1e-2]))
    gc = torch.tensor(rng.standard_normal((4, N, 2 * K)), device=cuda)
    td = torch.from_numpy(t).to(cuda)
    st = torch.cuda.current_stream().cuda_stream
    g_generic = torch.empty((N, K), dtype=torch.complex128, device=cuda)
    _lib.call("few_spline_adjoint", td.data_ptr(), 0, gc.clone().data_ptr(), g_generic.data_ptr(), 2 * K, 2, K, 1,
              2 * K, N, 0, st)
    fac = spline_factor_table(t, cuda)
    g_fact = torch.empty_like(g_generic)
    _lib.call("few_spline_adjoint_factored", fac.data_ptr(), gc.clone().data_ptr(), g_fact.data_ptr(), 2 * K, 2, K,
              1, 2 * K, N, 0, st)
    a, b = g_fact.cpu().numpy(), g_generic.cpu().numpy()
    assert np.abs(a - b).max() <= 1e-11 * np.abs(b).max()
