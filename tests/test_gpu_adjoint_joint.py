"""The joint FP64 adjoint (few_adjoint_joint: eleven moments per key and
work unit, from which G and the phase-coefficient gradients both follow) against
the two separate FP64 adjoint kernels (few_adjoint_G, few_adjoint_phase and its
reduction).  The joint pass regroups the same sums, so the two agree to
rounding; the cases cover the theta phase on and off, several row and column
groups, segments without samples and phase knots offset from the amplitude
knots (the basis terms then become shifted polynomials)."""
import numpy as np
import pytest
import torch

from fastemriwaveforms_b200 import InterpolatedModeSum
from fastemriwaveforms_b200 import _lib
from fastemriwaveforms_b200 import synthetic as S
from fastemriwaveforms_b200.summation import _ptr

pytestmark = pytest.mark.gpu

TOL_G = 1e-13    # G, max |difference| / max |G| (measured <= 2.1e-15)
TOL_PC = 1e-13   # phase-coefficient gradients, max |difference| / max |gradient| (measured <= 2.9e-15)


def _shifted_phase_knots():
    inp = S.small_case(K=30, N=40, out_len=30000, seed=17, theta=True)
    inp.phase_t = inp.t + 0.3 * np.diff(inp.t).min()
    return inp


CASES = {
    "small_theta": lambda: S.small_case(K=40, N=30, out_len=20000, seed=5, theta=True),
    "small_no_theta": lambda: S.small_case(K=40, N=30, out_len=20000, seed=6, theta=False),
    "plain_small": lambda: S.plain_small(seed=1),
    "many_rows": lambda: S.many_rows_case(),                                # 63 rows: several row groups
    "wide_n": lambda: S.many_rows_case(mmax=2, kmax=0, nmax=60, seed=13),  # NN = 121: two column groups
    "dense_knots": lambda: S.small_case(K=12, N=400, out_len=300, seed=8),  # segments without samples
    "shifted_phase_knots": _shifted_phase_knots,
}


def _plan(inp, cuda):
    teuk = torch.tensor(inp.teuk_modes, device=cuda, requires_grad=True)
    h = InterpolatedModeSum(precision="exact")(inp.t, teuk, inp.ylms, inp.phase_t, inp.phase_coeffs, inp.l, inp.m,
                                               inp.k, inp.n, T=inp.T, dt=inp.dt)
    rng = np.random.default_rng(3)
    g = rng.standard_normal(h.shape[0]) + 1j * rng.standard_normal(h.shape[0])
    p = h.grad_fn.prep
    return p, torch.tensor(g[: p.out_len], device=cuda).contiguous()


def _separate(p, grad):
    fold, seg = p.fold, p.seg
    seg_start, seg_units = seg.backward_tables()
    G = torch.empty((max(seg.nseg, 1), fold.R, fold.NN, 4), dtype=torch.complex128, device=grad.device)
    _lib.call("few_adjoint_G", _ptr(grad), _ptr(p.pc), p.N, _ptr(seg.d_seg_info), _ptr(seg_start), seg.nseg,
              _ptr(fold.d_row_m), _ptr(fold.d_row_k), fold.R, fold.nlo, fold.NN, p.dt, fold.use_theta, _ptr(G), p.st)
    partial = torch.empty((max(seg.nunits, 1), 24), dtype=torch.float64, device=grad.device)
    _lib.call("few_adjoint_phase", _ptr(grad), _ptr(p.W), _ptr(p.pc), p.N, _ptr(seg.d_seg_info), _ptr(seg.d_units),
              seg.nunits, _ptr(fold.d_row_m), _ptr(fold.d_row_k), fold.R, fold.nlo, fold.NN, p.dt, fold.use_theta,
              _ptr(partial), p.st)
    g_pc = torch.zeros((p.N - 1, 3, 8), dtype=torch.float64, device=grad.device)
    _lib.call("few_adjoint_phase_reduce", _ptr(partial), _ptr(seg_units), seg.nseg, _ptr(g_pc), p.st)
    return G.cpu().numpy()[: seg.nseg], g_pc.cpu().numpy()


def _joint(p, grad, want_G=True, want_pc=True, balanced=True):
    fold, seg = p.fold, p.seg
    if balanced:
        units, seg_units, nunits = seg.balanced_units()
    else:
        units, nunits = seg.d_units, seg.nunits
        _, seg_units = seg.backward_tables()
    G = torch.full((max(seg.nseg, 1), fold.R, fold.NN, 4), np.nan, dtype=torch.complex128, device=grad.device)
    g_pc = torch.zeros((p.N - 1, 3, 8), dtype=torch.float64, device=grad.device)
    n = int(_lib.load().few_adjoint_joint_scratch(max(nunits, 1), fold.R, fold.NN))
    scratch = torch.full((max(n, 1),), np.nan, dtype=torch.float64, device=grad.device)
    _lib.call("few_adjoint_joint", _ptr(grad), _ptr(p.W), _ptr(p.pc), p.N, _ptr(seg.d_seg_info), _ptr(units),
              nunits, _ptr(seg_units), seg.nseg, _ptr(fold.d_row_m), _ptr(fold.d_row_k), fold.R, fold.nlo, fold.NN,
              p.dt, fold.use_theta, _ptr(G) if want_G else 0, _ptr(g_pc) if want_pc else 0, _ptr(scratch), p.st)
    return G.cpu().numpy()[: seg.nseg], g_pc.cpu().numpy()


@pytest.mark.parametrize("name", sorted(CASES))
def test_joint_adjoint_matches_separate_kernels(cuda, name):
    inp = CASES[name]()
    p, grad = _plan(inp, cuda)
    G_ref, pc_ref = _separate(p, grad)
    G, pc = _joint(p, grad)
    assert np.isfinite(G).all()
    eg = float(np.abs(G - G_ref).max() / np.abs(G_ref).max())
    ep = float(np.abs(pc - pc_ref).max() / np.abs(pc_ref).max())
    print(f"\n{name}: R={p.fold.R} NN={p.fold.NN} nseg={p.seg.nseg}: G max/max {eg:.2e}, phase grads max/max {ep:.2e}")
    assert eg <= TOL_G
    assert ep <= TOL_PC
    assert not pc[p.seg.nseg:].any()
    if not p.fold.use_theta:
        assert not pc[:, 1, :].any()


def test_joint_adjoint_single_outputs_and_determinism(cuda):
    """G alone (the five-moment form) and the phase gradients alone equal the
    combined call's, and a repeated call gives the same bits."""
    p, grad = _plan(S.small_case(K=30, N=25, out_len=8000, seed=10, theta=True), cuda)
    G, pc = _joint(p, grad)
    G2, pc2 = _joint(p, grad)
    assert np.array_equal(G, G2) and np.array_equal(pc, pc2)
    G_only, _ = _joint(p, grad, want_pc=False)
    _, pc_only = _joint(p, grad, want_G=False)
    assert np.array_equal(G_only, G)
    assert np.array_equal(pc_only, pc)
    # the forward's work units (a short remainder per segment) regroup the same sums
    G_u, pc_u = _joint(p, grad, balanced=False)
    assert np.abs(G_u - G).max() <= TOL_G * np.abs(G).max()
    assert np.abs(pc_u - pc).max() <= TOL_PC * np.abs(pc).max()


def test_joint_adjoint_argument_errors(cuda):
    p, grad = _plan(S.small_case(K=8, N=12, out_len=3000, seed=2), cuda)
    fold, seg = p.fold, p.seg
    _, seg_units = seg.backward_tables()
    scratch = torch.empty(16, dtype=torch.float64, device=cuda)
    common = (_ptr(grad), _ptr(p.W), _ptr(p.pc), p.N, _ptr(seg.d_seg_info), _ptr(seg.d_units), seg.nunits,
              _ptr(seg_units), seg.nseg, _ptr(fold.d_row_m), _ptr(fold.d_row_k), fold.R, fold.nlo, fold.NN, p.dt,
              fold.use_theta)
    with pytest.raises(ValueError, match="neither"):
        _lib.call("few_adjoint_joint", *common, 0, 0, _ptr(scratch), p.st)
    g_pc = torch.zeros((p.N - 1, 3, 8), dtype=torch.float64, device=cuda)
    with pytest.raises(ValueError, match="null pointer"):  # the scratch rows are required
        _lib.call("few_adjoint_joint", *common, 0, _ptr(g_pc), 0, p.st)


@pytest.mark.parametrize("name", ["small_theta", "many_rows", "wide_n", "dense_knots"])
def test_joint_G_alone_matches_G_kernel(cuda, name):
    """G alone (five moments per key, used when only the amplitude gradient is
    wanted) against few_adjoint_G."""
    p, grad = _plan(CASES[name](), cuda)
    G_ref, _ = _separate(p, grad)
    G, _ = _joint(p, grad, want_pc=False)
    assert np.isfinite(G).all()
    assert np.abs(G - G_ref).max() <= TOL_G * np.abs(G_ref).max()

