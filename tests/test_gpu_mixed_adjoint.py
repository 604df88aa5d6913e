"""The tensor-core adjoint: the per-segment G contraction and the phase
adjoint against the FP64 adjoint kernels, and the gradients of a mixed
forward + mixed backward against the FP64 backward.  Both contractions run in
exact integer arithmetic on the tensor cores (FP64 operands as four int8
digits, int32 accumulation), so the only differences from FP64 are the 2^-32
representation of the operands; the relative errors are printed."""
import numpy as np
import pytest
import torch

from fastemriwaveforms_b200 import InterpolatedModeSum
from fastemriwaveforms_b200 import _lib
from fastemriwaveforms_b200 import synthetic as S
from fastemriwaveforms_b200.summation import _ptr

pytestmark = pytest.mark.gpu

REL_G = 1e-8           # G array (nseg, R, NN, 4) vs the FP64 kernel, relative L2 (measured <= 9e-10)
REL_GRAD_TEUK = 3e-8   # dL/d teuk_modes vs the FP64 backward, relative L2 (measured <= 4.2e-9)
REL_GRAD_PC = 3e-8     # dL/d phase_interp_coeffs vs the FP64 backward, relative L2 (measured <= 1.5e-9)


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def upstream(inp, cuda, seed=11):
    """torch's upstream gradient conj(h_ref + w), w white with sigma 0.1 rms(h_ref)."""
    with torch.no_grad():
        h = InterpolatedModeSum(precision="exact")(inp.t, inp.teuk_modes, inp.ylms, inp.phase_t, inp.phase_coeffs,
                                                   inp.l, inp.m, inp.k, inp.n, T=inp.T, dt=inp.dt)
    rng = np.random.default_rng(seed)
    href = h.cpu().numpy()
    rms = np.sqrt(np.mean(np.abs(href) ** 2))
    w = (rng.standard_normal(href.shape) + 1j * rng.standard_normal(href.shape)) * 0.1 * rms / np.sqrt(2.0)
    return torch.tensor(np.conj(href + w), device=cuda)


def gradients(inp, cuda, precision, backward, G):
    teuk = torch.tensor(inp.teuk_modes, device=cuda, requires_grad=True)
    pc = torch.tensor(inp.phase_coeffs, device=cuda, requires_grad=True)
    ims = InterpolatedModeSum(precision=precision, backward=backward)
    h = ims(inp.t, teuk, inp.ylms, inp.phase_t, pc, inp.l, inp.m, inp.k, inp.n, T=inp.T, dt=inp.dt)
    h.backward(G)
    torch.cuda.synchronize()
    assert not ims.mixed_error()
    return teuk.grad.cpu().numpy(), pc.grad.cpu().numpy()


CASES = {
    "plain_small": lambda: S.plain_small(seed=1),
    "plain_full": lambda: S.plain_full(seed=2),
    "small_theta": lambda: S.small_case(K=40, N=30, out_len=20000, seed=5, theta=True),
    "many_rows": lambda: S.many_rows_case(),  # 63 rows: two MMA column groups in the phase adjoint
    # n' = -60..60 (NN = 121): eight K steps of 16 n' in the phase adjoint, two 64-n' blocks in G
    "wide_n": lambda: S.many_rows_case(mmax=2, kmax=0, nmax=60, seed=13),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_mixed_G_matches_fp64(cuda, name):
    inp = CASES[name]()
    G_t = upstream(inp, cuda)
    ims = InterpolatedModeSum(precision="mixed")
    teuk = torch.tensor(inp.teuk_modes, device=cuda, requires_grad=True)
    h = ims(inp.t, teuk, inp.ylms, inp.phase_t, inp.phase_coeffs, inp.l, inp.m, inp.k, inp.n, T=inp.T, dt=inp.dt)
    p = h.grad_fn.prep if hasattr(h.grad_fn, "prep") else None
    assert p is not None
    fold, seg = p.fold, p.seg
    grad = G_t[: p.out_len].contiguous()
    seg_start, _ = seg.backward_tables()
    out = []
    for mixed in (False, True):
        Gk = torch.empty((max(seg.nseg, 1), fold.R, fold.NN, 4), dtype=torch.complex128, device=cuda)
        if mixed:
            _lib.call("few_adjoint_G_mixed", _ptr(grad), _ptr(p.pc), p.N, _ptr(seg.d_seg_info), _ptr(p.t_dev),
                      _ptr(seg_start), seg.nseg, _ptr(fold.d_row_m), _ptr(fold.d_row_k), fold.R, fold.nlo, fold.NN,
                      p.dt, fold.use_theta, _ptr(Gk), _ptr(p.err), p.st)
        else:
            _lib.call("few_adjoint_G", _ptr(grad), _ptr(p.pc), p.N, _ptr(seg.d_seg_info), _ptr(seg_start), seg.nseg,
                      _ptr(fold.d_row_m), _ptr(fold.d_row_k), fold.R, fold.nlo, fold.NN, p.dt, fold.use_theta,
                      _ptr(Gk), p.st)
        out.append(Gk.cpu().numpy())
    assert not ims.mixed_error()
    e = rel(out[1], out[0])
    emax = float(np.abs(out[1] - out[0]).max() / np.abs(out[0]).max())
    print(f"\n{name}: G mixed vs FP64 rel L2 {e:.3e}, max/max {emax:.3e}")
    assert e <= REL_G


@pytest.mark.parametrize("name", sorted(CASES))
def test_mixed_backward_matches_fp64(cuda, name):
    inp = CASES[name]()
    G_t = upstream(inp, cuda)
    ref_t, ref_p = gradients(inp, cuda, "exact", "fp64", G_t)
    got_t, got_p = gradients(inp, cuda, "mixed", "mixed", G_t)
    et, ep = rel(got_t, ref_t), rel(got_p, ref_p)
    per_field = [rel(got_p[:, f, :], ref_p[:, f, :]) for f in range(3) if np.any(ref_p[:, f, :])]
    print(f"\n{name}: grad teuk rel L2 {et:.3e}, grad phase coeffs rel L2 {ep:.3e} (per field {per_field})")
    assert et <= REL_GRAD_TEUK
    assert ep <= REL_GRAD_PC


def test_mixed_backward_deterministic(cuda):
    inp = S.small_case(K=30, N=25, out_len=8000, seed=10, theta=True)
    G_t = upstream(inp, cuda)
    a = gradients(inp, cuda, "mixed", "mixed", G_t)
    b = gradients(inp, cuda, "mixed", "mixed", G_t)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
