"""Batched persistent launch: many waveforms of uneven length, knot count and
mode count in one sum kernel, against one InterpolatedModeSum call per
waveform; CUDA-graph capture and replay; the autotuner's cache."""
import json

import numpy as np
import pytest
import torch

from fastemriwaveforms_b200 import InterpolatedModeSum
from fastemriwaveforms_b200 import synthetic as S
from fastemriwaveforms_b200.batched import BatchedInterpolatedModeSum

pytestmark = pytest.mark.gpu


def uneven_batch(count=6, seed=3):
    rng = np.random.default_rng(seed)
    out = []
    for w in range(count):
        K = int(rng.integers(20, 700))
        N = int(rng.integers(8, 120))
        T_samples = int(np.exp(rng.uniform(np.log(5e3), np.log(1.2e5))))
        span = (T_samples - 1) * 10.0
        out.append(S.make_inputs(K=K, N=N, span=span, t_c=span * 1.05, lmax=10, nmax=30,
                                 seed=int(rng.integers(1 << 30)), name=f"w{w}"))
    return out


def single(inp, precision):
    wf = InterpolatedModeSum(precision=precision)(*inp.call_args(), T=inp.T, dt=inp.dt)
    torch.cuda.synchronize()
    return wf.cpu().numpy()


@pytest.mark.parametrize("precision", ["exact", "faithful", "mixed"])
def test_batched_equals_single(cuda, tmp_path, monkeypatch, precision):
    monkeypatch.setenv("FEW_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    batch = uneven_batch()
    b = BatchedInterpolatedModeSum(precision=precision).setup(batch)
    outs = [o.cpu().numpy() for o in b.forward()]
    torch.cuda.synchronize()
    if precision == "mixed":
        assert not b.mixed_error()
    for inp, got in zip(batch, outs):
        ref = single(inp, precision)
        assert got.shape == ref.shape
        # each sample is computed the same way whatever unit it falls in
        assert np.array_equal(got, ref)
    cache = json.loads((tmp_path / "tune.json").read_text())
    assert b._key in cache and cache[b._key]["chunk"] in (256, 512, 1024)
    if precision == "mixed":  # the tensor-core shape search includes the operand pipeline
        assert cache[b._key]["astages"] in (1, 2) and cache[b._key]["bstages"] in (2, 3, 4)
        tried = cache[b._key]["tried"]
        assert {(t["astages"], t["bstages"]) for t in tried} == {(a, c) for a in (1, 2) for c in (2, 3, 4)}


def test_mixed_pipeline_shape_does_not_change_results(cuda, tmp_path, monkeypatch):
    """Every operand pipeline shape and CTA count gives bitwise the same waveforms."""
    monkeypatch.setenv("FEW_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    batch = uneven_batch(count=5, seed=9)
    ref = None
    for ast, bst, per_sm in ((1, 2, 2), (1, 3, 2), (1, 4, 1), (2, 2, 2), (2, 3, 2), (2, 4, 1)):
        b = BatchedInterpolatedModeSum(precision="mixed", chunk=512, ctas_per_sm=per_sm, astages=ast,
                                       bstages=bst).setup(batch)
        outs = [o.cpu().numpy() for o in b.forward()]
        torch.cuda.synchronize()
        assert not b.mixed_error()
        if ref is None:
            ref = outs
        for a, c in zip(ref, outs):
            assert np.array_equal(a, c), (ast, bst, per_sm)


def test_graph_capture_replay_and_update(cuda, tmp_path, monkeypatch):
    monkeypatch.setenv("FEW_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    batch = uneven_batch(count=4, seed=5)
    b = BatchedInterpolatedModeSum(precision="mixed", chunk=512, ctas_per_sm=2).setup(batch)
    first = [o.cpu().numpy() for o in b.forward()]
    b.capture()
    again = [o.cpu().numpy() for o in b.replay()]
    for x, y in zip(first, again):
        assert np.array_equal(x, y)
    # new amplitudes for waveform 2, replayed through the graph
    new = batch[2].teuk_modes * (0.5 - 0.25j)
    b.update(2, teuk_modes=new)
    replayed = [o.cpu().numpy() for o in b.replay()]
    changed = S.ModeSumInputs(**{**batch[2].__dict__})
    changed.teuk_modes = new
    assert np.array_equal(replayed[2], single(changed, "mixed"))
    assert np.array_equal(replayed[0], first[0])


@pytest.mark.parametrize("precision", ["exact", "mixed"])
def test_batched_backward_matches_single(cuda, tmp_path, monkeypatch, precision):
    """The batched graph's adjoint (FP64, or the tensor-core one for the mixed
    form) equals the single-waveform autograd backward bit for bit."""
    monkeypatch.setenv("FEW_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    batch = uneven_batch(count=3, seed=7)
    rng = np.random.default_rng(1)
    grads = [torch.tensor(rng.standard_normal(len(single(w, "exact"))) + 0j, device=cuda) for w in batch]
    b = BatchedInterpolatedModeSum(precision=precision, chunk=1024, ctas_per_sm=2).setup(batch, requires_grad=True)
    b.forward()
    b.capture(backward=True, grads=grads)
    b.replay()
    torch.cuda.synchronize()
    for inp, g, (gt, gp) in zip(batch, grads, b.grad_out):
        teuk = torch.tensor(inp.teuk_modes, device=cuda, requires_grad=True)
        pc = torch.tensor(inp.phase_coeffs, device=cuda, requires_grad=True)
        h = InterpolatedModeSum(precision=precision)(inp.t, teuk, inp.ylms, inp.phase_t, pc, inp.l, inp.m, inp.k,
                                                     inp.n, T=inp.T, dt=inp.dt)
        h.backward(g)
        assert not b.mixed_error()
        assert torch.equal(gt, teuk.grad)
        assert torch.equal(gp, pc.grad)


def test_per_waveform_completion_times(cuda, tmp_path, monkeypatch):
    """The time stamps behind the batched p50/p99: every waveform's sum
    completes after the forward's start, within the forward's span, and its
    backward after every forward completion (the backward starts once the
    persistent sum is done)."""
    monkeypatch.setenv("FEW_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    batch = uneven_batch(count=5, seed=11)
    b = BatchedInterpolatedModeSum(precision="mixed", chunk=1024, ctas_per_sm=2).setup(batch, requires_grad=True)
    outs = b.forward()
    b.backward([torch.conj(o).clone() for o in outs])
    torch.cuda.synchronize()
    fwd, bwd = b.latencies()
    assert fwd.shape == (5,) and bwd is not None and bwd.shape == (5,)
    assert np.all(fwd > 0) and np.all(np.isfinite(fwd))
    assert np.all(bwd >= fwd.max())
    assert bwd.max() < 60e3  # ms: the stamps are nanoseconds of the same clock


def test_backward_tables_reach_the_side_stream(cuda):
    """Many short forward + backward calls through one module (both gradients,
    so the phase branch runs on the side stream): every call's gradients equal
    a second run's bit for bit.  The side stream reads segment tables that the
    backward uploads; they must be in place before it forks."""
    rng = np.random.default_rng(4)
    cases = []
    for w in range(24):
        K = int(rng.integers(5, 60))
        N = int(rng.integers(6, 40))
        cases.append(S.small_case(K=K, N=N, out_len=int(rng.integers(2000, 9000)), seed=100 + w, theta=False))
    ims = InterpolatedModeSum(precision="exact")

    def grads(inp):
        teuk = torch.tensor(inp.teuk_modes, device=cuda, requires_grad=True)
        pc = torch.tensor(inp.phase_coeffs, device=cuda, requires_grad=True)
        h = ims(inp.t, teuk, inp.ylms, inp.phase_t, pc, inp.l, inp.m, inp.k, inp.n, T=inp.T, dt=inp.dt)
        h.backward(torch.conj(h.detach()))
        return teuk.grad, pc.grad

    first = [grads(c) for c in cases]
    torch.cuda.synchronize()
    for c, (gt, gp) in zip(cases, first):
        gt2, gp2 = grads(c)
        assert torch.equal(gt, gt2) and torch.equal(gp, gp2)
