"""The producers of ylms and of the mode list on the GPU against the
reference (golden vectors from its own GetYlms and ModeSelector, made by
tests/golden/make_fd_golden.py):

* GetYlms: every (l, m) with l <= 10 at seven viewing angles (poles included)
  within 1e-13 of the largest harmonic (the reference spells each (l, m) out
  in closed form; the kernel sums Goldberg's series, so the roundings differ);
* ModeSelector: the threshold form keeps exactly the reference's modes, in its
  order, with the same amplitudes and harmonics; the 'all' and list forms."""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from fastemriwaveforms_b200 import GetYlms, ModeSelector
from fastemriwaveforms_b200 import synthetic as S

pytestmark = pytest.mark.gpu

REL_YLM = 1e-13


def close(a, b, rel=REL_YLM):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and np.abs(a - b).max() <= rel * max(np.abs(b).max(), 1e-300)


def test_ylms_match_reference(cuda):
    d = np.load(os.path.join(GOLDEN, "ylm.npz"))
    gen = GetYlms()
    for i, (th, ph) in enumerate(d["angles"]):
        got = gen(d["l"], d["m"], th, ph).cpu().numpy()
        assert close(got, d["ylm"][i]), (th, ph, np.abs(got - d["ylm"][i]).max())
    # the (+m, -m) doubling of include_minus_m, scalars, and the range check
    l = np.array([2, 3, 4], dtype=np.int32)
    m = np.array([0, 1, 4], dtype=np.int32)
    both = GetYlms(include_minus_m=True)(l, m, 0.8, 0.3).cpu().numpy()
    assert np.allclose(both[3:], gen(l, -m, 0.8, 0.3).cpu().numpy(), rtol=0, atol=0)
    assert np.allclose(both[:3], gen(l, m, 0.8, 0.3).cpu().numpy(), rtol=0, atol=0)
    yp, ym = gen(2, 2, 0.8, 0.3, include_minus_m=True)
    assert yp == gen(2, 2, 0.8, 0.3) and ym == gen(2, -2, 0.8, 0.3)
    assert isinstance(gen(3, -1, 0.8, 0.3), complex)
    with pytest.raises(ValueError):
        gen(np.array([2]), np.array([3]), 0.8, 0.3)


def test_mode_selector_matches_reference(cuda):
    d = np.load(os.path.join(GOLDEN, "modeselector.npz"))
    gen = S.FixedAmplitudes()
    sel = ModeSelector(gen)
    t = d["t"]
    for tag, thr in (("thr5", 1e-5), ("thr2", 1e-2)):
        out = sel(t, 0.5, None, None, None, 1.1, 0.7, mode_selection_threshold=thr, return_sort_inds=True)
        teuk, ylms, l, m, k, n, inv = (v.cpu().numpy() for v in out)
        for name, got in (("l", l), ("m", m), ("k", k), ("n", n), ("inv", inv)):
            assert np.array_equal(got, d[f"{tag}_{name}"]), (tag, name)
        assert np.array_equal(teuk, d[f"{tag}_teuk"])
        assert close(ylms, d[f"{tag}_ylms"])
        print(f"\n{tag}: kept {len(l)} of {gen.teuk.shape[1]} modes, as the reference")
    out = sel(t, 0.5, None, None, None, 0.4, 2.0, mode_selection="all")
    assert close(out[1].cpu().numpy(), d["all_ylms"])
    out = sel(t, 0.5, None, None, None, 0.4, 2.0, mode_selection=[(2, 2, 0, 0), (3, 1, 0, -2), (4, 0, 0, 3)])
    assert np.array_equal(out[0].cpu().numpy(), d["list_teuk"])
    assert close(out[1].cpu().numpy(), d["list_ylms"])
    with pytest.raises(ValueError):
        sel(t, 0.5, None, None, None, 0.4, 2.0, mode_selection=[(2, 3, 0, 0)])
    with pytest.raises(ValueError):
        sel(t, 0.5, None, None, None, 0.4, 2.0, mode_selection="some")
