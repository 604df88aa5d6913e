"""DirectModeSum on the GPU against the reference's own DirectModeSum (golden
vectors, tests/golden/make_fd_golden.py) and the reference test's dummy case
(tests/test_mode_summation.py:152-200): relative L2 <= 1e-12 (the sums over
modes are ordered differently; phases reach ~1e6 rad)."""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from fastemriwaveforms_b200 import DirectModeSum
from fastemriwaveforms_b200 import synthetic as S

pytestmark = pytest.mark.gpu


def test_direct_sum_matches_reference(cuda):
    d = np.load(os.path.join(GOLDEN, "direct_sum.npz"))
    t, teuk, ylms, phases, l, m, k, n = S.direct_case()
    got = DirectModeSum()(t, teuk, ylms, t, phases, l, m, k, n).cpu().numpy()
    assert got.shape == d["waveform"].shape
    e = float(np.linalg.norm(got - d["waveform"]) / np.linalg.norm(d["waveform"]))
    print(f"\nDirectModeSum vs reference: rel L2 {e:.2e}")
    assert e <= 1e-12


def test_direct_sum_reference_test_case(cuda):
    rng = np.random.default_rng(3)
    t = np.linspace(0, 1000, 10001)
    K = 10
    amp = np.linspace(rng.uniform(-1, 1, (2, K)), rng.uniform(-1, 1, (2, K)), t.size, axis=-1)
    a = (amp[0] + 1j * amp[1]).T
    phases = np.asarray([np.pi / 3 + 1e-2 * t, np.pi / 6 + 2e-2 * t, np.pi / 4 + 3e-3 * t])
    l = np.ones(K) * 2
    m = rng.integers(2, 5, K)
    k = rng.integers(0, 2, K)
    n = rng.integers(-3, 3, K)
    ylms = np.ones(2 * K)
    ylms[K:] = 0
    manual = (a * np.exp(-1j * (phases[0][:, None] * m + phases[1][:, None] * k + phases[2][:, None] * n))).sum(-1)
    got = DirectModeSum()(t, a, ylms, t, phases, l, m, k, n).cpu().numpy()
    np.testing.assert_allclose(got, manual, rtol=1e-10, atol=1e-12)
