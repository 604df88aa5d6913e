import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TESTS = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, TESTS):
    if _p not in sys.path:
        sys.path.insert(0, _p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA kernels")


@pytest.fixture(scope="session")
def oracle():
    """The CPU oracle (C restatement, plus the reference build when present)."""
    from oracle import oracle as O

    O.build(ref=None)
    return O


@pytest.fixture(scope="session")
def cuda():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch.device("cuda", 0)


GOLDEN = os.path.join(ROOT, "tests", "golden")


def load_case(name):
    """A golden mode-sum case as (ModeSumInputs, reference waveform)."""
    import numpy as np

    from fastemriwaveforms_b200.synthetic import ModeSumInputs

    d = np.load(os.path.join(GOLDEN, name))
    inp = ModeSumInputs(t=d["t"], teuk_modes=d["teuk_modes"], ylms=d["ylms"], phase_t=d["phase_t"],
                        phase_coeffs=d["phase_coeffs"], l=d["l"], m=d["m"], k=d["k"], n=d["n"],
                        dt=float(d["dt"]), T=float(d["T"]), name=name)
    return inp, d["waveform"]
