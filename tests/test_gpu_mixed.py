"""The mixed-precision (tcgen05, split-BF16) sum against the FP64 sum:
waveform mismatch (1 - overlap, src/few/utils/utility.py:16-95) <= 1e-8 and
relative L2 error <= 1e-4; the max relative error is printed."""
import numpy as np
import pytest
import torch

from conftest import load_case
from fastemriwaveforms_b200 import InterpolatedModeSum, get_mismatch
from fastemriwaveforms_b200 import synthetic as S

pytestmark = pytest.mark.gpu

MISMATCH_MAX = 1e-8
REL_L2_MAX = 1e-4


def run(inp, precision):
    ims = InterpolatedModeSum(precision=precision)
    wf = ims(*inp.call_args(), T=inp.T, dt=inp.dt)
    torch.cuda.synchronize()
    if precision == "mixed":
        assert not ims.mixed_error(), "a tensor-core wait timed out"
    return wf.cpu().numpy()


@pytest.mark.parametrize("case", ["theta", "m0", "plain_small", "plain_full", "many_rows", "wide_n"])
def test_mixed_matches_fp64(cuda, case):
    if case == "theta":
        inp, _ = load_case("sum_small_theta.npz")
    elif case == "m0":
        inp, _ = load_case("sum_small_m0.npz")
    elif case == "plain_small":
        inp = S.plain_small()
    elif case == "many_rows":
        inp = S.many_rows_case()  # 63 (m', k') rows: two MMA column groups
    elif case == "wide_n":
        inp = S.many_rows_case(mmax=2, kmax=0, nmax=60, seed=13)  # NN = 121: eight K chunks
    else:
        inp = S.plain_full()
    ref = run(inp, "exact")
    got = run(inp, "mixed")
    mm = get_mismatch(got, ref)
    rel = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    maxrel = float(np.abs(got - ref).max() / np.abs(ref).max())
    print(f"{case}: mismatch {mm:.3e}, relative L2 {rel:.3e}, max |dh| / max |h| {maxrel:.3e}")
    assert mm <= MISMATCH_MAX
    assert rel <= REL_L2_MAX


def test_mixed_deterministic(cuda):
    inp = S.plain_small()
    a = run(inp, "mixed")
    b = run(inp, "mixed")
    assert np.array_equal(a, b)


def test_mixed_row_limit(cuda):
    """More than 64 (m', k') rows: the mixed form refuses (the FP64 forms do not)."""
    inp = S.many_rows_case(mmax=12)  # 75 rows
    with pytest.raises(ValueError):
        run(inp, "mixed")
    assert np.isfinite(run(inp, "exact")).all()
