"""Host-side logic, no GPU: the C ABI's planners, the output-length contract,
the synthetic workloads and the cubic -> 8-term phase basis map."""
import numpy as np
import pytest

from fastemriwaveforms_b200 import _lib
from fastemriwaveforms_b200 import synthetic as S


def fold_plan_host(m, k, n, max_rows=256):
    m, k, n = (np.ascontiguousarray(a, dtype=np.int32) for a in (m, k, n))
    K = len(m)
    nmax = int(np.abs(n).max())
    max_keys = max_rows * (2 * nmax + 1)
    row_m = np.zeros(max_rows, np.int32)
    row_k = np.zeros(max_rows, np.int32)
    dims = np.zeros(3, np.int32)
    key_ptr = np.zeros(max_keys + 1, np.int32)
    key_list = np.zeros(2 * K, np.int32)
    _lib.call("few_fold_plan", m.ctypes.data, k.ctypes.data, n.ctypes.data, K, max_rows, max_keys,
              row_m.ctypes.data, row_k.ctypes.data, dims.ctypes.data, key_ptr.ctypes.data, key_list.ctypes.data)
    R, nlo, NN = dims.tolist()
    return row_m[:R], row_k[:R], nlo, NN, key_ptr[: R * NN + 1], key_list


def test_fold_plan_covers_every_term_once():
    l, m, k, n = S.mode_list(10, 30)
    row_m, row_k, nlo, NN, key_ptr, key_list = fold_plan_host(m, k, n)
    assert len(row_m) == 21 and nlo == -30 and NN == 61
    assert list(row_m) == list(range(-10, 11)) and not row_k.any()
    nterms = len(m) + int(np.count_nonzero(m))
    assert key_ptr[-1] == nterms
    codes = key_list[:nterms]
    assert len(np.unique(codes)) == nterms
    # every contributor sits under the key of its phase
    for q in range(len(row_m) * NN):
        r, c = divmod(q, NN)
        for code in codes[key_ptr[q]:key_ptr[q + 1]]:
            j, minus = divmod(int(code), 2)
            sgn = -1 if minus else 1
            assert (sgn * m[j], sgn * k[j], sgn * n[j]) == (row_m[r], row_k[r], nlo + c)


def test_fold_plan_sparse_modes_with_theta():
    m = np.array([2, 3, 4, 0, 2])
    k = np.array([0, 1, 1, 1, 0])
    n = np.array([-4, 3, 0, 2, -4])
    row_m, row_k, nlo, NN, key_ptr, key_list = fold_plan_host(m, k, n)
    assert sorted(zip(row_m.tolist(), row_k.tolist())) == list(zip(row_m.tolist(), row_k.tolist()))
    assert (0, 1) in zip(row_m.tolist(), row_k.tolist())
    assert nlo == -4 and NN == 9
    assert key_ptr[-1] == 5 + 4
    # modes 0 and 4 share the key (2, 0, -4): listed in mode order
    q = list(zip(row_m.tolist(), row_k.tolist())).index((2, 0)) * NN + (-4 - nlo)
    assert key_list[key_ptr[q]:key_ptr[q + 1]].tolist() == [0, 8]


def test_fold_plan_limits():
    m = np.arange(0, 300) % 300
    with pytest.raises(ValueError):
        fold_plan_host(m, np.zeros(300), np.zeros(300), max_rows=256)


def segment_plan_host(h_t, phase_t, out_len, dt, chunk):
    h_t = np.ascontiguousarray(h_t, np.float64)
    phase_t = np.ascontiguousarray(phase_t, np.float64)
    N = len(h_t)
    max_units = N + out_len // chunk + 1
    seg_start = np.zeros(N, np.int32)
    seg_info = np.zeros(3 * (N - 1))
    units = np.zeros(3 * max_units, np.int32)
    counts = np.zeros(2, np.int32)
    _lib.call("few_segment_plan", h_t.ctypes.data, phase_t.ctypes.data, N, out_len, dt, chunk, max_units,
              seg_start.ctypes.data, seg_info.ctypes.data, units.ctypes.data, counts.ctypes.data)
    nseg, nu = counts.tolist()
    return seg_start[: nseg + 1], seg_info[: 3 * nseg].reshape(-1, 3), units[: 3 * nu].reshape(-1, 3)


def test_segment_plan_matches_find_start_inds(oracle):
    inp = S.plain_small()
    out_len = inp.out_len
    start, info, units = segment_plan_host(inp.t, inp.phase_t, out_len, inp.dt, 1024)
    ostart, nseg = oracle.find_start_inds(inp.t, inp.dt, out_len)
    assert start.tolist() == ostart.tolist()
    # units tile [0, out_len) exactly, in order, within their segments, <= chunk long
    assert units[0, 1] == 0 and units[-1, 2] == out_len
    assert (units[1:, 1] == units[:-1, 2]).all()
    assert ((units[:, 2] - units[:, 1]) <= 1024).all()
    assert (units[:, 1] >= start[units[:, 0]]).all() and (units[:, 2] <= start[units[:, 0] + 1]).all()
    np.testing.assert_array_equal(info[:, 0], inp.t[:nseg])
    np.testing.assert_array_equal(info[:, 2], np.diff(inp.phase_t)[:nseg])


def test_segment_plan_truncated_and_errors():
    t = np.array([0.0, 15.0, 30.0, 45.5, 70.0])
    start, info, units = segment_plan_host(t, t, 6, 10.0, 4)
    assert start.tolist() == [0, 2, 3, 5, 6]
    assert units.tolist() == [[0, 0, 2], [1, 2, 3], [2, 3, 5], [3, 5, 6]]
    with pytest.raises(ValueError):  # knots never reach the last sample
        segment_plan_host(t, t, 20, 10.0, 4)
    with pytest.raises(ValueError):  # not increasing
        segment_plan_host(np.array([0.0, 20.0, 10.0, 70.0]), t[:4], 6, 10.0, 4)


def test_output_length_contract():
    t = np.array([0.0, 1e3, 1e6])
    # T beyond the trajectory: output ends at the last knot
    assert S.output_length(t, 2e6 / S.YRSID_SI, 10.0) == (100001, 0)
    assert S.output_length(t, 2e6 / S.YRSID_SI, 10.0, pad_output=True)[1] > 0
    # T inside the trajectory
    n, pad = S.output_length(t, 5e5 / S.YRSID_SI, 10.0)
    assert pad == 0 and n in (50000, 50001)
    n, pad = S.output_length(t, 2e6 / S.YRSID_SI, 10.0, odd_len=True)
    assert (n + pad) % 2 == 1


def test_synthetic_workloads():
    a = S.plain_small()
    assert a.num_modes == 200 and a.num_knots == 100 and a.out_len == 100001
    assert np.diff(a.t).min() >= 1e3 - 1e-6
    l, m, k, n = S.mode_list(10, 30)
    assert len(l) == 3843
    inp = S.make_inputs(K=300, N=60, span=3e6, t_c=3.2e6, lmax=10, nmax=30, seed=3)
    assert inp.phase_coeffs.shape == (59, 3, 8) and not inp.phase_coeffs[:, 1].any()


def test_cubic_to_basis_reproduces_cubic():
    rng = np.random.default_rng(0)
    y0, c1, c2, c3 = rng.standard_normal(4)
    h = 3.7
    b = S.cubic_to_basis(y0, c1, c2, c3, h)
    for x in np.linspace(0, h, 7):
        s = x / h
        s1 = 1 - s
        v = b[0] + s * (b[1] + s1 * (b[2] + s * (b[3] + s1 * (b[4] + s * (b[5] + s1 * (b[6] + s * b[7]))))))
        assert abs(v - (y0 + c1 * x + c2 * x * x + c3 * x ** 3)) < 1e-12


def test_mismatch_known_answer():
    # tests/test_few.py:232-245 of the reference
    from fastemriwaveforms_b200 import get_mismatch, get_overlap

    t = np.arange(10000) * 1.0
    x0 = np.sin(t) + 1j * np.sin(t)
    x2 = np.sin(t) + 1j * np.cos(t)
    assert abs(get_overlap(x0, x0) - 1.0) < 1e-12
    assert abs(get_overlap(x0, x2) - 0.499981442642142) < 1e-7
    assert abs(get_mismatch(x0, x0)) < 1e-12


def test_fd_dense_grid_is_numpy_linspace():
    """The turnover search rebuilds numpy.linspace's points on the device from
    (start, step, stop): y_j = j*step + start, the last point = stop."""
    from fastemriwaveforms_b200.fdinterp import DENSE_POINTS, _linspace_params

    rng = np.random.default_rng(3)
    for _ in range(20):
        t = np.sort(rng.uniform(0, rng.uniform(1e4, 1e8), 40))
        t0, step, t1 = _linspace_params(t.min(), t.max(), DENSE_POINTS)
        mine = np.arange(DENSE_POINTS) * step + t0
        mine[-1] = t1
        assert np.array_equal(mine, np.linspace(t.min(), t.max(), DENSE_POINTS))


def test_mode_selector_list_checks():
    """ModeSelector's list checks and messages (the reference's
    modeselector.py:144-171): bad strings, empty lists, duplicates, |m| > l,
    l < 2; a negative m in the constructor's list only warns and sets the flag
    that makes a later include_minus_mkn call fail."""
    from fastemriwaveforms_b200 import ModeSelector

    gen = S.FixedAmplitudes()
    for bad, text in (("some", "must be either 'all', 'threshold', or None"),
                      ([], "cannot be empty"),
                      ([(2, 2, 0, 0), (2, 2, 0, 0)], "duplicate modes"),
                      ([(2, 3, 0, 0)], "|m| > l"),
                      ([(1, 0, 0, 0)], "l < 2")):
        with pytest.raises(ValueError) as err:
            ModeSelector(gen, mode_selection=bad, device="cpu")
        assert text in str(err.value), (bad, str(err.value))
    sel = ModeSelector(gen, mode_selection=[(2, -2, 0, 0)], device="cpu")
    assert sel.negative_m_flag
    with pytest.raises(ValueError, match="m >= 0 when include_minus_mkn = True"):
        sel(np.zeros(4), 0.5, None, None, None, 1.0, 0.5)


def test_autotune_shape_search_and_cache(tmp_path, monkeypatch):
    """The tuner's shape lists (the tensor-core sum's operand pipeline included)
    and its JSON cache: the fastest candidate is kept with every timing."""
    from fastemriwaveforms_b200 import autotune

    mixed = autotune.candidates_for("mixed")
    assert {(c["astages"], c["bstages"]) for c in mixed} == {(a, b) for a in (1, 2) for b in (2, 3, 4)}
    assert all(set(c) == {"chunk", "ctas_per_sm", "astages", "bstages"} for c in mixed)
    fp64 = autotune.candidates_for("exact")
    assert len(fp64) == len(autotune.CHUNKS) * len(autotune.CTAS_PER_SM)
    assert all(set(c) == {"chunk", "ctas_per_sm"} for c in fp64)

    monkeypatch.setenv("FEW_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    monkeypatch.setattr(autotune, "time_ms", lambda fn, reps=3: fn())
    cost = {1: 3.0, 2: 1.0, 3: 2.0}
    choice = autotune.tune("k", lambda chunk, ctas_per_sm: (lambda: cost[ctas_per_sm] + chunk * 1e-6), fp64)
    assert choice["ctas_per_sm"] == 2 and choice["chunk"] == min(autotune.CHUNKS)
    assert len(choice["tried"]) == len(fp64)
    assert autotune.lookup("k")["ctas_per_sm"] == 2


def test_balanced_work_units_tile_every_segment():
    """The joint adjoint's work units: each segment's samples cut into
    ceil(len / 1024) parts whose lengths differ by at most one, covering the
    segment exactly once and in order; segments without samples get none."""
    from fastemriwaveforms_b200.summation import _SegmentPlan

    class Plan:
        _device = "cpu"

    rng = np.random.default_rng(3)
    lens = np.concatenate([[0, 1, 1023, 1024, 1025, 3150], rng.integers(0, 5000, 40)])
    plan = Plan()
    plan.seg_start = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    plan.nseg = len(lens)
    units, seg_units, total = _SegmentPlan.balanced_units(plan)
    units = units.numpy().reshape(-1, 3)
    seg_units = seg_units.numpy()
    assert total == len(units) == seg_units[-1]
    for s, n in enumerate(lens):
        part = units[seg_units[s]: seg_units[s + 1]]
        assert len(part) == -(-int(n) // 1024)
        assert (part[:, 0] == s).all()
        if len(part):
            assert part[0, 1] == plan.seg_start[s] and part[-1, 2] == plan.seg_start[s + 1]
            assert (part[1:, 1] == part[:-1, 2]).all()
            sizes = part[:, 2] - part[:, 1]
            assert sizes.max() - sizes.min() <= 1 and sizes.max() <= 1024 and sizes.min() >= 1
