"""The oracle pinned against the reference: golden vectors made by the
reference's own CPU build, scipy's CubicSpline (the reference's spline test,
tests/test_mode_summation.py:23-52) and, where the reference sources are
present, the reference build itself."""
import os

import numpy as np
import pytest
from scipy.interpolate import CubicSpline

from conftest import GOLDEN, load_case
from fastemriwaveforms_b200 import synthetic as S


def test_spline_matches_golden_bitwise(oracle):
    d = np.load(os.path.join(GOLDEN, "spline_cos_sin.npz"))
    got = oracle.interpolate_arrays(d["t"], d["y"])
    assert np.array_equal(got, d["coeffs"])
    d = np.load(os.path.join(GOLDEN, "spline_rows2d.npz"))
    got = oracle.interpolate_arrays(d["t"], d["y"])
    assert np.array_equal(got, d["coeffs"])


def test_spline_matches_scipy_like_reference_test(oracle):
    # tests/test_mode_summation.py:23-52 with its rtol 1e-10
    t = np.linspace(0, 100, 1000)
    f = np.vstack((np.cos(t), np.sin(t)))
    coeffs = oracle.spline_coeffs(t, f)
    cs = CubicSpline(t, f, axis=-1)
    np.testing.assert_allclose(oracle.spline_eval(t, coeffs, t), f, rtol=1e-10)
    for nu in range(1, 4):
        np.testing.assert_allclose(oracle.spline_eval(t, coeffs, t, nu), cs(t, nu=nu), rtol=1e-10)
    te = np.linspace(0, 100, 1852)
    for nu in range(4):
        np.testing.assert_allclose(oracle.spline_eval(t, coeffs, te, nu), cs(te, nu=nu), rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("name", ["sum_small_theta.npz", "sum_small_m0.npz", "sum_small_truncated.npz"])
def test_mode_sum_matches_golden_bitwise(oracle, name):
    inp, ref = load_case(name)
    got = oracle.mode_sum(inp)
    assert got.shape == ref.shape
    assert np.array_equal(got, ref)


def test_extended_oracle_within_reference_rounding(oracle):
    inp, ref = load_case("sum_small_theta.npz")
    ext = oracle.mode_sum(inp, extended=True)
    # the reference rounds each mode phase; at |phase| ~ 1e2 rad that is ~1e-14
    assert oracle.rel_l2(ext, ref) < 1e-12


def test_plain_small_inputs_and_reference_values(oracle):
    d = np.load(os.path.join(GOLDEN, "plain_small_ref.npz"))
    inp = S.plain_small(int(d["seed"]))
    from golden.make_golden import inputs_digest

    assert inputs_digest(inp) == str(d["digest"]), "synthetic generator drifted from the golden inputs"
    idx = d["idx"]
    wf = oracle.mode_sum(inp, window=(0, int(idx.max()) + 1))
    assert np.array_equal(wf[idx], d["values"])


def test_window_is_a_restriction(oracle):
    inp, ref = load_case("sum_small_m0.npz")
    part = oracle.mode_sum(inp, window=(1000, 2500))
    assert np.array_equal(part[1000:2500], ref[1000:2500])
    assert not part[:1000].any() and not part[2500:].any()


def test_find_start_inds_semantics(oracle):
    t = np.array([0.0, 15.0, 30.0, 45.5, 70.0])
    start, nseg = oracle.find_start_inds(t, 10.0, 6)  # T = 50: knot 70 closes the plan
    assert nseg == 4
    assert start.tolist() == [0, 2, 3, 5, 6]
    with pytest.raises(ValueError):
        oracle.find_start_inds(t, 10.0, 20)  # no knot reaches T = 190


@pytest.mark.skipif(not os.path.isfile(os.path.join(os.path.dirname(GOLDEN), "..", "oracle", "_ref", "libfew_ref.so")),
                    reason="reference build absent (sources not on this machine)")
def test_restatement_equals_reference_build(oracle):
    inp = S.small_case(K=25, N=30, out_len=7000, seed=11)
    assert np.array_equal(oracle.mode_sum(inp), oracle.mode_sum(inp, impl="ref"))
    t = np.sort(np.random.default_rng(3).uniform(0, 10, 64))
    y = np.random.default_rng(4).standard_normal((7, 64))
    assert np.array_equal(oracle.interpolate_arrays(t, y), oracle.interpolate_arrays(t, y, impl="ref"))


def test_interp2d_oracle_matches_reference_golden_and_scipy(oracle):
    """The restated FITPACK evaluation (interp2D, AmpInterp2D.cu) equals the
    reference's own output bit for bit, and scipy's bisplev (the same FITPACK
    routine) on clamped points."""
    from scipy.interpolate import bisplev

    d = np.load(os.path.join(GOLDEN, "amp_interp2d.npz"))
    for tag, kx, ky in (("k33", 3, 3), ("k15", 1, 5)):
        tx, ty, c, x, y = (d[f"{tag}_{q}"] for q in ("tx", "ty", "c", "x", "y"))
        z = oracle.interp2d(tx, ty, c, kx, ky, x, y)
        assert np.array_equal(z, d[f"{tag}_z"]), tag
        xs = np.clip(x, tx[kx], tx[len(tx) - kx - 1])
        ys = np.clip(y, ty[ky], ty[len(ty) - ky - 1])
        zs = np.array([[bisplev(a, b, (tx, ty, cg, kx, ky)) for a, b in zip(xs, ys)] for cg in c])
        assert np.abs(z - zs).max() <= 1e-14 * np.abs(zs).max(), tag


FD_CASES = {
    "fd_schwarzschild": dict(),
    "fd_single_turnover": dict(),
    "fd_kerr_farr": dict(f_arr=True),
    "fd_generic_pos": dict(include_minus_m=False, mask_positive=True),
}


@pytest.mark.parametrize("name", sorted(FD_CASES))
def test_fd_oracle_matches_reference_golden(oracle, name):
    """The FD restatement (numpy bin plan + few_oracle.c stationary-phase
    kernel) against the reference's own FD sum (golden vectors from
    tests/golden/make_fd_golden.py): the plan bit for bit, the waveform to the
    last places (the SPA series coefficients are generated by recurrence here;
    the reference writes them as decimals)."""
    opts = FD_CASES[name]
    d = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    inp = S.ModeSumInputs(t=d["t"], teuk_modes=d["teuk_modes"], ylms=d["ylms"], phase_t=d["phase_t"],
                          phase_coeffs=d["phase_coeffs"], l=d["l"], m=d["m"], k=d["k"], n=d["n"], dt=float(d["dt"]),
                          T=float(d["T"]))
    L = int(d["num_pts"]) + int(d["num_pts_pad"])
    kw = dict(L=L, f_arr=d["f_arr"] if opts.get("f_arr") else None,
              include_minus_m=opts.get("include_minus_m", True), mask_positive=opts.get("mask_positive", False))
    wf, freq, start, end = oracle.fd_sum(inp, d["fknots"], impl="oracle", **kw)
    assert np.array_equal(freq, d["frequency"])
    assert np.array_equal(start.reshape(-1), d["start_inds"]) and np.array_equal(end.reshape(-1), d["end_inds"])
    assert np.linalg.norm(wf - d["waveform"]) <= 1e-13 * np.linalg.norm(d["waveform"])
    raw = oracle.fd_kernel(d["interp_array"], d["phase_t"], d["phase_kernel"], d["m"], d["k"], d["n"], d["t"],
                           d["frequency"], d["start_inds"], d["end_inds"], d["ylms_signed"], int(d["zero_index"]),
                           kw["include_minus_m"])
    assert np.linalg.norm(raw - d["raw"]) <= 1e-13 * np.linalg.norm(d["raw"])
    if oracle.have_ref():  # the reference's kernel behind the restated plan reproduces the golden exactly
        wf_ref, *_ = oracle.fd_sum(inp, d["fknots"], impl="ref", **kw)
        assert np.array_equal(wf_ref, d["waveform"])


def test_aak_oracle_matches_reference_golden(oracle):
    """The AAK restatement (numpy, scipy's Bessel functions) against the
    reference's own AAK kernel (golden vectors from its CPU path): the
    difference is the reference's Numerical Recipes Bessel approximations
    (~1e-7 of the waveform); the reference build reproduces its golden file."""
    d = np.load(os.path.join(GOLDEN, "aak_ref.npz"))
    inp = S.aak_case(N=40, span=3e5)
    assert np.array_equal(inp.interp_coeffs, d["interp_coeffs"])
    L = int(d["L"])
    for mich in (0, 1):
        ref = d[f"wf_mich{mich}"]
        got = oracle.aak_waveform(inp.t, inp.interp_coeffs, inp.m1, inp.a, inp.m2, inp.qS, inp.phiS, inp.qK,
                                  inp.phiK, inp.dist, inp.nmodes, bool(mich), L, inp.dt)
        e = np.linalg.norm(got - ref) / np.linalg.norm(ref)
        assert e <= 3e-7, e
        if oracle.have_ref():
            again = oracle.aak_waveform(inp.t, inp.interp_coeffs, inp.m1, inp.a, inp.m2, inp.qS, inp.phiS, inp.qK,
                                        inp.phiK, inp.dist, inp.nmodes, bool(mich), L, inp.dt, impl="ref")
            assert np.array_equal(again, ref)


def test_direct_sum_oracle_matches_reference_golden(oracle):
    import hashlib

    d = np.load(os.path.join(GOLDEN, "direct_sum.npz"))
    t, teuk, ylms, phases, l, m, k, n = S.direct_case()
    h = hashlib.sha256()
    for a in (t, teuk, ylms, phases, l, m, k, n):
        h.update(np.ascontiguousarray(a).tobytes())
    assert h.hexdigest() == str(d["digest"])  # the inputs the golden output was made from
    got = oracle.direct_sum(teuk, ylms, phases, l, m, k, n)
    assert np.linalg.norm(got - d["waveform"]) <= 1e-13 * np.linalg.norm(d["waveform"])


def test_dopr853_dense_output_oracle_matches_reference_golden(oracle):
    """The numpy restatement of DOPR853.prep_evaluate, batched over all the
    steps at once, against the reference's own prep_evaluate_single run
    after each step (tests/golden/make_dopr853_golden.py): bit for bit."""
    d = np.load(os.path.join(GOLDEN, "dopr853_dense.npz"))
    stages = np.transpose(d["stages"], (1, 2, 0))  # (10, node, nsys)
    got = oracle.dopr853_prep_evaluate(d["x0"], d["y0"].T.copy(), d["h0"], d["x1"], d["y1"].T.copy(), stages,
                                       S.toy_inspiral_ode(np))
    assert np.array_equal(got, d["rcont"])


def test_adjoint_fd_fixture_inputs_are_reproduced():
    """The finite-difference fixture belongs to synthetic.adjoint_case's inputs."""
    import hashlib

    fx = np.load(os.path.join(GOLDEN, "adjoint_fd.npz"))
    inp = S.adjoint_case(seed=int(fx["input_seed"]))
    h = hashlib.sha256()
    for a in (inp.t, inp.teuk_modes, inp.ylms, inp.phase_knots, inp.phase_coeffs, inp.m, inp.n):
        h.update(np.ascontiguousarray(a).tobytes())
    assert h.hexdigest()[:32] == str(fx["digest"])
    assert len(fx["fd"]) == 64 and set(fx["family"].tolist()) == {0, 1, 2, 3}
