"""Generates tests/golden/dopr853_dense.npz from the reference's own DOPR853
(src/few/trajectory/dopr853.py, imported from the reference sources; it needs
only numpy).

    python tests/golden/make_dopr853_golden.py

The reference stepper integrates ``synthetic.toy_inspiral_ode`` (an 8-component
inspiral-like system whose right-hand side uses only +, -, *, / and sqrt) from
t = 0 to 5e5 s the way the reference's trajectory drives it
(src/few/trajectory/integrate.py:283-337: take_step_single, then
prep_evaluate_single after every accepted step).  For each accepted step the
file keeps the step's end points, its size, the ten stage slots take_step left
behind (copied before prep_evaluate overwrites three of them) and the 8-term
dense-output basis prep_evaluate returned.  It also keeps DOPR853.eval and
eval_derivative (orders 1-3) of that basis at 400 random times plus the knots'
end points.
"""
import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from fastemriwaveforms_b200 import synthetic as S  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = os.path.join(HERE, "dopr853_dense.npz")
Y0 = np.array([12.0, 0.4, 0.7, 0.0, 0.0, 0.0, 1.0, 0.0])
T_END = 5e5
H0 = 10.0


def reference_module():
    path = os.path.join(O.REFERENCE_ROOT, "src", "few", "trajectory", "dopr853.py")
    spec = importlib.util.spec_from_file_location("reference_dopr853", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def main():
    ref = reference_module()
    dopr = ref.DOPR853(S.toy_inspiral_ode(np))
    t, h, y = 0.0, H0, Y0.copy()
    x0s, h0s, x1s, y0s, y1s, stages, rconts = [], [], [], [], [], [], []
    while t < T_END:
        t_old, h_old, y_old = t, h, y.copy()
        ok, t, h = dopr.take_step_single(t_old, h_old, y, None)
        if not ok:
            continue
        st = np.stack([k[:, 0].copy() for k in dopr.k_coefficient_storage])  # (10, node)
        rc = dopr.prep_evaluate_single(t_old, y_old, h_old, t, y, None)      # (node, 8)
        x0s.append(t_old)
        h0s.append(h_old)
        x1s.append(t)
        y0s.append(y_old)
        y1s.append(y.copy())
        stages.append(st)
        rconts.append(rc)
    t_knots = np.array(x0s + [x1s[-1]])
    coeffs = np.stack(rconts)                                               # (nsteps, node, 8)
    rng = np.random.default_rng(3)
    t_new = np.concatenate([[t_knots[0], t_knots[-1]], t_knots[1:-1:37],
                            np.sort(rng.uniform(t_knots[0], t_knots[-1], 400))])
    evals = [dopr.eval(t_new, t_knots, coeffs)]
    for order in (1, 2, 3):
        evals.append(dopr.eval_derivative(t_new, t_knots, coeffs, order=order))
    np.savez_compressed(OUT, x0=np.array(x0s), h0=np.array(h0s), x1=np.array(x1s), y0=np.stack(y0s),
                        y1=np.stack(y1s), stages=np.stack(stages), rcont=coeffs, t_knots=t_knots, t_new=t_new,
                        evals=np.stack(evals), abstol=dopr.abstol)
    print(f"wrote {OUT}: {len(x0s)} steps, {len(t_new)} evaluation times")


if __name__ == "__main__":
    main()
