"""The tight FP64 oracle (the reference's Radau at rtol 1e-12, atol 1e-20) used by
the precision tests, cross-checked against an independent integrator:
scipy.integrate.solve_ivp (Radau and BDF at rtol 1e-12) on a small subsample,
with the oracle's own dydt / Jacobian as the right-hand side."""
import numpy as np
import pytest

import accelerint_b200 as A

scipy_integrate = pytest.importorskip("scipy.integrate")


def _solve(oracle, mech, y0, var, t1, method):
    f = lambda t, y: oracle.dydt(mech, y, var, t)
    jac = lambda t, y: oracle.jacob(mech, y, var, t)
    r = scipy_integrate.solve_ivp(f, (0.0, t1), y0, method=method, jac=jac, rtol=1e-12, atol=1e-20)
    assert r.success
    return r.y[:, -1]


@pytest.mark.parametrize("which", ["vdp", "ma14"])
def test_tight_oracle_agrees_with_scipy(oracle, which):
    if which == "vdp":
        mech = A.VanDerPol()
        y, var = A.vdp_initial_conditions(3, seed=81)
        t1 = 0.05
    else:
        mech = A.mechanism_13()
        y, var = A.mass_action_initial_conditions(mech, 2, seed=82)
        t1 = 2e-7
    yt, codes, _ = oracle.run("radau2a", mech, y, var, 0.0, t1, t1, rtol=1e-12, atol=1e-20)
    assert (codes == 0).all()
    for i in range(y.shape[1]):
        for method in ("Radau", "BDF"):
            ys = _solve(oracle, mech, y[:, i], var[i], t1, method)
            big = np.abs(ys) > 1e-12 * np.max(np.abs(ys))
            rel = np.max(np.abs(yt[big, i] - ys[big]) / np.abs(ys[big]))
            assert rel < 1e-7, (which, i, method, rel)
