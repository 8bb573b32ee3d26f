"""Radau with the finite-difference Jacobian (generic/fd_jacob.c semantics) on the
GPU against the oracle's restatement, which tests/test_fd_jacobian.py pins to the
reference's own fd_jacob.c.  Same parity criterion as the analytic runs."""
import numpy as np
import pytest

import accelerint_b200 as A
from tests.helpers import check_parity, perturbed

pytestmark = pytest.mark.gpu


def _run_fd(mech, y, var, t0, t1, dt, lu=A.LU_FP64):
    integ = A.Integrator(y.shape[1], mech, lu=lu)
    try:
        integ.set_jacobian(True)
        return integ.integrate(t0, t1, dt, y, var)
    finally:
        integ.close()


@pytest.mark.parametrize("which", ["vdp", "ma14", "ma54"])
def test_fd_jacobian_radau_matches_oracle(oracle, which):
    if which == "vdp":
        mech = A.VanDerPol()
        y, var = A.vdp_initial_conditions(512, seed=61)
        t1, dt = 0.1, 0.01
    elif which == "ma14":
        mech = A.mechanism_13()
        y, var = A.mass_action_initial_conditions(mech, 64, seed=62)
        t1, dt = 2e-6, 1e-6
    else:
        mech = A.mechanism_53()
        y, var = A.mixed_stiffness_initial_conditions(mech, 16, seed=63)
        t1, dt = 1e-6, 1e-6
    yg, cg, _ = _run_fd(mech, y, var, 0.0, t1, dt)
    yo, co, _ = oracle.run("radau2a", mech, y, var, 0.0, t1, dt, fd_jacobian=True)
    yp, cp, _ = oracle.run("radau2a", mech, perturbed(y), var, 0.0, t1, dt, fd_jacobian=True)
    assert (cg == co).all()
    ok = (cg == 0) & (co == 0) & (cp == 0)
    check_parity(yg[:, ok], yo[:, ok], yp[:, ok], slack=max(0.1, 1.0 / ok.sum() + 1e-9))


def test_fd_jacobian_needs_fp64_radau():
    mech = A.mechanism_13()
    y, var = A.mass_action_initial_conditions(mech, 8, seed=64)
    with pytest.raises(RuntimeError):
        _run_fd(mech, y, var, 0.0, 1e-6, 1e-6, lu=A.LU_FP32)
