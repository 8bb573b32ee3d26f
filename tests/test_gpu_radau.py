"""GPU parity of the Radau IIA kernels against the oracle (C restatement of
radau2a/radau2a.c), through the C-ABI (accelerInt_integrate_status)."""
import numpy as np
import pytest

from accelerint_b200 import (LU_FP32, LU_FP32_ALL, LU_FP64, Integrator, VanDerPol, mechanism_13, mechanism_53,
                             mass_action_initial_conditions, mixed_stiffness_initial_conditions,
                             vdp_initial_conditions)
from tests.helpers import check_parity, per_system_error, perturbed, weighted_error

pytestmark = pytest.mark.gpu


def run_gpu(mech, y, var, t0, t1, dt, solver="radau2a", lu=LU_FP64):
    integ = Integrator(y.shape[1], mech, solver=solver, lu=lu)
    try:
        yo, codes, rc = integ.integrate(t0, t1, dt, y, var)
    finally:
        integ.close()
    return yo, codes


@pytest.mark.parametrize("lu", [LU_FP64, LU_FP32])
def test_van_der_pol(oracle, lu):
    y, var = vdp_initial_conditions(4096, seed=3)
    yg, cg = run_gpu(VanDerPol(), y, var, 0.0, 0.1, 1e-2, lu=lu)
    yo, co, _ = oracle.run("radau2a", VanDerPol(), y, var, 0.0, 0.1, 1e-2)
    assert (co == 0).all() and (cg == 0).all()
    if lu == LU_FP64:
        # same step sequence as the CPU reference: agreement far inside rtol 1e-6
        assert weighted_error(yg, yo) < 1.0
    else:
        # FP32 factors change Newton convergence, hence step sizes; accuracy against
        # a tight oracle must stay that of the FP64 solver
        yt, _, _ = oracle.run("radau2a", VanDerPol(), y, var, 0.0, 0.1, 1e-2, rtol=1e-12, atol=1e-20)
        eg, eo = per_system_error(yg, yt), per_system_error(yo, yt)
        print(f"\nvan der Pol lu={lu}: weighted error vs tight median {np.median(eg):.3g} (oracle {np.median(eo):.3g}), "
              f"max {eg.max():.3g} ({eo.max():.3g})")
        # slack of 0.1: a weighted error below 0.1 is a tenth of the tolerance
        assert np.median(eg) <= 2.0 * np.median(eo) + 0.1
        assert eg.max() <= 3.0 * eo.max() + 0.1


def check_mass_action(yg, yo, yp, yt, lu):
    """FP64: agreement with the reference CPU solver within its own perturbation envelope.
    Single-precision factorisations change Newton convergence, hence the step sequence;
    they must then be as accurate as the FP64 reference against the tight oracle."""
    if lu == LU_FP64:
        check_parity(yg, yo, yp)
    eg, eo = per_system_error(yg, yt), per_system_error(yo, yt)
    assert not np.isnan(yg).any()
    print(f"\nmass action lu={lu}: weighted error vs tight median {np.median(eg):.3g} (oracle {np.median(eo):.3g}), "
          f"max {eg.max():.3g} ({eo.max():.3g})")
    assert np.median(eg) <= 1.5 * np.median(eo) + 0.1
    assert eg.max() <= 2.0 * eo.max() + 0.1


@pytest.mark.parametrize("lu", [LU_FP64, LU_FP32, LU_FP32_ALL])
def test_mass_action_14(oracle, lu):
    mech = mechanism_13()
    y, var = mass_action_initial_conditions(mech, 256, seed=11)
    yg, cg = run_gpu(mech, y, var, 0.0, 5e-6, 1e-6, lu=lu)
    yo, co, _ = oracle.run("radau2a", mech, y, var, 0.0, 5e-6, 1e-6)
    yp, _, _ = oracle.run("radau2a", mech, perturbed(y), var, 0.0, 5e-6, 1e-6)
    yt, _, _ = oracle.run("radau2a", mech, y, var, 0.0, 5e-6, 1e-6, rtol=1e-12, atol=1e-20)
    assert (co == 0).all() and (cg == 0).all()
    check_mass_action(yg, yo, yp, yt, lu)


@pytest.mark.parametrize("lu", [LU_FP64, LU_FP32, LU_FP32_ALL])
def test_mass_action_54(oracle, lu):
    mech = mechanism_53()
    y, var = mixed_stiffness_initial_conditions(mech, 64, seed=5)
    yg, cg = run_gpu(mech, y, var, 0.0, 2e-6, 1e-6, lu=lu)
    yo, co, _ = oracle.run("radau2a", mech, y, var, 0.0, 2e-6, 1e-6)
    yp, _, _ = oracle.run("radau2a", mech, perturbed(y), var, 0.0, 2e-6, 1e-6)
    yt, _, _ = oracle.run("radau2a", mech, y, var, 0.0, 2e-6, 1e-6, rtol=1e-12, atol=1e-20)
    assert (co == 0).all() and (cg == 0).all()
    check_mass_action(yg, yo, yp, yt, lu)
