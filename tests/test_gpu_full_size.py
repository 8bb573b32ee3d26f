"""Size-independent properties at the bench's batch size (65,536 systems of the
53-species mixed-stiffness workload), where the oracle would take hours:

* every system finishes (code 0) with a finite state;
* mass conservation: the synthetic mechanism conserves mass, so sum_k Y_k = 1
  holds for the exact solution; Runge-Kutta methods preserve linear invariants,
  so the FP64 solver keeps it to roundoff (measured 2.2e-15); with FP32 factors
  the Newton iterates stop at their tolerance and the sum drifts within rtol
  (measured max 1.0e-7, median 1.9e-9);
* composition: one call over two global steps equals two consecutive one-step
  calls bit for bit (each global step restarts the integrator).
"""
import numpy as np
import pytest

import accelerint_b200 as A

pytestmark = pytest.mark.gpu

NUM = 65536


def _run(mech, y, var, lu, spans):
    import torch
    integ = A.Integrator(NUM, mech, lu=lu)
    try:
        yd = torch.from_numpy(y).cuda()
        vd = torch.from_numpy(var).cuda()
        cd = torch.zeros(NUM, dtype=torch.int32, device="cuda")
        for (t0, t1, dt) in spans:
            integ.integrate_device(t0, t1, dt, yd, vd, cd)
        torch.cuda.synchronize()
        return yd.cpu().numpy(), cd.cpu().numpy()
    finally:
        integ.close()


@pytest.fixture(scope="module")
def workload():
    mech = A.mechanism_53()
    y, var = A.mixed_stiffness_initial_conditions(mech, NUM, 2024)
    return mech, y, var


@pytest.mark.parametrize("lu,bound,median_bound", [(A.LU_FP64, 1e-12, 1e-14), (A.LU_FP32_ALL, 1e-6, 1e-8)])
def test_full_batch_finishes_and_conserves_mass(workload, lu, bound, median_bound):
    mech, y, var = workload
    yg, cg = _run(mech, y, var, lu, [(0.0, 1e-6, 1e-6)])
    assert (cg == 0).all()
    assert np.isfinite(yg).all()
    drift = np.abs(yg[1:].sum(axis=0) - 1.0)
    print(f"\nLU mode {lu}: max |sum Y - 1| = {drift.max():.3e}, median {np.median(drift):.3e}")
    assert drift.max() < bound
    assert np.median(drift) < median_bound


def test_full_batch_composition(workload):
    mech, y, var = workload
    y_one, _ = _run(mech, y, var, A.LU_FP32_ALL, [(0.0, 2e-6, 1e-6)])
    y_two, _ = _run(mech, y, var, A.LU_FP32_ALL, [(0.0, 1e-6, 1e-6), (1e-6, 2e-6, 1e-6)])
    assert np.array_equal(y_one, y_two)
