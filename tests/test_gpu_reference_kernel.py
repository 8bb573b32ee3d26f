"""The reference's own GPU Radau IIA (radau2a/radau2a.cu under generic/solver_generic.cu's
intDriver), compiled for sm_100a by oracle/build.py and driven by oracle.ReferenceGPU; the
bench times it beside the library.

* As shipped it fails every system: RK_ErrorEstimate (radau2a.cu:612) back-substitutes
  with the raw Jacobian as if it were the factored E1.  Van der Pol's Jacobian has a zero
  diagonal entry (df1/dy1 = 0), the error norm is infinite, the step-size controller sets
  H to zero and the integrator returns EC_h_plus_t_equals_h (3).
* With that line fixed (the build oracle/build.py makes with Q3_FIX) it integrates: its
  results agree with the oracle (the CPU algorithm) to within the spread the oracle
  itself shows under a 1e-15 perturbation of its inputs, which checks the harness and
  the mass-action callbacks written in the reference's INDEX() convention.
"""
import numpy as np
import pytest

import accelerint_b200 as A
from tests.helpers import check_parity, perturbed

pytestmark = pytest.mark.gpu


def _ref(n, fix):
    from oracle import ReferenceGPU, reference_gpu_available
    if not reference_gpu_available(n, q3_fix=fix):
        pytest.skip("reference GPU build missing (oracle/build.py needs the reference checkout)")
    return ReferenceGPU(n, q3_fix=fix)


def test_shipped_error_estimate_fails_van_der_pol():
    y, var = A.vdp_initial_conditions(64, seed=3)
    _, codes, _ = _ref(2, False).run(y, var, 0.0, 1e-2, 1e-2)
    assert (codes == 3).all(), np.bincount(codes)


def test_fixed_van_der_pol_matches_oracle(oracle):
    y, var = A.vdp_initial_conditions(256, seed=3)
    yg, cg, _ = _ref(2, True).run(y, var, 0.0, 0.1, 1e-2)
    yo, co, _ = oracle.run("radau2a", A.VanDerPol(), y, var, 0.0, 0.1, 1e-2)
    yp, _, _ = oracle.run("radau2a", A.VanDerPol(), perturbed(y), var, 0.0, 0.1, 1e-2)
    assert (cg == 0).all() and (co == 0).all()
    frac, worst, env = check_parity(yg, yo, yp, slack=0.02, factor=5.0)
    print(f"\nreference GPU (fixed), van der Pol: {frac:.3f} within tolerance, worst {worst:.3g}, envelope {env:.3g}")


def test_fixed_mass_action_matches_oracle(oracle):
    mech = A.mechanism_53()
    y, var = A.mixed_stiffness_initial_conditions(mech, 64, seed=5)
    r = _ref(54, True)
    r.set_mechanism(mech)
    yg, cg, _ = r.run(y, var, 0.0, 1e-6, 1e-6)
    yo, co, _ = oracle.run("radau2a", mech, y, var, 0.0, 1e-6, 1e-6)
    yp, _, _ = oracle.run("radau2a", mech, perturbed(y), var, 0.0, 1e-6, 1e-6)
    assert (cg == 0).all() and (co == 0).all()
    frac, worst, env = check_parity(yg, yo, yp, slack=0.05, factor=5.0)
    print(f"\nreference GPU (fixed), 53 species: {frac:.3f} within tolerance, worst {worst:.3g}, envelope {env:.3g}")
