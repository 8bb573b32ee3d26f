"""Edge cases of the C-ABI's integrate semantics on the GPU, against the oracle.

* NUM = 0 is a no-op that succeeds.
* stepsize < 0 means one global step of t_end - t_start (solver_interface.cuh).
* Global steps are measured from t_start, the documented CLI-loop semantics
  (generic/solver_main.c:196-209), also when t_start != 0 (quirk Q2 of the
  reference's library loop is not reproduced).
* The legacy void accelerInt_integrate records its status for
  accelerInt_last_status and the per-system codes for accelerInt_get_codes.
* A batch whose size is no multiple of any block or team size.
"""
import ctypes

import numpy as np
import pytest

import accelerint_b200 as A
from tests.helpers import weighted_error

pytestmark = pytest.mark.gpu


def test_empty_batch_is_a_noop():
    integ = A.Integrator(4, A.VanDerPol())
    try:
        y = np.zeros((2, 0))
        var = np.zeros(0)
        yo, codes, rc = integ.integrate(0.0, 0.1, 0.01, y, var)
        assert rc == A.ACCELERINT_OK and yo.shape == (2, 0) and codes.shape == (0,)
    finally:
        integ.close()


def test_negative_stepsize_is_one_step(oracle):
    y, var = A.vdp_initial_conditions(256, seed=71)
    integ = A.Integrator(256, A.VanDerPol())
    try:
        y1, _, _ = integ.integrate(0.0, 0.05, -1.0, y, var)
        y2, _, _ = integ.integrate(0.0, 0.05, 0.05, y, var)
    finally:
        integ.close()
    assert np.array_equal(y1, y2)
    yo, _, _ = oracle.run("radau2a", A.VanDerPol(), y, var, 0.0, 0.05, 0.05)
    assert weighted_error(y1, yo) < 1.0


def test_steps_measured_from_t_start(oracle):
    mech = A.mechanism_13()
    y, var = A.mass_action_initial_conditions(mech, 64, seed=72)
    integ = A.Integrator(64, mech)
    try:
        yg, cg, _ = integ.integrate(1e-3, 1e-3 + 2.5e-6, 1e-6, y, var)
    finally:
        integ.close()
    # the oracle's loop: [t0, t0 + dt], [t0 + dt, t0 + 2 dt], [t0 + 2 dt, t_end]
    yo, co, _ = oracle.run("radau2a", mech, y, var, 1e-3, 1e-3 + 2.5e-6, 1e-6)
    assert (cg == co).all()
    assert np.median(np.max(np.abs(yg - yo) / (1e-10 + 1e-6 * np.abs(yo)), axis=0)) < 1.0


def test_legacy_void_calls_record_status():
    lib = A.load_library()
    dp = ctypes.POINTER(ctypes.c_double)
    y, var = A.vdp_initial_conditions(100, seed=73)
    y = np.ascontiguousarray(y)
    lib.accelerInt_set_solver(0)
    lib.accelerInt_set_mechanism_van_der_pol()
    lib.accelerInt_initialize(100, 0)
    try:
        assert lib.accelerInt_last_status() == 0
        lib.accelerInt_integrate(100, 0.0, 0.02, 0.01, y.ctypes.data_as(dp), var.ctypes.data_as(dp))
        assert lib.accelerInt_last_status() == 0
        codes = np.full(100, -7, dtype=np.int32)
        assert lib.accelerInt_get_codes(codes.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), 100) == 0
        assert (codes == 0).all()
        assert np.isfinite(y).all()
    finally:
        lib.accelerInt_cleanup()
    # after cleanup the library refuses to integrate instead of crashing
    lib.accelerInt_integrate(100, 0.0, 0.01, 0.01, y.ctypes.data_as(dp), var.ctypes.data_as(dp))
    assert lib.accelerInt_last_status() == A._lib.ACCELERINT_ERR_STATE


@pytest.mark.parametrize("num", [1, 37, 741])
def test_ragged_batch_sizes(oracle, num):
    mech = A.mechanism_13()
    y, var = A.mass_action_initial_conditions(mech, num, seed=74)
    integ = A.Integrator(num, mech, lu=A.LU_FP32_ALL)
    try:
        yg, cg, _ = integ.integrate(0.0, 1e-6, 1e-6, y, var)
    finally:
        integ.close()
    yt, _, _ = oracle.run("radau2a", mech, y, var, 0.0, 1e-6, 1e-6)
    assert (cg == 0).all() and np.isfinite(yg).all()
    # every system integrated: FP32 factors take their own step sequence (weighted
    # differences of a few tens against the FP64 oracle), while a system left at
    # its initial state would differ by orders of magnitude more
    e = np.max(np.abs(yg - yt) / (1e-10 + 1e-6 * np.abs(yt)), axis=0)
    e0 = np.max(np.abs(y - yt) / (1e-10 + 1e-6 * np.abs(yt)), axis=0)
    assert np.median(e) < 100.0
    assert (e < 1e-2 * e0).all()
