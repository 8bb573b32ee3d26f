"""accelerInt_integrate_device_noalloc: the entry point for callers that cannot let a
library allocate device memory during a run (a host code that plans or pools all of its
device memory itself, or that must avoid the device-wide synchronisation cudaMalloc and
cudaFree can cause).  Its scratch lives in a fixed array inside the library instead.

The test calls it through the C-ABI twice in a row -- the second call continues the
integration from the first call's output, so a work-queue counter or Jacobian left in
the shared array by the first call would show -- and checks both results against the
allocating entry point accelerInt_integrate_device, within the tolerance of the other
parity tests (|x - x_ref| < atol + rtol |x_ref|, rtol 1e-6, atol 1e-10; the kernels are
the same, so the results are expected to be identical).  Collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

import accelerint_b200 as A
from tests.helpers import weighted_error

pytestmark = pytest.mark.gpu


def _noalloc(integ, t0, t1, dt, y_dev, var_dev, codes_dev):
    return integ.lib.accelerInt_integrate_device_noalloc(
        y_dev.shape[1], t0, t1, dt, ctypes.c_void_p(y_dev.data_ptr()), ctypes.c_void_p(var_dev.data_ptr()),
        ctypes.c_void_p(codes_dev.data_ptr()), None)


def _compare_two_calls(mech, y, var, lu=A.LU_FP64, finite_difference=False):
    import torch
    num = y.shape[1]
    integ = A.Integrator(num, mech, lu=lu)
    try:
        if finite_difference:
            integ.set_jacobian(True)
        var_d = torch.from_numpy(var).cuda()
        y_ref = torch.from_numpy(y).cuda()
        y_new = torch.from_numpy(y).cuda()
        c_ref = torch.zeros(num, dtype=torch.int32, device="cuda")
        c_new = torch.zeros(num, dtype=torch.int32, device="cuda")
        for (t0, t1) in [(0.0, 1e-6), (1e-6, 2e-6)]:
            integ.integrate_device(t0, t1, 1e-6, y_ref, var_d, c_ref)
            rc = _noalloc(integ, t0, t1, 1e-6, y_new, var_d, c_new)
            assert rc == A.ACCELERINT_OK
            torch.cuda.synchronize()
            assert torch.equal(c_ref, c_new)
            assert int(c_new.abs().max()) == 0
            a, b = y_new.cpu().numpy(), y_ref.cpu().numpy()
            assert not np.isnan(a).any()
            assert weighted_error(a, b) < 1.0
    finally:
        integ.close()


@pytest.mark.parametrize("which,lu", [("ma14", A.LU_FP64), ("ma54", A.LU_FP64), ("ma54", A.LU_FP32),
                                      ("ma54", A.LU_FP32_ALL)])
def test_noalloc_matches_allocating_entry_point(which, lu):
    if which == "ma14":
        mech = A.mechanism_13()
        y, var = A.mass_action_initial_conditions(mech, 96, seed=21)
    else:
        mech = A.mechanism_53()
        y, var = A.mixed_stiffness_initial_conditions(mech, 24, seed=22)
    _compare_two_calls(mech, y, var, lu=lu)


def test_noalloc_capped_grid_drains_the_queue():
    """2,048 53-species systems: more than the 719 whose Jacobians fit the static array at
    N = 54, so fewer teams than systems are in flight and the work queue must hand every
    system out exactly once."""
    mech = A.mechanism_53()
    y, var = A.mixed_stiffness_initial_conditions(mech, 2048, seed=23)
    _compare_two_calls(mech, y, var, lu=A.LU_FP32_ALL)


def test_noalloc_finite_difference_jacobian():
    """With the finite-difference Jacobian selected, both entry points run it."""
    mech = A.mechanism_13()
    y, var = A.mass_action_initial_conditions(mech, 32, seed=24)
    _compare_two_calls(mech, y, var, finite_difference=True)


def test_noalloc_refuses_step_recording():
    """Step recording (and learned proposals) have no allocation-free kernels: the call is refused."""
    import torch
    mech = A.mechanism_13()
    y, var = A.mass_action_initial_conditions(mech, 8, seed=25)
    integ = A.Integrator(8, mech)
    try:
        rec = torch.zeros((16, 240), dtype=torch.float32, device="cuda")
        cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
        assert integ.lib.accelerInt_set_step_recording(rec.data_ptr(), cnt.data_ptr(), 16) == A.ACCELERINT_OK
        yd, vd = torch.from_numpy(y).cuda(), torch.from_numpy(var).cuda()
        cd = torch.zeros(8, dtype=torch.int32, device="cuda")
        assert _noalloc(integ, 0.0, 1e-6, 1e-6, yd, vd, cd) == A._lib.ACCELERINT_ERR_UNSUPPORTED
        assert integ.lib.accelerInt_set_step_recording(None, None, 0) == A.ACCELERINT_OK
    finally:
        integ.close()


def test_noalloc_rejects_unsupported_state():
    """Van der Pol runs on the thread-per-system kernel, which has no allocation-free form."""
    import torch
    integ = A.Integrator(8, A.VanDerPol())
    try:
        y, var = A.vdp_initial_conditions(8)
        yd, vd = torch.from_numpy(y).cuda(), torch.from_numpy(var).cuda()
        cd = torch.zeros(8, dtype=torch.int32, device="cuda")
        assert _noalloc(integ, 0.0, 1e-2, 1e-2, yd, vd, cd) == A._lib.ACCELERINT_ERR_STATE
    finally:
        integ.close()
