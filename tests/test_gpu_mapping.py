"""The launch mappings the autotuner chooses between (accelerInt_set_mapping /
accelerInt_autotune), through the C-ABI, against the oracle (the plain-C
restatement of the reference's CPU radau2a, radau2a/radau2a.c:520-736, one system
at a time as the reference's intDriver thread does, generic/solver_generic.cu:28-42).

* Two systems per warp (team_lanes 16) for the 13-species mechanism (state length
  14): FP64 within the oracle's own perturbation envelope, FP32_ALL as accurate as
  the oracle against an rtol-1e-10 solution.
* Queue granularity: the systems a team claims per atomic change which team runs a
  system, not its arithmetic, so grain 1, 4 and 8 give bit-identical states and codes
  (53 species, FP32_ALL, on a batch larger than one wave of teams).
* The autotuner's pick is one of the candidates and its results agree with the oracle.
"""
import numpy as np
import pytest

import accelerint_b200 as A
from tests.helpers import check_parity, per_system_error, perturbed

pytestmark = pytest.mark.gpu


def _run(mech, y, var, t_end, dt, lu, team_lanes=0, grain=1):
    integ = A.Integrator(y.shape[1], mech, lu=lu)
    try:
        integ.set_mapping(team_lanes, grain)
        yo, codes, stats = integ.integrate(0.0, t_end, dt, y, var)
        assert integ.mapping()[:2] == (team_lanes, grain)
    finally:
        integ.close()
    return yo, codes, stats


@pytest.fixture(scope="module")
def ma14(oracle):
    mech = A.mechanism_13()
    y, var = A.mass_action_initial_conditions(mech, 512, seed=1414)
    t_end, dt = 3e-6, 1e-6
    yo, co, _ = oracle.run("radau2a", mech, y, var, 0.0, t_end, dt)
    yp, _, _ = oracle.run("radau2a", mech, perturbed(y), var, 0.0, t_end, dt)
    yt, _, _ = oracle.run("radau2a", mech, y, var, 0.0, t_end, dt, rtol=1e-10, atol=1e-16)
    assert (co == 0).all()
    return mech, y, var, t_end, dt, yo, yp, yt


def test_half_warp_teams_fp64(ma14):
    mech, y, var, t_end, dt, yo, yp, _ = ma14
    yg, cg, _ = _run(mech, y, var, t_end, dt, A.LU_FP64, team_lanes=16)
    assert (cg == 0).all()
    frac, worst, env = check_parity(yg, yo, yp)
    print(f"\n13 species, two systems per warp, FP64: {frac:.4f} within rtol 1e-6 / atol 1e-10 of the oracle; "
          f"worst {worst:.3g}, envelope {env:.3g}")


def test_half_warp_teams_fp32_all(ma14):
    mech, y, var, t_end, dt, yo, _, yt = ma14
    yg, cg, _ = _run(mech, y, var, t_end, dt, A.LU_FP32_ALL, team_lanes=16)
    yd, cd, _ = _run(mech, y, var, t_end, dt, A.LU_FP32_ALL, team_lanes=0)
    assert (cg == 0).all() and (cd == 0).all()
    eg, ed, eo = per_system_error(yg, yt), per_system_error(yd, yt), per_system_error(yo, yt)
    print(f"\n13 species FP32_ALL vs rtol-1e-10: median {np.median(eg):.3g} (one-warp team {np.median(ed):.3g}, "
          f"oracle {np.median(eo):.3g}), max {eg.max():.3g} ({ed.max():.3g}, {eo.max():.3g})")
    assert np.median(eg) <= 1.25 * np.median(eo) + 1e-3
    assert np.quantile(eg, 0.9) <= 1.5 * np.quantile(eo, 0.9) + 1e-3


def test_queue_grain_is_bit_identical():
    mech = A.mechanism_53()
    y, var = A.mixed_stiffness_initial_conditions(mech, 2048, seed=77)
    ref = _run(mech, y, var, 1e-6, 1e-6, A.LU_FP32_ALL, grain=1)
    for grain in (4, 8):
        out = _run(mech, y, var, 1e-6, 1e-6, A.LU_FP32_ALL, grain=grain)
        assert np.array_equal(out[0], ref[0]) and np.array_equal(out[1], ref[1])
        assert out[2] == ref[2]   # the call's status


def test_autotuned_mapping_agrees_with_oracle(ma14):
    import torch
    mech, y, var, t_end, dt, yo, yp, _ = ma14
    integ = A.Integrator(y.shape[1], mech, lu=A.LU_FP64)
    try:
        yd = torch.from_numpy(np.ascontiguousarray(y)).cuda()
        vd = torch.from_numpy(np.ascontiguousarray(var)).cuda()
        integ.autotune(0.0, dt / 4, dt / 4, yd, vd, 512)
        lanes, grain, occ = integ.mapping()
        assert lanes in (0, 16) and grain in (1, 2, 4, 8) and occ > 0
        integ.integrate_device(0.0, t_end, dt, yd, vd)
        yg = yd.cpu().numpy()
    finally:
        integ.close()
    frac, worst, env = check_parity(yg, yo, yp)
    print(f"\nautotuned mapping (team lanes {lanes}, grain {grain}): {frac:.4f} within tolerance, worst {worst:.3g}")
