"""GPU Radau with the collocation starting values (accelerInt_set_stage_extrapolation(1)),
through the C-ABI, against the oracle run with the same option (oracle/radau2a.c,
or_config.stage_extrap) on the same seeded inputs.

* FP64, 13 species (256 systems, three global steps) and 53 species (64 mixed-stiffness
  systems, two global steps): within the envelope of three oracle runs on inputs perturbed
  by 1e-15 (tests/helpers.check_parity: share within rtol 1e-6 / atol 1e-10 no lower than
  the envelope's less 0.02, the worst system within 3x of it).
* FP32_ALL on the 1,024-system 53-species sample of tests/golden/tight (three global
  steps): about as accurate against the rtol-1e-12 solution as the FP64 oracle with the
  same starting values (median within 1.5x, 90th percentile within 2x: single-precision
  factors change the Newton iterates, hence the step sequence, and the errors are now a
  quarter of what they are with the reference's start), more accurate than the oracle
  with the reference's starting values, and fewer Radau steps than the same GPU run with
  the reference's starting values.
"""
import os

import numpy as np
import pytest

import accelerint_b200 as A
from tests.helpers import check_parity, per_system_error, perturbed

pytestmark = pytest.mark.gpu

TIGHT = os.path.join(os.path.dirname(__file__), "golden", "tight", "ma54_tight.npz")


def _gpu(mech, y, var, t_end, dt, lu, mode):
    """Device-buffer path with the per-system counters: (y_out, codes, stats[num, NSTATS])."""
    import torch
    num = y.shape[1]
    integ = A.Integrator(num, mech, lu=lu, stage_extrapolation=mode)
    try:
        yd = torch.from_numpy(np.ascontiguousarray(y)).cuda()
        vd = torch.from_numpy(np.ascontiguousarray(var)).cuda()
        codes = torch.zeros(num, dtype=torch.int32, device="cuda")
        stats = torch.zeros((num, A.NSTATS), dtype=torch.int32, device="cuda")
        integ.integrate_device(0.0, t_end, dt, yd, vd, codes, stats)
        torch.cuda.synchronize()
        return yd.cpu().numpy(), codes.cpu().numpy(), stats.cpu().numpy()
    finally:
        integ.close()


def _parity(oracle, mech, y, var, t_end, dt, name):
    yg, cg, _ = _gpu(mech, y, var, t_end, dt, A.LU_FP64, 1)
    yo, co, _ = oracle.run("radau2a", mech, y, var, 0.0, t_end, dt, stage_extrapolation=1)
    pert = [oracle.run("radau2a", mech, perturbed(y, seed=s), var, 0.0, t_end, dt, stage_extrapolation=1)[0]
            for s in range(3)]
    assert (cg == 0).all() and (co == 0).all()
    frac, worst, env = check_parity(yg, yo, pert)
    print(f"\n{name}, collocation starting values, FP64: {frac:.4f} within rtol 1e-6 / atol 1e-10 of the oracle; "
          f"worst {worst:.3g}, envelope {env:.3g}")


def test_fp64_13_species_matches_oracle(oracle):
    mech = A.mechanism_13()
    y, var = A.mass_action_initial_conditions(mech, 256, seed=1717)
    _parity(oracle, mech, y, var, 3e-6, 1e-6, "13 species")


def test_fp64_53_species_matches_oracle(oracle):
    mech = A.mechanism_53()
    y, var = A.mixed_stiffness_initial_conditions(mech, 64, seed=5353)
    _parity(oracle, mech, y, var, 2e-6, 1e-6, "53 species")


def test_fp32_all_accuracy_and_work(oracle):
    d = np.load(TIGHT)
    mech = A.mechanism_53()
    y, var = A.mixed_stiffness_initial_conditions(mech, int(d["num"]), int(d["seed"]))
    t_end, dt, yt = float(d["t_end"]), float(d["dt"]), np.array(d["y"])
    y1, c1, s1 = _gpu(mech, y, var, t_end, dt, A.LU_FP32_ALL, 1)
    y0, c0, s0 = _gpu(mech, y, var, t_end, dt, A.LU_FP32_ALL, 0)
    yo1, co1, _ = oracle.run("radau2a", mech, y, var, 0.0, t_end, dt, stage_extrapolation=1)
    yo0, co0, _ = oracle.run("radau2a", mech, y, var, 0.0, t_end, dt)
    assert (c1 == 0).all() and (c0 == 0).all() and (co1 == 0).all() and (co0 == 0).all()
    assert np.isfinite(y1).all()
    e1, eo1, eo0 = per_system_error(y1, yt), per_system_error(yo1, yt), per_system_error(yo0, yt)
    q = lambda e, p: float(np.quantile(e, p))  # noqa: E731
    steps1, steps0 = float(s1[:, 0].sum()), float(s0[:, 0].sum())
    print(f"\nFP32_ALL, collocation start: weighted error vs rtol-1e-12 median {q(e1, .5):.3g} p90 {q(e1, .9):.3g} "
          f"(oracle, same start {q(eo1, .5):.3g} / {q(eo1, .9):.3g}; oracle, reference start {q(eo0, .5):.3g} / "
          f"{q(eo0, .9):.3g}); Radau steps {steps1:.0f} against {steps0:.0f} with the reference start")
    assert q(e1, 0.5) <= 1.5 * q(eo1, 0.5)
    assert q(e1, 0.9) <= 2.0 * q(eo1, 0.9)
    assert q(e1, 0.5) < q(eo0, 0.5)
    assert steps1 < steps0
