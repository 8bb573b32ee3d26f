"""Radau starting values after an accepted step (RK_Interpolate, radau2a/radau2a.c:302-314),
on the oracle (the plain-C restatement of the reference's CPU radau2a, CPU only).

The reference evaluates the third stage's starting value with x2 in its outer factor
(radau2a.c:312) where the collocation polynomial of the last step, evaluated at the third
new node, has x3.  Mode 0 keeps the reference's form (the plain form's parity); mode 1,
the library's accelerInt_set_stage_extrapolation(1), evaluates the polynomial at all three
nodes.  Only the Newton iteration's start changes; the error estimate accepts or rejects
every step in both.  On 13-species systems the reference's start makes most Newton
iterations fail: mode 1 takes several times fewer steps and is closer to the rtol-1e-12
solution.
"""
import numpy as np

import accelerint_b200 as A
from tests.helpers import per_system_error


def test_collocation_start_fewer_steps_and_more_accurate(oracle):
    mech = A.mechanism_13()
    y, var = A.mass_action_initial_conditions(mech, 64, seed=99)
    t_end, dt = 2e-6, 1e-6
    y0, c0, s0 = oracle.run("radau2a", mech, y, var, 0.0, t_end, dt, stage_extrapolation=0)
    y1, c1, s1 = oracle.run("radau2a", mech, y, var, 0.0, t_end, dt, stage_extrapolation=1)
    yt, ct, _ = oracle.run("radau2a", mech, y, var, 0.0, t_end, dt, rtol=1e-12, atol=1e-20, max_steps=20_000_000)
    assert (c0 == 0).all() and (c1 == 0).all() and (ct == 0).all()
    steps0, steps1 = s0[:, 0].sum(), s1[:, 0].sum()
    e0, e1 = per_system_error(y0, yt), per_system_error(y1, yt)
    print(f"\nsteps {steps0:.0f} -> {steps1:.0f}, rejected {s0[:, 2].sum():.0f} -> {s1[:, 2].sum():.0f}; "
          f"weighted error vs tight median {np.median(e0):.3g} -> {np.median(e1):.3g}, max {e0.max():.3g} -> {e1.max():.3g}")
    assert steps1 < 0.5 * steps0
    assert np.median(e1) < np.median(e0) and e1.max() < e0.max()


def test_reference_start_is_the_default(oracle):
    mech = A.mechanism_13()
    y, var = A.mass_action_initial_conditions(mech, 8, seed=5)
    ya, ca, sa = oracle.run("radau2a", mech, y, var, 0.0, 1e-6, 1e-6)
    yb, cb, sb = oracle.run("radau2a", mech, y, var, 0.0, 1e-6, 1e-6, stage_extrapolation=0)
    assert np.array_equal(ya, yb) and np.array_equal(sa, sb)
