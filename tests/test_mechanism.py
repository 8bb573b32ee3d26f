"""Mechanism callbacks: analytic Jacobian against finite differences (the
reference's FD Jacobian, generic/fd_jacob.c:24-127, is forward-difference; a
central form is used here for accuracy), conservation properties of the
synthetic model, equilibrium initial conditions."""
import numpy as np
import pytest

from accelerint_b200 import mechanism as M


def fd_jacobian(oracle, mech, y, var):
    n = y.shape[0]
    J = np.zeros((n, n))
    for j in range(n):
        h = 1e-6 * max(abs(y[j]), 1e-8)
        yp, ym = y.copy(), y.copy()
        yp[j] += h
        ym[j] -= h
        J[:, j] = (oracle.dydt(mech, yp, var) - oracle.dydt(mech, ym, var)) / (2 * h)
    return J


@pytest.mark.parametrize("which", ["vdp", "ma14", "ma54"])
def test_jacobian_matches_finite_differences(oracle, which):
    if which == "vdp":
        mech = M.VanDerPol()
        y, var = M.vdp_initial_conditions(4, seed=1)
    elif which == "ma14":
        mech = M.mechanism_13()
        y, var = M.mass_action_initial_conditions(mech, 4, seed=1)
    else:
        mech = M.mechanism_53()
        y, var = M.mixed_stiffness_initial_conditions(mech, 4, seed=1)
    for s in range(4):
        J = oracle.jacob(mech, y[:, s], var[s])
        Jfd = fd_jacobian(oracle, mech, y[:, s], var[s])
        assert np.max(np.abs(J - Jfd)) < 1e-4 * np.max(np.abs(J))


def test_mass_and_energy_conservation(oracle):
    """Unit-conserving reactions conserve mass (sum dY/dt = 0); the energy equation conserves
    total enthalpy: sum_k h_k dY_k/dt / W_k + cp_mix dT/dt = 0."""
    mech = M.mechanism_53()
    y, var = M.mixed_stiffness_initial_conditions(mech, 8, seed=2)
    for s in range(8):
        f = oracle.dydt(mech, y[:, s], var[s])
        assert abs(f[1:].sum()) < 1e-9 * np.max(np.abs(f[1:]))
        T = y[0, s]
        h = mech.h_form + mech.cp * (T - M.T_REF)
        cpm = np.sum(y[1:, s] * mech.cp / mech.mw)
        assert abs(np.sum(h * f[1:] / mech.mw) + cpm * f[0]) < 1e-9 * np.sum(np.abs(h * f[1:] / mech.mw))


def test_equilibrium_initial_conditions_are_near_equilibrium(oracle):
    mech = M.mechanism_53()
    T = np.array([900.0, 1100.0])
    x = M.equilibrium_mole_fractions(mech, T)
    yr, var = M.mass_action_initial_conditions(mech, 2, seed=3)
    for s in range(2):
        yk = x[:, s] * mech.mw
        y = np.concatenate([[T[s]], yk / yk.sum()])
        f = oracle.dydt(mech, y, M.P_ATM)
        yr[0, s] = T[s]
        fr = oracle.dydt(mech, yr[:, s], M.P_ATM)
        # net rates cancel: the residual is a tiny fraction of a random composition's rates
        assert np.max(np.abs(f)) < 1e-10 * np.max(np.abs(fr))


def test_generator_is_seeded_and_unit_conserving():
    a, b = M.mechanism_53(), M.mechanism_53()
    assert np.array_equal(a.reac, b.reac) and np.array_equal(a.log_a, b.log_a)
    units = np.round(a.mw / 16e-3).astype(int)
    for r in range(a.n_reactions):
        assert sum(units[s] for s in a.reac[r] if s >= 0) == sum(units[s] for s in a.prod[r] if s >= 0)
    assert a.n_species == 53 and a.n_reactions == 325
    m13 = M.mechanism_13()
    assert m13.n_species == 13 and m13.n_reactions == 27
