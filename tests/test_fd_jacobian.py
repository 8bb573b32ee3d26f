"""Finite-difference Jacobian (generic/fd_jacob.c, first order).

The oracle's restatement must reproduce the reference's own fd_jacob.c (compiled
into oracle/_ref) to the last bits.  On van der Pol both agree with the analytic
Jacobian to the accuracy of a forward difference.  On the mass-action mechanism
they do not: fd_jacob.c weights the RHS norm by ewt (sum (ewt_i dy_i)^2, where a
weighted RMS norm divides by ewt), so the increment r0 / ewt_j of a small mass
fraction is many times the fraction itself.  That is the reference's behaviour,
kept for parity.  The GPU form runs in tests/test_gpu_fd_jacobian.py."""
import numpy as np
import pytest

import accelerint_b200 as A


def _states(mech, num, seed):
    if mech.n_state == 2:
        return A.vdp_initial_conditions(num, seed=seed)
    return A.mixed_stiffness_initial_conditions(mech, num, seed)


@pytest.mark.parametrize("which", ["vdp", "ma14", "ma54"])
def test_oracle_fd_matches_reference_fd(oracle, which):
    from oracle import Reference, reference_available
    mech = {"vdp": A.VanDerPol(), "ma14": A.mechanism_13(), "ma54": A.mechanism_53()}[which]
    if not reference_available("radau2a", mech.n_state):
        pytest.skip("reference build absent")
    ref = Reference("radau2a", mech.n_state)
    ref.set_mechanism(mech)
    y, var = _states(mech, 6, 31)
    for i in range(y.shape[1]):
        jo = oracle.jacob(mech, y[:, i], var[i], fd=(1e-10, 1e-6))
        jr = ref.fd_jacob(y[:, i], var[i])
        assert np.all(np.abs(jo - jr) <= 1e-13 * np.abs(jr) + 1e-300)


@pytest.mark.parametrize("which", ["vdp"])
def test_fd_close_to_analytic(oracle, which):
    mech = {"vdp": A.VanDerPol()}[which]
    y, var = _states(mech, 6, 32)
    for i in range(y.shape[1]):
        ja = oracle.jacob(mech, y[:, i], var[i])
        jf = oracle.jacob(mech, y[:, i], var[i], fd=(1e-10, 1e-6))
        scale = np.max(np.abs(ja), axis=0, keepdims=True) + 1e-300
        assert np.max(np.abs(jf - ja) / scale) < 1e-3
