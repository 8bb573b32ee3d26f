"""The oracle (oracle/*.c) against the reference's own CPU integrators.

Golden fixtures in tests/golden/ were produced by the reference's unmodified
radau2a.c / rkc.c / exprb43.c / exp4.c (tests/golden/make_golden.py); the oracle
must reproduce them to the last bit (same operation order, same LU semantics),
given the reference's poles for the exponential methods.  A relative slack of
1e-13 covers a host whose libm rounds exp/log/pow differently.
"""
import glob
import os

import numpy as np
import pytest

from accelerint_b200 import mechanism as M

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def _mech(name):
    return {"vdp": M.VanDerPol(), "ma14": M.mechanism_13(), "ma54": M.mechanism_53()}[name]


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_reproduces_reference(oracle, path):
    g = np.load(path)
    mech = _mech(str(g["mech"]))
    poles = (g["poles"], g["res"]) if "poles" in g else None
    y, codes, _ = oracle.run(str(g["solver"]), mech, g["y0"], g["var"], 0.0, float(g["t_end"]), float(g["dt"]),
                             poles=poles)
    assert np.array_equal(codes, g["codes"])
    ok = g["codes"] == 0
    ref = g["y"][:, ok]
    assert np.all(np.abs(y[:, ok] - ref) <= 1e-13 * np.abs(ref) + 1e-300)


def test_oracle_matches_reference_live(oracle):
    """Same check against the reference build itself (skipped where it was not built)."""
    from oracle import Reference, reference_available
    if not reference_available("radau2a", 14):
        pytest.skip("reference build absent")
    mech = M.mechanism_13()
    y, var = M.mass_action_initial_conditions(mech, 24, seed=77)
    ref = Reference("radau2a", 14)
    ref.set_mechanism(mech)
    yr, cr = ref.run(y, var, 0.0, 2e-6, 1e-6, nthreads=2)
    yo, co, _ = oracle.run("radau2a", mech, y, var, 0.0, 2e-6, 1e-6)
    assert np.array_equal(cr, co)
    assert np.array_equal(yr, yo)


@pytest.mark.parametrize("solver", ["exprb43", "exp4"])
def test_reference_exponential_methods_live(solver):
    """The reference's exponential integrators as the bench drives them (oracle.Reference):
    constructing one computes its CF poles (rational_approximant.c:23-44), and a run on a
    golden fixture's inputs reproduces the fixture (made by the same reference build)."""
    from oracle import Reference, reference_available
    if not reference_available(solver, 14):
        pytest.skip("reference build absent")
    ref = Reference(solver, 14)
    poles, _ = ref.poles()
    assert np.all(np.abs(poles) > 1.0)
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", f"ma14_{solver}.npz"))
    ref.set_mechanism(M.mechanism_13())
    yr, cr = ref.run(np.array(g["y0"]), np.array(g["var"]), 0.0, float(g["t_end"]), float(g["dt"]), nthreads=1)
    assert np.array_equal(cr, g["codes"])
    ok = g["codes"] == 0
    assert np.array_equal(yr[:, ok], g["y"][:, ok])


def test_cf_poles_match_reference_cf():
    """numpy restatement of cf.c (oracle/cf.py) against the reference's cf() with the FFTW
    shim and LAPACK from OpenBLAS; both carry the ill-conditioning of the Hankel SVD + roots."""
    from oracle import cf_poles
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "vdp_exprb43.npz"))
    p, r = cf_poles()
    assert np.max(np.abs(p - g["poles"]) / np.abs(g["poles"])) < 1e-7
    assert np.max(np.abs(r - g["res"]) / np.abs(g["res"])) < 1e-6
