"""Known-answer tests of the oracle's Krylov building blocks, re-instantiated
from the reference's tests/unit_tests.c (which no longer builds there):
  * LUTests (unit_tests.c:42-61): Hessenberg LU of [[1,2,3],[4,5,6],[0,8,9]];
  * InverseTests (:104-160): the Hessenberg inverse agrees with a general
    inverse to ATOL = 1e-10;
  * PhiTests (:304-318): expAc of the same Hessenberg matrix at c = 1e-8/3
    against nine listed values -- this pins the whole Caratheodory-Fejer
    pole/residue pipeline end to end.
"""
import numpy as np

from oracle import cf_poles

ATOL = 1e-10
H = np.array([[1.0, 2.0, 3.0], [4.0, 5.0, 6.0], [0.0, 8.0, 9.0]])


def test_hessenberg_lu_known_answer(oracle):
    info, f, piv = oracle.hessenberg_lu(H.astype(complex))
    assert info == 0
    # unit_tests.c:53-61, column-major listing
    expect = np.array([4, 0, 1.0 / 4.0, 5, 8, 3.0 / 32.0, 6, 9, 21.0 / 32.0])
    got = f.reshape(-1, order="F")
    assert np.array_equal(got.real, expect) and np.all(got.imag == 0)


def test_hessenberg_inverse_matches_general_inverse(oracle):
    # unit_tests.c:108-127 (testMatrix, column-major)
    col = np.array([1 + 1e3j, 4 - 0.001j, 0, 16e5, 0.0001j, 80000 + 5j, 3 - 5j, 9j, 9j])
    A = col.reshape(3, 3, order="F")
    info, inv = oracle.inverse_hessenberg(A)
    assert info == 0
    assert np.max(np.abs(inv - np.linalg.inv(A))) < ATOL


def test_hessenberg_inverse_random(oracle):
    rng = np.random.default_rng(1)
    for n in (5, 14, 30):
        A = np.triu(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)), -1) + 4 * np.eye(n)
        info, inv = oracle.inverse_hessenberg(A)
        assert info == 0
        assert np.max(np.abs(inv @ A - np.eye(n))) < 1e-10


EXP_KAT = np.array([1.000000003333333e+00, 1.333333346666667e-08, 1.777777807407407e-16,
                    6.666666866666669e-09, 1.000000016666667e+00, 2.666666728888890e-08,
                    1.000000023333334e-08, 2.000000053333334e-08, 1.000000030000001e+00])


def test_expAc_known_answer(oracle):
    """The listed values are exp(cH) to 16 digits (scipy's expm reproduces them to 4e-16).
    The (10,10) Caratheodory-Fejer approximant itself is off by 2.72e-10 at the origin, so
    the reference's own pipeline misses its stated ATOL = 1e-10 on the diagonal (with its own
    poles and with these); the pin is the approximant's error, 3e-10, and ATOL off the diagonal."""
    info, E = oracle.phi(0, H, 1e-8 / 3.0)
    assert info == 0
    got = E.reshape(-1, order="F")
    assert np.max(np.abs(got - EXP_KAT)) < 3e-10
    off = np.array([1, 2, 3, 5, 6, 7])
    assert np.max(np.abs(got[off] - EXP_KAT[off])) < ATOL


def test_expAc_against_expm(oracle):
    from scipy.linalg import expm
    rng = np.random.default_rng(3)
    # upper Hessenberg with a small subdiagonal: eigenvalues near the negative real axis,
    # where the approximant is accurate to ~1e-10
    A = np.triu(rng.standard_normal((8, 8)), 1) + np.diag(-rng.uniform(0.5, 20.0, 8)) \
        + np.diag(0.01 * rng.standard_normal(7), -1)
    for c in (1e-3, 0.1, 1.0):
        info, E = oracle.phi(0, A, c)
        assert info == 0
        assert np.max(np.abs(E - expm(c * A))) < 1e-9


def test_phi1_against_closed_form(oracle):
    """phi_1(cA) = (cA)^-1 (exp(cA) - I) for an invertible A."""
    from scipy.linalg import expm
    rng = np.random.default_rng(4)
    A = np.triu(rng.standard_normal((6, 6)), -1) - 3 * np.eye(6)
    c = 0.5
    info, P1 = oracle.phi(1, A, c)
    assert info == 0
    ref = np.linalg.solve(c * A, expm(c * A) - np.eye(6))
    assert np.max(np.abs(P1 - ref)) < 1e-8


def test_cf_poles_conjugate_pairs():
    p, r = cf_poles()
    assert p.shape == (10,)
    for q in range(0, 10, 2):
        assert abs(p[q] - np.conj(p[q + 1])) < 1e-12 * abs(p[q])
        assert abs(r[q] - np.conj(r[q + 1])) < 1e-9 * abs(r[q])
