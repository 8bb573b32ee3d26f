"""The Radau iteration-matrix factorisations in isolation (RK_Decomp,
radau2a/radau2a.c:256-278), through the diagnostic C-ABI call
accelerInt_radau_decomp, against LAPACK-semantics dgetrf / zgetrf (the oracle's
plain-C restatement, oracle/lapack_plain.c).

* FP64: the same pivots as the oracle on every matrix, and factors equal to
  1e-12 relative to the largest entry (the GPU contracts multiply-adds into FMAs,
  so the last bits may differ).
* FP32 (E2 in single precision, the shared-memory LU) and FP32_ALL (both in
  single precision: the shared-memory LU at N = 54, the register-resident
  shifting-row LU of one-warp teams at N = 14): P E = L U holds to
  2e-5 relative to the largest entry of E, and every multiplier is bounded as
  partial pivoting bounds it (|l| <= 1 for the real matrix; |l| <= sqrt(2) for
  the complex one, whose pivots are chosen by |Re| + |Im|), up to rounding.  The
  pivot sequence itself is not compared with FP64's: the mechanism Jacobians
  have columns with proportional entries, and entries that tie to single-
  precision rounding go either way (about one matrix in seven at N = 14).
* A zero pivot reports info = k + 1 in every precision.

The matrices are E1 = (gamma/h) I - J and E2 = ((alpha + i beta)/h) I - J for
Jacobians of the synthetic mechanisms at seeded states and step sizes of
1e-9 .. 1e-5 s, plus Gaussian random Jacobians.
"""
import ctypes

import numpy as np
import pytest

import accelerint_b200 as A

pytestmark = pytest.mark.gpu

GAMMA = 3.637834252744495732208418513577775
ALPHA = 2.681082873627752133895790743211112
BETA = 3.050430199247410569426377624787569


def _jacobians(orc, n, count, seed):
    rng = np.random.default_rng(seed)
    if n == 54:
        mech = A.mechanism_53()
        y, var = A.mixed_stiffness_initial_conditions(mech, count // 2, seed=seed)
    else:
        mech = A.mechanism_13()
        y, var = A.mass_action_initial_conditions(mech, count // 2, seed=seed)
    jacs = [orc.jacob(mech, y[:, i], var[i]) for i in range(count // 2)]
    scale = np.median([np.abs(j).max() for j in jacs])
    jacs += [rng.standard_normal((n, n)) * scale * 10.0 ** rng.uniform(-3, 0) for _ in range(count - count // 2)]
    h = 10.0 ** rng.uniform(-9, -5, count)
    return np.stack(jacs), h


def _lapack(orc, E, cplx):
    n = E.shape[0]
    a = np.asfortranarray(E.astype(np.complex128 if cplx else np.float64))
    ipiv = np.zeros(n, dtype=np.int32)
    info = ctypes.c_int(0)
    nn = ctypes.c_int(n)
    f = orc.lib.zgetrf_ if cplx else orc.lib.dgetrf_
    f(ctypes.byref(nn), ctypes.byref(nn), a.ctypes.data_as(ctypes.c_void_p), ctypes.byref(nn),
      ipiv.ctypes.data_as(ctypes.c_void_p), ctypes.byref(info))
    perm = np.arange(n)
    for k in range(n):
        p = ipiv[k] - 1
        perm[k], perm[p] = perm[p], perm[k]
    return a, perm, info.value


def _gpu(n, precision, jacs, h):
    import torch
    lib = A.load_library()
    count = len(h)
    # column-major per matrix: J[i + j n] = jacs[m, i, j]
    jd = torch.from_numpy(np.ascontiguousarray(jacs.transpose(0, 2, 1))).cuda()
    hd = torch.from_numpy(h).cuda()
    f1 = torch.float32 if precision == A.LU_FP32_ALL else torch.float64
    f2 = torch.float64 if precision == A.LU_FP64 else torch.float32
    e1 = torch.zeros(count * n * n, dtype=f1, device="cuda")
    e2 = torch.zeros(count * n * n * 2, dtype=f2, device="cuda")
    perm = torch.zeros(count * 2 * n, dtype=torch.int32, device="cuda")
    info = torch.zeros(count * 2, dtype=torch.int32, device="cuda")
    rc = lib.accelerInt_radau_decomp(n, precision, count, jd.data_ptr(), hd.data_ptr(), e1.data_ptr(),
                                     e2.data_ptr(), perm.data_ptr(), info.data_ptr(), None)
    assert rc == A.ACCELERINT_OK
    torch.cuda.synchronize()
    e1 = e1.cpu().numpy().astype(np.float64).reshape(count, n, n).transpose(0, 2, 1)
    e2 = e2.cpu().numpy().astype(np.float64).reshape(count, n, n, 2)
    e2 = (e2[..., 0] + 1j * e2[..., 1]).transpose(0, 2, 1)
    perm = perm.cpu().numpy().reshape(count, 2, n)
    info = info.cpu().numpy().reshape(count, 2)
    return e1, e2, perm, info


def _matrices(J, h):
    n = J.shape[0]
    return (GAMMA / h) * np.eye(n) - J, ((ALPHA + 1j * BETA) / h) * np.eye(n) - J


def _residual(E, F, perm):
    n = E.shape[0]
    L = np.tril(F, -1) + np.eye(n)
    U = np.triu(F)
    return float(np.abs(E[perm] - L @ U).max() / np.abs(E).max())


@pytest.mark.parametrize("n", [14, 54])
def test_fp64_factors_match_lapack(oracle, n):
    jacs, h = _jacobians(oracle, n, 256, seed=100 + n)
    e1, e2, perm, info = _gpu(n, A.LU_FP64, jacs, h)
    for m in range(len(h)):
        E1, E2 = _matrices(jacs[m], h[m])
        f1, p1, i1 = _lapack(oracle, E1, False)
        f2, p2, i2 = _lapack(oracle, E2, True)
        assert np.array_equal(perm[m, 0], p1) and np.array_equal(perm[m, 1], p2), f"matrix {m}: pivots differ"
        assert info[m, 0] == i1 and info[m, 1] == i2
        assert np.abs(e1[m] - f1).max() <= 1e-12 * np.abs(E1).max()
        assert np.abs(e2[m] - f2).max() <= 1e-12 * np.abs(E2).max()


@pytest.mark.parametrize("n", [14, 54])
@pytest.mark.parametrize("precision", [A.LU_FP32, A.LU_FP32_ALL])
def test_single_precision_factors(oracle, n, precision):
    jacs, h = _jacobians(oracle, n, 256, seed=200 + n)
    _, _, perm64, _ = _gpu(n, A.LU_FP64, jacs, h)
    e1, e2, perm, info = _gpu(n, precision, jacs, h)
    assert (info == 0).all()
    r1, r2 = [], []
    for m in range(len(h)):
        E1, E2 = _matrices(jacs[m], h[m])
        r1.append(_residual(E1, e1[m], perm[m, 0]))
        r2.append(_residual(E2, e2[m], perm[m, 1]))
    # E1 stays in FP64 in the FP32 mode
    assert max(r1) <= (1e-13 if precision == A.LU_FP32 else 2e-5), max(r1)
    assert max(r2) <= 2e-5, max(r2)
    l1 = max(float(np.abs(np.tril(e1[m], -1)).max()) for m in range(len(h)))
    l2 = max(float(np.abs(np.tril(e2[m], -1)).max()) for m in range(len(h)))
    assert l1 <= 1.0 + 1e-6, l1
    assert l2 <= np.sqrt(2.0) * (1.0 + 1e-6), l2
    same = [float(np.mean([np.array_equal(perm[m, i], perm64[m, i]) for m in range(len(h))])) for i in (0, 1)]
    print(f"n={n} precision={precision}: residual E1 {max(r1):.2e} E2 {max(r2):.2e}, max |l| {l1:.4f} {l2:.4f}, "
          f"pivots as FP64 on {same[0]:.3f} / {same[1]:.3f} of the matrices")


@pytest.mark.parametrize("n", [14, 54])
@pytest.mark.parametrize("precision", [A.LU_FP64, A.LU_FP32, A.LU_FP32_ALL])
def test_zero_pivot_info(oracle, n, precision):
    """A column of E1 that is zero from the start gives a zero pivot at its step:
    info = k + 1 (xGETF2), and E2 of the same Jacobian is regular."""
    jacs, h = _jacobians(oracle, n, 8, seed=300 + n)
    k = 3
    for m in range(len(h)):
        jacs[m][:, k] = 0.0
        jacs[m][k, k] = GAMMA / h[m]
    _, _, _, info = _gpu(n, precision, jacs, h)
    assert (info[:, 0] == k + 1).all(), info
    assert (info[:, 1] == 0).all(), info
