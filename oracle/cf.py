"""ORACLE / TEST INFRASTRUCTURE: Caratheodory-Fejer poles and residues in numpy.

Restates exponential_integrators/cf.c:41-312 (reference repository) step by
step: Chebyshev coefficients of exp transplanted to [-1, 1] by an FFT of
length 1024, SVD of the K=75 Hankel matrix, roots of the singular vector
polynomial, numerator coefficients by a second FFT, residues by deflated
polynomial evaluation, then the map back to the z-plane.  numpy's FFT uses
the same sign convention as FFTW_FORWARD; numpy.roots builds the same
companion matrix as linear-algebra.c:141-199 and uses LAPACK dgeev, so the
roots come out in the same conjugate-pair order the reference relies on
(phiAHessenberg.c sums q = 0, 2, 4, ...).
"""
import numpy as np


def cf_poles_residues(n: int = 10, atol: float = 1e-10):
    K, nf = 75, 1024
    w = np.exp(2.0j * np.pi * np.arange(nf) / nf)
    t = w.real
    scl = 9.0
    F = np.exp(scl * (t - 1.0) / (t + 1.0 + atol))
    c = np.fft.fft(F).real / nf
    # analytic part f = sum_{j=K..0} c_j w^j  (cf.c:89-93)
    f = np.zeros(nf, dtype=complex)
    for j in range(K, -1, -1):
        f += c[j] * w ** j
    # Hankel matrix H[r, s] = c[r + s + 1] for r + s <= K - 1  (cf.c:103-107)
    H = np.zeros((K, K))
    for i in range(K):
        for j in range(i + 1):
            H[i - j, j] = c[i + 1]
    U, S, Vh = np.linalg.svd(H)
    V = Vh.T
    s_val = S[n]
    u = np.zeros(nf, dtype=complex)
    v = np.zeros(nf, dtype=complex)
    u[:K] = U[K - 1 - np.arange(K), n]
    v[:K] = V[:K, n]
    b = np.fft.fft(u) / np.fft.fft(v)
    rt = f - s_val * w ** K * b
    zr = np.roots(v[:K].real)
    qk = zr[np.abs(zr) > 1.0]
    assert qk.shape[0] == n, f"expected {n} poles outside the unit disc, got {qk.shape[0]}"
    qc = np.zeros(n + 1, dtype=complex)
    qc[0] = 1.0
    for j in range(n):
        old1 = qc[0]
        for i in range(1, j + 2):
            old2 = qc[i]
            qc[i] = qc[i] - qk[j] * old1
            old1 = old2
    qc = qc.real
    pt = np.zeros(nf, dtype=complex)
    for j in range(n + 1):
        pt += qc[j] * w ** (n - j)
    pt *= rt
    ptc_i = np.fft.fft(pt)
    ptc = np.array([ptc_i[n - i].real / nf for i in range(n + 1)])
    res = np.zeros(n, dtype=complex)
    for k in range(n):
        q = qk[k]
        others = np.array([qk[i] for i in range(n) if i != k])
        q2 = np.zeros(n, dtype=complex)
        q2[0] = 1.0
        for j in range(n - 1):
            old1 = q2[0]
            for i in range(1, j + 2):
                old2 = q2[i]
                q2[i] = q2[i] - others[j] * old1
                old1 = old2
        ck1 = sum(ptc[i] * q ** (n - i) for i in range(n + 1))
        ck2 = sum(q2[i] * q ** (n - 1 - i) for i in range(n))
        res[k] = ck1 / ck2
    poles = scl * (qk - 1.0) ** 2 / ((qk + 1.0) ** 2)
    res = 4.0 * res * poles / (qk * qk - 1.0)
    return poles, res
