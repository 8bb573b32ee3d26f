// Caratheodory-Fejer (CF) rational approximation of exp(z) on (-inf, 0]: the
// (n, n) approximant's poles and residues that the exponential integrators use
// in phi_k(cH) = sum_q 2 Re(r_q theta_q^-k (cH - theta_q I)^-1).
//
// Follows the steps of exponential_integrators/cf.c:41-312 (which follows
// Trefethen, Weideman and Schmelzer, "Talbot quadratures and rational
// approximations", BIT 46 (2006)):
//   1. Chebyshev coefficients c_0..c_K of exp(9 (t - 1) / (t + 1)), t on [-1, 1],
//      from a length-1024 FFT of samples on the unit circle (cf.c:64-81);
//   2. the K x K Hankel matrix H[r][s] = c[r + s + 1] (r + s <= K - 1) and its
//      (n+1)-th singular pair (cf.c:99-115);
//   3. the roots of the singular-vector polynomial outside the unit disc are
//      the poles in the transplanted variable (cf.c:168-190);
//   4. the numerator by a second FFT, the residues by deflated polynomial
//      evaluation, and the map back z = 9 (q - 1)^2 / (q + 1)^2 (cf.c:192-300).
// The reference calls FFTW, LAPACK dgesvd and dgeev (companion-matrix roots);
// here the FFT is a radix-2 transform, the Hankel matrix (symmetric) is
// diagonalised by cyclic Jacobi rotations (singular values = |eigenvalues|),
// and the roots come from the Aberth-Ehrlich simultaneous iteration polished
// by Newton steps.  The poles are returned in conjugate pairs, ordered by
// decreasing real part with the positive imaginary part first -- the order
// dgeev produces for this polynomial, which the phi sums (q = 0, 2, 4, ...)
// rely on.
#include <algorithm>
#include <cmath>
#include <complex>
#include <vector>

namespace aib_cf {

using cd = std::complex<double>;

// In-place iterative radix-2 FFT, X_j = sum_k x_k exp(-2 pi i j k / n).
static void fft(std::vector<cd>& a) {
    const size_t n = a.size();
    for (size_t i = 1, j = 0; i < n; ++i) {
        size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    for (size_t len = 2; len <= n; len <<= 1) {
        const double ang = -2.0 * M_PI / double(len);
        for (size_t i = 0; i < n; i += len) {
            for (size_t k = 0; k < len / 2; ++k) {
                const cd wk(std::cos(ang * double(k)), std::sin(ang * double(k)));
                const cd u = a[i + k], v = a[i + k + len / 2] * wk;
                a[i + k] = u + v;
                a[i + k + len / 2] = u - v;
            }
        }
    }
}

// Cyclic Jacobi eigen-decomposition of a symmetric K x K matrix (row-major a),
// eigenvectors in the columns of v (row-major).
static void jacobi_eigen(int K, std::vector<double>& a, std::vector<double>& v, std::vector<double>& lam) {
    v.assign(size_t(K) * K, 0.0);
    for (int i = 0; i < K; ++i) v[size_t(i) * K + i] = 1.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0, tot = 0.0;
        for (int i = 0; i < K; ++i)
            for (int j = 0; j < K; ++j) {
                const double x = a[size_t(i) * K + j] * a[size_t(i) * K + j];
                tot += x;
                if (i != j) off += x;
            }
        if (off <= 1e-32 * tot) break;
        for (int p = 0; p < K - 1; ++p) {
            for (int q = p + 1; q < K; ++q) {
                const double apq = a[size_t(p) * K + q];
                if (apq == 0.0) continue;
                const double app = a[size_t(p) * K + p], aqq = a[size_t(q) * K + q];
                const double theta = (aqq - app) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < K; ++k) {
                    const double akp = a[size_t(k) * K + p], akq = a[size_t(k) * K + q];
                    a[size_t(k) * K + p] = c * akp - s * akq;
                    a[size_t(k) * K + q] = s * akp + c * akq;
                }
                for (int k = 0; k < K; ++k) {
                    const double apk = a[size_t(p) * K + k], aqk = a[size_t(q) * K + k];
                    a[size_t(p) * K + k] = c * apk - s * aqk;
                    a[size_t(q) * K + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < K; ++k) {
                    const double vkp = v[size_t(k) * K + p], vkq = v[size_t(k) * K + q];
                    v[size_t(k) * K + p] = c * vkp - s * vkq;
                    v[size_t(k) * K + q] = s * vkp + c * vkq;
                }
            }
        }
    }
    lam.resize(K);
    for (int i = 0; i < K; ++i) lam[i] = a[size_t(i) * K + i];
}

// p(x) = sum_i c[i] x^(d - i), d = c.size() - 1, and p'(x), by Horner's rule.
static void horner(const std::vector<cd>& c, cd x, cd& p, cd& dp) {
    p = c[0];
    dp = 0.0;
    for (size_t i = 1; i < c.size(); ++i) {
        dp = dp * x + p;
        p = p * x + c[i];
    }
}

// All roots of sum_i c[i] x^(d - i) (c[0] != 0) by the Aberth-Ehrlich iteration.
static std::vector<cd> poly_roots(std::vector<cd> c) {
    while (c.size() > 1 && c[0] == 0.0) c.erase(c.begin());
    const int d = int(c.size()) - 1;
    std::vector<cd> z(d);
    if (d <= 0) return z;
    // initial guesses on a circle of the Cauchy-bound-like radius
    double r = 0.0;
    for (int i = 1; i <= d; ++i) r = std::max(r, std::pow(std::abs(c[i] / c[0]), 1.0 / i));
    r = std::max(r, 1e-3);
    for (int k = 0; k < d; ++k) {
        const double ang = 2.0 * M_PI * (k + 0.25) / d + 0.4;
        z[k] = r * cd(std::cos(ang), std::sin(ang));
    }
    for (int it = 0; it < 2000; ++it) {
        double worst = 0.0;
        for (int k = 0; k < d; ++k) {
            cd p, dp;
            horner(c, z[k], p, dp);
            if (p == 0.0) continue;
            const cd ratio = p / dp;
            cd s = 0.0;
            for (int j = 0; j < d; ++j)
                if (j != k) s += 1.0 / (z[k] - z[j]);
            const cd delta = ratio / (1.0 - ratio * s);
            z[k] -= delta;
            worst = std::max(worst, std::abs(delta) / std::max(1.0, std::abs(z[k])));
        }
        if (worst < 1e-15) break;
    }
    for (int k = 0; k < d; ++k) {   // Newton polish
        for (int it = 0; it < 3; ++it) {
            cd p, dp;
            horner(c, z[k], p, dp);
            if (dp == 0.0) break;
            z[k] -= p / dp;
        }
    }
    return z;
}

// Coefficients (highest power first) of prod_j (x - roots[j]).
static std::vector<cd> poly_from_roots(const std::vector<cd>& roots) {
    std::vector<cd> q(roots.size() + 1, 0.0);
    q[0] = 1.0;
    for (size_t j = 0; j < roots.size(); ++j) {
        cd old1 = q[0];
        for (size_t i = 1; i <= j + 1; ++i) {
            const cd old2 = q[i];
            q[i] = q[i] - roots[j] * old1;
            old1 = old2;
        }
    }
    return q;
}

// Returns 0 on success; n poles and residues in pr/pi, rr/ri.
int poles_residues(int n, double atol, double* pr, double* pi, double* rr, double* ri) {
    const int K = 75, nf = 1024;
    const double scl = 9.0;
    std::vector<cd> w(nf), F(nf);
    for (int k = 0; k < nf; ++k) {
        const double ang = 2.0 * M_PI * double(k) / double(nf);
        w[k] = cd(std::cos(ang), std::sin(ang));
        const double t = w[k].real();
        F[k] = std::exp(scl * (t - 1.0) / (t + 1.0 + atol));
    }
    std::vector<cd> Fh = F;
    fft(Fh);
    std::vector<double> c(nf);
    for (int k = 0; k < nf; ++k) c[k] = Fh[k].real() / nf;
    // analytic part f(w) = sum_{j=K..0} c_j w^j
    std::vector<cd> f(nf, 0.0);
    for (int k = 0; k < nf; ++k) {
        cd acc = 0.0;
        for (int j = K; j >= 0; --j) acc = acc * w[k] + c[j];
        f[k] = acc;
    }
    // Hankel matrix and its singular pairs (symmetric: from the eigenpairs)
    std::vector<double> H(size_t(K) * K, 0.0), V, lam;
    for (int r = 0; r < K; ++r)
        for (int s = 0; r + s <= K - 1; ++s) H[size_t(r) * K + s] = c[r + s + 1];
    jacobi_eigen(K, H, V, lam);
    std::vector<int> order(K);
    for (int i = 0; i < K; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return std::fabs(lam[a]) > std::fabs(lam[b]); });
    const int col = order[n];
    const double sval = std::fabs(lam[col]);
    const double sgn = lam[col] >= 0 ? 1.0 : -1.0;
    std::vector<cd> u(nf, 0.0), v(nf, 0.0);
    for (int k = 0; k < K; ++k) {
        v[k] = V[size_t(k) * K + col];
        u[k] = sgn * V[size_t(K - 1 - k) * K + col];
    }
    std::vector<cd> uf = u, vf = v;
    fft(uf);
    fft(vf);
    std::vector<cd> rt(nf);
    for (int k = 0; k < nf; ++k) {
        const double ang = 2.0 * M_PI * double((long(k) * K) % nf) / double(nf);   // w_k^K
        rt[k] = f[k] - sval * cd(std::cos(ang), std::sin(ang)) * (uf[k] / vf[k]);
    }
    // poles in the transplanted variable: roots of v outside the unit disc
    std::vector<cd> pc(K);
    for (int k = 0; k < K; ++k) pc[k] = v[k];
    std::vector<cd> zr = poly_roots(pc), qk;
    for (const cd& z : zr)
        if (std::abs(z) > 1.0) qk.push_back(z);
    if (int(qk.size()) != n) return 1;
    // conjugate pairs: exact conjugates, ordered as the reference's phi sums expect
    std::vector<cd> up;
    for (const cd& z : qk)
        if (z.imag() > 0) up.push_back(z);
    if (int(up.size()) * 2 != n) return 2;
    // order by the real part of the z-plane pole, descending; in each pair the
    // member whose z-plane image has the positive imaginary part comes first
    auto zplane = [&](cd q) { return scl * (q - 1.0) * (q - 1.0) / ((q + 1.0) * (q + 1.0)); };
    std::sort(up.begin(), up.end(), [&](cd a, cd b) { return zplane(a).real() > zplane(b).real(); });
    qk.clear();
    for (const cd& z : up) {
        const bool first = zplane(z).imag() >= 0;
        qk.push_back(first ? z : std::conj(z));
        qk.push_back(first ? std::conj(z) : z);
    }
    std::vector<cd> qc = poly_from_roots(qk);
    std::vector<cd> pt(nf);
    for (int k = 0; k < nf; ++k) {
        cd acc = 0.0;
        for (int j = 0; j <= n; ++j) acc = acc * w[k] + qc[j].real();
        pt[k] = acc * rt[k];
    }
    fft(pt);
    std::vector<double> ptc(n + 1);
    for (int i = 0; i <= n; ++i) ptc[i] = pt[n - i].real() / nf;
    for (int k = 0; k < n; ++k) {
        const cd q = qk[k];
        std::vector<cd> others;
        for (int i = 0; i < n; ++i)
            if (i != k) others.push_back(qk[i]);
        std::vector<cd> q2 = poly_from_roots(others);
        cd ck1 = 0.0, ck2 = 0.0;
        for (int i = 0; i <= n; ++i) ck1 = ck1 * q + ptc[i];
        for (int i = 0; i < n; ++i) ck2 = ck2 * q + q2[i];
        const cd resq = ck1 / ck2;
        const cd pole = zplane(q);
        const cd r = 4.0 * resq * pole / (q * q - 1.0);
        pr[k] = pole.real();
        pi[k] = pole.imag();
        rr[k] = r.real();
        ri[k] = r.imag();
    }
    return 0;
}

}  // namespace aib_cf
