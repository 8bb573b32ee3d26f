// Runge-Kutta-Chebyshev (second order, stabilised explicit) for one system per
// team, after rkc/rkc.c:41-362 -- the CPU semantics: the work array (h,
// spectral radius, previous error, eigenvector estimate) starts from zero on
// every call (rkc.c:212), the spectral-radius convergence test compares
// against the previous sigma (rkc.c:90-92) and hmin follows the step
// (rkc.c:292).  The GPU reference keeps work[] across calls and tests against
// an overwritten norm (rkc.cu:81,231); neither is reproduced.
#pragma once
#include "common.cuh"

namespace aib {

namespace rkcc {
constexpr double UROUND = 2.22e-16;   // rkc/rkc_props.h:394
}

template <int N, int TS, class Mech>
struct Rkc {
    using V = Vec<N, TS>;
    using TM = Team<TS>;
    static constexpr int S = V::S;
    const Mech& mech;
    double* scratch;
    double atol, rtol, pr;
    Stats& stats;

    __device__ __forceinline__ void rhs(double t, const V& y, V& f) {
        mech.template dydt<TS>(t, pr, y, f, scratch);
        stats.c[ST_RHS]++;
    }

    __device__ __forceinline__ double dot(const V& a, const V& b) const {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < S; ++k)
            if (V::ok(k)) s += a[k] * b[k];
        return TM::sum(s);
    }

    // rkc.c:41-110
    __device__ double spec_rad(double t, double hmax, const V& y, const V& F, V& v, V& Fv) {
        const int itmax = 50;
        const double small = 1.0 / hmax;
        double nrm1 = sqrt(dot(y, y));
        double nrm2 = sqrt(dot(v, v));
        double dynrm;
        if (nrm1 != 0.0 && nrm2 != 0.0) {
            dynrm = nrm1 * sqrt(rkcc::UROUND);
#pragma unroll
            for (int k = 0; k < S; ++k) v[k] = y[k] + v[k] * (dynrm / nrm2);
        } else if (nrm1 != 0.0) {
            dynrm = nrm1 * sqrt(rkcc::UROUND);
#pragma unroll
            for (int k = 0; k < S; ++k) v[k] = y[k] * (1.0 + sqrt(rkcc::UROUND));
        } else if (nrm2 != 0.0) {
            dynrm = rkcc::UROUND;
#pragma unroll
            for (int k = 0; k < S; ++k) v[k] *= (dynrm / nrm2);
        } else {
            dynrm = rkcc::UROUND;
#pragma unroll
            for (int k = 0; k < S; ++k) v[k] = rkcc::UROUND;
        }
        double sigma = 0.0;
        for (int iter = 1; iter <= itmax; ++iter) {
            rhs(t, v, Fv);
            double d = 0.0;
#pragma unroll
            for (int k = 0; k < S; ++k)
                if (V::ok(k)) d += (Fv[k] - F[k]) * (Fv[k] - F[k]);
            nrm1 = sqrt(TM::sum(d));
            nrm2 = sigma;
            sigma = nrm1 / dynrm;
            if (iter >= 2 && fabs(sigma - nrm2) <= fmax(sigma, small) * 0.01) {
#pragma unroll
                for (int k = 0; k < S; ++k) v[k] = v[k] - y[k];
                return 1.2 * sigma;
            }
            if (nrm1 != 0.0) {
#pragma unroll
                for (int k = 0; k < S; ++k) v[k] = y[k] + (Fv[k] - F[k]) * (dynrm / nrm1);
            } else {
                const int ind = iter % N;
#pragma unroll
                for (int k = 0; k < S; ++k)
                    if (V::idx(k) == ind) v[k] = y[k] - (v[k] - y[k]);
            }
        }
        return 1.2 * sigma;
    }

    // rkc.c:125-196
    __device__ void step(double t, double h, const V& y0, const V& F0, int s, V& yj) {
        const double w0 = 1.0 + 2.0 / (13.0 * double(s * s));
        const double temp1 = w0 * w0 - 1.0;
        const double temp2 = sqrt(temp1);
        const double arg = double(s) * log(w0 + temp2);
        const double w1 = sinh(arg) * temp1 / (cosh(arg) * double(s) * temp2 - w0 * sinh(arg));
        double b_jm1 = 1.0 / (4.0 * (w0 * w0));
        double b_jm2 = b_jm1;
        V yjm1, yjm2;
        double mu_t = w1 * b_jm1;
#pragma unroll
        for (int k = 0; k < S; ++k) {
            yjm2[k] = y0[k];
            yjm1[k] = y0[k] + mu_t * h * F0[k];
        }
        double c_jm2 = 0.0, c_jm1 = mu_t, zjm1 = w0, zjm2 = 1.0, dzjm1 = 1.0, dzjm2 = 0.0, d2zjm1 = 0.0,
               d2zjm2 = 0.0;
        for (int j = 2; j <= s; ++j) {
            const double zj = 2.0 * w0 * zjm1 - zjm2;
            const double dzj = 2.0 * w0 * dzjm1 - dzjm2 + 2.0 * zjm1;
            const double d2zj = 2.0 * w0 * d2zjm1 - d2zjm2 + 4.0 * dzjm1;
            const double b_j = d2zj / (dzj * dzj);
            const double gamma_t = 1.0 - zjm1 * b_jm1;
            const double nu = -b_j / b_jm2;
            const double mu = 2.0 * b_j * w0 / b_jm1;
            mu_t = mu * w1 / w0;
            rhs(t + h * c_jm1, yjm1, yj);
#pragma unroll
            for (int k = 0; k < S; ++k)
                yj[k] = (1.0 - mu - nu) * y0[k] + mu * yjm1[k] + nu * yjm2[k] + h * mu_t * (yj[k] - gamma_t * F0[k]);
            const double c_j = mu * c_jm1 + nu * c_jm2 + mu_t * (1.0 - gamma_t);
            if (j < s) {
#pragma unroll
                for (int k = 0; k < S; ++k) {
                    yjm2[k] = yjm1[k];
                    yjm1[k] = yj[k];
                }
            }
            c_jm2 = c_jm1;
            c_jm1 = c_j;
            b_jm2 = b_jm1;
            b_jm1 = b_j;
            zjm2 = zjm1;
            zjm1 = zj;
            dzjm2 = dzjm1;
            dzjm1 = dzj;
            d2zjm2 = d2zjm1;
            d2zjm1 = d2zj;
        }
    }

    // rkc.c:209-362
    __device__ int integrate(double t, double tEnd, V& y) {
        int nstep = 0;
        double w0 = 0.0, w1 = 0.0, w2 = 0.0, w3 = 0.0;   // work[0..3]
        V ev;                                            // work[4..]
        int m_max = int(round(sqrt(rtol / (10.0 * rkcc::UROUND))));
        if (m_max < 2) m_max = 2;
        V yn, Fn;
#pragma unroll
        for (int k = 0; k < S; ++k) yn[k] = y[k];
        rhs(t, yn, Fn);
#pragma unroll
        for (int k = 0; k < S; ++k) ev[k] = Fn[k];
        const double hmax = fabs(tEnd - t);
        double hmin = 10.0 * rkcc::UROUND * fmax(fabs(t), hmax);
        while (t < tEnd) {
            V tmp, tmp2;
            double err;
            if ((nstep % 25) == 0) w3 = spec_rad(t, hmax, yn, Fn, ev, tmp2);
            if (w2 < rkcc::UROUND) {
                w2 = hmax;
                if (w3 * w2 > 1.0) w2 = 1.0 / w3;
                w2 = fmax(w2, hmin);
#pragma unroll
                for (int k = 0; k < S; ++k) tmp[k] = yn[k] + w2 * Fn[k];
                rhs(t + w2, tmp, tmp2);
                double e = 0.0;
#pragma unroll
                for (int k = 0; k < S; ++k) {
                    if (V::ok(k)) {
                        const double est = (tmp2[k] - Fn[k]) / (atol + rtol * fabs(yn[k]));
                        e += est * est;
                    }
                }
                err = w2 * sqrt(TM::sum(e) / N);
                if (0.1 * w2 < hmax * sqrt(err)) w2 = fmax(0.1 * w2 / sqrt(err), hmin);
                else w2 = hmax;
            }
            if (1.1 * w2 >= fabs(tEnd - t)) w2 = fabs(tEnd - t);
            int m = 1 + int(sqrt(1.54 * w2 * w3 + 1.0));
            if (m > m_max) {
                m = m_max;
                w2 = double(m * m - 1) / (1.54 * w3);
            }
            hmin = 10.0 * rkcc::UROUND * fmax(fabs(t), fabs(t + w2));
            stats.c[ST_STEPS]++;
            stats.c[ST_NEWTON] += m;
            step(t, w2, yn, Fn, m, y);
            rhs(t + w2, y, tmp);
            double e = 0.0;
#pragma unroll
            for (int k = 0; k < S; ++k) {
                if (V::ok(k)) {
                    double est = 0.8 * (yn[k] - y[k]) + 0.4 * w2 * (Fn[k] + tmp[k]);
                    est /= (atol + rtol * fmax(fabs(y[k]), fabs(yn[k])));
                    e += est * est;
                }
            }
            err = sqrt(TM::sum(e) / double(N));
            if (err > 1.0) {
                w2 = 0.8 * w2 / pow(err, 1.0 / 3.0);
                w3 = spec_rad(t, hmax, yn, Fn, ev, tmp2);
                stats.c[ST_REJECT]++;
            } else {
                t += w2;
                nstep++;
                stats.c[ST_ACCEPT]++;
                double fac = 10.0, t1, t2;
                if (w1 < rkcc::UROUND) {
                    t2 = pow(err, 1.0 / 3.0);
                    if (0.8 < fac * t2) fac = 0.8 / t2;
                } else {
                    t1 = 0.8 * w2 * pow(w0, 1.0 / 3.0);
                    t2 = w1 * pow(err, 2.0 / 3.0);
                    if (t1 < fac * t2) fac = t1 / t2;
                }
                w0 = err;
                w1 = w2;
#pragma unroll
                for (int k = 0; k < S; ++k) {
                    yn[k] = y[k];
                    Fn[k] = tmp[k];
                }
                w2 *= fmax(0.1, fac);
                w2 = fmax(hmin, fmin(hmax, w2));
            }
        }
        return EC_success;
    }
};

}  // namespace aib
