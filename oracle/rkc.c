/*
 * ORACLE / TEST INFRASTRUCTURE.  RKC restated from rkc/rkc.c (line numbers
 * below refer to that file), the CPU semantics: work[] is zeroed per call.
 */
#include <math.h>
#include <string.h>
#include "oracle.h"

#define UROUND (2.22e-16)   /* rkc/rkc_props.h:394 */

typedef struct {
    const or_mech* m;
    double pr;
    double* st;
} rctx;

static void rhs(rctx* x, double t, const double* y, double* f)
{
    or_dydt(x->m, t, x->pr, y, f);
    x->st[ST_RHS] += 1;
}

/* rkc.c:41-110 */
static double spec_rad(rctx* x, int n, double t, double hmax, const double* y, const double* F,
                       double* v, double* Fv)
{
    const int itmax = 50;
    double small = 1.0 / hmax;
    double nrm1 = 0.0, nrm2 = 0.0;
    for (int i = 0; i < n; ++i) {
        nrm1 += (y[i] * y[i]);
        nrm2 += (v[i] * v[i]);
    }
    nrm1 = sqrt(nrm1);
    nrm2 = sqrt(nrm2);
    double dynrm;
    if ((nrm1 != 0.0) && (nrm2 != 0.0)) {
        dynrm = nrm1 * sqrt(UROUND);
        for (int i = 0; i < n; ++i) v[i] = y[i] + v[i] * (dynrm / nrm2);
    } else if (nrm1 != 0.0) {
        dynrm = nrm1 * sqrt(UROUND);
        for (int i = 0; i < n; ++i) v[i] = y[i] * (1.0 + sqrt(UROUND));
    } else if (nrm2 != 0.0) {
        dynrm = UROUND;
        for (int i = 0; i < n; ++i) v[i] *= (dynrm / nrm2);
    } else {
        dynrm = UROUND;
        for (int i = 0; i < n; ++i) v[i] = UROUND;
    }
    double sigma = 0.0;
    for (int iter = 1; iter <= itmax; ++iter) {
        rhs(x, t, v, Fv);
        nrm1 = 0.0;
        for (int i = 0; i < n; ++i) nrm1 += ((Fv[i] - F[i]) * (Fv[i] - F[i]));
        nrm1 = sqrt(nrm1);
        nrm2 = sigma;
        sigma = nrm1 / dynrm;
        if ((iter >= 2) && (fabs(sigma - nrm2) <= (fmax(sigma, small) * 0.01))) {
            for (int i = 0; i < n; ++i) v[i] = v[i] - y[i];
            return (1.2 * sigma);
        }
        if (nrm1 != 0.0) {
            for (int i = 0; i < n; ++i) v[i] = y[i] + ((Fv[i] - F[i]) * (dynrm / nrm1));
        } else {
            int ind = (iter % n);
            v[ind] = y[ind] - (v[ind] - y[ind]);
        }
    }
    return (1.2 * sigma);
}

/* rkc.c:125-196 */
static void rkc_step(rctx* x, int n, double t, double h, const double* y_0, const double* F_0, int s,
                     double* y_j)
{
    const double w0 = 1.0 + 2.0 / (13.0 * (double)(s * s));
    double temp1 = (w0 * w0) - 1.0;
    double temp2 = sqrt(temp1);
    double arg = (double)(s) * log(w0 + temp2);
    const double w1 = sinh(arg) * temp1 / (cosh(arg) * (double)(s) * temp2 - w0 * sinh(arg));
    double b_jm1 = 1.0 / (4.0 * (w0 * w0));
    double b_jm2 = b_jm1;
    double y_jm1[OR_NMAX], y_jm2[OR_NMAX];
    double mu_t = w1 * b_jm1;
    for (int i = 0; i < n; ++i) {
        y_jm2[i] = y_0[i];
        y_jm1[i] = y_0[i] + (mu_t * h * F_0[i]);
    }
    double c_jm2 = 0.0, c_jm1 = mu_t, zjm1 = w0, zjm2 = 1.0, dzjm1 = 1.0, dzjm2 = 0.0;
    double d2zjm1 = 0.0, d2zjm2 = 0.0;
    for (int j = 2; j <= s; ++j) {
        double zj = 2.0 * w0 * zjm1 - zjm2;
        double dzj = 2.0 * w0 * dzjm1 - dzjm2 + 2.0 * zjm1;
        double d2zj = 2.0 * w0 * d2zjm1 - d2zjm2 + 4.0 * dzjm1;
        double b_j = d2zj / (dzj * dzj);
        double gamma_t = 1.0 - (zjm1 * b_jm1);
        double nu = -b_j / b_jm2;
        double mu = 2.0 * b_j * w0 / b_jm1;
        mu_t = mu * w1 / w0;
        rhs(x, t + (h * c_jm1), y_jm1, y_j);
        for (int i = 0; i < n; ++i) {
            y_j[i] = (1.0 - mu - nu) * y_0[i] + (mu * y_jm1[i]) + (nu * y_jm2[i])
                     + h * mu_t * (y_j[i] - (gamma_t * F_0[i]));
        }
        double c_j = (mu * c_jm1) + (nu * c_jm2) + mu_t * (1.0 - gamma_t);
        if (j < s) {
            for (int i = 0; i < n; ++i) {
                y_jm2[i] = y_jm1[i];
                y_jm1[i] = y_j[i];
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

/* rkc.c:209-362 */
int or_rkc(const or_config* c, const or_mech* m, double t, double tEnd, double pr, double* y, double* st)
{
    rctx x = {m, pr, st};
    const int n = m->n;
    const double ATOL = c->atol, RTOL = c->rtol;
    int nstep = 0;
    double work[4 + OR_NMAX];
    memset(work, 0, sizeof(work));
    int m_max = (int)(round(sqrt(RTOL / (10.0 * UROUND))));
    if (m_max < 2) m_max = 2;
    double y_n[OR_NMAX], F_n[OR_NMAX];
    for (int i = 0; i < n; ++i) y_n[i] = y[i];
    rhs(&x, t, y_n, F_n);
    if (work[2] < UROUND) {
        for (int i = 0; i < n; ++i) work[4 + i] = F_n[i];
    }
    const double hmax = fabs(tEnd - t);
    double hmin = 10.0 * UROUND * fmax(fabs(t), hmax);
    while (t < tEnd) {
        double temp_arr[OR_NMAX], temp_arr2[OR_NMAX];
        double err;
        if ((nstep % 25) == 0) work[3] = spec_rad(&x, n, t, hmax, y_n, F_n, &work[4], temp_arr2);
        if (work[2] < UROUND) {
            work[2] = hmax;
            if ((work[3] * work[2]) > 1.0) work[2] = 1.0 / work[3];
            work[2] = fmax(work[2], hmin);
            for (int i = 0; i < n; ++i) temp_arr[i] = y_n[i] + (work[2] * F_n[i]);
            rhs(&x, t + work[2], temp_arr, temp_arr2);
            err = 0.0;
            for (int i = 0; i < n; ++i) {
                double est = (temp_arr2[i] - F_n[i]) / (ATOL + RTOL * fabs(y_n[i]));
                err += est * est;
            }
            err = work[2] * sqrt(err / n);
            if ((0.1 * work[2]) < (hmax * sqrt(err))) {
                work[2] = fmax(0.1 * work[2] / sqrt(err), hmin);
            } else {
                work[2] = hmax;
            }
        }
        if ((1.1 * work[2]) >= fabs(tEnd - t)) work[2] = fabs(tEnd - t);
        int ms = 1 + (int)(sqrt(1.54 * work[2] * work[3] + 1.0));
        if (ms > m_max) {
            ms = m_max;
            work[2] = (double)(ms * ms - 1) / (1.54 * work[3]);
        }
        hmin = 10.0 * UROUND * fmax(fabs(t), fabs(t + work[2]));
        st[ST_STEPS] += 1;
        st[ST_NEWTON] += ms;           /* stage count, reported in the Newton column for RKC */
        rkc_step(&x, n, t, work[2], y_n, F_n, ms, y);
        rhs(&x, t + work[2], y, temp_arr);
        err = 0.0;
        for (int i = 0; i < n; ++i) {
            double est = 0.8 * (y_n[i] - y[i]) + 0.4 * work[2] * (F_n[i] + temp_arr[i]);
            est /= (ATOL + RTOL * fmax(fabs(y[i]), fabs(y_n[i])));
            err += est * est;
        }
        err = sqrt(err / ((double)n));
        if (err > 1.0) {
            work[2] = 0.8 * work[2] / (pow(err, (1.0 / 3.0)));
            work[3] = spec_rad(&x, n, t, hmax, y_n, F_n, &work[4], temp_arr2);
            st[ST_REJECT] += 1;
        } else {
            t += work[2];
            nstep++;
            st[ST_ACCEPT] += 1;
            double fac = 10.0;
            double t1, t2;
            if (work[1] < UROUND) {
                t2 = pow(err, (1.0 / 3.0));
                if (0.8 < (fac * t2)) fac = 0.8 / t2;
            } else {
                t1 = 0.8 * work[2] * pow(work[0], (1.0 / 3.0));
                t2 = work[1] * pow(err, (2.0 / 3.0));
                if (t1 < (fac * t2)) fac = t1 / t2;
            }
            work[0] = err;
            work[1] = work[2];
            for (int i = 0; i < n; ++i) {
                y_n[i] = y[i];
                F_n[i] = temp_arr[i];
            }
            work[2] *= fmax(0.1, fac);
            work[2] = fmax(hmin, fmin(hmax, work[2]));
        }
    }
    return 0;
}
