/*
 * ORACLE / TEST INFRASTRUCTURE.  Analytic Jacobian of the synthetic mass-action
 * mechanism for the reference GPU build, jac[INDEX(i + NSP * j)] = d f_i / d y_j
 * (the slot and convention of examples/van_der_pol/jacob.cu:29-41); the
 * arithmetic of oracle/mech.c's ma_jacob.
 */
#include "ma_common.cuh"
#include "jacob.cuh"

__device__ void eval_jacob(const double t, const double pres, const double* __restrict__ y, double* __restrict__ jac,
                           const mechanism_memory* __restrict__ d_mem)
{
    const ma_tables tb = d_mem->tb;
    const int n = NSP;
    ma_point s;
    ma_point_at(tb, pres, y, s);
    double wdot[MA_K], wT[MA_K], G[MA_K * MA_K];   /* G[k + K m] = d wdot_k / d C_m */
    for (int k = 0; k < MA_K; ++k) wdot[k] = wT[k] = 0.0;
    for (int k = 0; k < MA_K * MA_K; ++k) G[k] = 0.0;
    for (int r = 0; r < tb.R; ++r) {
        double kf, kr;
        int dnu;
        ma_rate_constants(tb, s, r, kf, kr, dnu);
        const int re[2] = {tb.reac[2 * r], tb.reac[2 * r + 1]};
        const int pd[2] = {tb.prod[2 * r], tb.prod[2 * r + 1]};
        const int nre = re[1] >= 0 ? 2 : 1, npd = pd[1] >= 0 ? 2 : 1;
        double fwd = kf * s.C[re[0]];
        if (nre == 2) fwd *= s.C[re[1]];
        double rev = kr * s.C[pd[0]];
        if (npd == 2) rev *= s.C[pd[1]];
        const double q = fwd - rev;
        double dH = 0.0;
        for (int a = 0; a < npd; ++a) dH += s.h[pd[a]];
        for (int a = 0; a < nre; ++a) dH -= s.h[re[a]];
        const double dlkf = (tb.beta[r] + tb.ta[r] / s.T) / s.T;
        const double dlkr = dlkf - dH / (MA_R_U * s.T * s.T) + dnu / s.T;
        const double dqdT = fwd * dlkf - rev * dlkr - (nre * fwd - npd * rev) / s.T;
        double dqdC[4];
        int sp[4];
        int ns = 0;
        for (int a = 0; a < nre; ++a) {
            dqdC[ns] = kf * (nre == 2 ? s.C[re[1 - a]] : 1.0);
            sp[ns++] = re[a];
        }
        for (int a = 0; a < npd; ++a) {
            dqdC[ns] = -kr * (npd == 2 ? s.C[pd[1 - a]] : 1.0);
            sp[ns++] = pd[a];
        }
        for (int a = 0; a < ns; ++a) {
            const int k = sp[a];
            const double nu = a < nre ? -1.0 : 1.0;
            wdot[k] += nu * q;
            wT[k] += nu * dqdT;
            for (int b = 0; b < ns; ++b) G[k + MA_K * sp[b]] += nu * dqdC[b];
        }
    }
    double x[MA_K], g[MA_K];
    for (int k = 0; k < MA_K; ++k) x[k] = (y[INDEX(1 + k)] / tb.mw[k]) / s.S;
    for (int k = 0; k < MA_K; ++k) {
        double acc = 0.0;
        for (int j = 0; j < MA_K; ++j) acc += G[k + MA_K * j] * x[j];
        g[k] = acc;
    }
    double Q = 0.0, dQT = 0.0, hg = 0.0;
    for (int k = 0; k < MA_K; ++k) {
        Q += s.h[k] * wdot[k];
        dQT += tb.cp[k] * wdot[k] + s.h[k] * wT[k];
    }
    for (int k = 0; k < MA_K; ++k) hg += s.h[k] * g[k];
    for (int k = 0; k < MA_K; ++k) {
        const double a = wdot[k] / s.c0 - g[k];
        for (int j = 0; j < MA_K; ++j)
            jac[INDEX((1 + k) + n * (1 + j))] = (tb.mw[k] / tb.mw[j]) * (a + G[k + MA_K * j]);
        jac[INDEX(1 + k)] = (tb.mw[k] * s.S / s.c0) * (wT[k] + wdot[k] / s.T);
    }
    const double f = -1.0 / (s.c0 * s.cpm);
    for (int j = 0; j < MA_K; ++j) {
        double hG = 0.0;
        for (int k = 0; k < MA_K; ++k) hG += s.h[k] * G[k + MA_K * j];
        const double dQ = (s.c0 / tb.mw[j]) * (hG - hg);
        jac[INDEX(n * (1 + j))] = f * (Q / tb.mw[j] - s.S * Q * tb.cp[j] / (tb.mw[j] * s.cpm) + dQ);
    }
    jac[INDEX(0)] = f * s.S * (Q / s.T + dQT);
    if (!(y[INDEX(0)] > MA_T_FLOOR))
        for (int i = 0; i < n; ++i) jac[INDEX(i)] = 0.0;
}
