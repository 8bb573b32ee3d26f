/*
 * ORACLE / TEST INFRASTRUCTURE.  The synthetic constant-pressure mass-action
 * mechanism (the model of accelerint_b200/mechanism.py, the arithmetic of
 * oracle/mech.c: ma_prepare / ma_rates) as one-thread device code in the
 * reference's GPU callback convention: every per-system array is strided by
 * the grid (INDEX(i) = thread + i * grid size, gpu_macros.cuh:19-23), as
 * pyJac-generated CUDA callbacks are.  The per-thread work arrays are local.
 */
#ifndef MA_COMMON_CUH
#define MA_COMMON_CUH
#include "header.cuh"

#define MA_K (NSP - 1)
#define MA_R_U 8.31446261815324
#define MA_P_ATM 101325.0
#define MA_T_REF 298.15
#define MA_T_FLOOR 100.0

struct ma_point {
    double T, S, c0, cpm, logT, log_catm;
    double C[MA_K], h[MA_K], grt[MA_K];
};

__device__ __forceinline__ void ma_point_at(const ma_tables& tb, double pr, const double* __restrict__ y,
                                            ma_point& s)
{
    const double T = fmax(y[INDEX(0)], MA_T_FLOOR);
    double S = 0.0, cpm = 0.0;
    for (int k = 0; k < MA_K; ++k) {
        const double yk = y[INDEX(1 + k)];
        S += yk / tb.mw[k];
        cpm += yk * tb.cp[k] / tb.mw[k];
    }
    s.T = T;
    s.S = S;
    s.cpm = cpm;
    s.c0 = 1e-6 * pr / (MA_R_U * T);
    s.logT = log(T);
    s.log_catm = log(1e-6 * MA_P_ATM / (MA_R_U * T));
    const double lnt = log(T / MA_T_REF);
    for (int k = 0; k < MA_K; ++k) {
        s.C[k] = s.c0 * (y[INDEX(1 + k)] / tb.mw[k]) / S;
        const double hk = tb.h_form[k] + tb.cp[k] * (T - MA_T_REF);
        const double sk = tb.s_ref[k] + tb.cp[k] * lnt;
        s.h[k] = hk;
        s.grt[k] = hk / (MA_R_U * T) - sk / MA_R_U;
    }
}

/* forward and reverse rate constants of reaction r; dnu = sum of the stoichiometric changes */
__device__ __forceinline__ void ma_rate_constants(const ma_tables& tb, const ma_point& s, int r, double& kf,
                                                  double& kr, int& dnu)
{
    double g = 0.0;
    int nu = 0;
    for (int a = 0; a < 2; ++a) {
        const int p = tb.prod[2 * r + a], q = tb.reac[2 * r + a];
        if (p >= 0) { g += s.grt[p]; ++nu; }
        if (q >= 0) { g -= s.grt[q]; --nu; }
    }
    const double lkf = tb.log_a[r] + tb.beta[r] * s.logT - tb.ta[r] / s.T;
    kf = exp(lkf);
    kr = exp(lkf + g - nu * s.log_catm);
    dnu = nu;
}

#endif
