/*
 * ORACLE / TEST INFRASTRUCTURE.  dydt of the synthetic mass-action mechanism for
 * the reference GPU build: y' = f(y) for the state (T, Y_1..Y_K) of the calling
 * thread's system, dy[INDEX(i)] (the slot of examples/van_der_pol/dydt.cu:31).
 */
#include "ma_common.cuh"
#include "dydt.cuh"

__device__ void dydt(const double t, const double pres, const double* __restrict__ y, double* __restrict__ dy,
                     const mechanism_memory* __restrict__ d_mem)
{
    const ma_tables tb = d_mem->tb;
    ma_point s;
    ma_point_at(tb, pres, y, s);
    double wdot[MA_K];
    for (int k = 0; k < MA_K; ++k) wdot[k] = 0.0;
    for (int r = 0; r < tb.R; ++r) {
        double kf, kr;
        int dnu;
        ma_rate_constants(tb, s, r, kf, kr, dnu);
        const int r0 = tb.reac[2 * r], r1 = tb.reac[2 * r + 1], p0 = tb.prod[2 * r], p1 = tb.prod[2 * r + 1];
        double fwd = kf * s.C[r0];
        if (r1 >= 0) fwd *= s.C[r1];
        double rev = kr * s.C[p0];
        if (p1 >= 0) rev *= s.C[p1];
        const double q = fwd - rev;
        wdot[r0] -= q;
        if (r1 >= 0) wdot[r1] -= q;
        wdot[p0] += q;
        if (p1 >= 0) wdot[p1] += q;
    }
    double Q = 0.0;
    for (int k = 0; k < MA_K; ++k) {
        Q += s.h[k] * wdot[k];
        dy[INDEX(1 + k)] = tb.mw[k] * s.S * wdot[k] / s.c0;
    }
    dy[INDEX(0)] = -s.S * Q / (s.c0 * s.cpm);
}
