/*
 * ORACLE / TEST INFRASTRUCTURE.  Mechanism callbacks for the oracle and for the
 * build of the reference's own sources (oracle/refshim/callbacks.c).
 *
 * van der Pol: examples/van_der_pol/dydt.c:88-95, jacob.c:129-141,
 *              sparse_multiplier.c:165-168.
 * Mass action: the synthetic constant-pressure mechanism documented in
 *              accelerint_b200/mechanism.py (no reference source; pyJac's
 *              generated code is absent from the reference repository).
 */
#include <math.h>
#include <float.h>
#include <string.h>
#include <string.h>
#include "oracle.h"

#define R_U 8.31446261815324
#define P_ATM 101325.0
#define T_REF 298.15
/* Rates and thermodynamics are evaluated at max(T, T_FLOOR): Newton iterates
 * of an over-long step can carry unphysical temperatures, and log(T) of a
 * negative value would turn the whole state into NaN (which the reference's
 * fmax()-based norms then accept as converged, radau2a.c:452). */
#define T_FLOOR 100.0

static void vdp_dydt(double mu, const double* y, double* dy)
{
    dy[0] = y[1];
    dy[1] = mu * (1 - y[0] * y[0]) * y[1] - y[0];
}

static void vdp_jacob(double mu, const double* y, double* jac)
{
    jac[0 * 2 + 0] = 0;
    jac[0 * 2 + 1] = -2 * mu * y[0] * y[1] - 1;
    jac[1 * 2 + 0] = 1;
    jac[1 * 2 + 1] = mu * (1 - y[0] * y[0]);
}

/* Common per-call quantities of the mass-action model. */
typedef struct {
    double T, S, c0, cpm, logT, log_catm;
    double C[OR_NMAX];
    double h[OR_NMAX];     /* J/mol */
    double grt[OR_NMAX];   /* g/(R T) */
} ma_state;

static void ma_prepare(const or_mech* m, double pr, const double* y, ma_state* s)
{
    const int K = m->n_species;
    const double T = fmax(y[0], T_FLOOR);
    double S = 0.0, cpm = 0.0;
    for (int k = 0; k < K; ++k) {
        S += y[1 + k] / m->mw[k];
        cpm += y[1 + k] * m->cp[k] / m->mw[k];
    }
    s->T = T;
    s->S = S;
    s->cpm = cpm;
    s->c0 = 1e-6 * pr / (R_U * T);
    s->logT = log(T);
    s->log_catm = log(1e-6 * P_ATM / (R_U * T));
    const double lnt = log(T / T_REF);
    for (int k = 0; k < K; ++k) {
        s->C[k] = s->c0 * (y[1 + k] / m->mw[k]) / S;
        double hk = m->h_form[k] + m->cp[k] * (T - T_REF);
        double sk = m->s_ref[k] + m->cp[k] * lnt;
        s->h[k] = hk;
        s->grt[k] = hk / (R_U * T) - sk / R_U;
    }
}

/* Forward / reverse rate constants of reaction r (log space combined to avoid overflow). */
static void ma_rates(const or_mech* m, const ma_state* s, int r, double* kf, double* kr,
                     double* dG, int* dnu)
{
    const int* re = m->reac + 2 * r;
    const int* pr = m->prod + 2 * r;
    double g = 0.0;
    int nu = 0;
    for (int a = 0; a < 2; ++a) {
        if (pr[a] >= 0) { g += s->grt[pr[a]]; ++nu; }
        if (re[a] >= 0) { g -= s->grt[re[a]]; --nu; }
    }
    const double lkf = m->log_a[r] + m->beta[r] * s->logT - m->ta[r] / s->T;
    *kf = exp(lkf);
    *kr = exp(lkf + g - nu * s->log_catm);
    *dG = g;
    *dnu = nu;
}

static void ma_dydt(const or_mech* m, double pr, const double* y, double* dy)
{
    const int K = m->n_species, R = m->n_reactions;
    ma_state s;
    ma_prepare(m, pr, y, &s);
    double wdot[OR_NMAX];
    memset(wdot, 0, sizeof(double) * K);
    for (int r = 0; r < R; ++r) {
        double kf, kr, dG;
        int dnu;
        ma_rates(m, &s, r, &kf, &kr, &dG, &dnu);
        const int* re = m->reac + 2 * r;
        const int* pd = m->prod + 2 * r;
        double fwd = kf * s.C[re[0]];
        if (re[1] >= 0) fwd *= s.C[re[1]];
        double rev = kr * s.C[pd[0]];
        if (pd[1] >= 0) rev *= s.C[pd[1]];
        const double q = fwd - rev;
        wdot[re[0]] -= q;
        if (re[1] >= 0) wdot[re[1]] -= q;
        wdot[pd[0]] += q;
        if (pd[1] >= 0) wdot[pd[1]] += q;
    }
    double Q = 0.0;
    for (int k = 0; k < K; ++k) {
        Q += s.h[k] * wdot[k];
        dy[1 + k] = m->mw[k] * s.S * wdot[k] / s.c0;
    }
    dy[0] = -s.S * Q / (s.c0 * s.cpm);
}

static void ma_jacob(const or_mech* m, double pr, const double* y, double* jac)
{
    const int K = m->n_species, R = m->n_reactions, n = K + 1;
    ma_state s;
    ma_prepare(m, pr, y, &s);
    double wdot[OR_NMAX], wT[OR_NMAX], G[OR_NMAX * OR_NMAX];   /* G[k + K*m] = d wdot_k / d C_m */
    memset(wdot, 0, sizeof(double) * K);
    memset(wT, 0, sizeof(double) * K);
    memset(G, 0, sizeof(double) * K * K);
    for (int r = 0; r < R; ++r) {
        double kf, kr, dG;
        int dnu;
        ma_rates(m, &s, r, &kf, &kr, &dG, &dnu);
        const int* re = m->reac + 2 * r;
        const int* pd = m->prod + 2 * r;
        const int nre = re[1] >= 0 ? 2 : 1, npd = pd[1] >= 0 ? 2 : 1;
        double fwd = kf * s.C[re[0]];
        if (nre == 2) fwd *= s.C[re[1]];
        double rev = kr * s.C[pd[0]];
        if (npd == 2) rev *= s.C[pd[1]];
        const double q = fwd - rev;
        double dH = 0.0;
        for (int a = 0; a < npd; ++a) dH += s.h[pd[a]];
        for (int a = 0; a < nre; ++a) dH -= s.h[re[a]];
        const double dlkf = (m->beta[r] + m->ta[r] / s.T) / s.T;
        const double dlkr = dlkf - dH / (R_U * s.T * s.T) + dnu / s.T;
        /* d q / d T at fixed Y: rate constants plus C_m ~ 1/T */
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
        /* nu_kr: -1 for reactants, +1 for products */
        for (int a = 0; a < ns; ++a) {
            const int k = sp[a];
            const double nu = a < nre ? -1.0 : 1.0;
            wdot[k] += nu * q;
            wT[k] += nu * dqdT;
            for (int b = 0; b < ns; ++b) G[k + K * sp[b]] += nu * dqdC[b];
        }
    }
    double x[OR_NMAX], g[OR_NMAX];
    for (int k = 0; k < K; ++k) x[k] = (y[1 + k] / m->mw[k]) / s.S;
    for (int k = 0; k < K; ++k) {
        double acc = 0.0;
        for (int j = 0; j < K; ++j) acc += G[k + K * j] * x[j];
        g[k] = acc;
    }
    double Q = 0.0, dQT = 0.0;
    for (int k = 0; k < K; ++k) {
        Q += s.h[k] * wdot[k];
        dQT += m->cp[k] * wdot[k] + s.h[k] * wT[k];
    }
    double hg = 0.0;
    for (int k = 0; k < K; ++k) hg += s.h[k] * g[k];
    /* species rows */
    for (int k = 0; k < K; ++k) {
        const double a = wdot[k] / s.c0 - g[k];
        for (int j = 0; j < K; ++j)
            jac[(1 + k) + n * (1 + j)] = (m->mw[k] / m->mw[j]) * (a + G[k + K * j]);
        jac[(1 + k) + n * 0] = (m->mw[k] * s.S / s.c0) * (wT[k] + wdot[k] / s.T);
    }
    /* temperature row */
    const double f = -1.0 / (s.c0 * s.cpm);
    for (int j = 0; j < K; ++j) {
        double hG = 0.0;
        for (int k = 0; k < K; ++k) hG += s.h[k] * G[k + K * j];
        const double dQ = (s.c0 / m->mw[j]) * (hG - hg);       /* S * dQ/dY_j */
        jac[0 + n * (1 + j)] = f * (Q / m->mw[j] - s.S * Q * m->cp[j] / (m->mw[j] * s.cpm) + dQ);
    }
    jac[0] = f * s.S * (Q / s.T + dQT);
    if (!(y[0] > T_FLOOR))            /* f does not depend on T below the floor */
        for (int i = 0; i < n; ++i) jac[i] = 0.0;
}

void or_dydt(const or_mech* m, double t, double pr, const double* y, double* dy)
{
    (void)t;
    if (m->kind == OR_MECH_VDP) vdp_dydt(pr, y, dy);
    else ma_dydt(m, pr, y, dy);
}

/* generic/fd_jacob.c:24-127 with FD_ORD 1: forward differences, increment
 * r_j = max(sqrt(eps) |y_j|, r0 / ewt_j), ewt = ATOL + RTOL |y|,
 * r0 = 1000 RTOL eps N sqrt(sum (ewt dy)^2 / N). */
static void fd_jacob(const or_mech* m, double t, double pr, const double* cy, double* jac)
{
    const int n = m->n;
    double y[OR_NMAX], dy[OR_NMAX], ftemp[OR_NMAX], ewt[OR_NMAX];
    memcpy(y, cy, n * sizeof(double));
    or_dydt(m, t, pr, y, dy);
    for (int i = 0; i < n; ++i) ewt[i] = m->fd_atol + (m->fd_rtol * fabs(y[i]));
    const double srur = sqrt(DBL_EPSILON);
    double sum = 0.0;
    for (int i = 0; i < n; ++i) sum += (ewt[i] * dy[i]) * (ewt[i] * dy[i]);
    const double fac = sqrt(sum / ((double)(n)));
    const double r0 = 1000.0 * m->fd_rtol * DBL_EPSILON * ((double)(n)) * fac;
    for (int j = 0; j < n; ++j) {
        const double yj_orig = y[j];
        const double r = fmax(srur * fabs(yj_orig), r0 / ewt[j]);
        y[j] = yj_orig + r;
        or_dydt(m, t, pr, y, ftemp);
        for (int i = 0; i < n; ++i) jac[i + n * j] = (ftemp[i] - dy[i]) / r;
        y[j] = yj_orig;
    }
}

void or_jacob(const or_mech* m, double t, double pr, const double* y, double* jac)
{
    if (m->jac_fd) {
        fd_jacob(m, t, pr, y, jac);
        return;
    }
    (void)t;
    if (m->kind == OR_MECH_VDP) vdp_jacob(pr, y, jac);
    else ma_jacob(m, pr, y, jac);
}

/* sparse_multiplier: w = A v (examples/van_der_pol/sparse_multiplier.c:165-168 for N = 2). */
void or_jacvec(const or_mech* m, const double* A, const double* v, double* w)
{
    const int n = m->n;
    if (m->kind == OR_MECH_VDP) {
        w[0] = A[0] * v[0] + A[2] * v[1];
        w[1] = A[1] * v[0] + A[2 + 1] * v[1];
        return;
    }
    for (int i = 0; i < n; ++i) {
        double acc = A[i] * v[0];
        for (int j = 1; j < n; ++j) acc += A[i + n * j] * v[j];
        w[i] = acc;
    }
}
