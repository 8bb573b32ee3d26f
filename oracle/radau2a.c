/*
 * ORACLE / TEST INFRASTRUCTURE.  Radau IIA restated from radau2a/radau2a.c
 * (line numbers below refer to that file).  Same arithmetic in the same order,
 * with the state length and tolerances taken at run time.
 */
#include <complex.h>
#include <math.h>
#include <float.h>
#include <string.h>
#include <stdbool.h>
#include "oracle.h"
#include "lapack_plain.h"

/* radau2a.c:38-65 */
#define MAX_NO_STEPS 200000
#define NEWTON_MAXIT 8
#define ROUNDOFF DBL_EPSILON
#define FAC_MIN 0.2
#define FAC_MAX 8
#define FAC_SAFE 0.9
#define FAC_REJ 0.1
#define THETA_MIN 0.001
#define NEWTON_TOL 0.03
#define Q_MIN 1.0
#define Q_MAX 1.2
#define MAX_CONSECUTIVE_ERRS 5

/* radau2a.c:101-231: tableau, classical error estimator, transformation */
static const double rkA[3][3] = {
    {1.968154772236604258683861429918299e-1, -6.55354258501983881085227825696087e-2,
     2.377097434822015242040823210718965e-2},
    {3.944243147390872769974116714584975e-1, 2.920734116652284630205027458970589e-1,
     -4.154875212599793019818600988496743e-2},
    {3.764030627004672750500754423692808e-1, 5.124858261884216138388134465196080e-1,
     1.111111111111111111111111111111111e-1}};
static const double rkC[3] = {1.550510257216821901802715925294109e-1,
                              6.449489742783178098197284074705891e-1, 1.0};
static const double rkE[4] = {0.05, -10.04880939982741556246032950764708 * 0.05,
                              1.382142733160748895793662840980412 * 0.05,
                              -0.3333333333333333333333333333333333 * 0.05};
static const double rkGamma = 3.637834252744495732208418513577775;
static const double rkAlpha = 2.681082873627752133895790743211112;
static const double rkBeta = 3.050430199247410569426377624787569;
static const double rkT[3][3] = {
    {9.443876248897524148749007950641664e-2, -1.412552950209542084279903838077973e-1,
     -3.00291941051474244918611170890539e-2},
    {2.502131229653333113765090675125018e-1, 2.041293522937999319959908102983381e-1,
     3.829421127572619377954382335998733e-1},
    {1.0, 1.0, 0.0e0}};
static const double rkTinvAinv[3][3] = {
    {1.520148562492775501049204957366528e+1, 1.192055789400527921212348994770778,
     1.903956760517560343018332287285119},
    {-9.669512977505946748632625374449567, -8.724028436822336183071773193986487,
     3.096043239482439656981667712714881},
    {-1.409513259499574544876303981551774e+1, 5.895975725255405108079130152868952,
     -1.441236197545344702389881889085515e-1}};
static const double rkELO = 4;

typedef struct {
    const or_config* c;
    const or_mech* m;
    int n;
    double pr;
    double* st;
} ctx;

static void rhs(ctx* x, double t, const double* y, double* f)
{
    or_dydt(x->m, t, x->pr, y, f);
    x->st[ST_RHS] += 1;
}

/* radau2a.c:256-278 */
static void decomp(ctx* x, double H, double* E1, double complex* E2, const double* Jac,
                   int* ipiv1, int* ipiv2, int* info)
{
    const int n = x->n;
    double complex temp2 = rkAlpha / H + I * rkBeta / H;
    double temp1 = rkGamma / H;
    for (int i = 0; i < n; i++) {
        for (int j = 0; j < n; j++) {
            E1[i + j * n] = -Jac[i + j * n];
            E2[i + j * n] = -Jac[i + j * n] + 0 * I;
        }
        E1[i + i * n] += temp1;
        E2[i + i * n] += temp2;
    }
    dgetrf_(&n, &n, E1, &n, ipiv1, info);
    x->st[ST_DECOMP] += 1;
    if (*info != 0) return;
    zgetrf_(&n, &n, E2, &n, ipiv2, info);
}

/* radau2a.c:283-297 */
static void make_interpolate(int n, const double* Z1, const double* Z2, const double* Z3, double* CONT)
{
    double den = (rkC[2] - rkC[1]) * (rkC[1] - rkC[0]) * (rkC[0] - rkC[2]);
    for (int i = 0; i < n; i++) {
        CONT[i] = ((-rkC[2] * rkC[2] * rkC[1] * Z1[i] + Z3[i] * rkC[1] * rkC[0] * rkC[0]
                    + rkC[1] * rkC[1] * rkC[2] * Z1[i] - rkC[1] * rkC[1] * rkC[0] * Z3[i]
                    + rkC[2] * rkC[2] * rkC[0] * Z2[i] - Z2[i] * rkC[2] * rkC[0] * rkC[0])
                   / den) - Z3[i];
        CONT[n + i] = -(rkC[0] * rkC[0] * (Z3[i] - Z2[i]) + rkC[1] * rkC[1] * (Z1[i] - Z3[i])
                        + rkC[2] * rkC[2] * (Z2[i] - Z1[i])) / den;
        CONT[n + n + i] = (rkC[0] * (Z3[i] - Z2[i]) + rkC[1] * (Z1[i] - Z3[i])
                           + rkC[2] * (Z2[i] - Z1[i])) / den;
    }
}

/* radau2a.c:302-314; Z3 uses x2 in the outer factor exactly as the reference does
 * (colloc = 0), or x3 (colloc = 1: the collocation polynomial at the third node) */
static void interpolate(int n, double H, double Hold, double* Z1, double* Z2, double* Z3, const double* CONT,
                        int colloc)
{
    double r = H / Hold;
    double x1 = 1.0 + rkC[0] * r;
    double x2 = 1.0 + rkC[1] * r;
    double x3 = 1.0 + rkC[2] * r;
    double x3o = colloc ? x3 : x2;
    for (int i = 0; i < n; i++) {
        Z1[i] = CONT[i] + x1 * (CONT[n + i] + x1 * CONT[n + n + i]);
        Z2[i] = CONT[i] + x2 * (CONT[n + i] + x2 * CONT[n + n + i]);
        Z3[i] = CONT[i] + x3o * (CONT[n + i] + x3 * CONT[n + n + i]);
    }
}

/* radau2a.c:353-383 */
static void prepare_rhs(ctx* x, double t, double H, const double* Y, const double* Z1,
                        const double* Z2, const double* Z3, double* R1, double* R2, double* R3)
{
    const int n = x->n;
    double TMP[OR_NMAX], F[OR_NMAX];
    for (int i = 0; i < n; i++) { R1[i] = Z1[i]; R2[i] = Z2[i]; R3[i] = Z3[i]; }
    const double* Zs[3] = {Z1, Z2, Z3};
    for (int s = 0; s < 3; ++s) {
        for (int i = 0; i < n; i++) TMP[i] = Y[i] + Zs[s][i];
        rhs(x, t + rkC[s] * H, TMP, F);
        double DA1 = -H * rkA[0][s], DA2 = -H * rkA[1][s], DA3 = -H * rkA[2][s];
        for (int i = 0; i < n; i++) {
            R1[i] += DA1 * F[i];
            R2[i] += DA2 * F[i];
            R3[i] += DA3 * F[i];
        }
    }
}

/* radau2a.c:388-441 */
static void solve(int n, double H, double* E1, double complex* E2, double* R1, double* R2, double* R3,
                  int* ipiv1, int* ipiv2)
{
    for (int i = 0; i < n; i++) {
        double x1 = R1[i] / H;
        double x2 = R2[i] / H;
        double x3 = R3[i] / H;
        R1[i] = rkTinvAinv[0][0] * x1 + rkTinvAinv[0][1] * x2 + rkTinvAinv[0][2] * x3;
        R2[i] = rkTinvAinv[1][0] * x1 + rkTinvAinv[1][1] * x2 + rkTinvAinv[1][2] * x3;
        R3[i] = rkTinvAinv[2][0] * x1 + rkTinvAinv[2][1] * x2 + rkTinvAinv[2][2] * x3;
    }
    int info = 0, one = 1;
    dgetrs_("N", &n, &one, E1, &n, ipiv1, R1, &n, &info);
    double complex temp[OR_NMAX];
    for (int i = 0; i < n; ++i) temp[i] = R2[i] + I * R3[i];
    zgetrs_("N", &n, &one, E2, &n, ipiv2, temp, &n, &info);
    for (int i = 0; i < n; ++i) { R2[i] = creal(temp[i]); R3[i] = cimag(temp[i]); }
    for (int i = 0; i < n; ++i) {
        double x1 = R1[i], x2 = R2[i], x3 = R3[i];
        R1[i] = rkT[0][0] * x1 + rkT[0][1] * x2 + rkT[0][2] * x3;
        R2[i] = rkT[1][0] * x1 + rkT[1][1] * x2 + rkT[1][2] * x3;
        R3[i] = rkT[2][0] * x1 + rkT[2][1] * x2 + rkT[2][2] * x3;
    }
}

/* radau2a.c:446-453 */
static double error_norm(int n, const double* scale, const double* DY)
{
    double sum = 0;
    for (int i = 0; i < n; ++i) sum += (scale[i] * scale[i] * DY[i] * DY[i]);
    return fmax(sqrt(sum / ((double)n)), 1e-10);
}

/* radau2a.c:458-508 */
static double error_estimate(ctx* x, double H, double t, const double* Y, const double* F0,
                             const double* Z1, const double* Z2, const double* Z3, const double* scale,
                             double* E1, int* ipiv1, bool FirstStep, bool Reject)
{
    const int n = x->n;
    double HrkE1 = rkE[1] / H, HrkE2 = rkE[2] / H, HrkE3 = rkE[3] / H;
    double F1[OR_NMAX], F2[OR_NMAX], TMP[OR_NMAX];
    for (int i = 0; i < n; ++i) F2[i] = HrkE1 * Z1[i] + HrkE2 * Z2[i] + HrkE3 * Z3[i];
    for (int i = 0; i < n; ++i) TMP[i] = rkE[0] * F0[i] + F2[i];
    int info = 0, one = 1;
    dgetrs_("N", &n, &one, E1, &n, ipiv1, TMP, &n, &info);
    x->st[ST_ERRSOLVE] += 1;
    double Err = error_norm(n, scale, TMP);
    if (Err >= 1.0 && (FirstStep || Reject)) {
        for (int i = 0; i < n; i++) TMP[i] += Y[i];
        rhs(x, t, TMP, F1);
        for (int i = 0; i < n; i++) TMP[i] = F1[i] + F2[i];
        dgetrs_("N", &n, &one, E1, &n, ipiv1, TMP, &n, &info);
        x->st[ST_ERRSOLVE] += 1;
        Err = error_norm(n, scale, TMP);
    }
    return Err;
}

/* radau2a.c:520-736 (adaptive branch; CONST_TIME_STEP is not part of the hot path) */
int or_radau2a(const or_config* c, const or_mech* m, double t_start, double t_end, double pr,
               double* y, double* st)
{
    ctx x = {c, m, m->n, pr, st};
    const int n = m->n;
    const double ATOL = c->atol, RTOL = c->rtol;
    double Hmin = 0, Hold = 0, Hacc = 0, ErrOld = 0;
    double H = fmin(5e-7, t_end - t_start);
    double Hnew;
    double t = t_start;
    bool Reject = false, FirstStep = true, SkipJac = false, SkipLU = false;
    double sc[OR_NMAX];
    double A[OR_NMAX * OR_NMAX] = {0.0};
    double E1[OR_NMAX * OR_NMAX] = {0};
    double complex E2[OR_NMAX * OR_NMAX] = {0};
    int ipiv1[OR_NMAX] = {0}, ipiv2[OR_NMAX] = {0};
    double Z1[OR_NMAX] = {0}, Z2[OR_NMAX] = {0}, Z3[OR_NMAX] = {0};
    double DZ1[OR_NMAX] = {0}, DZ2[OR_NMAX] = {0}, DZ3[OR_NMAX] = {0};
    double CONT[OR_NMAX * 3] = {0};
    for (int i = 0; i < n; ++i) sc[i] = 1.0 / (ATOL + fabs(y[i]) * RTOL);
    double y0[OR_NMAX];
    memcpy(y0, y, n * sizeof(double));
    double F0[OR_NMAX];
    int info = 0, Nconsecutive = 0, Nsteps = 0;
    double NewtonRate = pow(2.0, 1.25);

    while (t + ROUNDOFF < t_end) {
        if (!Reject) rhs(&x, t, y, F0);
        if (!SkipLU) {
            if (!SkipJac) {
                or_jacob(m, t, pr, y, A);
                st[ST_JAC] += 1;
            }
            decomp(&x, H, E1, E2, A, ipiv1, ipiv2, &info);
            if (info != 0) {
                Nconsecutive += 1;
                if (Nconsecutive >= MAX_CONSECUTIVE_ERRS) return 1;  /* EC_consecutive_steps */
                H *= 0.5;
                Reject = true;
                SkipJac = true;
                SkipLU = false;
                st[ST_REJECT] += 1;
                continue;
            } else {
                Nconsecutive = 0;
            }
        }
        Nsteps += 1;
        st[ST_STEPS] += 1;
        if (Nsteps >= (c->max_steps > 0 ? c->max_steps : MAX_NO_STEPS)) return 2;   /* EC_max_steps_exceeded */
        if (0.1 * fabs(H) <= fabs(t) * ROUNDOFF) return 3;           /* EC_h_plus_t_equals_h */
        if (FirstStep) {
            memset(Z1, 0, n * sizeof(double));
            memset(Z2, 0, n * sizeof(double));
            memset(Z3, 0, n * sizeof(double));
        } else {
            interpolate(n, H, Hold, Z1, Z2, Z3, CONT, c->stage_extrap);
        }
        bool NewtonDone = false;
        double NewtonIncrementOld = 0;
        double Fac = 0.5;
        int NewtonIter = 0;
        double Theta = 0;
        NewtonRate = pow(fmax(NewtonRate, DBL_EPSILON), 0.8);
        for (; NewtonIter < NEWTON_MAXIT; NewtonIter++) {
            st[ST_NEWTON] += 1;
            prepare_rhs(&x, t, H, y, Z1, Z2, Z3, DZ1, DZ2, DZ3);
            solve(n, H, E1, E2, DZ1, DZ2, DZ3, ipiv1, ipiv2);
            double d1 = error_norm(n, sc, DZ1);
            double d2 = error_norm(n, sc, DZ2);
            double d3 = error_norm(n, sc, DZ3);
            double NewtonIncrement = sqrt((d1 * d1 + d2 * d2 + d3 * d3) / 3.0);
            Theta = THETA_MIN;
            if (NewtonIter > 0) {
                Theta = NewtonIncrement / NewtonIncrementOld;
                if (Theta < 0.99) {
                    NewtonRate = Theta / (1.0 - Theta);
                } else {
                    break;
                }
                if (NewtonIter < NEWTON_MAXIT) {
                    double NewtonPredictedErr =
                        (NewtonIncrement * pow(Theta, (NEWTON_MAXIT - NewtonIter - 1))) / (1.0 - Theta);
                    if (NewtonPredictedErr >= NEWTON_TOL) {
                        double Qnewton = fmin(10.0, NewtonPredictedErr / NEWTON_TOL);
                        Fac = 0.8 * pow(Qnewton, -1.0 / ((double)(NEWTON_MAXIT - NewtonIter)));
                        break;
                    }
                }
            }
            NewtonIncrementOld = fmax(NewtonIncrement, ROUNDOFF);
            for (int i = 0; i < n; i++) {
                Z1[i] -= DZ1[i];
                Z2[i] -= DZ2[i];
                Z3[i] -= DZ3[i];
            }
            NewtonDone = (NewtonRate * NewtonIncrement <= NEWTON_TOL);
            if (NewtonDone) break;
            if (NewtonIter == NEWTON_MAXIT - 1) return 4;           /* EC_newton_max_iterations_exceeded */
        }
        if (!NewtonDone) {
            H = Fac * H;
            Reject = true;
            SkipJac = true;
            SkipLU = false;
            st[ST_REJECT] += 1;
            continue;
        }
        double Err = error_estimate(&x, H, t, y, F0, Z1, Z2, Z3, sc, E1, ipiv1, FirstStep, Reject);
        Fac = pow(Err, (-1.0 / rkELO)) * (1.0 + 2 * NEWTON_MAXIT) / (NewtonIter + 1.0 + 2 * NEWTON_MAXIT);
        Fac = fmin(FAC_MAX, fmax(FAC_MIN, Fac));
        Hnew = Fac * H;
        if (Err < 1.0) {
            if (!FirstStep) {
                double FacGus = FAC_SAFE * (H / Hacc) * pow(Err * Err / ErrOld, -0.25);
                FacGus = fmin(FAC_MAX, fmax(FAC_MIN, FacGus));
                Fac = fmin(Fac, FacGus);
                Hnew = Fac * H;
            }
            Hacc = H;
            ErrOld = fmax(1e-2, Err);
            FirstStep = false;
            Hold = H;
            t += H;
            st[ST_ACCEPT] += 1;
            for (int i = 0; i < n; i++) y[i] += Z3[i];
            make_interpolate(n, Z1, Z2, Z3, CONT);
            for (int i = 0; i < n; ++i) sc[i] = 1.0 / (ATOL + fmax(fabs(y[i]), fabs(y0[i])) * RTOL);
            memcpy(y0, y, n * sizeof(double));
            Hnew = fmin(fmax(Hnew, Hmin), t_end - t);
            if (Reject) Hnew = fmin(Hnew, H);
            Reject = false;
            if (t + Hnew / Q_MIN - t_end >= 0.0) {
                H = t_end - t;
            } else {
                double Hratio = Hnew / H;
                SkipLU = (Theta <= THETA_MIN) && (Hratio >= Q_MIN) && (Hratio <= Q_MAX);
                if (!SkipLU) H = Hnew;
            }
            SkipJac = NewtonIter == 1 || NewtonRate <= THETA_MIN;
        } else {
            if (FirstStep || Reject) {
                H = FAC_REJ * H;
            } else {
                H = Hnew;
            }
            Reject = true;
            SkipJac = true;
            SkipLU = false;
            st[ST_REJECT] += 1;
        }
    }
    return 0;
}
