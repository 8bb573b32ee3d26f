/*
 * ORACLE / TEST INFRASTRUCTURE.  The Krylov exponential integrators restated
 * from the reference (paths relative to its repository):
 *   exponential_integrators/arnoldi.h:26-141            arnoldi()
 *   exponential_integrators/phiAHessenberg.c:83-184     phiAc_variable / expAc_variable
 *   generic/complexInverse.c:35-248                     Hessenberg LU and inverse
 *   exponential_integrators/exponential_linear_algebra.h:28-402  vector helpers
 *   exponential_integrators/exprb43/exprb43.c:47-309    EXPRB43
 *   exponential_integrators/exp4/exp4.c:46-320          EXP4
 * The state length is a run-time value; Hm/phiHm use the leading dimension
 * STRIDE = n + P exactly as the reference (P = 4 for exprb43, 1 for exp4).
 */
#include <complex.h>
#include <math.h>
#include <float.h>
#include <string.h>
#include <stdbool.h>
#include "oracle.h"

/* arnoldi.h:26 */
static const int index_list[23] = {1, 2, 3, 4, 5, 6, 7, 9, 11, 14, 17, 21, 27, 34, 42, 53, 67, 84,
                                   106, 133, 167, 211, 265};

/* complexInverse.c:35-74 */
int or_hessenberg_lu(int n, int stride, double complex* A, int* indPivot)
{
    int last_pivot = 0;
    for (int i = 0; i < n - 1; i++) {
        if (cabs(A[i * stride + i]) < cabs(A[i * stride + i + 1])) {
            for (int k = last_pivot; k < n; ++k) {
                double complex temp = A[k * stride + i];
                A[k * stride + i] = A[k * stride + i + 1];
                A[k * stride + i + 1] = temp;
            }
            indPivot[i] = i + 1;
        } else {
            indPivot[i] = i;
            last_pivot = i;
        }
        if (cabs(A[i * stride + i]) > 0.0) {
            double complex tau = A[i * stride + i + 1] / A[i * stride + i];
            for (int j = i + 1; j < n; j++) A[j * stride + i + 1] -= tau * A[j * stride + i];
            A[i * stride + i + 1] = tau;
        } else {
            return i;
        }
    }
    indPivot[n - 1] = n - 1;
    return 0;
}

/* complexInverse.c:108-123 */
static void upper_mv(int n, double complex* x, int lda, const double complex* A)
{
    for (int j = 0; j < n; ++j) {
        if (cabs(x[j]) > 0.0) {
            double complex temp = x[j];
            for (int i = 0; i < j; ++i) x[i] += temp * A[i + (lda * j)];
            x[j] *= A[j + (lda * j)];
        }
    }
}

/* complexInverse.c:146-164 */
static void cgemv(int m, int n, int lda, double alpha, const double complex* A, const double complex* x,
                  double complex* y)
{
    for (int j = 0; j < n - 1; ++j) {
        if (cabs(x[j]) > 0.0) {
            double complex temp = alpha * x[j];
            for (int i = 0; i < m; ++i) y[i] += temp * A[i + (lda * j)];
        }
    }
}

/* complexInverse.c:178-227 */
static int inverse_hessenberg_lu(int n, int stride, double complex* A, const int* indPivot)
{
    double complex work[OR_STRIDE_MAX] = {0};
    for (int j = 0; j < n; ++j) {
        if (cabs(A[j + (stride * j)]) == 0) return j;
        A[j + (stride * j)] = 1.0 / A[j + (stride * j)];
        double complex Ajj = -A[j + (stride * j)];
        upper_mv(j, &A[stride * j], stride, A);
        for (int i = 0; i < j; ++i) A[stride * j + i] *= Ajj;
    }
    for (int j = n - 1; j >= 0; --j) {
        for (int i = j + 1; i < n; ++i) {
            work[i] = A[i + stride * j];
            A[i + (stride * j)] = 0;
        }
        if (j < n - 1) cgemv(n, n - j, stride, -1, &A[stride * (j + 1)], &work[j + 1], &A[stride * j]);
    }
    for (int j = n - 2; j >= 0; --j) {
        if (indPivot[j] != j) {
            for (int i = 0; i < n; ++i) {
                double complex temp = A[stride * j + i];
                A[stride * j + i] = A[stride * indPivot[j] + i];
                A[stride * indPivot[j] + i] = temp;
            }
        }
    }
    return 0;
}

/* complexInverse.c:238-248 */
int or_complex_inverse_hessenberg(int n, int stride, double complex* A, int* ipiv)
{
    int info = or_hessenberg_lu(n, stride, A, ipiv);
    if (info != 0) return info;
    return inverse_hessenberg_lu(n, stride, A, ipiv);
}

/* phiAHessenberg.c:83-127 (order 1) and :140-184 (order 0) */
int or_phi_ac(const or_config* c, int order, int m, int stride, const double* A, double cs, double* phiA)
{
    int ipiv[OR_STRIDE_MAX] = {0};
    double complex invA[OR_STRIDE_MAX * OR_STRIDE_MAX];
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) phiA[i + j * stride] = 0.0;
    for (int q = 0; q < OR_NRA; q += 2) {
        const double complex pole = c->poles_re[q] + c->poles_im[q] * I;
        const double complex res = c->res_re[q] + c->res_im[q] * I;
        for (int i = 0; i < m; ++i) {
            for (int j = 0; j < m; ++j) {
                if (i == j) invA[i + j * stride] = cs * A[i + j * stride] - pole;
                else invA[i + j * stride] = cs * A[i + j * stride];
            }
        }
        int info = or_complex_inverse_hessenberg(m, stride, invA, ipiv);
        if (info != 0) return info;
        for (int i = 0; i < m; ++i) {
            for (int j = 0; j < m; ++j) {
                if (order == 0) phiA[i + j * stride] += 2.0 * creal(res * invA[i + j * stride]);
                else phiA[i + j * stride] += 2.0 * creal((res / pole) * invA[i + j * stride]);
            }
        }
    }
    return 0;
}

/* ---- exponential_linear_algebra.h helpers (n = state length) ---- */
static double sc_norm(int n, const double* nums, const double* sc)
{
    double norm = 0.0;
    for (int i = 0; i < n; ++i) norm += nums[i] * nums[i] * sc[i] * sc[i];
    return sqrt(norm / n);
}

static double two_norm(int n, const double* v)
{
    double norm = 0.0;
    for (int i = 0; i < n; ++i) norm += v[i] * v[i];
    return sqrt(norm);
}

static double normalize(int n, const double* v, double* v_out)
{
    double norm = two_norm(n, v);
    if (norm == 0) norm = 1;
    double m_norm = 1.0 / norm;
    for (int i = 0; i < n; ++i) v_out[i] = v[i] * m_norm;
    return norm;
}

static double dotproduct(int n, const double* w, const double* Vm)
{
    double sum = 0;
    for (int i = 0; i < n; i++) sum += w[i] * Vm[i];
    return sum;
}

/* matvec_m_by_m (:28-40) and its (A + I) form (:54-70) */
static void matvec_m_by_m(int m, int stride, const double* A, const double* V, double* Av, bool plus_eye)
{
    for (int i = 0; i < m; ++i) {
        Av[i] = A[i] * V[0];
        for (int j = 1; j < m; ++j) Av[i] += A[j * stride + i] * V[j];
        if (plus_eye) Av[i] += V[i];
    }
}

/* matvec_n_by_m_scale (:84-100), _scale_add (:193-208), _scale_add_subtract (:227-244) */
static void matvec_n_by_m(int n, int m, double scale, const double* A, const double* V, double* Av,
                          const double* add, const double* sub)
{
    for (int i = 0; i < n; ++i) {
        Av[i] = A[i] * V[0];
        for (int j = 1; j < m; ++j) Av[i] += A[j * n + i] * V[j];
        if (!add) Av[i] *= scale;
        else if (!sub) Av[i] = Av[i] * scale + add[i];
        else Av[i] = Av[i] * scale + 2.0 * add[i] - sub[i];
    }
}

/* arnoldi.h:45-141.  stride = n + P of the calling method; order 0 (exprb43) or 1 (exp4). */
static int arnoldi(const or_config* c, const or_mech* mech, int order, int stride, double scale, int p,
                   double h, const double* A, const double* v, const double* sc, double* beta,
                   double* Vm, double* Hm, double* phiHm)
{
    const int n = mech->n;
    double w[OR_NMAX];
    *beta = normalize(n, v, Vm);
    double store = 0;
    int index = 0;
    int j = 0;
    double err = 2.0;
    while (err > 1.0) {
        for (; j < index_list[index] && j + p < stride; j++) {
            or_jacvec(mech, A, &Vm[j * n], w);
            for (int i = 0; i <= j; i++) {
                Hm[j * stride + i] = dotproduct(n, w, &Vm[i * n]);
                const double s = Hm[j * stride + i];
                for (int k = 0; k < n; k++) w[k] -= s * Vm[i * n + k];
            }
            Hm[j * stride + j + 1] = two_norm(n, w);
            if (fabs(Hm[j * stride + j + 1]) < c->atol) {
                j++;
                break;
            }
            const double s = 1.0 / Hm[j * stride + j + 1];
            for (int k = 0; k < n; k++) Vm[(j + 1) * n + k] = w[k] * s;
        }
        if (j + p >= stride) return j;
        index++;
        store = Hm[(j - 1) * stride + j];
        Hm[(j - 1) * stride + j] = 0.0;
        memset(&Hm[j * stride], 0, (j + 2) * sizeof(double));
        Hm[(j)*stride] = 1.0;
        for (int i = 1; i < p; i++) {
            memset(&Hm[(j + i) * stride], 0, (j + i + 2) * sizeof(double));
            Hm[(j + i) * stride + (j + i - 1)] = 1.0;
        }
        int info = or_phi_ac(c, order, j + p, stride, Hm, h * scale, phiHm);
        if (info != 0) return -info;
        err = h * (*beta) * fabs(store * phiHm[(j)*stride + (j)-1]) * sc_norm(n, &Vm[(j)*n], sc);
        Hm[(j - 1) * stride + j] = store;
        Hm[(j)*stride] = 0.0;
    }
    return j;
}

#define MAX_CONSECUTIVE_ERRORS 5

/* exprb43.c:47-309 (P = 4, ORD = 3, MAX_STEPS = 100000; exprb43_props.h:334-343) */
int or_exprb43(const or_config* c, const or_mech* mech, double t_start, double t_end, double pr,
               double* y, double* st)
{
    const int n = mech->n, P = 4, stride = n + 4;
    const double ORD = 3.0, ATOL = c->atol, RTOL = c->rtol;
    double h = fmin(1.0e-8, t_end - t_start);
    double h_new, err_old = 1.0, h_old = h;
    bool reject = false;
    int failures = 0, steps = 0;
    double t = t_start;
    double sc[OR_NMAX];
    for (int i = 0; i < n; ++i) sc[i] = 1.0 / (ATOL + fabs(y[i]) * RTOL);
    double beta = 0;
    double temp[OR_NMAX], f_temp[OR_NMAX], y1[OR_NMAX], fy[OR_NMAX], gy[OR_NMAX];
    double A[OR_NMAX * OR_NMAX] = {0.0};
    double Hm[OR_STRIDE_MAX * OR_STRIDE_MAX];
    for (int i = 0; i < OR_STRIDE_MAX * OR_STRIDE_MAX; ++i) Hm[i] = 0.0;
    /* zero-initialised: arnoldi() reads basis column j after a happy breakdown
     * without writing it (arnoldi.h:118); the reference leaves it uninitialised */
    double Vm[OR_NMAX * OR_STRIDE_MAX], phiHm[OR_STRIDE_MAX * OR_STRIDE_MAX];
    for (int i = 0; i < OR_NMAX * OR_STRIDE_MAX; ++i) Vm[i] = 0.0;
    for (int i = 0; i < OR_STRIDE_MAX * OR_STRIDE_MAX; ++i) phiHm[i] = 0.0;
    double err = 0.0;
    double savedActions[OR_NMAX * 5];
    (void)P;
    while ((t < t_end) && (t + h > t)) {
        if (failures >= 5) return 1;
        if (steps++ >= 100000) return 2;
        if (t + h <= t) return 3;
        st[ST_STEPS] += 1;
        if (!reject) {
            or_dydt(mech, t, pr, y, fy);
            or_jacob(mech, t, pr, y, A);
            st[ST_RHS] += 1;
            st[ST_JAC] += 1;
            or_jacvec(mech, A, y, gy);
            for (int i = 0; i < n; ++i) gy[i] = fy[i] - gy[i];
        }
        int m = arnoldi(c, mech, 0, stride, 0.5, 1, h, A, fy, sc, &beta, Vm, Hm, phiHm);
        st[ST_ARNOLDI] += 1;
        st[ST_KRYLOV] += m > 0 ? m : 0;
        if (m + 1 >= stride || m < 0) {
            h /= 5.0;
            failures++;
            reject = true;
            st[ST_REJECT] += 1;
            continue;
        }
        matvec_m_by_m(m, stride, phiHm, &phiHm[m * stride], temp, true);
        matvec_n_by_m(n, m, beta, Vm, temp, savedActions, NULL, NULL);
        matvec_n_by_m(n, m, beta, Vm, &phiHm[m * stride], temp, y, NULL);
        or_dydt(mech, t, pr, temp, &savedActions[n]);
        st[ST_RHS] += 1;
        or_jacvec(mech, A, temp, f_temp);
        for (int i = 0; i < n; ++i) temp[i] = savedActions[n + i] - f_temp[i] - gy[i];
        int m1 = arnoldi(c, mech, 0, stride, 1.0, 4, h, A, temp, sc, &beta, Vm, Hm, phiHm);
        st[ST_ARNOLDI] += 1;
        st[ST_KRYLOV] += m1 > 0 ? m1 : 0;
        if (m1 + 4 >= stride || m1 < 0) {
            h /= 5.0;
            failures++;
            reject = true;
            st[ST_REJECT] += 1;
            continue;
        }
        /* matvec_n_by_m_scale_special (exponential_linear_algebra.h:118-139) */
        {
            const double* in0 = &phiHm[(m1 + 2) * stride];
            const double* in1 = &phiHm[(m1 + 3) * stride];
            const double* in2 = &phiHm[m1 * stride];
            double s0 = beta / (h * h), s1 = beta / (h * h * h), s2 = beta;
            for (int i = 0; i < n; ++i) {
                double a0 = Vm[i] * in0[0], a1 = Vm[i] * in1[0], a2 = Vm[i] * in2[0];
                for (int j = 1; j < m1; ++j) {
                    a0 += Vm[j * n + i] * in0[j];
                    a1 += Vm[j * n + i] * in1[j];
                    a2 += Vm[j * n + i] * in2[j];
                }
                savedActions[n + i] = a0 * s0;
                savedActions[2 * n + i] = a1 * s1;
                temp[i] = a2 * s2 + savedActions[i] + y[i];
            }
        }
        or_dydt(mech, t, pr, temp, &savedActions[3 * n]);
        st[ST_RHS] += 1;
        or_jacvec(mech, A, temp, f_temp);
        for (int i = 0; i < n; ++i) temp[i] = savedActions[3 * n + i] - f_temp[i] - gy[i];
        int m2 = arnoldi(c, mech, 0, stride, 1.0, 4, h, A, temp, sc, &beta, Vm, Hm, phiHm);
        st[ST_ARNOLDI] += 1;
        st[ST_KRYLOV] += m2 > 0 ? m2 : 0;
        if (m2 + 4 >= stride || m2 < 0) {
            h /= 5.0;
            failures++;
            reject = true;
            st[ST_REJECT] += 1;
            continue;
        }
        /* matvec_n_by_m_scale_special2 (:158-176) */
        {
            const double* in0 = &phiHm[(m2 + 2) * stride];
            const double* in1 = &phiHm[(m2 + 3) * stride];
            double s0 = beta / (h * h), s1 = beta / (h * h * h);
            for (int i = 0; i < n; ++i) {
                double a0 = Vm[i] * in0[0], a1 = Vm[i] * in1[0];
                for (int j = 1; j < m2; ++j) {
                    a0 += Vm[j * n + i] * in0[j];
                    a1 += Vm[j * n + i] * in1[j];
                }
                savedActions[3 * n + i] = a0 * s0;
                savedActions[4 * n + i] = a1 * s1;
            }
        }
        for (int i = 0; i < n; ++i) {
            y1[i] = y[i] + savedActions[i] + 16.0 * savedActions[n + i] - 48.0 * savedActions[2 * n + i]
                    + -2.0 * savedActions[3 * n + i] + 12.0 * savedActions[4 * n + i];
            temp[i] = 48.0 * savedActions[2 * n + i] - 12.0 * savedActions[4 * n + i];
        }
        for (int i = 0; i < n; ++i) f_temp[i] = 1.0 / (ATOL + fmax(fabs(y[i]), fabs(y1[i])) * RTOL);
        err = fmax(DBL_EPSILON, sc_norm(n, temp, f_temp));
        h_new = pow(err, -1.0 / ORD);
        failures = 0;
        if (err <= 1.0) {
            memcpy(sc, f_temp, n * sizeof(double));
            h_new = fmin(h_new, (h / h_old) * pow((err_old / (err * err)), (1.0 / ORD)));
            h_new = h * fmax(fmin(0.9 * h_new, 8.0), 0.2);
            for (int i = 0; i < n; ++i) y[i] = y1[i];
            t += h;
            st[ST_ACCEPT] += 1;
            err_old = fmax(1.0e-2, err);
            h_old = h;
            if (reject) {
                reject = false;
                h_new = fmin(h, h_new);
            }
            h = fmin(h_new, t_end - t);
        } else {
            h_new = h * fmax(fmin(0.9 * h_new, 8.0), 0.2);
            h_new = fmin(h_new, t_end - t);
            reject = true;
            st[ST_REJECT] += 1;
            h = fmin(h, h_new);
        }
    }
    return 0;
}

/* exp4.c:46-320 (P = 1, ORD = 3, MAX_STEPS = 100000 on the CPU; exp4_props.h:600-610) */
int or_exp4(const or_config* c, const or_mech* mech, double t_start, double t_end, double pr,
            double* y, double* st)
{
    const int n = mech->n, P = 1, stride = n + 1;
    const double ORD = 3.0, ATOL = c->atol, RTOL = c->rtol;
    double h = fmin(1.0e-8, t_end - t_start);
    double h_new, err_old = 1.0, h_old = h;
    bool reject = false;
    int failures = 0, steps = 0;
    double t = t_start;
    double sc[OR_NMAX];
    for (int i = 0; i < n; ++i) sc[i] = 1.0 / (ATOL + fabs(y[i]) * RTOL);
    double beta = 0;
    double fy[OR_NMAX];
    double A[OR_NMAX * OR_NMAX] = {0.0};
    double temp[OR_NMAX], f_temp[OR_NMAX], y1[OR_NMAX];
    double Hm[OR_STRIDE_MAX * OR_STRIDE_MAX];
    for (int i = 0; i < OR_STRIDE_MAX * OR_STRIDE_MAX; ++i) Hm[i] = 0.0;
    double Vm[OR_NMAX * OR_STRIDE_MAX], phiHm[OR_STRIDE_MAX * OR_STRIDE_MAX];
    for (int i = 0; i < OR_NMAX * OR_STRIDE_MAX; ++i) Vm[i] = 0.0;   /* see or_exprb43 */
    for (int i = 0; i < OR_STRIDE_MAX * OR_STRIDE_MAX; ++i) phiHm[i] = 0.0;
    double err = 0.0;
    double k1[OR_NMAX], k2[OR_NMAX], k3[OR_NMAX], k4[OR_NMAX], k5[OR_NMAX], k6[OR_NMAX], k7[OR_NMAX];
    while ((t < t_end) && (t + h > t)) {
        if (failures >= MAX_CONSECUTIVE_ERRORS) return 1;
        if (steps++ >= 100000) return 2;
        if (t + h <= t) return 3;
        st[ST_STEPS] += 1;
        if (!reject) {
            or_dydt(mech, t, pr, y, fy);
            or_jacob(mech, t, pr, y, A);
            st[ST_RHS] += 1;
            st[ST_JAC] += 1;
        }
        int m = arnoldi(c, mech, 1, stride, 1.0 / 3.0, P, h, A, fy, sc, &beta, Vm, Hm, phiHm);
        st[ST_ARNOLDI] += 1;
        st[ST_KRYLOV] += m > 0 ? m : 0;
        if (m + P >= stride || m < 0) {
            h /= 5.0;
            failures++;
            reject = true;
            st[ST_REJECT] += 1;
            continue;
        }
        matvec_n_by_m(n, m, beta, Vm, phiHm, k1, NULL, NULL);
        matvec_m_by_m(m, stride, phiHm, phiHm, temp, false);
        matvec_m_by_m(m, stride, Hm, temp, f_temp, false);
        matvec_n_by_m(n, m, beta * (h / 6.0), Vm, f_temp, k2, k1, NULL);
        matvec_m_by_m(m, stride, phiHm, f_temp, temp, false);
        matvec_m_by_m(m, stride, Hm, temp, f_temp, false);
        matvec_n_by_m(n, m, beta * (h * h / 27.0), Vm, f_temp, k3, k2, k1);
        for (int i = 0; i < n; ++i) {
            f_temp[i] = h * ((-7.0 / 300.0) * k1[i] + (97.0 / 150.0) * k2[i] - (37.0 / 300.0) * k3[i]);
            k4[i] = y[i] + f_temp[i];
        }
        or_dydt(mech, t, pr, k4, temp);
        st[ST_RHS] += 1;
        or_jacvec(mech, A, f_temp, k4);
        for (int i = 0; i < n; ++i) k4[i] = temp[i] - fy[i] - k4[i];
        int m1 = arnoldi(c, mech, 1, stride, 1.0 / 3.0, P, h, A, k4, sc, &beta, Vm, Hm, phiHm);
        st[ST_ARNOLDI] += 1;
        st[ST_KRYLOV] += m1 > 0 ? m1 : 0;
        if (m1 + P >= stride || m1 < 0) {
            h /= 5.0;
            failures++;
            reject = true;
            st[ST_REJECT] += 1;
            continue;
        }
        matvec_n_by_m(n, m1, beta, Vm, phiHm, k4, NULL, NULL);
        matvec_m_by_m(m1, stride, phiHm, phiHm, temp, false);
        matvec_m_by_m(m1, stride, Hm, temp, f_temp, false);
        matvec_n_by_m(n, m1, beta * (h / 6.0), Vm, f_temp, k5, k4, NULL);
        matvec_m_by_m(m1, stride, phiHm, f_temp, temp, false);
        matvec_m_by_m(m1, stride, Hm, temp, f_temp, false);
        matvec_n_by_m(n, m1, beta * (h * h / 27.0), Vm, f_temp, k6, k5, k4);
        for (int i = 0; i < n; ++i) {
            f_temp[i] = h * ((59.0 / 300.0) * k1[i] - (7.0 / 75.0) * k2[i] + (269.0 / 300.0) * k3[i]
                             + (2.0 / 3.0) * (k4[i] + k5[i] + k6[i]));
            k7[i] = y[i] + f_temp[i];
        }
        or_dydt(mech, t, pr, k7, temp);
        st[ST_RHS] += 1;
        or_jacvec(mech, A, f_temp, k7);
        for (int i = 0; i < n; ++i) k7[i] = temp[i] - fy[i] - k7[i];
        int m2 = arnoldi(c, mech, 1, stride, 1.0 / 3.0, P, h, A, k7, sc, &beta, Vm, Hm, phiHm);
        st[ST_ARNOLDI] += 1;
        st[ST_KRYLOV] += m2 > 0 ? m2 : 0;
        if (m2 + P >= stride || m2 < 0) {
            h /= 5.0;
            failures++;
            reject = true;
            st[ST_REJECT] += 1;
            continue;
        }
        matvec_n_by_m(n, m2, beta / (h / 3.0), Vm, &phiHm[m2 * stride], k7, NULL, NULL);
        for (int i = 0; i < n; ++i)
            y1[i] = y[i] + h * (k3[i] + k4[i] - (4.0 / 3.0) * k5[i] + k6[i] + (1.0 / 6.0) * k7[i]);
        for (int i = 0; i < n; ++i) f_temp[i] = 1.0 / (ATOL + fmax(fabs(y[i]), fabs(y1[i])) * RTOL);
        for (int i = 0; i < n; ++i)
            temp[i] = k3[i] - (2.0 / 3.0) * k5[i] + 0.5 * (k6[i] + k7[i] - k4[i]) - (y1[i] - y[i]) / h;
        err = h * sc_norm(n, temp, f_temp);
        for (int i = 0; i < n; ++i) temp[i] = -k1[i] + 2.0 * k2[i] - k4[i] + k7[i] - (y1[i] - y[i]) / h;
        err = fmax(DBL_EPSILON, fmin(err, h * sc_norm(n, temp, f_temp)));
        h_new = pow(err, -1.0 / ORD);
        failures = 0;
        if (err <= 1.0) {
            h_new = fmin(h_new, (h / h_old) * pow((err_old / (err * err)), (1.0 / ORD)));
            h_new = h * fmax(fmin(0.9 * h_new, 8.0), 0.2);
            memcpy(sc, f_temp, n * sizeof(double));
            memcpy(y, y1, n * sizeof(double));
            t += h;
            st[ST_ACCEPT] += 1;
            err_old = fmax(1.0e-2, err);
            h_old = h;
            if (reject) {
                reject = false;
                h_new = fmin(h, h_new);
            }
            h = fmin(h_new, t_end - t);
        } else {
            h_new = h * fmax(fmin(0.9 * h_new, 8.0), 0.2);
            h_new = fmin(h_new, t_end - t);
            reject = true;
            st[ST_REJECT] += 1;
            h = fmin(h, h_new);
        }
    }
    return 0;
}
