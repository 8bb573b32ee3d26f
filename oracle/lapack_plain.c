/*
 * ORACLE / TEST INFRASTRUCTURE -- not part of the product path.
 *
 * Plain-C LU factorisation and solve with LAPACK semantics (unblocked
 * right-looking partial pivoting, as LAPACK's xGETF2 + xGETRS):
 *
 *   dgetrf_ / zgetrf_  : pivot = first index of max |a| (real) or
 *                        max |Re a| + |Im a| (complex, LAPACK izamax/dcabs1);
 *                        rows swapped physically; column scaled by the
 *                        reciprocal of the pivot; rank-1 update column by
 *                        column, skipping zero multipliers of the pivot row.
 *   dgetrs_ / zgetrs_  : 'N' only, one or more right-hand sides; apply the
 *                        interchanges, unit-lower forward then upper backward
 *                        substitution, column oriented, skipping zero entries.
 *
 * accelerInt calls these through generic/lapack_dfns.h:353-356 from
 * radau2a/radau2a.c:273,277,404,417,479,498.  The reference links MKL by
 * default (SConstruct:124-129, unversioned); this unblocked form is used both
 * by the oracle restatement and by the build of the reference's own C sources
 * under oracle/_ref, so the two agree operation for operation.
 */
#include <complex.h>
#include <math.h>
#include <float.h>
#include "lapack_plain.h"

void dgetrf_(const int* m_, const int* n_, double* A, const int* lda_, int* ipiv, int* info)
{
    const int m = *m_, n = *n_, lda = *lda_;
    const int mn = m < n ? m : n;
    *info = 0;
    for (int j = 0; j < mn; ++j) {
        int jp = j;
        double amax = fabs(A[j + j * lda]);
        for (int i = j + 1; i < m; ++i) {
            double a = fabs(A[i + j * lda]);
            if (a > amax) { amax = a; jp = i; }
        }
        ipiv[j] = jp + 1;
        if (A[jp + j * lda] != 0.0) {
            if (jp != j) {
                for (int k = 0; k < n; ++k) {
                    double t = A[j + k * lda];
                    A[j + k * lda] = A[jp + k * lda];
                    A[jp + k * lda] = t;
                }
            }
            if (fabs(A[j + j * lda]) >= DBL_MIN) {
                double r = 1.0 / A[j + j * lda];
                for (int i = j + 1; i < m; ++i) A[i + j * lda] *= r;
            } else {
                for (int i = j + 1; i < m; ++i) A[i + j * lda] /= A[j + j * lda];
            }
        } else if (*info == 0) {
            *info = j + 1;
        }
        for (int k = j + 1; k < n; ++k) {
            double u = A[j + k * lda];
            if (u != 0.0) {
                double t = -u;
                for (int i = j + 1; i < m; ++i) A[i + k * lda] += A[i + j * lda] * t;
            }
        }
    }
}

static inline double cabs1(double complex z) { return fabs(creal(z)) + fabs(cimag(z)); }

void zgetrf_(const int* m_, const int* n_, double complex* A, const int* lda_, int* ipiv, int* info)
{
    const int m = *m_, n = *n_, lda = *lda_;
    const int mn = m < n ? m : n;
    *info = 0;
    for (int j = 0; j < mn; ++j) {
        int jp = j;
        double amax = cabs1(A[j + j * lda]);
        for (int i = j + 1; i < m; ++i) {
            double a = cabs1(A[i + j * lda]);
            if (a > amax) { amax = a; jp = i; }
        }
        ipiv[j] = jp + 1;
        if (A[jp + j * lda] != 0.0) {
            if (jp != j) {
                for (int k = 0; k < n; ++k) {
                    double complex t = A[j + k * lda];
                    A[j + k * lda] = A[jp + k * lda];
                    A[jp + k * lda] = t;
                }
            }
            double complex r = 1.0 / A[j + j * lda];
            for (int i = j + 1; i < m; ++i) A[i + j * lda] *= r;
        } else if (*info == 0) {
            *info = j + 1;
        }
        for (int k = j + 1; k < n; ++k) {
            double complex u = A[j + k * lda];
            if (u != 0.0) {
                double complex t = -u;
                for (int i = j + 1; i < m; ++i) A[i + k * lda] += A[i + j * lda] * t;
            }
        }
    }
}

void dgetrs_(const char* trans, const int* n_, const int* nrhs_, double* A, const int* lda_,
             int* ipiv, double* B, const int* ldb_, int* info)
{
    (void)trans;
    const int n = *n_, nrhs = *nrhs_, lda = *lda_, ldb = *ldb_;
    *info = 0;
    for (int c = 0; c < nrhs; ++c) {
        double* b = B + c * ldb;
        for (int i = 0; i < n; ++i) {
            int p = ipiv[i] - 1;
            if (p != i) { double t = b[i]; b[i] = b[p]; b[p] = t; }
        }
        for (int j = 0; j < n; ++j) {
            if (b[j] != 0.0) {
                for (int i = j + 1; i < n; ++i) b[i] -= b[j] * A[i + j * lda];
            }
        }
        for (int j = n - 1; j >= 0; --j) {
            if (b[j] != 0.0) {
                b[j] /= A[j + j * lda];
                for (int i = 0; i < j; ++i) b[i] -= b[j] * A[i + j * lda];
            }
        }
    }
}

void zgetrs_(const char* trans, const int* n_, const int* nrhs_, double complex* A, const int* lda_,
             int* ipiv, double complex* B, const int* ldb_, int* info)
{
    (void)trans;
    const int n = *n_, nrhs = *nrhs_, lda = *lda_, ldb = *ldb_;
    *info = 0;
    for (int c = 0; c < nrhs; ++c) {
        double complex* b = B + c * ldb;
        for (int i = 0; i < n; ++i) {
            int p = ipiv[i] - 1;
            if (p != i) { double complex t = b[i]; b[i] = b[p]; b[p] = t; }
        }
        for (int j = 0; j < n; ++j) {
            if (b[j] != 0.0) {
                for (int i = j + 1; i < n; ++i) b[i] -= b[j] * A[i + j * lda];
            }
        }
        for (int j = n - 1; j >= 0; --j) {
            if (b[j] != 0.0) {
                b[j] /= A[j + j * lda];
                for (int i = 0; i < j; ++i) b[i] -= b[j] * A[i + j * lda];
            }
        }
    }
}
