/* ORACLE / TEST INFRASTRUCTURE: plain-C LAPACK-semantics LU (see lapack_plain.c). */
#ifndef ORACLE_LAPACK_PLAIN_H
#define ORACLE_LAPACK_PLAIN_H
#include <complex.h>

void dgetrf_(const int* m, const int* n, double* A, const int* lda, int* ipiv, int* info);
void zgetrf_(const int* m, const int* n, double complex* A, const int* lda, int* ipiv, int* info);
void dgetrs_(const char* trans, const int* n, const int* nrhs, double* A, const int* lda,
             int* ipiv, double* B, const int* ldb, int* info);
void zgetrs_(const char* trans, const int* n, const int* nrhs, double complex* A, const int* lda,
             int* ipiv, double complex* B, const int* ldb, int* info);

#endif
