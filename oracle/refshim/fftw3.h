/*
 * ORACLE / TEST INFRASTRUCTURE.  Minimal FFTW3 API used by the reference's
 * exponential_integrators/cf.c (fftw_alloc_complex, fftw_plan_dft_1d,
 * fftw_execute, fftw_free, fftw_destroy_plan, fftw_cleanup).  FFTW is absent
 * here; the transform is a plain O(n^2) DFT with FFTW's forward sign
 * convention, X_k = sum_j x_j exp(-2 pi i j k / n), evaluated in long double.
 */
#ifndef ORACLE_FFTW3_SHIM_H
#define ORACLE_FFTW3_SHIM_H
#include <complex.h>
typedef double complex fftw_complex;
typedef struct oracle_fftw_plan_s* fftw_plan;
#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)
fftw_complex* fftw_alloc_complex(size_t n);
void fftw_free(void* p);
fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
void fftw_cleanup(void);
#endif
