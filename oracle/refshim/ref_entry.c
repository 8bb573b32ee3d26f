/*
 * ORACLE / TEST INFRASTRUCTURE.  Entry points of oracle/_ref/libref_<solver>_n<N>.so,
 * a build of the reference's own unmodified CPU sources.
 *
 *   ref_integrate_batch : OpenMP loop over systems calling the reference's
 *                         integrate() (radau2a.c:520, rkc.c:209, exprb43.c:47,
 *                         exp4.c:294); records each return code instead of the
 *                         reference's exit() in check_error().
 *   ref_int_driver      : the reference's own batch driver intDriver
 *                         (generic/solver_generic.c:159), timed as the stock
 *                         CPU path.
 *   ref_poles           : poles/residues computed by the reference's cf()
 *                         (exp methods only).
 */
#include <string.h>
#include <complex.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "header.h"
#include "solver.h"

#if defined(RB43) || defined(EXP4)
#include "rational_approximant.h"
extern double complex poles[N_RA];
extern double complex res[N_RA];
#endif

int ref_nsp(void) { return NSP; }

void ref_init(void)
{
#if defined(RB43) || defined(EXP4)
    find_poles_and_residuals();
#endif
}

int ref_poles(double* pr, double* pi, double* rr, double* ri)
{
#if defined(RB43) || defined(EXP4)
    for (int i = 0; i < N_RA; ++i) {
        pr[i] = creal(poles[i]); pi[i] = cimag(poles[i]);
        rr[i] = creal(res[i]); ri[i] = cimag(res[i]);
    }
    return N_RA;
#else
    (void)pr; (void)pi; (void)rr; (void)ri;
    return 0;
#endif
}

int ref_integrate_batch(int num, double t0, double t1, const double* var, double* y, int* codes, int nthreads)
{
    int nfail = 0;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads) reduction(+ : nfail)
#else
    (void)nthreads;
#endif
    for (int tid = 0; tid < num; ++tid) {
        double yl[NSP];
        for (int i = 0; i < NSP; ++i) yl[i] = y[tid + (size_t)i * num];
        int code = integrate(t0, t1, var[tid], yl);
        for (int i = 0; i < NSP; ++i) y[tid + (size_t)i * num] = yl[i];
        if (codes) codes[tid] = code;
        nfail += code != 0;
    }
    return nfail;
}

void ref_int_driver(int num, double t0, double t1, const double* var, double* y, int nthreads)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    intDriver(num, t0, t1, var, y);
}
