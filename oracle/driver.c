/*
 * ORACLE / TEST INFRASTRUCTURE.  Batch driver restated from
 * generic/solver_generic.c:28-58: gather each system from the column-major
 * global array, integrate, scatter back.  OpenMP with dynamic scheduling (the
 * reference uses the default static schedule; the result per system does not
 * depend on the schedule).  Failures are recorded per system instead of
 * calling exit().
 */
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "oracle.h"

int or_integrate_batch(int solver, const or_config* c, const or_mech* m, int num, double t0, double t1,
                       const double* var, double* y, int* codes, double* stats, int nthreads)
{
    const int n = m->n;
    int nfail = 0;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads) reduction(+ : nfail)
#else
    (void)nthreads;
#endif
    for (int tid = 0; tid < num; ++tid) {
        double yl[OR_NMAX];
        double st[OR_NSTATS];
        memset(st, 0, sizeof(st));
        for (int i = 0; i < n; ++i) yl[i] = y[tid + (size_t)i * num];
        int code = 0;
        switch (solver) {
            case OR_RADAU2A: code = or_radau2a(c, m, t0, t1, var[tid], yl, st); break;
            case OR_EXPRB43: code = or_exprb43(c, m, t0, t1, var[tid], yl, st); break;
            case OR_EXP4: code = or_exp4(c, m, t0, t1, var[tid], yl, st); break;
            case OR_RKC: code = or_rkc(c, m, t0, t1, var[tid], yl, st); break;
            default: code = -1; break;
        }
        for (int i = 0; i < n; ++i) y[tid + (size_t)i * num] = yl[i];
        if (codes) codes[tid] = code;
        if (stats)
            for (int s = 0; s < OR_NSTATS; ++s) stats[(size_t)tid * OR_NSTATS + s] += st[s];
        nfail += code != 0;
    }
    return nfail;
}
