/*
 * ORACLE / TEST INFRASTRUCTURE -- a plain-C restatement of the reference's CPU
 * integrators, used only by tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg as the checker.  Nothing in the product library links it.
 *
 * Restated from accelerInt (paths relative to the reference repository):
 *   radau2a/radau2a.c:38-736          Radau IIA            -> oracle/radau2a.c
 *   rkc/rkc.c:41-362                  RKC                  -> oracle/rkc.c
 *   exponential_integrators/exprb43/exprb43.c:47-309,
 *   exponential_integrators/exp4/exp4.c:46-320,
 *   exponential_integrators/arnoldi.h:46-141,
 *   exponential_integrators/phiAHessenberg.c:27-184,
 *   exponential_integrators/exponential_linear_algebra.h:28-402,
 *   generic/complexInverse.c:35-248   Krylov methods       -> oracle/krylov.c
 *   generic/solver_generic.c:28-58    batch driver         -> oracle/driver.c
 *   examples/van_der_pol/{dydt,jacob,sparse_multiplier}.c  -> oracle/mech.c
 *
 * Differences from the reference, all deliberate:
 *   - the state length N and the tolerances are runtime values (the reference
 *     fixes NSP/ATOL/RTOL at compile time); the arithmetic is the same;
 *   - failures return a code per system instead of exit() (check_error,
 *     radau2a/radau2a_props.c:13-32);
 *   - per-system event counters are recorded (steps, rejections, LU count ...).
 */
#ifndef ACCELERINT_ORACLE_H
#define ACCELERINT_ORACLE_H

#include <complex.h>

#define OR_NMAX 64            /* largest state length the oracle handles */
#define OR_PMAX 4             /* largest phi order (exprb43) */
#define OR_STRIDE_MAX (OR_NMAX + OR_PMAX)
#define OR_NRA 10             /* rational approximant size, SConstruct N_RA default */

enum { OR_RADAU2A = 0, OR_EXPRB43 = 1, OR_EXP4 = 2, OR_RKC = 3 };
enum { OR_MECH_VDP = 0, OR_MECH_MASS_ACTION = 1 };

typedef struct {
    int kind;                 /* OR_MECH_* */
    int n;                    /* state length */
    int n_species, n_reactions;
    const double *mw, *cp, *h_form, *s_ref, *log_a, *beta, *ta;
    const int *reac, *prod;   /* [R*2], -1 = empty slot */
    int jac_fd;               /* 1: Jacobian by first-order finite differences (generic/fd_jacob.c) */
    double fd_atol, fd_rtol;  /* the ATOL / RTOL the difference increments use */
} or_mech;

typedef struct {
    double atol, rtol;
    /* rational-approximant poles and residues (exp methods) */
    double poles_re[OR_NRA], poles_im[OR_NRA], res_re[OR_NRA], res_im[OR_NRA];
    /* Radau step limit per integrate call; 0: the reference's MAX_NO_STEPS (200000).
     * A tight-tolerance oracle run raises it: at rtol 1e-12 a few ignition systems
     * take more steps than the reference allows at its own tolerance. */
    int max_steps;
    /* Radau starting values after an accepted step: 0 the reference's (radau2a.c:312,
     * x2 in the outer factor of Z3); 1 the collocation polynomial at all three nodes
     * (x3 there), the library's accelerInt_set_stage_extrapolation(1). */
    int stage_extrap;
} or_config;

/* Per-system counters; one row of OR_NSTATS doubles per system. */
enum {
    ST_STEPS = 0,     /* attempted steps (loop iterations that ran the stage logic) */
    ST_ACCEPT,        /* accepted steps */
    ST_REJECT,        /* error-test or Newton rejections */
    ST_JAC,           /* Jacobian evaluations */
    ST_DECOMP,        /* Radau: E1/E2 factorisations */
    ST_NEWTON,        /* Radau: Newton iterations */
    ST_RHS,           /* right-hand-side evaluations */
    ST_ERRSOLVE,      /* Radau: extra E1 solves in the error estimate */
    ST_KRYLOV,        /* exp methods: sum of Krylov dimensions over Arnoldi calls */
    ST_ARNOLDI,       /* exp methods: Arnoldi calls */
    OR_NSTATS = 16
};

/* mechanism callbacks (pyJac convention: column-major jac[i + j*n] = d f_i / d y_j) */
void or_dydt(const or_mech* m, double t, double pr, const double* y, double* dy);
void or_jacob(const or_mech* m, double t, double pr, const double* y, double* jac);
void or_jacvec(const or_mech* m, const double* jac, const double* v, double* out);

/* single-system integrators: advance y from t0 to t1; return the reference EC_* code */
int or_radau2a(const or_config* c, const or_mech* m, double t0, double t1, double pr, double* y, double* st);
int or_rkc(const or_config* c, const or_mech* m, double t0, double t1, double pr, double* y, double* st);
int or_exprb43(const or_config* c, const or_mech* m, double t0, double t1, double pr, double* y, double* st);
int or_exp4(const or_config* c, const or_mech* m, double t0, double t1, double pr, double* y, double* st);

/* Krylov building blocks exposed for the known-answer tests */
int or_hessenberg_lu(int n, int stride, double complex* A, int* piv);
int or_complex_inverse_hessenberg(int n, int stride, double complex* A, int* piv);
int or_phi_ac(const or_config* c, int order, int m, int stride, const double* A, double cscale, double* phiA);

/* batch driver over a column-major y[i*num + sys]; returns the number of failed systems */
int or_integrate_batch(int solver, const or_config* c, const or_mech* m, int num,
                       double t0, double t1, const double* var, double* y, int* codes,
                       double* stats, int nthreads);

#endif
