/*
 * ORACLE / TEST INFRASTRUCTURE.  The reference's mechanism callback slot
 * (dydt / eval_jacob / sparse_multiplier, examples/van_der_pol/*.h) filled with
 * the synthetic mass-action mechanism of oracle/mech.c, for building the
 * reference's own integrators under oracle/_ref.  The mechanism tables are set
 * once through refshim_set_mass_action() before integrating.
 */
#include "header.h"
#include "dydt.h"
#include "jacob.h"
#include "sparse_multiplier.h"
#include "oracle.h"

static or_mech g_mech;

void refshim_set_mass_action(int K, int R, const double* mw, const double* cp, const double* h_form,
                             const double* s_ref, const int* reac, const int* prod, const double* log_a,
                             const double* beta, const double* ta)
{
    g_mech.kind = OR_MECH_MASS_ACTION;
    g_mech.n = K + 1;
    g_mech.n_species = K;
    g_mech.n_reactions = R;
    g_mech.mw = mw; g_mech.cp = cp; g_mech.h_form = h_form; g_mech.s_ref = s_ref;
    g_mech.reac = reac; g_mech.prod = prod; g_mech.log_a = log_a; g_mech.beta = beta; g_mech.ta = ta;
}

void dydt(const double t, const double pres, const double* __restrict__ y, double* __restrict__ dy)
{
    or_dydt(&g_mech, t, pres, y, dy);
}

void eval_jacob(const double t, const double pres, const double* __restrict__ y, double* __restrict__ jac)
{
    or_jacob(&g_mech, t, pres, y, jac);
}

void sparse_multiplier(const double* A, const double* v, double* w)
{
    or_jacvec(&g_mech, A, v, w);
}

void set_same_initial_conditions(int NUM, double** y_host, double** var_host) { (void)NUM; (void)y_host; (void)var_host; }
void apply_mask(double* y_host) { (void)y_host; }
void apply_reverse_mask(double* y_host) { (void)y_host; }
