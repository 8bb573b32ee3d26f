/* ORACLE / TEST INFRASTRUCTURE: callback prototypes (examples/van_der_pol/jacob.h form). */
#ifndef JACOB_H
#define JACOB_H
void eval_jacob(const double t, const double pres, const double* __restrict__ y, double* __restrict__ jac);
#endif
