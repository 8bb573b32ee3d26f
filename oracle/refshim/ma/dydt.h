/* ORACLE / TEST INFRASTRUCTURE: callback prototypes (examples/van_der_pol/dydt.h form). */
#ifndef DYDT_H
#define DYDT_H
void dydt(const double t, const double pres, const double* __restrict__ y, double* __restrict__ dy);
#endif
