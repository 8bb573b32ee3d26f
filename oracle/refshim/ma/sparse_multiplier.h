/* ORACLE / TEST INFRASTRUCTURE: callback prototypes (examples/van_der_pol/sparse_multiplier.h form). */
#ifndef SPARSE_HEAD
#define SPARSE_HEAD
#include "header.h"
void sparse_multiplier(const double*, const double*, double*);
#endif
