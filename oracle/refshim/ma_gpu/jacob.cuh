/* ORACLE / TEST INFRASTRUCTURE.  eval_jacob of the reference's GPU callback slot
 * (examples/van_der_pol/jacob.cuh:21) for the synthetic mass-action mechanism. */
#ifndef JACOB_CUH
#define JACOB_CUH
#include "header.cuh"
__device__ void eval_jacob(const double t, const double pres, const double* __restrict__ y, double* __restrict__ jac,
                           const mechanism_memory* __restrict__ d_mem);
#endif
