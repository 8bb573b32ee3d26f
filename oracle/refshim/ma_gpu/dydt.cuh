/* ORACLE / TEST INFRASTRUCTURE.  dydt of the reference's GPU callback slot
 * (examples/van_der_pol/dydt.cuh:22-23) for the synthetic mass-action mechanism. */
#ifndef DYDT_CUH
#define DYDT_CUH
#include "header.cuh"
__device__ void dydt(const double t, const double pres, const double* __restrict__ y, double* __restrict__ dy,
                     const mechanism_memory* __restrict__ d_mem);
#endif
