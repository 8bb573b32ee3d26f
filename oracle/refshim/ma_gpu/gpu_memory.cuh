/*
 * ORACLE / TEST INFRASTRUCTURE.  Mechanism memory of the synthetic mass-action
 * mechanism for the build of the reference's own GPU Radau (radau2a/radau2a.cu
 * with generic/solver_generic.cu), in the layout of the reference's
 * mechanism_memory slot (examples/van_der_pol/gpu_memory.cuh:29-34): the state,
 * dydt and Jacobian arrays the solver reads (mech->y, ->dy, ->jac), each strided
 * by the padded number of threads (INDEX(i) = thread + i * grid size), plus the
 * mechanism's tables.
 */
#ifndef GPU_MEM_CUH
#define GPU_MEM_CUH

#include "header.cuh"

struct ma_tables {
    int K, R;
    const double *mw, *cp, *h_form, *s_ref;    /* [K] */
    const double *log_a, *beta, *ta;           /* [R] */
    const int *reac, *prod;                    /* [2R], -1 = empty slot */
};

struct mechanism_memory {
    double* y;
    double* dy;
    double* var;
    double* jac;
    ma_tables tb;
};

size_t required_mechanism_size();
void initialize_gpu_memory(int padded, mechanism_memory** h_mem, mechanism_memory** d_mem);
void free_gpu_memory(mechanism_memory** h_mem, mechanism_memory** d_mem);

/* host side: copy the mechanism's tables to the device (before initialize_gpu_memory) */
extern "C" int refgpu_set_mass_action(int K, int R, const double* mw, const double* cp, const double* h_form,
                                      const double* s_ref, const int* reac, const int* prod, const double* log_a,
                                      const double* beta, const double* ta);

#endif
