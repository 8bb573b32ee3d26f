/*
 * ORACLE / TEST INFRASTRUCTURE.  Host entry of the reference's own GPU Radau IIA
 * (radau2a/radau2a.cu, generic/solver_generic.cu intDriver, radau2a_init.cu
 * memory), built unmodified by oracle/build.py into oracle/_ref so that its
 * kernel can be timed beside the library's.
 *
 * It does what the reference's library entry does (generic/solver_interface.cu:
 * memory for `padded` threads, one intDriver launch of padded/64 blocks of 64
 * threads per global step, PreferL1), with three differences.  The reference's
 * accelerInt_initialize stores the padded size in a local that shadows the
 * global `padded` (solver_interface.cu:128 vs :18), so its integrate loop takes
 * min(NUM - num_solved, padded) = 0 systems per pass and never ends; here the
 * padded size is passed along.  The global steps are measured from t_start (the
 * reference's loops measure them from 0, solver_main.cu:301-346 and
 * solver_interface.cu:166-209; for t_start = 0 they agree).  And the per-system
 * codes of every step are kept (maximum over steps) instead of exit()ing
 * (radau2a_props.cu:15-37).
 */
#include <stdlib.h>
#include <string.h>
#include "header.cuh"
#include "solver.cuh"
#include "solver_init.cuh"
#include "launch_bounds.cuh"

extern "C" int refgpu_run(int num, double t0, double t_end, double dt, double* y_host, const double* var_host,
                          int* codes_host, double* kernel_ms)
{
    if (num <= 0) return 0;
    const int padded = (num + TARGET_BLOCK_SIZE - 1) / TARGET_BLOCK_SIZE * TARGET_BLOCK_SIZE;
    // the reference's initialisation prefers L1 device-wide (generic/solver_interface.cu:118);
    // the caller's preference is put back on return
    cudaFuncCache prev = cudaFuncCachePreferNone;
    if (cudaDeviceGetCacheConfig(&prev) != cudaSuccess) return -2;
    if (cudaDeviceSetCacheConfig(cudaFuncCachePreferL1) != cudaSuccess) return -2;
    mechanism_memory* h_mech = (mechanism_memory*)calloc(1, sizeof(mechanism_memory));
    solver_memory* h_sol = (solver_memory*)calloc(1, sizeof(solver_memory));
    mechanism_memory* d_mech = nullptr;
    solver_memory* d_sol = nullptr;
    initialize_gpu_memory(padded, &h_mech, &d_mech);
    initialize_solver(padded, &h_sol, &d_sol);
    int rc = 0;
    int* step_codes = (int*)malloc(num * sizeof(int));
    memset(codes_host, 0, num * sizeof(int));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float total = 0.0f;
    if (cudaMemcpy2D(h_mech->y, padded * sizeof(double), y_host, num * sizeof(double), num * sizeof(double), NSP,
                     cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(h_mech->var, var_host, num * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
        rc = -2;
    double t = t0;
    for (int k = 0; rc == 0 && t + EPS < t_end; ++k) {
        const double t_next = fmin(t_end, t0 + (k + 1) * dt);
        cudaEventRecord(e0);
        intDriver<<<padded / TARGET_BLOCK_SIZE, TARGET_BLOCK_SIZE, SHARED_SIZE>>>(num, t, t_next, h_mech->var,
                                                                                 h_mech->y, d_mech, d_sol);
        cudaEventRecord(e1);
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
            rc = -3;
            break;
        }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        total += ms;
        if (cudaMemcpy(step_codes, h_sol->result, num * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) {
            rc = -2;
            break;
        }
        for (int i = 0; i < num; ++i)
            if (step_codes[i] > codes_host[i]) codes_host[i] = step_codes[i];
        t = t_next;
    }
    if (rc == 0 && cudaMemcpy2D(y_host, num * sizeof(double), h_mech->y, padded * sizeof(double),
                                num * sizeof(double), NSP, cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = -2;
    *kernel_ms = total;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    free(step_codes);
    free_gpu_memory(&h_mech, &d_mech);
    cleanup_solver(&h_sol, &d_sol);
    free(h_mech);
    free(h_sol);
    cudaDeviceSetCacheConfig(prev);
    return rc;
}
