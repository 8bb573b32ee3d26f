/*
 * ORACLE / TEST INFRASTRUCTURE.  Allocation of the mass-action mechanism memory
 * for the reference GPU build, after the reference's slot
 * (examples/van_der_pol/gpu_memory.cu:21-68: y, dy, var and the Jacobian,
 * padded per thread, dy and the Jacobian zeroed).
 */
#include "gpu_memory.cuh"

static ma_tables g_tb;          /* device pointers of the tables */
static void* g_tb_mem = nullptr;

extern "C" int refgpu_set_mass_action(int K, int R, const double* mw, const double* cp, const double* h_form,
                                      const double* s_ref, const int* reac, const int* prod, const double* log_a,
                                      const double* beta, const double* ta)
{
    if (K + 1 != NSP) return -1;
    if (g_tb_mem) cudaFree(g_tb_mem);
    g_tb_mem = nullptr;
    const size_t nd = size_t(4 * K + 3 * R), ni = size_t(4 * R);
    if (cudaMalloc(&g_tb_mem, nd * sizeof(double) + ni * sizeof(int)) != cudaSuccess) return -2;
    double* d = static_cast<double*>(g_tb_mem);
    int* i = reinterpret_cast<int*>(d + nd);
    const double* src[7] = {mw, cp, h_form, s_ref, log_a, beta, ta};
    const size_t len[7] = {size_t(K), size_t(K), size_t(K), size_t(K), size_t(R), size_t(R), size_t(R)};
    const double* dst[7];
    double* p = d;
    for (int a = 0; a < 7; ++a) {
        if (cudaMemcpy(p, src[a], len[a] * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) return -2;
        dst[a] = p;
        p += len[a];
    }
    if (cudaMemcpy(i, reac, 2 * R * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess) return -2;
    if (cudaMemcpy(i + 2 * R, prod, 2 * R * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess) return -2;
    g_tb.K = K;
    g_tb.R = R;
    g_tb.mw = dst[0]; g_tb.cp = dst[1]; g_tb.h_form = dst[2]; g_tb.s_ref = dst[3];
    g_tb.log_a = dst[4]; g_tb.beta = dst[5]; g_tb.ta = dst[6];
    g_tb.reac = i;
    g_tb.prod = i + 2 * R;
    return 0;
}

size_t required_mechanism_size()
{
    /* y, dy, the Jacobian and the pressure, per thread */
    return (2 * NSP + NSP * NSP + 1) * sizeof(double);
}

void initialize_gpu_memory(int padded, mechanism_memory** h_mem, mechanism_memory** d_mem)
{
    cudaErrorCheck(cudaMalloc(d_mem, sizeof(mechanism_memory)));
    cudaErrorCheck(cudaMalloc(&((*h_mem)->y), NSP * padded * sizeof(double)));
    cudaErrorCheck(cudaMalloc(&((*h_mem)->dy), NSP * padded * sizeof(double)));
    cudaErrorCheck(cudaMalloc(&((*h_mem)->var), padded * sizeof(double)));
    cudaErrorCheck(cudaMalloc(&((*h_mem)->jac), NSP * NSP * padded * sizeof(double)));
    cudaErrorCheck(cudaMemset((*h_mem)->dy, 0, NSP * padded * sizeof(double)));
    cudaErrorCheck(cudaMemset((*h_mem)->jac, 0, NSP * NSP * padded * sizeof(double)));
    (*h_mem)->tb = g_tb;
    cudaErrorCheck(cudaMemcpy(*d_mem, *h_mem, sizeof(mechanism_memory), cudaMemcpyHostToDevice));
}

void free_gpu_memory(mechanism_memory** h_mem, mechanism_memory** d_mem)
{
    cudaErrorCheck(cudaFree((*h_mem)->y));
    cudaErrorCheck(cudaFree((*h_mem)->dy));
    cudaErrorCheck(cudaFree((*h_mem)->var));
    cudaErrorCheck(cudaFree((*h_mem)->jac));
    cudaErrorCheck(cudaFree(*d_mem));
}
