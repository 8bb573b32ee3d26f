// Training and batched inference of the step-proposal MLP (mlp.cuh) on the
// tensor cores: BF16 operands (weights and activations rounded to BF16 as the
// tiles are loaded), FP32 accumulation (mma.sync m16n8k16), FP32 master weights
// and Adam moments.  The network is tiny (64 -> 128 -> 128 -> 128 -> 176), so
// the GEMMs are a few hundred 16 x 8 output tiles; the batch dimension is split
// across blocks (atomic FP32 accumulation) for the weight gradients.
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cstdio>
#include "../../include/accelerint_b200.h"
#include "mlp.cuh"

using namespace aib;

namespace {

__device__ __forceinline__ unsigned pack_bf16(float lo, float hi) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const unsigned*>(&h);
}

// C(m, n) (+)= sum_k A(m, k) B(k, n); element (r, c) of X at X[r * s_r + c * s_c].
// One warp per 16 x 8 tile of C; blockIdx.y selects a k range of k_chunk
// (k_chunk, M multiples of 16, N of 8).  atomic: accumulate into C.
__global__ void __launch_bounds__(128) gemm_bf16_kernel(int M, int N, int K, const float* __restrict__ A, long sam,
                                                        long sak, const float* __restrict__ B, long sbk, long sbn,
                                                        float* __restrict__ C, long scm, long scn, int k_chunk,
                                                        bool atomic)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int tn = N / 8, tiles = (M / 16) * tn;
    if (warp >= tiles) return;
    const int m0 = (warp / tn) * 16, n0 = (warp % tn) * 8;
    const int g = lane >> 2, q = lane & 3;
    const int k_begin = blockIdx.y * k_chunk;
    const int k_end = min(K, k_begin + k_chunk);
    float c0 = 0.f, c1 = 0.f, c2 = 0.f, c3 = 0.f;
    const float* Ar0 = A + long(m0 + g) * sam;
    const float* Ar1 = A + long(m0 + g + 8) * sam;
    const float* Bc = B + long(n0 + g) * sbn;
    for (int k0 = k_begin; k0 < k_end; k0 += 16) {
        const long ka = k0 + 2 * q, kb = ka + 8;
        const unsigned a0 = pack_bf16(Ar0[ka * sak], Ar0[(ka + 1) * sak]);
        const unsigned a1 = pack_bf16(Ar1[ka * sak], Ar1[(ka + 1) * sak]);
        const unsigned a2 = pack_bf16(Ar0[kb * sak], Ar0[(kb + 1) * sak]);
        const unsigned a3 = pack_bf16(Ar1[kb * sak], Ar1[(kb + 1) * sak]);
        const unsigned b0 = pack_bf16(Bc[ka * sbk], Bc[(ka + 1) * sbk]);
        const unsigned b1 = pack_bf16(Bc[kb * sbk], Bc[(kb + 1) * sbk]);
        asm volatile(
            "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
            "{%0,%1,%2,%3};\n"
            : "+f"(c0), "+f"(c1), "+f"(c2), "+f"(c3)
            : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
    }
    float* C0 = C + long(m0 + g) * scm + long(n0 + 2 * q) * scn;
    float* C1 = C + long(m0 + g + 8) * scm + long(n0 + 2 * q) * scn;
    if (atomic) {
        atomicAdd(C0, c0);
        atomicAdd(C0 + scn, c1);
        atomicAdd(C1, c2);
        atomicAdd(C1 + scn, c3);
    } else {
        C0[0] = c0;
        C0[scn] = c1;
        C1[0] = c2;
        C1[scn] = c3;
    }
}

void gemm(int M, int N, int K, const float* A, long sam, long sak, const float* B, long sbk, long sbn, float* C,
          long scm, long scn, bool split, cudaStream_t s) {
    const int tiles = (M / 16) * (N / 8);
    const int blocks = (tiles + 3) / 4;
    int chunk = K, splits = 1;
    if (split) {
        chunk = 1024;
        splits = (K + chunk - 1) / chunk;
    }
    gemm_bf16_kernel<<<dim3(blocks, splits), 128, 0, s>>>(M, N, K, A, sam, sak, B, sbk, sbn, C, scm, scn, chunk,
                                                           split);
}

__device__ __forceinline__ float gelu_grad(float z) {
    const float cdf = 0.5f * (1.0f + erff(z * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * __expf(-0.5f * z * z);
    return cdf + z * pdf;
}

// x_std = (x - mu) / sd
__global__ void standardize_kernel(int M, int D, const float* x, const float* mu, const float* sd, float* out) {
    const long i = blockIdx.x * long(blockDim.x) + threadIdx.x;
    if (i >= long(M) * D) return;
    const int j = int(i % D);
    out[i] = (x[i] - mu[j]) / sd[j];
}

// Z += b; A = gelu(Z) (hidden) or A = Z (output)
__global__ void bias_act_kernel(int M, int D, float* Z, const float* b, float* Aout, bool act) {
    const long i = blockIdx.x * long(blockDim.x) + threadIdx.x;
    if (i >= long(M) * D) return;
    const float z = Z[i] + b[i % D];
    Z[i] = z;
    if (Aout) Aout[i] = act ? gelu_f(z) : z;
}

// y = y * sd + mu
__global__ void destandardize_kernel(int M, int D, float* y, const float* mu, const float* sd) {
    const long i = blockIdx.x * long(blockDim.x) + threadIdx.x;
    if (i >= long(M) * D) return;
    const int j = int(i % D);
    y[i] = y[i] * sd[j] + mu[j];
}

// loss = sum_m sum_j w_j (y - t)^2 / M;  dY = 2 w_j (y - t) / M
__global__ void loss_kernel(int M, const float* Y, const float* T, const float* w, float* dY, float* loss) {
    const long i = blockIdx.x * long(blockDim.x) + threadIdx.x;
    float l = 0.f;
    if (i < long(M) * MLP_D4) {
        const int j = int(i % MLP_D4);
        const float d = Y[i] - T[i];
        dY[i] = 2.0f * w[j] * d / float(M);
        l = w[j] * d * d / float(M);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, l);
}

// dZ = dA * gelu'(Z)
__global__ void gelu_back_kernel(long n, const float* Z, float* dA) {
    const long i = blockIdx.x * long(blockDim.x) + threadIdx.x;
    if (i < n) dA[i] *= gelu_grad(Z[i]);
}

// db_j += sum_m dZ[m, j]; one thread per column over a slice of rows
__global__ void colsum_kernel(int M, int D, const float* dZ, float* db) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= D) return;
    const int rows = (M + gridDim.y - 1) / gridDim.y;
    const int r0 = blockIdx.y * rows, r1 = min(M, r0 + rows);
    float s = 0.f;
    for (int r = r0; r < r1; ++r) s += dZ[long(r) * D + j];
    atomicAdd(db + j, s);
}

__global__ void adam_kernel(int n, float* p, const float* g, float* m, float* v, float lr, float b1, float b2,
                            float eps, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

__global__ void to_bf16_kernel(const float* p, __nv_bfloat16* w) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= MLP_NWEIGHT) return;
    int l = 0;
    while (l + 1 < MLP_LAYERS && i >= mlp_wq(l + 1)) ++l;
    w[i] = __float2bfloat16_rn(p[mlp_woff(l) + (i - mlp_wq(l))]);
}

inline int nblk(long n, int b = 256) { return int((n + b - 1) / b); }

// activations of one batch: Z_l (pre-activation, FP32) and A_l (post), dZ scratch
struct Work {
    int M = 0;
    float* buf = nullptr;
    float* Z[MLP_LAYERS];
    float* A[MLP_LAYERS];
    float* x;
    float* d0;
    float* d1;
};
Work g_work;

int ensure_work(int M) {
    if (g_work.M >= M) return 0;
    if (g_work.buf) cudaFree(g_work.buf);
    g_work.buf = nullptr;
    size_t n = size_t(M) * MLP_D0;
    for (int l = 0; l < MLP_LAYERS; ++l) n += 2 * size_t(M) * mlp_dout(l);
    n += 2 * size_t(M) * MLP_D4;
    if (cudaMalloc(&g_work.buf, n * sizeof(float)) != cudaSuccess) return ACCELERINT_ERR_CUDA;
    float* p = g_work.buf;
    g_work.x = p;
    p += size_t(M) * MLP_D0;
    for (int l = 0; l < MLP_LAYERS; ++l) {
        g_work.Z[l] = p;
        p += size_t(M) * mlp_dout(l);
        g_work.A[l] = p;
        p += size_t(M) * mlp_dout(l);
    }
    g_work.d0 = p;
    p += size_t(M) * MLP_D4;
    g_work.d1 = p;
    g_work.M = M;
    return 0;
}

// forward pass on standardised inputs xs [M x D0]; output (standardised) in A[L-1]
void forward(const float* params, const float* xs, int M, cudaStream_t s) {
    const float* in = xs;
    for (int l = 0; l < MLP_LAYERS; ++l) {
        const int din = mlp_din(l), dout = mlp_dout(l);
        gemm(M, dout, din, in, din, 1, params + mlp_woff(l), 1, din, g_work.Z[l], dout, 1, false, s);
        bias_act_kernel<<<nblk(long(M) * dout), 256, 0, s>>>(M, dout, g_work.Z[l], params + mlp_boff(l), g_work.A[l],
                                                             l < MLP_LAYERS - 1);
        in = g_work.A[l];
    }
}

// MLP features of whole states (the layout the solver's records use): x[m] = (T,
// log10 max(Y_k, 1e-20), log10 h, log10(P / 1 atm), 0...) for system m of
// y[N * num] (column-major); rows num..M-1 zero.
__global__ void state_features_kernel(int num, int M, int n, const double* y, const double* var, double h,
                                      float* x) {
    const long e = blockIdx.x * long(blockDim.x) + threadIdx.x;
    if (e >= long(M) * MLP_D0) return;
    const int m = int(e / MLP_D0), j = int(e % MLP_D0);
    float v = 0.f;
    if (m < num) {
        if (j == 0) v = float(y[m]);
        else if (j < n) v = float(log10(fmax(y[size_t(j) * num + m], 1e-20)));
        else if (j == n) v = float(log10(h));
        else if (j == n + 1) v = float(log10(var[m] / 101325.0));
    }
    x[e] = v;
}

__global__ void column0_kernel(int num, const float* y, float* key) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < num) key[i] = y[size_t(i) * MLP_D4];
}

}  // namespace

namespace aib_mlp {
// release the activation / gradient workspace (accelerInt_cleanup)
void free_work() {
    if (g_work.buf) cudaFree(g_work.buf);
    g_work = Work{};
}

// bf16 copy of the weights for the solver (api.cu)
int to_bf16(const float* params, void* w_bf16, cudaStream_t s) {
    to_bf16_kernel<<<nblk(MLP_NWEIGHT), 256, 0, s>>>(params, static_cast<__nv_bfloat16*>(w_bf16));
    return cudaGetLastError() == cudaSuccess ? 0 : ACCELERINT_ERR_CUDA;
}

// Predicted cost (output 0 of the model) of every system of y, into key[num]
// (a float per system); x and out: scratch of M x 64 and M x 176 floats,
// M = num rounded up to 16.  Returns the number of kernels launched, < 0 on error.
int predict_cost(const float* params, const float* norm, int num, int n, const double* y, const double* var,
                 double h, float* x, float* out, float* key, cudaStream_t s) {
    const int M = (num + 15) / 16 * 16;
    if (ensure_work(M)) return -1;
    state_features_kernel<<<nblk(long(M) * MLP_D0), 256, 0, s>>>(num, M, n, y, var, h, x);
    standardize_kernel<<<nblk(long(M) * MLP_D0), 256, 0, s>>>(M, MLP_D0, x, norm, norm + MLP_D0, g_work.x);
    forward(params, g_work.x, M, s);
    cudaMemcpyAsync(out, g_work.A[MLP_LAYERS - 1], size_t(M) * MLP_D4 * sizeof(float), cudaMemcpyDeviceToDevice, s);
    destandardize_kernel<<<nblk(long(M) * MLP_D4), 256, 0, s>>>(M, MLP_D4, out, norm + 2 * MLP_D0,
                                                                norm + 2 * MLP_D0 + MLP_D4);
    column0_kernel<<<nblk(num), 256, 0, s>>>(num, out, key);
    return cudaGetLastError() == cudaSuccess ? 5 + 2 * MLP_LAYERS : -1;
}
}  // namespace aib_mlp

extern "C" {

int accelerInt_mlp_forward(const float* params_dev, const float* norm_dev, const float* x_dev, int M, float* y_dev,
                           void* stream) {
    if (!params_dev || !norm_dev || !x_dev || !y_dev || M <= 0 || M % 16) return ACCELERINT_ERR_ARGUMENT;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (ensure_work(M)) return ACCELERINT_ERR_CUDA;
    standardize_kernel<<<nblk(long(M) * MLP_D0), 256, 0, s>>>(M, MLP_D0, x_dev, norm_dev, norm_dev + MLP_D0,
                                                              g_work.x);
    forward(params_dev, g_work.x, M, s);
    cudaMemcpyAsync(y_dev, g_work.A[MLP_LAYERS - 1], size_t(M) * MLP_D4 * sizeof(float), cudaMemcpyDeviceToDevice, s);
    destandardize_kernel<<<nblk(long(M) * MLP_D4), 256, 0, s>>>(M, MLP_D4, y_dev, norm_dev + 2 * MLP_D0,
                                                                norm_dev + 2 * MLP_D0 + MLP_D4);
    return cudaGetLastError() == cudaSuccess ? ACCELERINT_OK : ACCELERINT_ERR_CUDA;
}

int accelerInt_mlp_loss_grad(const float* params_dev, const float* xs_dev, const float* ts_dev, const float* w_dev,
                             int M, float* grad_dev, float* loss_dev, void* stream) {
    if (!params_dev || !xs_dev || !ts_dev || !w_dev || !grad_dev || !loss_dev || M <= 0 || M % 16)
        return ACCELERINT_ERR_ARGUMENT;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (ensure_work(M)) return ACCELERINT_ERR_CUDA;
    forward(params_dev, xs_dev, M, s);
    cudaMemsetAsync(grad_dev, 0, size_t(MLP_NPARAM) * sizeof(float), s);
    cudaMemsetAsync(loss_dev, 0, sizeof(float), s);
    float* dZ = g_work.d0;   // gradient w.r.t. the current layer's pre-activation
    float* dA = g_work.d1;
    loss_kernel<<<nblk(long(M) * MLP_D4), 256, 0, s>>>(M, g_work.A[MLP_LAYERS - 1], ts_dev, w_dev, dZ, loss_dev);
    for (int l = MLP_LAYERS - 1; l >= 0; --l) {
        const int din = mlp_din(l), dout = mlp_dout(l);
        const float* Ain = l > 0 ? g_work.A[l - 1] : xs_dev;
        // dW_l [dout x din] = dZ^T Ain (reduction over the batch)
        gemm(dout, din, M, dZ, 1, dout, Ain, din, 1, grad_dev + mlp_woff(l), din, 1, true, s);
        colsum_kernel<<<dim3(nblk(dout, 128), 32), 128, 0, s>>>(M, dout, dZ, grad_dev + mlp_boff(l));
        if (l > 0) {
            // dA_{l-1} [M x din] = dZ W_l, then through GELU
            gemm(M, din, dout, dZ, dout, 1, params_dev + mlp_woff(l), din, 1, dA, din, 1, false, s);
            gelu_back_kernel<<<nblk(long(M) * din), 256, 0, s>>>(long(M) * din, g_work.Z[l - 1], dA);
            float* t = dZ;
            dZ = dA;
            dA = t;
        }
    }
    return cudaGetLastError() == cudaSuccess ? ACCELERINT_OK : ACCELERINT_ERR_CUDA;
}

int accelerInt_mlp_adam_step(float* params_dev, const float* grad_dev, float* m_dev, float* v_dev, int step,
                             float lr, float beta1, float beta2, float eps, void* stream) {
    if (!params_dev || !grad_dev || !m_dev || !v_dev || step < 1) return ACCELERINT_ERR_ARGUMENT;
    const float c1 = 1.f - powf(beta1, float(step)), c2 = 1.f - powf(beta2, float(step));
    adam_kernel<<<nblk(MLP_NPARAM), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        MLP_NPARAM, params_dev, grad_dev, m_dev, v_dev, lr, beta1, beta2, eps, c1, c2);
    return cudaGetLastError() == cudaSuccess ? ACCELERINT_OK : ACCELERINT_ERR_CUDA;
}

int accelerInt_mlp_sizes(int* nparam, int* nnorm, int* d_in, int* d_out) {
    if (nparam) *nparam = MLP_NPARAM;
    if (nnorm) *nnorm = MLP_NNORM;
    if (d_in) *d_in = MLP_D0;
    if (d_out) *d_out = MLP_D4;
    return ACCELERINT_OK;
}

}  // extern "C"
