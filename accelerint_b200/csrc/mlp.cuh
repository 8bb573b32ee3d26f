// Learned step proposals for Radau IIA: a small MLP maps the state at the start
// of a step to (a) initial Newton stage values and (b) a step size.
//
//   input  (D0 = 64, first N + 2 used): T, log10 max(Y_k, 1e-20) (k = 1..N-1),
//          log10 h (the last accepted step size), log10 (P / 1 atm)
//   hidden 3 x 128, GELU (erf form)
//   output (D4 = 176, first 3N + 1 used): symlog(Z_c,i / s_i) for the three
//          stages c and elements i, s_i = atol + rtol |y_i|, then log10 of the
//          accepted step size over the previous accepted one.
// Inputs and outputs are standardised with per-feature mean / spread stored with
// the model.  Weights are BF16 (the solver's copy); accumulation is FP32.
//
// Inside the solver one team runs one system, so inference is a batch of one:
// a matrix-vector product per layer on the FP32 pipe (a tensor-core tile would
// be 15/16 padding).  Training and batched inference run on the tensor cores
// (mlp.cu).
#pragma once
#include <cuda_bf16.h>
#include "common.cuh"

namespace aib {

constexpr int MLP_D0 = 64, MLP_DH = 128, MLP_D4 = 176, MLP_LAYERS = 4;
__host__ __device__ constexpr int mlp_din(int l) { return l == 0 ? MLP_D0 : MLP_DH; }
__host__ __device__ constexpr int mlp_dout(int l) { return l == MLP_LAYERS - 1 ? MLP_D4 : MLP_DH; }
// FP32 parameter vector: W0 b0 W1 b1 W2 b2 W3 b3, W_l row-major [dout x din]
__host__ __device__ constexpr int mlp_woff(int l) {
    int o = 0;
    for (int i = 0; i < l; ++i) o += mlp_dout(i) * mlp_din(i) + mlp_dout(i);
    return o;
}
__host__ __device__ constexpr int mlp_boff(int l) { return mlp_woff(l) + mlp_dout(l) * mlp_din(l); }
constexpr int MLP_NPARAM = mlp_woff(MLP_LAYERS);
// normalisation vector: in_mu[D0] in_sd[D0] out_mu[D4] out_sd[D4]
constexpr int MLP_NNORM = 2 * MLP_D0 + 2 * MLP_D4;

// What the solver does with the proposals (bit flags).
enum : int { MLP_USE_H = 1, MLP_USE_Z = 2 };

// Device copy the solver reads (bf16 weights in one block, FP32 biases and norms).
struct MlpDevice {
    const __nv_bfloat16* w;   // weights at mlp_woff-like offsets without the biases: see mlp_wq
    const float* p;           // FP32 parameter vector (biases read from here)
    const float* norm;        // MLP_NNORM floats
    int flags;
    double growth_floor;      // the step-size proposal never holds the step below this x the last accepted
};
__host__ __device__ constexpr int mlp_wq(int l) {   // offset of W_l in the bf16 weight block
    int o = 0;
    for (int i = 0; i < l; ++i) o += mlp_dout(i) * mlp_din(i);
    return o;
}
constexpr int MLP_NWEIGHT = mlp_wq(MLP_LAYERS);

__device__ __forceinline__ float gelu_f(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ double symlog(double z) { return z >= 0 ? log1p(z) : -log1p(-z); }
__device__ __forceinline__ double symexp(double v) { return v >= 0 ? expm1(v) : -expm1(-v); }

// One inference for the calling team.  x (D0 floats, raw features, entries past
// N + 2 zero) and the two ping-pong buffers (MLP_D4 floats each) live in shared
// memory; the raw (de-standardised) outputs end in `out` (one of the buffers,
// returned).  only >= 0: the last layer computes that output alone (the step-size
// proposal needs one of its MLP_D4 rows).  Every thread of the team must call.
template <int TS>
__device__ __noinline__ float* mlp_infer_team(const MlpDevice& m, float* x, float* b0, float* b1, int only = -1)
{
    using TM = Team<TS>;
    const int lane = TM::lane();
    for (int i = lane; i < MLP_D0; i += TS) x[i] = (x[i] - m.norm[i]) / m.norm[MLP_D0 + i];
    TM::sync();
    const float* in = x;
    for (int l = 0; l < MLP_LAYERS; ++l) {
        float* out = (l & 1) ? b1 : b0;
        const int din = mlp_din(l), dout = mlp_dout(l);
        const __nv_bfloat16* W = m.w + mlp_wq(l);
        const float* b = m.p + mlp_boff(l);
        const bool last = l == MLP_LAYERS - 1;
        for (int j = (last && only >= 0) ? only + lane : lane; j < ((last && only >= 0) ? only + 1 : dout); j += TS) {
            const uint4* row = reinterpret_cast<const uint4*>(W + size_t(j) * din);
            float acc = b[j];
            for (int k8 = 0; k8 < din / 8; ++k8) {
                const uint4 q = __ldg(row + k8);
                const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&q);
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const float2 f = __bfloat1622float2(h[e]);
                    acc = fmaf(f.x, in[k8 * 8 + 2 * e], acc);
                    acc = fmaf(f.y, in[k8 * 8 + 2 * e + 1], acc);
                }
            }
            out[j] = (l < MLP_LAYERS - 1) ? gelu_f(acc) : acc;
        }
        TM::sync();
        in = out;
    }
    float* y = ((MLP_LAYERS - 1) & 1) ? b1 : b0;
    for (int j = only >= 0 ? only + lane : lane; j < (only >= 0 ? only + 1 : MLP_D4); j += TS)
        y[j] = y[j] * m.norm[2 * MLP_D0 + MLP_D4 + j] + m.norm[2 * MLP_D0 + j];
    TM::sync();
    return y;
}

// Learned mode and step-record capture of the Radau kernel (both optional).
struct LearnArgs {
    MlpDevice mlp;        // mlp.flags == 0: proposals off
    float* rec;           // step records [cap][MLP_D0 + MLP_D4] (raw features, raw targets), or null
    int* rec_count;       // records claimed so far (atomic)
    int rec_cap;
};
constexpr int MLP_REC = MLP_D0 + MLP_D4;

}  // namespace aib
