// C-ABI of libaccelerint_b200.so: the reference's accelerInt_initialize /
// accelerInt_integrate / accelerInt_cleanup (generic/solver_interface.cu:88-225)
// plus run-time selection of solver, mechanism, Jacobian, tolerances and
// precision, the device-buffer / graph / allocation-free entry points, the
// launch mapping (persistent queue, queue order, autotuner) and the learned
// proposals.  One process-wide instance, as in the reference.
#include <cuda_runtime.h>
#include <cstdio>
#include <cstring>
#include <cmath>
#include <vector>
#include <algorithm>
#include "../../include/accelerint_b200.h"
#include "kernels.cuh"

using namespace aib;

namespace aib_cf {
int poles_residues(int n, double atol, double* pr, double* pi, double* rr, double* ri);
}
namespace aib_mlp {
void free_work();
int to_bf16(const float* params, void* w_bf16, cudaStream_t s);
int predict_cost(const float* params, const float* norm, int num, int n, const double* y, const double* var,
                 double h, float* x, float* out, float* key, cudaStream_t s);
}

namespace {

// FMA throughput probe: 8 independent dependency chains per thread.
__global__ void fma_peak_kernel2(float2* out, int iters, float2 m) {
    float2 a[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) a[c] = make_float2(float(threadIdx.x + c) * 1e-3f, float(c) * 1e-3f);
    const float2 d = make_float2(1e-7f, 1e-7f);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < 8; ++c) a[c] = __ffma2_rn(a[c], m, d);
    }
    float2 s = make_float2(0.f, 0.f);
#pragma unroll
    for (int c = 0; c < 8; ++c) { s.x += a[c].x; s.y += a[c].y; }
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}
template <typename T>
__global__ void fma_peak_kernel(T* out, int iters, T m) {
    T a[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) a[c] = T(threadIdx.x + c) * T(1e-3);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < 8; ++c) a[c] = fma(a[c], m, T(1e-7));
    }
    T s = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) s += a[c];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

struct MechTablesHost {
    int K = 0, R = 0;
    std::vector<double> inv_mw, mw, cp, h_form, s_ref, log_a, beta, ta;
    std::vector<int4> rsp;
    std::vector<int> sp_ptr, sp_ent;
};

struct State {
    bool initialized = false;
    int device = 0;
    int num_sms = 0;
    int capacity = 0;          // systems per device batch (legacy path)
    int solver = ACCELERINT_RADAU2A;
    int mech_kind = 0;         // 0 van der Pol, 1 mass action
    int lu = ACCELERINT_LU_FP64;
    double atol = 1e-10, rtol = 1e-6;
    MechTablesHost mt;
    MassActionTables dev_tb{};
    void* dev_tb_mem = nullptr;
    double* y_dev = nullptr;
    double* var_dev = nullptr;
    int* codes_dev = nullptr;
    int* queue = nullptr;
    double* jac = nullptr;
    size_t jac_doubles = 0;
    cudaStream_t stream = nullptr;
    int last_status = ACCELERINT_OK;
    std::vector<int> codes;
    double poles[4][10] = {};
    double poles_atol = -1.0;     // ATOL the poles were computed for (< 0: not yet)
    int poles_device = -1;        // device whose c_cf holds them
    long long launches = 0;       // kernels this library launched
    LearnArgs learn{};            // learned proposals / step records for the Radau block teams
    void* mlp_w = nullptr;        // bf16 weight copy of the installed model
    // launch mapping (autotuned): resident blocks per SM cap (0: occupancy maximum)
    // for the persistent team kernels, block size of the thread-per-system kernels
    int occ_cap = 0;
    int tps_block = 128;
    // team mapping of mass-action Radau: 0 the default team (one warp up to 32 state
    // elements, two warps up to 64); 16: two systems per warp (16 lanes each), for
    // state lengths up to 16 (analytic Jacobian, no learned mode)
    int team_lanes = 0;
    int grain = 1;                // work-queue slots a team claims per atomic
    int stage_extrap = 0;         // Radau starting values: 0 the reference's, 1 collocation
    int last_occ = 0;             // resident blocks per SM of the last team launch
    bool graph = false;           // device-buffer launches through a captured CUDA graph
    bool persistent = true;       // team kernels: persistent grid + work queue (else one team per system)
    int jac_mode = 0;             // 0 analytic Jacobian, 1 finite differences (fd_jacob.c)
    int order_mode = 0;           // work-queue order: 0 index, 1 by y_0 (descending), 2 by last call's steps
    int order_cap = 0;            // systems the order buffers hold
    int* order_buf = nullptr;     // [order_cap] queue slot -> system
    int* cost_buf = nullptr;      // [order_cap] steps of the last call per system (-1: unknown)
    float* key_buf = nullptr;     // [order_cap] sort keys
    int* hist_buf = nullptr;      // [ORDER_BUCKETS] histogram / offsets, then 2 floats (key min, max)
    const float* cost_params = nullptr;   // learned cost model (order_mode 3)
    const float* cost_norm = nullptr;
    float* cost_x = nullptr;      // [round16(order_cap) x 64] features
    float* cost_out = nullptr;    // [round16(order_cap) x 176] outputs
    cudaGraphExec_t gexec = nullptr;
    cudaStream_t cap_stream = nullptr;
};

State g;

constexpr int kMaxDevices = 64;
void noalloc_forget();   // allocation-free entry point: drops its cached scratch addresses

#define CK(x)                                                                                  \
    do {                                                                                       \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess) {                                                               \
            fprintf(stderr, "accelerint_b200: %s failed: %s (%s:%d)\n", #x, cudaGetErrorString(e_), \
                    __FILE__, __LINE__);                                                       \
            return ACCELERINT_ERR_CUDA;                                                        \
        }                                                                                      \
    } while (0)

int state_n() { return g.mech_kind == 0 ? 2 : g.mt.K + 1; }

int ensure_jac(size_t doubles) {
    if (doubles <= g.jac_doubles) return ACCELERINT_OK;
    if (g.jac) cudaFree(g.jac);
    g.jac = nullptr;
    g.jac_doubles = 0;
    CK(cudaMalloc(&g.jac, doubles * sizeof(double)));
    g.jac_doubles = doubles;
    return ACCELERINT_OK;
}

// CF poles and residues of the (10, 10) approximant for the current ATOL
// (rational_approximant.c:23-44 computes them once at start-up).
int compute_poles() {
    if (g.poles_atol == g.atol) return ACCELERINT_OK;
    if (aib_cf::poles_residues(CF_NRA, g.atol, g.poles[0], g.poles[1], g.poles[2], g.poles[3]) != 0)
        return ACCELERINT_ERR_UNSUPPORTED;
    g.poles_atol = g.atol;
    g.poles_device = -1;
    return ACCELERINT_OK;
}

int upload_poles() {
    int rc = compute_poles();
    if (rc) return rc;
    if (g.poles_device == g.device) return ACCELERINT_OK;
    CfTable tb;
    for (int i = 0; i < CF_NRA; ++i) {
        tb.pr[i] = g.poles[0][i];
        tb.pi[i] = g.poles[1][i];
        tb.rr[i] = g.poles[2][i];
        tb.ri[i] = g.poles[3][i];
    }
    CK(cudaMemcpyToSymbol(c_cf, &tb, sizeof(tb)));
    g.poles_device = g.device;
    return ACCELERINT_OK;
}

// Species count of the kernels that serve a mechanism of K species: K itself for the
// instantiated sizes (13, 53), else the next padded size (K + 1 rounded up to 16, 32,
// 48 or 64 state elements).  Padding species have no reactions, unit molar mass and
// zero heat capacity and enthalpy: their mass fractions stay zero and their rows and
// columns leave the real ones unchanged (only the error norms need the real length).
int device_species(int K) {
    if (K == 13 || K == 53) return K;
    const int n = K + 1;
    return n <= 16 ? 15 : n <= 32 ? 31 : n <= 48 ? 47 : 63;
}

int upload_mass_action() {
    MechTablesHost m = g.mt;
    const int kd = device_species(m.K);
    for (int k = m.K; k < kd; ++k) {
        m.mw.push_back(1.0);
        m.inv_mw.push_back(1.0);
        m.cp.push_back(0.0);
        m.h_form.push_back(0.0);
        m.s_ref.push_back(0.0);
        m.sp_ptr.push_back(m.sp_ptr.back());
    }
    m.K = kd;
    if (g.dev_tb_mem) cudaFree(g.dev_tb_mem);
    g.dev_tb_mem = nullptr;
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    const size_t nK = size_t(m.K) * sizeof(double), nR = size_t(m.R) * sizeof(double);
    size_t total = 5 * al(nK) + 3 * al(nR) + al(m.R * sizeof(int4)) + al((m.K + 1) * sizeof(int)) +
                   al(m.sp_ent.size() * sizeof(int));
    CK(cudaMalloc(&g.dev_tb_mem, total));
    char* p = static_cast<char*>(g.dev_tb_mem);
    auto put = [&](const void* src, size_t bytes) {
        void* dst = p;
        cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice);
        p += al(bytes);
        return dst;
    };
    MassActionTables t;
    t.K = m.K;
    t.R = m.R;
    t.inv_mw = static_cast<const double*>(put(m.inv_mw.data(), nK));
    t.mw = static_cast<const double*>(put(m.mw.data(), nK));
    t.cp = static_cast<const double*>(put(m.cp.data(), nK));
    t.h_form = static_cast<const double*>(put(m.h_form.data(), nK));
    t.s_ref = static_cast<const double*>(put(m.s_ref.data(), nK));
    t.log_a = static_cast<const double*>(put(m.log_a.data(), nR));
    t.beta = static_cast<const double*>(put(m.beta.data(), nR));
    t.ta = static_cast<const double*>(put(m.ta.data(), nR));
    t.rsp = static_cast<const int4*>(put(m.rsp.data(), m.R * sizeof(int4)));
    t.sp_ptr = static_cast<const int*>(put(m.sp_ptr.data(), (m.K + 1) * sizeof(int)));
    t.sp_ent = static_cast<const int*>(put(m.sp_ent.data(), m.sp_ent.size() * sizeof(int)));
    CK(cudaGetLastError());
    g.dev_tb = t;
    CK(cudaMemcpyToSymbol(c_ma, &t, sizeof(t)));
    return ACCELERINT_OK;
}

// ------------------------------------------------------------------ dispatch
template <class K> int persistent_grid(K kernel, int block, size_t smem, int num_teams_needed, int teams_per_block,
                                       int* grid) {
    if (smem > 48 * 1024) CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    // the whole carveout for shared memory, whatever cache preference the host set for the
    // device (the reference's own initialisation sets cudaFuncCachePreferL1 device-wide,
    // generic/solver_interface.cu:118, which would leave room for one or two teams per SM)
    CK(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, int(cudaSharedmemCarveoutMaxShared)));
    int nb = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, block, smem));
    if (nb <= 0) return ACCELERINT_ERR_UNSUPPORTED;
    if (g.occ_cap > 0) nb = std::min(nb, g.occ_cap);
    g.last_occ = nb;
    const int need = (num_teams_needed + teams_per_block - 1) / teams_per_block;
    *grid = std::max(1, std::min(nb * g.num_sms, need));
    return ACCELERINT_OK;
}

// Longest-first queue order for this launch (order_mode 1 or 2), on stream s.
int build_order(BatchArgs& a, cudaStream_t s) {
    if (a.num > g.order_cap) {
        if (g.order_buf) cudaFree(g.order_buf);
        if (g.cost_buf) cudaFree(g.cost_buf);
        if (g.key_buf) cudaFree(g.key_buf);
        if (g.hist_buf) cudaFree(g.hist_buf);
        g.order_buf = g.cost_buf = g.hist_buf = nullptr;
        g.key_buf = nullptr;
        g.order_cap = 0;
        CK(cudaMalloc(&g.order_buf, size_t(a.num) * sizeof(int)));
        CK(cudaMalloc(&g.cost_buf, size_t(a.num) * sizeof(int)));
        CK(cudaMalloc(&g.key_buf, size_t(a.num) * sizeof(float)));
        CK(cudaMalloc(&g.hist_buf, (ORDER_BUCKETS + 2) * sizeof(int)));
        if (g.cost_x) cudaFree(g.cost_x);
        if (g.cost_out) cudaFree(g.cost_out);
        g.cost_x = g.cost_out = nullptr;
        const size_t M = size_t(a.num + 15) / 16 * 16;
        CK(cudaMalloc(&g.cost_x, M * MLP_D0 * sizeof(float)));
        CK(cudaMalloc(&g.cost_out, M * MLP_D4 * sizeof(float)));
        CK(cudaMemsetAsync(g.cost_buf, 0xff, size_t(a.num) * sizeof(int), s));   // -1: unknown
        g.order_cap = a.num;
    }
    float* kmin = reinterpret_cast<float*>(g.hist_buf + ORDER_BUCKETS);
    float* kmax = kmin + 1;
    CK(cudaMemsetAsync(g.hist_buf, 0, ORDER_BUCKETS * sizeof(int), s));
    CK(cudaMemsetAsync(kmin, 0x7f, sizeof(float), s));   // 0x7f7f7f7f: a large positive float
    CK(cudaMemsetAsync(kmax, 0, sizeof(float), s));
    const int b = 256, nb = (a.num + b - 1) / b;
    const int* cost = g.order_mode == 2 ? g.cost_buf : nullptr;
    const float* ext = nullptr;
    if (g.order_mode == 3 && g.cost_params) {
        // learned cost of every system from its state (batched MLP on the tensor cores)
        const int k = aib_mlp::predict_cost(g.cost_params, g.cost_norm, a.num, state_n(), a.y, a.var,
                                            a.t_end - a.t_start, g.cost_x, g.cost_out, g.key_buf, s);
        if (k < 0) return ACCELERINT_ERR_CUDA;
        g.launches += k;
        ext = g.key_buf;
    }
    order_keys_kernel<<<nb, b, 0, s>>>(a.num, a.y, cost, ext, g.key_buf, kmin, kmax);
    order_hist_kernel<<<nb, b, 0, s>>>(a.num, g.key_buf, kmin, kmax, g.hist_buf);
    order_scan_kernel<<<1, ORDER_BUCKETS, 0, s>>>(g.hist_buf);
    order_scatter_kernel<<<nb, b, 0, s>>>(a.num, g.key_buf, kmin, kmax, g.hist_buf, g.order_buf);
    CK(cudaGetLastError());
    g.launches += 4;
    a.order = g.order_buf;
    a.cost = g.order_mode == 2 ? g.cost_buf : nullptr;
    return ACCELERINT_OK;
}

template <int SK, class Mech, int TS, typename LT, typename L1 = LT, int LEARN = 0>
int launch_team(BatchArgs a, const Mech& mech, TeamLayout lay, cudaStream_t s) {
    constexpr int N = Mech::N;
    const int block = TS >= 32 ? TS : 32, tpb = block / TS;
    const size_t smem = size_t(lay.total) * tpb;
    auto kern = team_kernel<SK, Mech, TS, LT, L1, LEARN>;
    int grid = 0;
    int rc = persistent_grid(kern, block, smem, a.num, tpb, &grid);
    if (rc) return rc;
    if (!g.persistent) {
        // plain form: one team per system over a full grid (the hardware block
        // scheduler balances), one Jacobian per system
        grid = (a.num + tpb - 1) / tpb;
        a.plain_grid = 1;
    }
    rc = ensure_jac(size_t(grid) * tpb * N * N);
    if (rc) return rc;
    a.jac = g.jac;
    if (g.persistent && g.order_mode != 0 && a.num > 0) {
        rc = build_order(a, s);
        if (rc) return rc;
    }
    if (g.persistent) CK(cudaMemsetAsync(a.queue, 0, sizeof(int), s));
    kern<<<grid, block, smem, s>>>(a, mech, lay);
    CK(cudaGetLastError());
    g.launches++;
    return ACCELERINT_OK;
}

// EXPRB43 (P = 4) or EXP4 (P = 1) on block teams of TS threads.
template <class Mech, int TS>
int launch_krylov(BatchArgs a, const Mech& mech, int rhs_doubles, int jac_doubles, cudaStream_t s) {
    constexpr int N = Mech::N;
    int rc = upload_poles();
    if (rc) return rc;
    if (g.solver == ACCELERINT_EXPRB43) {
        TeamLayout lay = TeamLayout::krylov(N, 4, rhs_doubles, jac_doubles);
        return launch_team<SK_EXPRB43, Mech, TS, double>(a, mech, lay, s);
    }
    TeamLayout lay = TeamLayout::krylov(N, 1, rhs_doubles, jac_doubles);
    return launch_team<SK_EXP4, Mech, TS, double>(a, mech, lay, s);
}

// Radau IIA on a mechanism padded to KP species (device_species): analytic
// Jacobian, no learned proposals; the caller's state has n_state = K + 1 rows.
template <int KP, int TS>
int launch_mass_action_padded(BatchArgs a, cudaStream_t s) {
    using M = MassAction<KP>;
    M mech;
    const int R = g.mt.R;
    constexpr int N = M::N;
    if (g.solver != ACCELERINT_RADAU2A || g.jac_mode != 0 || a.learn.mlp.flags || a.learn.rec)
        return ACCELERINT_ERR_UNSUPPORTED;
    a.n_state = g.mt.K + 1;
    if (g.lu == ACCELERINT_LU_FP32) {
        TeamLayout lay = TeamLayout::radau(N, 4, M::smem_rhs(R), M::smem_jac(R), 8);
        return launch_team<SK_RADAU, M, TS, float, double>(a, mech, lay, s);
    }
    if (g.lu == ACCELERINT_LU_FP32_ALL) {
        TeamLayout lay = TeamLayout::radau(N, 4, M::smem_rhs(R), M::smem_jac(R), 4);
        return launch_team<SK_RADAU, M, TS, float, float>(a, mech, lay, s);
    }
    TeamLayout lay = TeamLayout::radau(N, 8, M::smem_rhs(R), M::smem_jac(R));
    return launch_team<SK_RADAU, M, TS, double>(a, mech, lay, s);
}

template <int K, int TS>
int launch_mass_action(BatchArgs a, cudaStream_t s) {
    using M = MassAction<K>;
    M mech;
    const int R = g.mt.R;
    constexpr int N = M::N;
    if (g.jac_mode == 1) {
        // finite-difference Jacobian: plain FP64 Radau (the form of the reference's
        // FINITE_DIFFERENCE build)
        if (g.solver != ACCELERINT_RADAU2A || g.lu != ACCELERINT_LU_FP64) return ACCELERINT_ERR_UNSUPPORTED;
        FdJacobian<M> fd;
        fd.atol = g.atol;
        fd.rtol = g.rtol;
        TeamLayout lay = TeamLayout::radau(N, 8, M::smem_rhs(R), M::smem_jac(R));
        return launch_team<SK_RADAU, FdJacobian<M>, TS, double>(a, fd, lay, s);
    }
    if (g.solver == ACCELERINT_RADAU2A) {
        // learned level: 2 with stage proposals, 1 with step-size proposals or records only
        const int learn = (a.learn.mlp.flags & MLP_USE_Z) ? 2 : (a.learn.rec != nullptr || a.learn.mlp.flags) ? 1 : 0;
        if (g.lu == ACCELERINT_LU_FP32) {
            TeamLayout lay = TeamLayout::radau(N, 4, M::smem_rhs(R), M::smem_jac(R), 8);
            if (learn == 2) return launch_team<SK_RADAU, M, TS, float, double, 2>(a, mech, lay, s);
            if (learn == 1) return launch_team<SK_RADAU, M, TS, float, double, 1>(a, mech, lay, s);
            return launch_team<SK_RADAU, M, TS, float, double>(a, mech, lay, s);
        }
        if (g.lu == ACCELERINT_LU_FP32_ALL) {
            TeamLayout lay = TeamLayout::radau(N, 4, M::smem_rhs(R), M::smem_jac(R), 4);
            if (learn == 2) return launch_team<SK_RADAU, M, TS, float, float, 2>(a, mech, lay, s);
            if (learn == 1) return launch_team<SK_RADAU, M, TS, float, float, 1>(a, mech, lay, s);
            return launch_team<SK_RADAU, M, TS, float, float>(a, mech, lay, s);
        }
        TeamLayout lay = TeamLayout::radau(N, 8, M::smem_rhs(R), M::smem_jac(R));
        if (learn == 2) return launch_team<SK_RADAU, M, TS, double, double, 2>(a, mech, lay, s);
        if (learn == 1) return launch_team<SK_RADAU, M, TS, double, double, 1>(a, mech, lay, s);
        return launch_team<SK_RADAU, M, TS, double>(a, mech, lay, s);
    }
    if (g.solver == ACCELERINT_RKC) {
        TeamLayout lay = TeamLayout::rkc(N, M::smem_rhs(R));
        return launch_team<SK_RKC, M, TS, double>(a, mech, lay, s);
    }
    if (g.solver == ACCELERINT_EXPRB43 || g.solver == ACCELERINT_EXP4)
        return launch_krylov<M, TS>(a, mech, M::smem_rhs(R), M::smem_jac(R), s);
    return ACCELERINT_ERR_UNSUPPORTED;
}

int launch_vdp(BatchArgs a, cudaStream_t s) {
    const int block = g.tps_block, grid = (a.num + block - 1) / block;
    if (g.jac_mode == 1) {
        if (g.solver != ACCELERINT_RADAU2A || g.lu != ACCELERINT_LU_FP64) return ACCELERINT_ERR_UNSUPPORTED;
        FdJacobian<VanDerPol> fd;
        fd.atol = g.atol;
        fd.rtol = g.rtol;
        tps_kernel<SK_RADAU, FdJacobian<VanDerPol>, double><<<grid, block, 0, s>>>(a, fd);
        CK(cudaGetLastError());
        g.launches++;
        return ACCELERINT_OK;
    }
    if (g.solver == ACCELERINT_RADAU2A) {
        // E2 in FP32 (E1 in FP64), or both in FP32
        if (g.lu == ACCELERINT_LU_FP32)
            tps_kernel<SK_RADAU, VanDerPol, float, double><<<grid, block, 0, s>>>(a, VanDerPol{});
        else if (g.lu == ACCELERINT_LU_FP32_ALL)
            tps_kernel<SK_RADAU, VanDerPol, float, float><<<grid, block, 0, s>>>(a, VanDerPol{});
        else tps_kernel<SK_RADAU, VanDerPol, double><<<grid, block, 0, s>>>(a, VanDerPol{});
    } else if (g.solver == ACCELERINT_RKC) {
        tps_kernel<SK_RKC, VanDerPol, double><<<grid, block, 0, s>>>(a, VanDerPol{});
    } else if (g.solver == ACCELERINT_EXPRB43 || g.solver == ACCELERINT_EXP4) {
        return launch_krylov<VanDerPol, 32>(a, VanDerPol{}, 0, 0, s);
    } else {
        return ACCELERINT_ERR_UNSUPPORTED;
    }
    CK(cudaGetLastError());
    g.launches++;
    return ACCELERINT_OK;
}

template <int K, int TS, typename LT, typename L1>
int launch_decomp(int count, const double* jac, const double* h, void* e1, void* e2, int* perm, int* info,
                  cudaStream_t s) {
    using M = MassAction<K>;
    constexpr int N = M::N;
    const TeamLayout lay = TeamLayout::radau(N, int(sizeof(LT)), M::smem_rhs(0), M::smem_jac(0), int(sizeof(L1)));
    auto kern = decomp_kernel<M, TS, LT, L1>;
    if (lay.total > 48 * 1024) CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, lay.total));
    CK(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, int(cudaSharedmemCarveoutMaxShared)));
    kern<<<count, TS, lay.total, s>>>(count, jac, h, static_cast<L1*>(e1), static_cast<cx<LT>*>(e2), perm, info, lay);
    CK(cudaGetLastError());
    g.launches++;
    return ACCELERINT_OK;
}

template <int K, int TS>
int launch_decomp_prec(int precision, int count, const double* jac, const double* h, void* e1, void* e2, int* perm,
                       int* info, cudaStream_t s) {
    if (precision == ACCELERINT_LU_FP64) return launch_decomp<K, TS, double, double>(count, jac, h, e1, e2, perm, info, s);
    if (precision == ACCELERINT_LU_FP32) return launch_decomp<K, TS, float, double>(count, jac, h, e1, e2, perm, info, s);
    return launch_decomp<K, TS, float, float>(count, jac, h, e1, e2, perm, info, s);
}

// Two systems per warp (team_lanes 16) serve analytic-Jacobian Radau without learned
// proposals; other settings run on the default team.
bool half_warp_teams(const BatchArgs& a) {
    return g.team_lanes == 16 && g.solver == ACCELERINT_RADAU2A && g.jac_mode == 0 && !a.learn.mlp.flags &&
           !a.learn.rec;
}

int launch(BatchArgs a, cudaStream_t s) {
    if (a.num <= 0) return ACCELERINT_OK;
    a.grain = g.grain;
    a.stage_extrap = g.stage_extrap;
    if (g.mech_kind == 0) return launch_vdp(a, s);
    switch (device_species(g.mt.K)) {
        case 13:
            if (half_warp_teams(a)) return launch_mass_action_padded<13, 16>(a, s);
            return launch_mass_action<13, 32>(a, s);
        case 53: return launch_mass_action<53, 64>(a, s);
        case 15:
            if (half_warp_teams(a)) return launch_mass_action_padded<15, 16>(a, s);
            return launch_mass_action_padded<15, 32>(a, s);
        case 31: return launch_mass_action_padded<31, 32>(a, s);
        case 47: return launch_mass_action_padded<47, 64>(a, s);
        case 63: return launch_mass_action_padded<63, 64>(a, s);
        default: return ACCELERINT_ERR_UNSUPPORTED;
    }
}

int run_chunked(int NUM, double t_start, double t_end, double stepsize, double* y_host, const double* var_host) {
    if (!g.initialized) return ACCELERINT_ERR_STATE;
    if (NUM < 0 || !y_host || !var_host) return ACCELERINT_ERR_ARGUMENT;
    const int N = state_n();
    const double step = stepsize < 0 ? t_end - t_start : stepsize;
    g.codes.assign(NUM, 0);
    cudaStream_t s = g.stream;
    for (int off = 0; off < NUM; off += g.capacity) {
        const int cnt = std::min(g.capacity, NUM - off);
        CK(cudaMemcpyAsync(g.var_dev, var_host + off, cnt * sizeof(double), cudaMemcpyHostToDevice, s));
        CK(cudaMemcpy2DAsync(g.y_dev, cnt * sizeof(double), y_host + off, size_t(NUM) * sizeof(double),
                             cnt * sizeof(double), N, cudaMemcpyHostToDevice, s));
        BatchArgs a{};
        a.num = cnt;
        a.t_start = t_start;
        a.t_end = t_end;
        a.step = step;
        a.y = g.y_dev;
        a.var = g.var_dev;
        a.codes = g.codes_dev;
        a.stats = nullptr;
        a.queue = g.queue;
        a.atol = g.atol;
        a.rtol = g.rtol;
        a.learn = g.learn;
        int rc = launch(a, s);
        if (rc) return rc;
        CK(cudaMemcpy2DAsync(y_host + off, size_t(NUM) * sizeof(double), g.y_dev, cnt * sizeof(double),
                             cnt * sizeof(double), N, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(g.codes.data() + off, g.codes_dev, cnt * sizeof(int), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
    }
    for (int c : g.codes)
        if (c != 0) return ACCELERINT_ERR_SYSTEMS;
    return ACCELERINT_OK;
}

// Record this call's launch sequence (queue reset + kernel) by stream capture,
// update the cached executable graph in place when only parameters changed,
// and launch it on the caller's stream.
int launch_graph(BatchArgs a, cudaStream_t s) {
    if (!g.cap_stream) CK(cudaStreamCreateWithFlags(&g.cap_stream, cudaStreamNonBlocking));
    CK(cudaStreamBeginCapture(g.cap_stream, cudaStreamCaptureModeRelaxed));
    const int rc = launch(a, g.cap_stream);
    cudaGraph_t graph = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(g.cap_stream, &graph);
    if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    CK(ec);
    bool updated = false;
    if (g.gexec) {
        cudaGraphExecUpdateResultInfo info;
        updated = cudaGraphExecUpdate(g.gexec, graph, &info) == cudaSuccess;
        if (!updated) {
            cudaGetLastError();
            cudaGraphExecDestroy(g.gexec);
            g.gexec = nullptr;
        }
    }
    if (!updated) {
        const cudaError_t ei = cudaGraphInstantiate(&g.gexec, graph, 0);
        if (ei != cudaSuccess) {
            cudaGraphDestroy(graph);
            CK(ei);
        }
    }
    cudaGraphDestroy(graph);
    CK(cudaGraphLaunch(g.gexec, s));
    return ACCELERINT_OK;
}

int alloc_batch(int capacity) {
    const int N = state_n();
    if (g.y_dev) cudaFree(g.y_dev);
    if (g.var_dev) cudaFree(g.var_dev);
    if (g.codes_dev) cudaFree(g.codes_dev);
    g.y_dev = nullptr;
    g.var_dev = nullptr;
    g.codes_dev = nullptr;
    CK(cudaMalloc(&g.y_dev, size_t(capacity) * N * sizeof(double)));
    CK(cudaMalloc(&g.var_dev, size_t(capacity) * sizeof(double)));
    CK(cudaMalloc(&g.codes_dev, size_t(capacity) * sizeof(int)));
    g.capacity = capacity;
    return ACCELERINT_OK;
}

}  // namespace

extern "C" {

void accelerInt_initialize(int NUM, int device) {
    g.last_status = ACCELERINT_OK;
    noalloc_forget();
    device = device < 0 ? 0 : device;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device >= ndev) {
        fprintf(stderr, "accelerint_b200: GPU device %d not available (%d devices)\n", device, ndev);
        g.last_status = ACCELERINT_ERR_ARGUMENT;
        return;
    }
    if (cudaSetDevice(device) != cudaSuccess) { g.last_status = ACCELERINT_ERR_CUDA; return; }
    g.device = device;
    cudaDeviceGetAttribute(&g.num_sms, cudaDevAttrMultiProcessorCount, device);
    if (!g.stream) cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking);
    if (!g.queue && cudaMalloc(&g.queue, 256) != cudaSuccess) { g.last_status = ACCELERINT_ERR_CUDA; return; }
    size_t free_mem = 0, total_mem = 0;
    cudaMemGetInfo(&free_mem, &total_mem);
    const size_t per = size_t(64 + 2) * sizeof(double) + sizeof(int);
    const size_t cap = std::min<size_t>(std::max(NUM, 1), size_t(0.5 * double(free_mem) / double(per)));
    g.initialized = true;
    if (g.mech_kind == 1 && g.mt.K > 0) {
        int rc = upload_mass_action();
        if (rc) { g.last_status = rc; return; }
    }
    g.last_status = alloc_batch(int(cap));
}

void accelerInt_integrate(const int NUM, const double t_start, const double t_end, const double stepsize,
                          double* y_host, const double* var_host) {
    g.last_status = run_chunked(NUM, t_start, t_end, stepsize, y_host, var_host);
}

void accelerInt_cleanup(void) {
    noalloc_forget();
    if (g.y_dev) cudaFree(g.y_dev);
    if (g.var_dev) cudaFree(g.var_dev);
    if (g.codes_dev) cudaFree(g.codes_dev);
    if (g.jac) cudaFree(g.jac);
    if (g.queue) cudaFree(g.queue);
    if (g.mlp_w) cudaFree(g.mlp_w);
    g.mlp_w = nullptr;
    aib_mlp::free_work();
    if (g.gexec) cudaGraphExecDestroy(g.gexec);
    g.gexec = nullptr;
    if (g.cap_stream) cudaStreamDestroy(g.cap_stream);
    g.cap_stream = nullptr;
    g.occ_cap = 0;
    g.tps_block = 128;
    g.team_lanes = 0;
    g.grain = 1;
    g.stage_extrap = 0;
    g.graph = false;
    g.persistent = true;
    g.jac_mode = 0;
    g.order_mode = 0;
    if (g.order_buf) cudaFree(g.order_buf);
    if (g.cost_buf) cudaFree(g.cost_buf);
    if (g.key_buf) cudaFree(g.key_buf);
    if (g.hist_buf) cudaFree(g.hist_buf);
    g.order_buf = g.cost_buf = g.hist_buf = nullptr;
    g.key_buf = nullptr;
    g.order_cap = 0;
    if (g.cost_x) cudaFree(g.cost_x);
    if (g.cost_out) cudaFree(g.cost_out);
    g.cost_x = g.cost_out = nullptr;
    g.cost_params = g.cost_norm = nullptr;
    g.learn = LearnArgs{};
    if (g.dev_tb_mem) cudaFree(g.dev_tb_mem);
    if (g.stream) cudaStreamDestroy(g.stream);
    g.y_dev = nullptr;
    g.var_dev = nullptr;
    g.codes_dev = nullptr;
    g.jac = nullptr;
    g.jac_doubles = 0;
    g.queue = nullptr;
    g.dev_tb_mem = nullptr;
    g.stream = nullptr;
    g.initialized = false;
    g.capacity = 0;
}

int accelerInt_set_solver(int solver) {
    if (solver < ACCELERINT_RADAU2A || solver > ACCELERINT_RKC) return ACCELERINT_ERR_ARGUMENT;
    g.solver = solver;
    return ACCELERINT_OK;
}

int accelerInt_set_mechanism_van_der_pol(void) {
    g.mech_kind = 0;
    if (g.initialized && g.capacity > 0) return alloc_batch(g.capacity);
    return ACCELERINT_OK;
}

int accelerInt_set_mechanism_mass_action(const accelerInt_mass_action* m) {
    if (!m || m->n_species < 1 || m->n_species > 63 || m->n_reactions < 1) return ACCELERINT_ERR_ARGUMENT;
    MechTablesHost t;
    t.K = m->n_species;
    t.R = m->n_reactions;
    for (int k = 0; k < t.K; ++k) {
        if (!(m->mw[k] > 0)) return ACCELERINT_ERR_ARGUMENT;
        t.mw.push_back(m->mw[k]);
        t.inv_mw.push_back(1.0 / m->mw[k]);
        t.cp.push_back(m->cp[k]);
        t.h_form.push_back(m->h_form[k]);
        t.s_ref.push_back(m->s_ref[k]);
    }
    std::vector<std::vector<int>> lists(t.K);
    for (int r = 0; r < t.R; ++r) {
        int4 q{m->reac[2 * r], m->reac[2 * r + 1], m->prod[2 * r], m->prod[2 * r + 1]};
        const int sl[4] = {q.x, q.y, q.z, q.w};
        if (q.x < 0 || q.z < 0) return ACCELERINT_ERR_ARGUMENT;
        for (int a = 0; a < 4; ++a) {
            if (sl[a] >= t.K) return ACCELERINT_ERR_ARGUMENT;
            if (sl[a] >= 0) lists[sl[a]].push_back(4 * r + a);
        }
        t.rsp.push_back(q);
        t.log_a.push_back(m->log_a[r]);
        t.beta.push_back(m->beta[r]);
        t.ta.push_back(m->ta[r]);
    }
    t.sp_ptr.push_back(0);
    for (int k = 0; k < t.K; ++k) {
        for (int e : lists[k]) t.sp_ent.push_back(e);
        t.sp_ptr.push_back(int(t.sp_ent.size()));
    }
    g.mt = t;
    g.mech_kind = 1;
    if (g.initialized) {
        int rc = upload_mass_action();
        if (rc) return rc;
        if (g.capacity > 0) return alloc_batch(g.capacity);
    }
    return ACCELERINT_OK;
}

int accelerInt_set_tolerances(double atol, double rtol) {
    if (!(atol > 0) || !(rtol > 0)) return ACCELERINT_ERR_ARGUMENT;
    g.atol = atol;
    g.rtol = rtol;
    return ACCELERINT_OK;
}

int accelerInt_set_lu_precision(int precision) {
    if (precision != ACCELERINT_LU_FP64 && precision != ACCELERINT_LU_FP32 && precision != ACCELERINT_LU_FP32_ALL)
        return ACCELERINT_ERR_ARGUMENT;
    g.lu = precision;
    return ACCELERINT_OK;
}

int accelerInt_integrate_status(int NUM, double t_start, double t_end, double stepsize, double* y_host,
                                const double* var_host) {
    g.last_status = run_chunked(NUM, t_start, t_end, stepsize, y_host, var_host);
    return g.last_status;
}

int accelerInt_integrate_device(int NUM, double t_start, double t_end, double stepsize, double* y_dev,
                                const double* var_dev, int* codes_dev, int* stats_dev, void* stream) {
    if (!g.initialized) return ACCELERINT_ERR_STATE;
    if (NUM < 0 || (NUM > 0 && (!y_dev || !var_dev))) return ACCELERINT_ERR_ARGUMENT;
    BatchArgs a{};
    a.num = NUM;
    a.t_start = t_start;
    a.t_end = t_end;
    a.step = stepsize < 0 ? t_end - t_start : stepsize;
    a.y = y_dev;
    a.var = var_dev;
    a.codes = codes_dev;
    a.stats = stats_dev;
    a.queue = g.queue;
    a.atol = g.atol;
    a.rtol = g.rtol;
    a.learn = g.learn;
    if (!g.graph) return launch(a, static_cast<cudaStream_t>(stream));
    if (g.solver == ACCELERINT_EXPRB43 || g.solver == ACCELERINT_EXP4) {
        const int rc = upload_poles();   // a synchronous copy: before the capture
        if (rc) return rc;
    }
    return launch_graph(a, static_cast<cudaStream_t>(stream));
}

int accelerInt_last_status(void) { return g.last_status; }

int accelerInt_get_codes(int* codes_host, int NUM) {
    if (!codes_host || NUM < 0 || size_t(NUM) > g.codes.size()) return ACCELERINT_ERR_ARGUMENT;
    std::memcpy(codes_host, g.codes.data(), size_t(NUM) * sizeof(int));
    return ACCELERINT_OK;
}

int accelerInt_get_poles(double* pr, double* pi, double* rr, double* ri) {
    if (!pr || !pi || !rr || !ri) return ACCELERINT_ERR_ARGUMENT;
    const int rc = compute_poles();
    if (rc) return rc;
    for (int i = 0; i < 10; ++i) {
        pr[i] = g.poles[0][i];
        pi[i] = g.poles[1][i];
        rr[i] = g.poles[2][i];
        ri[i] = g.poles[3][i];
    }
    return ACCELERINT_OK;
}

long long accelerInt_kernel_launches(void) { return g.launches; }

int accelerInt_radau_decomp(int n, int precision, int count, const double* jac_dev, const double* h_dev,
                            void* e1_dev, void* e2_dev, int* perm_dev, int* info_dev, void* stream) {
    if (count < 0 || (count > 0 && (!jac_dev || !h_dev || !e1_dev || !e2_dev || !perm_dev || !info_dev)))
        return ACCELERINT_ERR_ARGUMENT;
    if (precision != ACCELERINT_LU_FP64 && precision != ACCELERINT_LU_FP32 && precision != ACCELERINT_LU_FP32_ALL)
        return ACCELERINT_ERR_ARGUMENT;
    if (count == 0) return ACCELERINT_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    switch (n) {
        case 14: return launch_decomp_prec<13, 32>(precision, count, jac_dev, h_dev, e1_dev, e2_dev, perm_dev,
                                                   info_dev, s);
        case 54: return launch_decomp_prec<53, 64>(precision, count, jac_dev, h_dev, e1_dev, e2_dev, perm_dev,
                                                   info_dev, s);
        default: return ACCELERINT_ERR_UNSUPPORTED;
    }
}

int accelerInt_set_learned(const float* params_dev, const float* norm_dev, int flags) {
    if (flags & ~(ACCELERINT_MLP_USE_H | ACCELERINT_MLP_USE_Z)) return ACCELERINT_ERR_ARGUMENT;
    if (flags == 0) {
        g.learn.mlp = MlpDevice{};
        return ACCELERINT_OK;
    }
    if (!params_dev || !norm_dev) return ACCELERINT_ERR_ARGUMENT;
    if (!g.initialized) return ACCELERINT_ERR_STATE;
    if (!g.mlp_w) CK(cudaMalloc(&g.mlp_w, size_t(MLP_NWEIGHT) * 2));
    if (aib_mlp::to_bf16(params_dev, g.mlp_w, nullptr)) return ACCELERINT_ERR_CUDA;
    CK(cudaDeviceSynchronize());
    g.learn.mlp.w = static_cast<const __nv_bfloat16*>(g.mlp_w);
    g.learn.mlp.p = params_dev;
    g.learn.mlp.norm = norm_dev;
    g.learn.mlp.flags = flags;
    if (!(g.learn.mlp.growth_floor > 1.0)) g.learn.mlp.growth_floor = 2.0;
    return ACCELERINT_OK;
}

int accelerInt_set_learned_growth_floor(double floor) {
    if (!(floor >= 1.05) || !(floor <= 8.0)) return ACCELERINT_ERR_ARGUMENT;
    g.learn.mlp.growth_floor = floor;
    return ACCELERINT_OK;
}

int accelerInt_set_persistent(int enable) {
    g.persistent = enable != 0;
    return ACCELERINT_OK;
}

int accelerInt_set_cost_model(const float* params_dev, const float* norm_dev) {
    if ((params_dev == nullptr) != (norm_dev == nullptr)) return ACCELERINT_ERR_ARGUMENT;
    g.cost_params = params_dev;
    g.cost_norm = norm_dev;
    return ACCELERINT_OK;
}

int accelerInt_set_jacobian(int mode) {
    if (mode != 0 && mode != 1) return ACCELERINT_ERR_ARGUMENT;
    g.jac_mode = mode;
    return ACCELERINT_OK;
}

int accelerInt_set_queue_order(int mode) {
    if (mode < 0 || mode > 3) return ACCELERINT_ERR_ARGUMENT;
    if (mode == 3 && !g.cost_params) return ACCELERINT_ERR_STATE;
    g.order_mode = mode;
    // the step-count history starts over: the next call orders by y_0 (after any
    // launch still writing step counts has finished)
    if (g.cost_buf) {
        CK(cudaDeviceSynchronize());
        CK(cudaMemset(g.cost_buf, 0xff, size_t(g.order_cap) * sizeof(int)));
    }
    return ACCELERINT_OK;
}

int accelerInt_set_graph_launch(int enable) {
    g.graph = enable != 0;
    return ACCELERINT_OK;
}

int accelerInt_set_launch_config(int occupancy_cap, int tps_block) {
    if (occupancy_cap < 0 || (tps_block != 0 && (tps_block < 32 || tps_block > 1024 || tps_block % 32)))
        return ACCELERINT_ERR_ARGUMENT;
    g.occ_cap = occupancy_cap;
    if (tps_block) g.tps_block = tps_block;
    return ACCELERINT_OK;
}

int accelerInt_set_stage_extrapolation(int mode) {
    if (mode != 0 && mode != 1) return ACCELERINT_ERR_ARGUMENT;
    g.stage_extrap = mode;
    return ACCELERINT_OK;
}

int accelerInt_set_mapping(int team_lanes, int grain) {
    if ((team_lanes != 0 && team_lanes != 16) || grain < 1 || grain > 64) return ACCELERINT_ERR_ARGUMENT;
    g.team_lanes = team_lanes;
    g.grain = grain;
    return ACCELERINT_OK;
}

int accelerInt_get_mapping(int* team_lanes, int* grain, int* occupancy) {
    if (team_lanes) *team_lanes = g.team_lanes;
    if (grain) *grain = g.grain;
    if (occupancy) *occupancy = g.last_occ;
    return ACCELERINT_OK;
}

int accelerInt_autotune(int NUM, double t_start, double t_end, double stepsize, const double* y_dev,
                        const double* var_dev, int sample, int* occupancy_cap_out, int* tps_block_out,
                        double* best_ms_out) {
    if (!g.initialized) return ACCELERINT_ERR_STATE;
    if (NUM <= 0 || !y_dev || !var_dev || sample <= 0) return ACCELERINT_ERR_ARGUMENT;
    sample = std::min(sample, NUM);
    const int N = state_n();
    double* ys = nullptr;
    CK(cudaMalloc(&ys, size_t(sample) * N * sizeof(double)));
    cudaStream_t s = g.stream;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto trial = [&](double* ms) -> int {
        CK(cudaMemcpy2DAsync(ys, sample * sizeof(double), y_dev, size_t(NUM) * sizeof(double),
                             sample * sizeof(double), N, cudaMemcpyDeviceToDevice, s));
        BatchArgs a{};
        a.num = sample;
        a.t_start = t_start;
        a.t_end = t_end;
        a.step = stepsize < 0 ? t_end - t_start : stepsize;
        a.y = ys;
        a.var = var_dev;
        a.queue = g.queue;
        a.atol = g.atol;
        a.rtol = g.rtol;
        a.learn = g.learn;
        CK(cudaEventRecord(e0, s));
        int rc = launch(a, s);
        if (rc) return rc;
        CK(cudaEventRecord(e1, s));
        CK(cudaEventSynchronize(e1));
        float f = 0;
        CK(cudaEventElapsedTime(&f, e0, e1));
        *ms = f;
        return ACCELERINT_OK;
    };
    int rc = ACCELERINT_OK;
    double best = 1e300, ms = 0;
    // a candidate replaces the current choice only when it is 3 % faster: on a sample the
    // launch's tail varies by a few per cent from trial to trial
    constexpr double kKeep = 0.97;
    if (g.mech_kind == 0 && (g.solver == ACCELERINT_RADAU2A || g.solver == ACCELERINT_RKC)) {
        // thread per system: block size
        int best_b = g.tps_block;
        for (int b : {32, 64, 128}) {   // the kernels' launch bound is 128 threads
            g.tps_block = b;
            if ((rc = trial(&ms))) break;
            if (ms < best) { best = ms; best_b = b; }
        }
        g.tps_block = best_b;
    } else {
        // persistent teams: resident blocks per SM, from the occupancy maximum down to half of it
        g.occ_cap = 0;
        rc = trial(&ms);   // also measures the maximum
        // a few systems per resident team time the slowest system rather than the
        // mapping: grow the sample to 16 per team (up to NUM) and measure again
        const int want = std::min(NUM, 16 * g.last_occ * g.num_sms);
        if (!rc && want > sample) {
            cudaFree(ys);
            ys = nullptr;
            sample = want;
            CK(cudaMalloc(&ys, size_t(sample) * N * sizeof(double)));
            rc = trial(&ms);
        }
        int best_c = 0;
        if (!rc) {
            best = ms;
            const int mx = g.last_occ;
            for (int c = mx - 1; c >= std::max(1, (mx + 1) / 2) && !rc; --c) {
                g.occ_cap = c;
                if ((rc = trial(&ms))) break;
                if (ms < kKeep * best) { best = ms; best_c = c; }
            }
        }
        g.occ_cap = best_c;
        // queue order: index order vs longest (hottest) first, at the chosen occupancy
        if (!rc && g.persistent) {
            const int keep = g.order_mode;
            int best_o = keep;
            for (int o : {0, 1}) {
                if (o == keep) continue;
                g.order_mode = o;
                if ((rc = trial(&ms))) break;
                if (ms < kKeep * best) { best = ms; best_o = o; }
            }
            g.order_mode = best_o;
        }
        // mapping: two systems per warp where the state fits 16 lanes (at the
        // occupancy maximum of that kernel), then the queue granularity
        if (!rc && g.mech_kind == 1 && g.mt.K + 1 <= 16 && g.solver == ACCELERINT_RADAU2A && g.jac_mode == 0 &&
            !g.learn.mlp.flags && !g.learn.rec) {
            const int keep_lanes = g.team_lanes, keep_cap = g.occ_cap;
            g.team_lanes = 16;
            g.occ_cap = 0;
            if (!(rc = trial(&ms)) && ms < kKeep * best) {
                best = ms;
            } else {
                g.team_lanes = keep_lanes;
                g.occ_cap = keep_cap;
            }
        }
        if (!rc && g.persistent) {
            int best_gr = g.grain;
            for (int gr : {1, 2, 4, 8}) {
                if (gr == best_gr) continue;
                const int keep = g.grain;
                g.grain = gr;
                if ((rc = trial(&ms))) break;
                if (ms < kKeep * best) { best = ms; best_gr = gr; }
                g.grain = keep;
            }
            g.grain = best_gr;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(ys);
    if (rc) return rc;
    if (occupancy_cap_out) *occupancy_cap_out = g.occ_cap | (g.order_mode << 16);
    if (tps_block_out) *tps_block_out = g.tps_block;
    if (best_ms_out) *best_ms_out = best;
    return ACCELERINT_OK;
}

int accelerInt_set_step_recording(float* rec_dev, int* count_dev, int capacity) {
    if (rec_dev && (!count_dev || capacity < 0)) return ACCELERINT_ERR_ARGUMENT;
    g.learn.rec = rec_dev;
    g.learn.rec_count = rec_dev ? count_dev : nullptr;
    g.learn.rec_cap = rec_dev ? capacity : 0;
    return ACCELERINT_OK;
}

const char* accelerInt_version(void) { return "accelerint_b200 0.1 (sm_100a)"; }

int accelerInt_measure_fma_peak(int fp64, double* tflops) {
    if (!tflops) return ACCELERINT_ERR_ARGUMENT;
    int dev = 0, sms = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    void* out = nullptr;
    const int block = 256, grid = sms * 8, iters = 4096;
    if (fp64 < 0 || fp64 > 2) return ACCELERINT_ERR_ARGUMENT;
    CK(cudaMalloc(&out, size_t(grid) * block * sizeof(double)));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(e0);
        if (fp64 == 1) fma_peak_kernel<double><<<grid, block>>>(static_cast<double*>(out), iters, 1.0000001);
        else if (fp64 == 2)
            fma_peak_kernel2<<<grid, block>>>(static_cast<float2*>(out), iters, make_float2(1.0000001f, 0.9999999f));
        else fma_peak_kernel<float><<<grid, block>>>(static_cast<float*>(out), iters, 1.0000001f);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0) best = std::min(best, ms);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    CK(cudaGetLastError());
    // 8 independent chains per thread; a packed FP32x2 FMA is two FMAs
    const double flops = 2.0 * 8.0 * double(iters) * grid * block * (fp64 == 2 ? 2.0 : 1.0);
    *tflops = flops / (best * 1e-3) / 1e12;
    return ACCELERINT_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free entry point.  Its device scratch (the work-queue counter and
// the per-team Jacobians of the mass-action Radau kernel) lives in this
// file-scope array instead of memory from cudaMalloc.  Every device that loads
// the library holds the array until the process exits.
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;   // 16 MiB
constexpr size_t kNoAllocQueueBytes = 256;                   // queue counter + padding
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

void* g_noalloc_ptr[kMaxDevices] = {};

// Forget the cached device addresses: after a device reset (the reference's
// solver_interface.cu:111,224 calls cudaDeviceReset) the module, and with it the
// array, may be loaded again at another address.
void noalloc_forget() {
    for (int d = 0; d < kMaxDevices; ++d) g_noalloc_ptr[d] = nullptr;
}

// Device address of the array for the current device, looked up once per device.
// In host code the array's name is only a host-side stand-in, never a device address.
int noalloc_scratch(void** out) {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return ACCELERINT_ERR_ARGUMENT;
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            fprintf(stderr, "accelerint_b200: cudaGetSymbolAddress of the static scratch failed: %s\n",
                    cudaGetErrorString(e));
            return ACCELERINT_ERR_CUDA;
        }
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return ACCELERINT_OK;
}

template <int SK, class Mech, int TS, typename LT, typename L1 = LT>
int launch_team_noalloc(BatchArgs a, const Mech& mech, TeamLayout lay, unsigned char* scratch, cudaStream_t s) {
    constexpr int N = Mech::N;
    const size_t per_team = size_t(N) * N * sizeof(double);
    const size_t fit = (kNoAllocScratchBytes - kNoAllocQueueBytes) / per_team;
    if (fit < 1) {
        fprintf(stderr, "accelerint_b200: state length %d needs %zu bytes of scratch per system in flight; "
                        "the allocation-free entry point holds %zu\n", N, per_team + kNoAllocQueueBytes,
                kNoAllocScratchBytes);
        return ACCELERINT_ERR_ARGUMENT;
    }
    const int block = TS >= 32 ? TS : 32, tpb = block / TS;
    const size_t smem = size_t(lay.total) * tpb;
    auto kern = team_kernel<SK, Mech, TS, LT, L1>;
    int grid = 0;
    int rc = persistent_grid(kern, block, smem, a.num, tpb, &grid);
    if (rc) return rc;
    // fewer teams in flight when the scratch cannot hold a Jacobian for each (the work queue keeps it correct)
    grid = int(std::min<size_t>(size_t(grid), fit / size_t(tpb)));
    if (grid < 1) return ACCELERINT_ERR_ARGUMENT;
    a.queue = reinterpret_cast<int*>(scratch);
    a.jac = reinterpret_cast<double*>(scratch + kNoAllocQueueBytes);
    CK(cudaMemsetAsync(a.queue, 0, sizeof(int), s));   // the counter must start at zero on every call
    kern<<<grid, block, smem, s>>>(a, mech, lay);
    CK(cudaGetLastError());
    g.launches++;
    return ACCELERINT_OK;
}

template <int K, int TS>
int launch_mass_action_noalloc(BatchArgs a, unsigned char* scratch, cudaStream_t s) {
    using M = MassAction<K>;
    M mech;
    const int R = g.mt.R;
    constexpr int N = M::N;
    if (g.solver != ACCELERINT_RADAU2A) return ACCELERINT_ERR_UNSUPPORTED;
    // learned proposals and step recording have no allocation-free kernels: refuse
    // rather than integrate differently from accelerInt_integrate_device
    if (g.learn.mlp.flags != 0 || g.learn.rec != nullptr) return ACCELERINT_ERR_UNSUPPORTED;
    if (g.jac_mode == 1) {
        // finite-difference Jacobian, as the allocating entry point runs it: plain FP64 only
        if (g.lu != ACCELERINT_LU_FP64) return ACCELERINT_ERR_UNSUPPORTED;
        FdJacobian<M> fd;
        fd.atol = g.atol;
        fd.rtol = g.rtol;
        TeamLayout lay = TeamLayout::radau(N, 8, M::smem_rhs(R), M::smem_jac(R));
        return launch_team_noalloc<SK_RADAU, FdJacobian<M>, TS, double>(a, fd, lay, scratch, s);
    }
    if (g.lu == ACCELERINT_LU_FP32) {
        TeamLayout lay = TeamLayout::radau(N, 4, M::smem_rhs(R), M::smem_jac(R), 8);
        return launch_team_noalloc<SK_RADAU, M, TS, float, double>(a, mech, lay, scratch, s);
    }
    if (g.lu == ACCELERINT_LU_FP32_ALL) {
        TeamLayout lay = TeamLayout::radau(N, 4, M::smem_rhs(R), M::smem_jac(R), 4);
        return launch_team_noalloc<SK_RADAU, M, TS, float, float>(a, mech, lay, scratch, s);
    }
    TeamLayout lay = TeamLayout::radau(N, 8, M::smem_rhs(R), M::smem_jac(R));
    return launch_team_noalloc<SK_RADAU, M, TS, double>(a, mech, lay, scratch, s);
}

}  // namespace

extern "C" int accelerInt_integrate_device_noalloc(int NUM, double t_start, double t_end, double stepsize,
                                                   double* y_dev, const double* var_dev, int* codes_dev,
                                                   void* stream) {
    if (!g.initialized || g.mech_kind != 1) return ACCELERINT_ERR_STATE;
    if (NUM < 0 || (NUM > 0 && (!y_dev || !var_dev))) return ACCELERINT_ERR_ARGUMENT;
    if (NUM == 0) return ACCELERINT_OK;
    void* scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc) return rc;
    BatchArgs a{};
    a.num = NUM;
    a.t_start = t_start;
    a.t_end = t_end;
    a.step = stepsize < 0 ? t_end - t_start : stepsize;
    a.y = y_dev;
    a.var = var_dev;
    a.codes = codes_dev;
    a.stats = nullptr;
    a.atol = g.atol;
    a.rtol = g.rtol;
    a.stage_extrap = g.stage_extrap;
    unsigned char* sp = static_cast<unsigned char*>(scratch);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    switch (g.mt.K) {
        case 13: return launch_mass_action_noalloc<13, 32>(a, sp, st);
        case 53: return launch_mass_action_noalloc<53, 64>(a, sp, st);
        default: return ACCELERINT_ERR_UNSUPPORTED;
    }
}
