// Batch kernels: the device side of accelerInt_integrate.
//
// The reference launches one thread per system over a padded grid
// (generic/solver_generic.cu:28-42, solver_interface.cu:189).  Here:
//   * thread-per-system kernels for the 2-state van der Pol workload, state in
//     registers, coalesced structure-of-arrays loads y[i*num + ivp];
//   * persistent team kernels for the mass-action mechanisms: one team of TS
//     lanes per system, its matrices in shared memory; teams pull systems from
//     a device work queue (one atomic per system), so systems with very
//     different stiffness do not hold each other up.  The queue can be taken
//     in a longest-first order (a counting sort of per-system cost keys,
//     order_*_kernel below) so that the launch does not end on one stiff
//     system; a plain-grid mode (one team per system) is the plain form.
// Every kernel integrates all global steps [t_k, t_{k+1}] of its systems in
// one launch; each step restarts the integrator exactly as a separate
// intDriver call of the reference would.
#pragma once
#include "common.cuh"
#include "mech.cuh"
#include "radau2a.cuh"
#include "rkc.cuh"
#include "krylov.cuh"

namespace aib {

struct BatchArgs {
    int num;
    double t_start, t_end, step;
    double* y;              // [N * num] column-major, IVP fastest
    const double* var;      // [num]
    int* codes;             // [num] or null
    int* stats;             // [num * NSTATS] or null
    int* queue;             // work-queue counter (zeroed before launch)
    double* jac;            // per-team Jacobian scratch [teams * N * N]
    double atol, rtol;
    LearnArgs learn;        // Radau block teams: learned proposals / step records (zero: off)
    int plain_grid;         // team kernels: one team per system over a full grid, no work queue
    const int* order;       // queue order (system index of each queue slot), or null: index order
    int* cost;              // per-system steps of this call (written), or null
    int n_state;            // the caller's state length (rows of y), when the kernel's N pads it; 0: N
    int grain;              // queue slots a team claims per atomic (0 or 1: one)
    int stage_extrap;       // Radau starting values after an accepted step (RadauParams::stage_extrap)
};

// The reference's global-step loop (generic/solver_main.c:196-209), measured from t_start.
struct StepLoop {
    double t, t_next, t_start, t_end, step;
    int k;
    __device__ StepLoop(double a, double b, double s) : t(a), t_start(a), t_end(b), step(s), k(0) {
        t_next = fmin(t_end, t_start + step);
    }
    __device__ bool more() const { return t + DBL_EPSILON < t_end; }
    __device__ void advance() {
        ++k;
        t = t_next;
        t_next = fmin(t_end, t_start + double(k + 1) * step);
    }
};

template <int N, int TS>
__device__ __forceinline__ void store_stats(const BatchArgs& a, int sys, const Stats& st) {
    if (a.stats && Team<TS>::lane() == 0) {
        int* o = a.stats + size_t(sys) * NSTATS;
#pragma unroll
        for (int k = 0; k < NSTATS; ++k) o[k] += st.c[k];
    }
}

// ------------------------------------------------------------- thread per system
enum SolverKind { SK_RADAU = 0, SK_EXPRB43 = 1, SK_EXP4 = 2, SK_RKC = 3 };

template <int SK, class Mech, typename LT, typename L1 = LT>
__global__ void __launch_bounds__(128) tps_kernel(BatchArgs a, Mech mech)
{
    constexpr int N = Mech::N;
    const int sys = blockIdx.x * blockDim.x + threadIdx.x;
    if (sys >= a.num) return;
    Vec<N, 1> y;
#pragma unroll
    for (int i = 0; i < N; ++i) y[i] = a.y[size_t(i) * a.num + sys];
    const double pr = a.var[sys];
    Stats st;
    st.clear();
    int code = EC_success;
    StepLoop L(a.t_start, a.t_end, a.step);
    if constexpr (SK == SK_RADAU) {
        RadauRegStore<N, LT, L1> store;
        Radau<N, 1, Mech, LT, RadauRegStore<N, LT, L1>> rad{mech, store, RadauParams{a.atol, a.rtol, 0, a.stage_extrap},
                                                            pr, st};
        while (L.more() && code == EC_success) {
            code = rad.integrate(L.t, L.t_next, y);
            L.advance();
        }
    } else if constexpr (SK == SK_RKC) {
        Rkc<N, 1, Mech> rk{mech, nullptr, a.atol, a.rtol, pr, st};
        while (L.more() && code == EC_success) {
            code = rk.integrate(L.t, L.t_next, y);
            L.advance();
        }
    }
#pragma unroll
    for (int i = 0; i < N; ++i) {
        a.y[size_t(i) * a.num + sys] = y[i];
        if (code == EC_success && !isfinite(y[i])) code = EC_nonfinite_state;
    }
    if (a.codes) a.codes[sys] = code;
    store_stats<N, 1>(a, sys, st);
}

// ------------------------------------------------------------- team per system
// Shared-memory layout of one team (bytes, 16-byte aligned pieces).
struct TeamLayout {
    int e1, e2, d1, d2, p1, p2, buf, rhs, inf, total;
    int vm, hm, phi, inv, cw, piv, mv, nv;   // Krylov methods
    __host__ __device__ static int al(int b) { return (b + 15) & ~15; }
    // lt_bytes: element size of E2's real type; l1_bytes: of E1
    __host__ __device__ static TeamLayout radau(int N, int lt_bytes, int rhs_doubles, int jac_doubles,
                                                int l1_bytes = 0) {
        TeamLayout L;
        int o = 0;
        if (l1_bytes == 0) l1_bytes = lt_bytes;
        const int NC = lu_cols(N);   // padded column count of the block-team factorisation
        L.e1 = o; o += al(N * NC * l1_bytes);
        L.e2 = o;
        const int e2b = N * NC * 2 * lt_bytes, jb = jac_doubles * 8;
        o += al(e2b > jb ? e2b : jb);
        L.d1 = o; o += al(N * l1_bytes);
        L.d2 = o; o += al(N * 2 * lt_bytes);
        L.p1 = o; o += al(N * 4);
        L.p2 = o; o += al(N * 4);
        L.buf = o; o += al(3 * N * 8);
        // dydt scratch; also holds the MLP input and activations in learned mode
        const int rb = rhs_doubles * 8 > (MLP_D0 + 2 * MLP_D4) * 4 ? rhs_doubles * 8 : (MLP_D0 + 2 * MLP_D4) * 4;
        L.rhs = o; o += al(rb);
        L.inf = o; o += al(4 * 4);   // factorisation status of E1, E2; pivot exchange slots of the LU
        L.total = o;
        return L;
    }
    // stride = N + P; the complex work matrix doubles as mechanism scratch
    __host__ __device__ static TeamLayout krylov(int N, int P, int rhs_doubles, int jac_doubles) {
        TeamLayout L{};
        const int S = N + P;
        int o = 0;
        L.vm = o; o += al(N * S * 8);
        L.hm = o; o += al(S * S * 8);
        L.phi = o; o += al(S * S * 8);
        L.inv = o;
        int ib = S * S * 16;
        if (rhs_doubles * 8 > ib) ib = rhs_doubles * 8;
        if (jac_doubles * 8 > ib) ib = jac_doubles * 8;
        o += al(ib);
        L.cw = o; o += al(S * 16);
        L.piv = o; o += al(S * 4);
        L.mv = o; o += al(2 * S * 8);
        L.nv = o; o += al(N * 8);
        L.total = o;
        return L;
    }
    __host__ __device__ static TeamLayout rkc(int N, int rhs_doubles) {
        TeamLayout L{};
        L.buf = 0;
        L.rhs = al(N * 8);
        L.total = L.rhs + al(rhs_doubles * 8);
        return L;
    }
};

template <int SK, class Mech, int TS, typename LT, typename L1 = LT, int LEARN = 0>
__global__ void __launch_bounds__(TS >= 32 ? TS : 32, (TS >= 64 && sizeof(L1) == 4) ? 5 : 1)
team_kernel(BatchArgs a, Mech mech, TeamLayout lay)
{
    constexpr int N = Mech::N;
    using TM = Team<TS>;
    extern __shared__ __align__(16) unsigned char smem[];
    const int tib = threadIdx.x / TS;
    const int tpb = blockDim.x / TS;
    const int gteam = blockIdx.x * tpb + tib;
    unsigned char* base = smem + size_t(tib) * lay.total;
    const int lane = TM::lane();
    // queue slots claimed by this team and not yet taken (lane 0's copy counts)
    const int grain = a.grain > 1 ? a.grain : 1;
    int next = 0, left = 0;
    for (int it = 0;; ++it) {
        int sys = 0;
        if (a.plain_grid) {
            if (it > 0) break;
            sys = gteam;
        } else {
            if (lane == 0) {
                if (left == 0) {
                    next = atomicAdd(a.queue, grain);
                    left = grain;
                }
                sys = next++;
                --left;
                if (sys >= a.num) sys = a.num;
                else if (a.order) sys = a.order[sys];
            }
            sys = TM::bcast(sys, 0);
        }
        if (sys >= a.num) break;
        // a padded mechanism (n_state < N) holds zeros in the rows past the caller's state
        const int nst = a.n_state > 0 ? a.n_state : N;
        Vec<N, TS> y;
#pragma unroll
        for (int s = 0; s < Vec<N, TS>::S; ++s)
            y[s] = (Vec<N, TS>::ok(s) && Vec<N, TS>::idx(s) < nst) ? a.y[size_t(Vec<N, TS>::idx(s)) * a.num + sys] : 0.0;
        const double pr = a.var[sys];
        Stats st;
        st.clear();
        int code = EC_success;
        StepLoop L(a.t_start, a.t_end, a.step);
        if constexpr (SK == SK_RADAU) {
            RadauTeamStore<N, LT, L1> store;
            store.J = a.jac + size_t(gteam) * N * N;
            store.E1 = reinterpret_cast<L1*>(base + lay.e1);
            store.E2 = reinterpret_cast<cx<LT>*>(base + lay.e2);
            store.d1 = reinterpret_cast<L1*>(base + lay.d1);
            store.d2 = reinterpret_cast<cx<LT>*>(base + lay.d2);
            store.p1 = reinterpret_cast<int*>(base + lay.p1);
            store.p2 = reinterpret_cast<int*>(base + lay.p2);
            store.buf = reinterpret_cast<double*>(base + lay.buf);
            store.rhs = reinterpret_cast<double*>(base + lay.rhs);
            store.inf = reinterpret_cast<int*>(base + lay.inf);
            const LearnArgs la = a.learn;
            Radau<N, TS, Mech, LT, RadauTeamStore<N, LT, L1>, LEARN> rad{mech, store,
                                                                         RadauParams{a.atol, a.rtol, nst, a.stage_extrap},
                                                                         pr, st, LEARN ? &la : nullptr};
            while (L.more() && code == EC_success) {
                code = rad.integrate(L.t, L.t_next, y);
                L.advance();
            }
        } else if constexpr (SK == SK_RKC) {
            Rkc<N, TS, Mech> rk{mech, reinterpret_cast<double*>(base + lay.rhs), a.atol, a.rtol, pr, st};
            while (L.more() && code == EC_success) {
                code = rk.integrate(L.t, L.t_next, y);
                L.advance();
            }
        } else if constexpr (SK == SK_EXPRB43 || SK == SK_EXP4) {
            constexpr int P = SK == SK_EXPRB43 ? 4 : 1;
            KrylovStore ks;
            ks.J = a.jac + size_t(gteam) * N * N;
            ks.Vm = reinterpret_cast<double*>(base + lay.vm);
            ks.Hm = reinterpret_cast<double*>(base + lay.hm);
            ks.phiHm = reinterpret_cast<double*>(base + lay.phi);
            ks.inv = reinterpret_cast<cxd*>(base + lay.inv);
            ks.cw = reinterpret_cast<cxd*>(base + lay.cw);
            ks.piv = reinterpret_cast<int*>(base + lay.piv);
            ks.mv0 = reinterpret_cast<double*>(base + lay.mv);
            ks.mv1 = ks.mv0 + (N + P);
            ks.nv = reinterpret_cast<double*>(base + lay.nv);
            Krylov<N, TS, Mech, P> kr{mech, ks, a.atol, a.rtol, pr, st};
            while (L.more() && code == EC_success) {
                if constexpr (SK == SK_EXPRB43) code = kr.integrate_exprb43(L.t, L.t_next, y);
                else code = kr.integrate_exp4(L.t, L.t_next, y);
                L.advance();
            }
        }
        double bad = 0.0;
#pragma unroll
        for (int s = 0; s < Vec<N, TS>::S; ++s)
            if (Vec<N, TS>::ok(s) && Vec<N, TS>::idx(s) < nst) {
                a.y[size_t(Vec<N, TS>::idx(s)) * a.num + sys] = y[s];
                if (!isfinite(y[s])) bad = 1.0;
            }
        if (code == EC_success && TM::sum(bad) > 0.0) code = EC_nonfinite_state;
        if (a.codes && lane == 0) a.codes[sys] = code;
        store_stats<N, TS>(a, sys, st);
        if (a.cost && lane == 0) a.cost[sys] = st.c[ST_STEPS];
        TM::sync();
    }
}

// ------------------------------------------------------------- factorisation only
// E1 = (gamma/h) I - J and E2 = ((alpha + i beta)/h) I - J of one Jacobian per
// block team, factored by the routine the Radau team kernels use at this
// precision (Radau::decomp); the factors are copied out column-major (leading
// dimension N) with perm[position] = original row and info[2] per matrix.
template <class Mech, int TS, typename LT, typename L1>
__global__ void __launch_bounds__(TS >= 32 ? TS : 32)
decomp_kernel(int count, const double* jac, const double* h, L1* e1_out, cx<LT>* e2_out, int* perm_out,
              int* info_out, TeamLayout lay)
{
    constexpr int N = Mech::N;
    extern __shared__ __align__(16) unsigned char smem[];
    const int m = blockIdx.x;
    if (m >= count) return;
    RadauTeamStore<N, LT, L1> store;
    store.J = const_cast<double*>(jac) + size_t(m) * N * N;
    store.E1 = reinterpret_cast<L1*>(smem + lay.e1);
    store.E2 = reinterpret_cast<cx<LT>*>(smem + lay.e2);
    store.d1 = reinterpret_cast<L1*>(smem + lay.d1);
    store.d2 = reinterpret_cast<cx<LT>*>(smem + lay.d2);
    store.p1 = reinterpret_cast<int*>(smem + lay.p1);
    store.p2 = reinterpret_cast<int*>(smem + lay.p2);
    store.buf = reinterpret_cast<double*>(smem + lay.buf);
    store.rhs = reinterpret_cast<double*>(smem + lay.rhs);
    store.inf = reinterpret_cast<int*>(smem + lay.inf);
    Stats st;
    st.clear();
    Mech mech{};
    Radau<N, TS, Mech, LT, RadauTeamStore<N, LT, L1>> rad{mech, store, RadauParams{1e-10, 1e-6}, 0.0, st};
    rad.decomp(h[m]);
    __syncthreads();
    const int t = threadIdx.x;
    for (int e = t; e < N * N; e += blockDim.x) {
        e1_out[size_t(m) * N * N + e] = store.E1[e];
        e2_out[size_t(m) * N * N + e] = store.E2[e];
    }
    for (int i = t; i < N; i += blockDim.x) {
        perm_out[size_t(m) * 2 * N + i] = store.p1[i];
        perm_out[size_t(m) * 2 * N + N + i] = store.p2[i];
    }
    __syncthreads();
    if (t == 0) {
        // Radau::decomp reports the first failing matrix; recompute both from the factors
        int i1 = 0, i2 = 0;
        for (int k = 0; k < N && (!i1 || !i2); ++k) {
            if (!i1 && store.E1[k + k * N] == L1(0)) i1 = k + 1;
            if (!i2 && store.E2[k + k * N].re == LT(0) && store.E2[k + k * N].im == LT(0)) i2 = k + 1;
        }
        info_out[2 * m] = i1;
        info_out[2 * m + 1] = i2;
    }
}

// ------------------------------------------------------------- queue order
// Longest-first order of the work queue by a per-system cost key: keys are
// mapped to ORDER_BUCKETS buckets between their minimum and maximum (largest
// key first) and systems are scattered by bucket (counting sort; the order
// inside a bucket is arbitrary).
constexpr int ORDER_BUCKETS = 1024;

// key[i]: the previous call's step count when it is known (>= 0), else y_0 (the
// temperature of the mass-action state).
// (ext: keys given per system, e.g. a learned cost prediction, used as they are.)
__global__ void order_keys_kernel(int num, const double* y, const int* cost, const float* ext, float* key,
                                  float* kmin, float* kmax) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float k = 0.f;
    if (i < num) {
        k = ext ? ext[i] : ((cost && cost[i] >= 0) ? float(cost[i]) : float(y[i]));
        if (!(k == k)) k = 0.f;
        key[i] = k;
    }
    float lo = i < num ? k : 3.0e38f, hi = i < num ? k : -3.0e38f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if ((threadIdx.x & 31) == 0) {
        // float min / max through the ordered integer images of non-negative keys
        atomicMin(reinterpret_cast<int*>(kmin), __float_as_int(fmaxf(lo, 0.f)));
        atomicMax(reinterpret_cast<int*>(kmax), __float_as_int(fmaxf(hi, 0.f)));
    }
}

__device__ __forceinline__ int order_bucket(float k, float lo, float hi) {
    const float span = hi - lo;
    int b = span > 0.f ? int((hi - fmaxf(k, 0.f)) / span * float(ORDER_BUCKETS - 1)) : 0;
    return min(max(b, 0), ORDER_BUCKETS - 1);
}

__global__ void order_hist_kernel(int num, const float* key, const float* kmin, const float* kmax, int* hist) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < num) atomicAdd(hist + order_bucket(key[i], *kmin, *kmax), 1);
}

// exclusive prefix sum of the histogram, one block of ORDER_BUCKETS threads
__global__ void order_scan_kernel(int* hist) {
    __shared__ int s[ORDER_BUCKETS];
    const int t = threadIdx.x;
    s[t] = hist[t];
    __syncthreads();
    for (int o = 1; o < ORDER_BUCKETS; o <<= 1) {
        const int v = t >= o ? s[t - o] : 0;
        __syncthreads();
        s[t] += v;
        __syncthreads();
    }
    hist[t] = t > 0 ? s[t - 1] : 0;
}

__global__ void order_scatter_kernel(int num, const float* key, const float* kmin, const float* kmax, int* next,
                                     int* order) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < num) order[atomicAdd(next + order_bucket(key[i], *kmin, *kmax), 1)] = i;
}

}  // namespace aib
