// Common device building blocks: teams of lanes that own one system, complex
// arithmetic, reductions.  sm_100a only.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cfloat>

namespace aib {

// Return codes of the integrators (radau2a/radau2a_props.h:288-296,
// exprb43_props.h:356-362, rkc_props.h:427).
enum : int {
    EC_success = 0,
    EC_consecutive_steps = 1,
    EC_max_steps_exceeded = 2,
    EC_h_plus_t_equals_h = 3,
    EC_newton_max_iterations_exceeded = 4,
    // not a reference code: the integrator reported success but the final state
    // holds a NaN or an infinity (the reference returns 0 for such a system)
    EC_nonfinite_state = 5,
};

// Per-system counters (stats_dev[ivp * NSTATS + k]).
enum : int {
    ST_STEPS = 0, ST_ACCEPT, ST_REJECT, ST_JAC, ST_DECOMP, ST_NEWTON, ST_RHS, ST_AUX,
    ST_KRYLOV,    // exponential methods: sum of Krylov dimensions over Arnoldi calls;
                  // Radau in learned mode: steps started from a learned proposal
    ST_ARNOLDI,   // exponential methods: Arnoldi calls;
                  // Radau in learned mode: fall-backs to the extrapolated guess
    NSTATS
};

struct Stats {
    int c[NSTATS];
    __device__ void clear() {
#pragma unroll
        for (int i = 0; i < NSTATS; ++i) c[i] = 0;
    }
};

// ------------------------------------------------------------------ complex
template <typename T> struct cx { T re, im; };
using cxd = cx<double>;

template <typename T> __device__ __forceinline__ cx<T> cmake(T r, T i) { return {r, i}; }
template <typename T> __device__ __forceinline__ cx<T> cadd(cx<T> a, cx<T> b) { return {a.re + b.re, a.im + b.im}; }
template <typename T> __device__ __forceinline__ cx<T> csub(cx<T> a, cx<T> b) { return {a.re - b.re, a.im - b.im}; }
template <typename T> __device__ __forceinline__ cx<T> cmul(cx<T> a, cx<T> b) {
    return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
// a - b * c
template <typename T> __device__ __forceinline__ cx<T> cfnma(cx<T> b, cx<T> c, cx<T> a) {
    return {a.re - b.re * c.re + b.im * c.im, a.im - b.re * c.im - b.im * c.re};
}
template <typename T> __device__ __forceinline__ T cabs1(cx<T> a) { return fabs(a.re) + fabs(a.im); }
// 1 / b by Smith's scaling (R. L. Smith, CACM 5(8), 1962)
template <typename T> __device__ __forceinline__ cx<T> crecip(cx<T> b) {
    if (fabs(b.re) >= fabs(b.im)) {
        T r = b.im / b.re, d = b.re + b.im * r;
        return {T(1) / d, -r / d};
    } else {
        T r = b.re / b.im, d = b.re * r + b.im;
        return {r / d, T(-1) / d};
    }
}
// a / b by Smith's algorithm
template <typename T> __device__ __forceinline__ cx<T> cdiv(cx<T> a, cx<T> b) {
    if (fabs(b.re) >= fabs(b.im)) {
        T r = b.im / b.re, d = b.re + b.im * r;
        return {(a.re + a.im * r) / d, (a.im - a.re * r) / d};
    } else {
        T r = b.re / b.im, d = b.re * r + b.im;
        return {(a.re * r + a.im) / d, (a.im * r - a.re) / d};
    }
}

// ------------------------------------------------------------------ teams
// A team of TS threads integrates one system.  TS = 1 is a thread per system
// (everything in registers); TS = 2..16 are lane groups inside one warp; TS =
// 32 or 64 is a whole thread block (one system per block) whose threads own
// one state element each and share the system's matrices in shared memory.
// Control decisions must be identical on every thread of a team, so every
// reduction ends with a broadcast of one value (a butterfly alone can leave
// lanes with differently rounded sums).
template <int TS> struct Team {
    static_assert(TS == 1 || TS == 2 || TS == 4 || TS == 8 || TS == 16 || TS == 32 || TS == 64, "team size");
    static constexpr int size = TS;
    static constexpr bool block = TS >= 32;        // one team per thread block
    static constexpr int W = TS >= 32 ? TS / 32 : 1;
    static constexpr int WS = TS < 32 ? TS : 32;   // width of the warp-level part
    __device__ __forceinline__ static int lane() { return TS == 1 ? 0 : int(threadIdx.x & (TS - 1)); }
    __device__ __forceinline__ static int warp() { return block ? int(threadIdx.x >> 5) : 0; }
    __device__ __forceinline__ static unsigned mask() {
        if constexpr (TS >= 32) {
            return 0xffffffffu;
        } else if constexpr (TS == 1) {
            return 1u << (threadIdx.x & 31);
        } else {
            const unsigned base = (threadIdx.x & 31) & ~unsigned(TS - 1);
            return ((1u << TS) - 1u) << base;
        }
    }
    __device__ __forceinline__ static void sync() {
        if (TS > 32) __syncthreads();
        else if (TS > 1) __syncwarp(mask());
    }
    __device__ __forceinline__ static double wsum(double v) {
#pragma unroll
        for (int o = WS / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask(), v, o, WS);
        return __shfl_sync(mask(), v, 0, WS);
    }
    __device__ __forceinline__ static double bcast(double v, int src) {
        if (TS == 1) return v;
        if (TS <= 32) return __shfl_sync(mask(), v, src, TS);
        __shared__ double b;
        __syncthreads();
        if (lane() == src) b = v;
        __syncthreads();
        return b;
    }
    __device__ __forceinline__ static int bcast(int v, int src) {
        if (TS == 1) return v;
        if (TS <= 32) return __shfl_sync(mask(), v, src, TS);
        __shared__ int b;
        __syncthreads();
        if (lane() == src) b = v;
        __syncthreads();
        return b;
    }
    __device__ __forceinline__ static double sum(double v) {
        if (TS == 1) return v;
        v = wsum(v);
        if (TS <= 32) return v;
        __shared__ double red[W];
        __syncthreads();
        if ((threadIdx.x & 31) == 0) red[warp()] = v;
        __syncthreads();
        double s = red[0];
#pragma unroll
        for (int w = 1; w < W; ++w) s += red[w];
        return s;
    }
    // argmax of v with ties to the smallest index (warp-level teams only); an
    // index of INT_MAX marks "no candidate on this lane"; NaN loses to a number
    __device__ __forceinline__ static int argmax(double v, int idx) {
        static_assert(TS <= 32, "warp-level argmax");
        if (TS == 1) return idx;
#pragma unroll
        for (int o = TS / 2; o > 0; o >>= 1) {
            double ov = __shfl_xor_sync(mask(), v, o, TS);
            int oi = __shfl_xor_sync(mask(), idx, o, TS);
            if (oi != 0x7fffffff && (idx == 0x7fffffff || ov > v || (ov == v && oi < idx) || (v != v && ov == ov))) {
                v = ov;
                idx = oi;
            }
        }
        return __shfl_sync(mask(), idx, 0, TS);
    }
};

// A length-N vector distributed over a team: lane l owns elements l, l + TS, ...
template <int N, int TS> struct Vec {
    static constexpr int S = (N + TS - 1) / TS;
    double v[S];
    __device__ __forceinline__ static int idx(int s) { return Team<TS>::lane() + TS * s; }
    __device__ __forceinline__ static bool ok(int s) { return (N % TS == 0) || idx(s) < N; }
    __device__ __forceinline__ double& operator[](int s) { return v[s]; }
    __device__ __forceinline__ const double& operator[](int s) const { return v[s]; }
};

template <int N, int TS> __device__ __forceinline__ void vfill(Vec<N, TS>& a, double x) {
#pragma unroll
    for (int s = 0; s < Vec<N, TS>::S; ++s) a[s] = x;
}

}  // namespace aib
