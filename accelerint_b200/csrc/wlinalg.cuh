// Warp-level dense LU factorisation and solves for block teams: rows
// i = lane + 32 r of a column-major matrix in shared memory.  A 32-thread team
// factors E1 and E2 on its one warp (wlu_real / wlu_cplx); a 64-thread team
// factors both overlapped on its two warps (tlu_pair).  Solves run E1 on warp 0
// and E2 on warp 1 (wsolve_real / wsolve_cplx), in the factors' precision.
//
// Semantics of LAPACK's unblocked xGETF2 / xGETRS as in linalg.cuh (first
// maximal pivot by |a| or |Re a| + |Im a|, reciprocal scaling of the
// multiplier column, info = k + 1 on a zero pivot), the radau2a/radau2a.c:
// 273-277 and :404-417 calls.  The routines are out of line so the team kernel
// holds one copy of each: a fully inlined integrator does not fit the
// instruction cache.
#pragma once
#include "common.cuh"

namespace aib {

template <int R, typename V> __device__ __forceinline__ double vsel(const V& x, int s) {
    double r = x[0];
#pragma unroll
    for (int k = 1; k < R; ++k)
        if (s == k) r = x[k];
    return r;
}
template <int R, typename V> __device__ __forceinline__ void vput(V& x, int s, double v) {
#pragma unroll
    for (int k = 0; k < R; ++k)
        if (s == k) x[k] = v;
}

// Columns of the stored E1/E2: N rounded up to a multiple of 8; the extra
// columns (leading dimension N) hold zeros so that factorisation chunks need no
// bounds tests.
__host__ __device__ constexpr int lu_cols(int n) { return (n + 7) & ~7; }

// Accumulation type of the triangular solves: the factors' precision (single-
// precision factors are solved in single precision; the Newton loop refines).
template <typename T> struct SolveType { using type = double; };
template <> struct SolveType<float> { using type = float; };
// Power of two near max |b| over the warp (1 when b is zero or not finite): a
// single-precision solve runs on b / scale, so the right-hand side (which
// carries a 1/h factor) stays inside the FP32 range.
__device__ __forceinline__ double warp_pow2_scale(double m) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (!(m > 0.0) || !(m < 1e300)) return 1.0;
    int e = 0;
    frexp(m, &e);
    return ldexp(1.0, e);
}

template <int R, typename AT> __device__ __forceinline__ AT vselt(const AT* x, int s) {
    AT r = x[0];
#pragma unroll
    for (int k = 1; k < R; ++k)
        if (s == k) r = x[k];
    return r;
}
template <int R, typename AT> __device__ __forceinline__ void vputt(AT* x, int s, AT v) {
#pragma unroll
    for (int k = 0; k < R; ++k)
        if (s == k) x[k] = v;
}

__device__ __forceinline__ double dbl(double a) { return a; }
__device__ __forceinline__ double dbl(float a) { return double(a); }

// First-maximum argmax over the warp for magnitudes m >= 0 (m < 0: no
// candidate; NaN counts as a candidate).  Two 32-bit warp reductions on the
// ordered bit pattern, then the smallest row index among the winners.
__device__ __forceinline__ int warp_pivot(double m, int idx) {
    unsigned long long b = 0;
    if (!(m < 0.0)) b = static_cast<unsigned long long>(__double_as_longlong(fabs(m))) + 1ull;
    const unsigned hi = unsigned(b >> 32), lo = unsigned(b);
    const unsigned mh = __reduce_max_sync(0xffffffffu, hi);
    const unsigned ml = __reduce_max_sync(0xffffffffu, hi == mh ? lo : 0u);
    const bool win = b != 0 && hi == mh && lo == ml;
    const int cand = win ? idx : 0x7fffffff;
    return int(__reduce_min_sync(0xffffffffu, unsigned(cand)));
}

// Real LU in place of an N x lu_cols(N) column-major array (zero columns past
// N); perm[i] = original row at position i, dinv[k] = 1 / U(k,k).
template <int N, typename T>
__device__ __noinline__ int wlu_real(T* A, int* perm, T* dinv)
{
    constexpr int R = (N + 31) / 32;
    constexpr int CB = 8;
    constexpr int NC = lu_cols(N);
    static_assert(NC % CB == 0, "column padding");
    const int lane = threadIdx.x & 31;
    int info = 0;
    for (int i = lane; i < N; i += 32) perm[i] = i;
    __syncwarp();
#pragma unroll 1
    for (int k = 0; k < N; ++k) {
        // pivot: first maximal |a| in column k, rows k..N-1
        double best = -1.0;
        int bi = 0x7fffffff;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int i = lane + 32 * r;
            if (i >= k && i < N) {
                const double a = fabs(dbl(A[i + k * N]));
                if (!(a <= best)) { best = a; bi = i; }   // NaN-safe: a row is always taken
            }
        }
        const int p = warp_pivot(best, bi);
        const T piv = A[p + k * N];
        if (piv != T(0)) {
            if (p != k) {
                for (int j = lane; j < N; j += 32) {
                    const T t = A[k + j * N];
                    A[k + j * N] = A[p + j * N];
                    A[p + j * N] = t;
                }
                if (lane == 0) { const int t = perm[k]; perm[k] = perm[p]; perm[p] = t; }
                __syncwarp();
            }
            const T rc = T(1) / piv;
            if (lane == 0) dinv[k] = rc;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int i = lane + 32 * r;
                if (i > k && i < N) A[i + k * N] *= rc;
            }
        } else {
            if (info == 0) info = k + 1;
            if (lane == 0) dinv[k] = T(0);
        }
        __syncwarp();
        T l[R];
        bool act[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int i = lane + 32 * r;
            act[r] = i > k && i < N;
            l[r] = act[r] ? A[i + k * N] : T(0);
        }
        // Trailing update in chunks of CB columns from a chunk boundary; the storage
        // is padded with zero columns to a multiple of CB (NC), columns j <= k carry
        // u = 0, so a chunk needs no bounds tests; only rows below k are written.
        T* colp = A + lane;
#pragma unroll 1
        for (int j0 = (k + 1) & ~(CB - 1); j0 < NC; j0 += CB) {
            T u[CB], a[R][CB];
            const T* pr = A + k + j0 * N;
            T* pc = colp + j0 * N;
#pragma unroll
            for (int c = 0; c < CB; ++c) u[c] = (j0 + c > k) ? pr[c * N] : T(0);
#pragma unroll
            for (int r = 0; r < R; ++r)
#pragma unroll
                for (int c = 0; c < CB; ++c) a[r][c] = act[r] ? pc[32 * r + c * N] : T(0);
#pragma unroll
            for (int r = 0; r < R; ++r)
#pragma unroll
                for (int c = 0; c < CB; ++c)
                    if (act[r]) pc[32 * r + c * N] = fma(l[r], -u[c], a[r][c]);
        }
        __syncwarp();
    }
    return info;
}

template <int N, typename T>
__device__ __noinline__ int wlu_cplx(cx<T>* A, int* perm, cx<T>* dinv)
{
    constexpr int R = (N + 31) / 32;
    constexpr int CB = 8;
    constexpr int NC = lu_cols(N);
    static_assert(NC % CB == 0, "column padding");
    const int lane = threadIdx.x & 31;
    const cx<T> z{T(0), T(0)};
    int info = 0;
    for (int i = lane; i < N; i += 32) perm[i] = i;
    __syncwarp();
#pragma unroll 1
    for (int k = 0; k < N; ++k) {
        double best = -1.0;
        int bi = 0x7fffffff;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int i = lane + 32 * r;
            if (i >= k && i < N) {
                const double a = dbl(cabs1(A[i + k * N]));
                if (!(a <= best)) { best = a; bi = i; }
            }
        }
        const int p = warp_pivot(best, bi);
        const cx<T> piv = A[p + k * N];
        if (piv.re != T(0) || piv.im != T(0)) {
            if (p != k) {
                for (int j = lane; j < N; j += 32) {
                    const cx<T> t = A[k + j * N];
                    A[k + j * N] = A[p + j * N];
                    A[p + j * N] = t;
                }
                if (lane == 0) { const int t = perm[k]; perm[k] = perm[p]; perm[p] = t; }
                __syncwarp();
            }
            const cx<T> rc = crecip(piv);
            if (lane == 0) dinv[k] = rc;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int i = lane + 32 * r;
                if (i > k && i < N) A[i + k * N] = cmul(A[i + k * N], rc);
            }
        } else {
            if (info == 0) info = k + 1;
            if (lane == 0) dinv[k] = z;
        }
        __syncwarp();
        cx<T> l[R];
        bool act[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int i = lane + 32 * r;
            act[r] = i > k && i < N;
            l[r] = act[r] ? A[i + k * N] : z;
        }
        cx<T>* colp = A + lane;
#pragma unroll 1
        for (int j0 = (k + 1) & ~(CB - 1); j0 < NC; j0 += CB) {
            cx<T> u[CB], a[R][CB];
            const cx<T>* pr = A + k + j0 * N;
            cx<T>* pc = colp + j0 * N;
#pragma unroll
            for (int c = 0; c < CB; ++c) u[c] = (j0 + c > k) ? pr[c * N] : z;
#pragma unroll
            for (int r = 0; r < R; ++r)
#pragma unroll
                for (int c = 0; c < CB; ++c) a[r][c] = act[r] ? pc[32 * r + c * N] : z;
#pragma unroll
            for (int r = 0; r < R; ++r)
#pragma unroll
                for (int c = 0; c < CB; ++c)
                    if (act[r]) pc[32 * r + c * N] = cfnma(l[r], u[c], a[r][c]);
        }
        __syncwarp();
    }
    return info;
}

// ---------------------------------------------------------------- two-warp LU
// Element helpers shared by the real and the complex factorisation.
template <typename T> __device__ __forceinline__ double emag(T a) { return fabs(dbl(a)); }
template <typename T> __device__ __forceinline__ double emag(cx<T> a) { return dbl(cabs1(a)); }
template <typename T> __device__ __forceinline__ bool ezero(T a) { return a == T(0); }
template <typename T> __device__ __forceinline__ bool ezero(cx<T> a) { return a.re == T(0) && a.im == T(0); }
template <typename T> __device__ __forceinline__ T erecip(T a) { return T(1) / a; }
template <typename T> __device__ __forceinline__ cx<T> erecip(cx<T> a) { return crecip(a); }
template <typename T> __device__ __forceinline__ T emul(T a, T b) { return a * b; }
template <typename T> __device__ __forceinline__ cx<T> emul(cx<T> a, cx<T> b) { return cmul(a, b); }
template <typename T> __device__ __forceinline__ T efnma(T l, T u, T a) { return fma(l, -u, a); }
template <typename T> __device__ __forceinline__ cx<T> efnma(cx<T> l, cx<T> u, cx<T> a) { return cfnma(l, u, a); }
template <typename E> __device__ __forceinline__ E ezero_value() { return E{}; }

// a - l u for single-precision complex elements as two packed FP32x2 FMAs
// (sm_100 FFMA2): (a.re - l.re u.re, a.im - l.re u.im), then + (l.im u.im, -l.im u.re).
__device__ __forceinline__ float2 cfnma2(float2 nlr, float2 lim, float2 u, float2 us, float2 a) {
    return __ffma2_rn(lim, us, __ffma2_rn(nlr, u, a));
}

// E1 and E2 together on the two warps of a 64-thread block team, overlapped:
// in elimination step k warp 1 finds the E2 pivot and writes the E2
// multipliers of column k while warp 0 performs the whole step k of E1 (the
// real factorisation is about a quarter of the complex one); after a block
// barrier both warps apply the E2 row interchange and trailing update to the
// columns they own (j % 2 == warp), and a second barrier closes the step.
// Semantics per matrix are those of wlu_real / wlu_cplx (xGETF2).  xchg: one
// shared int for the E2 pivot row.  Returns (info of E1, info of E2).
template <int N, typename T1, typename T2>
__device__ __noinline__ int2 tlu_pair(T1* A1, int* perm1, T1* dinv1, T2* A2, int* perm2, T2* dinv2, int* xchg)
{
    constexpr int R = (N + 31) / 32;
    constexpr int CB1 = 8;
    constexpr int CB = 4;
    constexpr int NC = lu_cols(N);
    constexpr int MH = NC / 2;
    static_assert(NC % CB1 == 0 && MH % CB == 0, "column padding");
    const int lane = threadIdx.x & 31;
    const int w = (threadIdx.x >> 5) & 1;
    const T2 z2 = ezero_value<T2>();
    int info1 = 0, info2 = 0;
    for (int i = lane; i < N; i += 32) {
        if (w == 0) perm1[i] = i;
        else perm2[i] = i;
    }
    __syncthreads();
#pragma unroll 1
    for (int k = 0; k < N; ++k) {
        if (w == 1) {
            // ---- E2: pivot and multipliers of column k (warp 1)
            double best = -1.0;
            int bi = 0x7fffffff;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int i = lane + 32 * r;
                if (i >= k && i < N) {
                    const double a = emag(A2[i + k * N]);
                    if (!(a <= best)) { best = a; bi = i; }
                }
            }
            int p = warp_pivot(best, bi);
            const T2 piv = A2[p + k * N];
            const bool nz = !ezero(piv);
            T2 rc = z2;
            if (nz) rc = erecip(piv);
            else { if (info2 == 0) info2 = k + 1; p = k; }
            const T2 akk = A2[k + k * N];
            T2 nv[R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int i = lane + 32 * r;
                T2 a = z2;
                if (i == k) a = nz ? piv : akk;
                else if (i > k && i < N) {
                    a = (i == p) ? akk : A2[i + k * N];
                    if (nz) a = emul(a, rc);
                }
                nv[r] = a;
            }
            __syncwarp();
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int i = lane + 32 * r;
                if (i >= k && i < N) A2[i + k * N] = nv[r];
            }
            if (lane == 0) {
                xchg[0] = p;
                dinv2[k] = nz ? rc : z2;
                if (p != k) { const int t = perm2[k]; perm2[k] = perm2[p]; perm2[p] = t; }
            }
        } else {
            // ---- E1: the whole elimination step k (warp 0)
            double best = -1.0;
            int bi = 0x7fffffff;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int i = lane + 32 * r;
                if (i >= k && i < N) {
                    const double a = emag(A1[i + k * N]);
                    if (!(a <= best)) { best = a; bi = i; }
                }
            }
            const int p = warp_pivot(best, bi);
            const T1 piv = A1[p + k * N];
            if (piv != T1(0)) {
                if (p != k) {
                    for (int j = lane; j < N; j += 32) {
                        const T1 t = A1[k + j * N];
                        A1[k + j * N] = A1[p + j * N];
                        A1[p + j * N] = t;
                    }
                    if (lane == 0) { const int t = perm1[k]; perm1[k] = perm1[p]; perm1[p] = t; }
                    __syncwarp();
                }
                const T1 rc = T1(1) / piv;
                if (lane == 0) dinv1[k] = rc;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int i = lane + 32 * r;
                    if (i > k && i < N) A1[i + k * N] *= rc;
                }
            } else {
                if (info1 == 0) info1 = k + 1;
                if (lane == 0) dinv1[k] = T1(0);
            }
            __syncwarp();
            T1 l[R];
            bool act[R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int i = lane + 32 * r;
                act[r] = i > k && i < N;
                l[r] = act[r] ? A1[i + k * N] : T1(0);
            }
            T1* colp = A1 + lane;
#pragma unroll 1
            for (int j0 = (k + 1) & ~(CB1 - 1); j0 < NC; j0 += CB1) {
                T1 u[CB1], a[R][CB1];
                const T1* pr = A1 + k + j0 * N;
                T1* pc = colp + j0 * N;
#pragma unroll
                for (int c = 0; c < CB1; ++c) u[c] = (j0 + c > k) ? pr[c * N] : T1(0);
#pragma unroll
                for (int r = 0; r < R; ++r)
#pragma unroll
                    for (int c = 0; c < CB1; ++c) a[r][c] = act[r] ? pc[32 * r + c * N] : T1(0);
                if constexpr (sizeof(T1) == sizeof(float) && R == 2) {
                    // the two rows of a lane as one packed FP32x2 FMA per column
                    const float2 nl = make_float2(-l[0], -l[1]);
#pragma unroll
                    for (int c = 0; c < CB1; ++c) {
                        const float2 v = __ffma2_rn(nl, make_float2(u[c], u[c]), make_float2(a[0][c], a[1][c]));
                        a[0][c] = v.x;
                        a[1][c] = v.y;
                    }
#pragma unroll
                    for (int r = 0; r < R; ++r)
#pragma unroll
                        for (int c = 0; c < CB1; ++c)
                            if (act[r]) pc[32 * r + c * N] = a[r][c];
                } else {
#pragma unroll
                    for (int r = 0; r < R; ++r)
#pragma unroll
                        for (int c = 0; c < CB1; ++c)
                            if (act[r]) pc[32 * r + c * N] = fma(l[r], -u[c], a[r][c]);
                }
            }
        }
        __syncthreads();
        // ---- E2: interchange and trailing update of the owned columns (both warps)
        const int p = xchg[0];
        if (p != k) {
            const int j = 2 * lane + w;
            if (j < N && j != k) {
                const T2 t = A2[k + j * N];
                A2[k + j * N] = A2[p + j * N];
                A2[p + j * N] = t;
            }
            __syncwarp();
        }
        T2 l[R];
        bool act[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int i = lane + 32 * r;
            act[r] = i > k && i < N;
            l[r] = act[r] ? A2[i + k * N] : z2;
        }
        const int mfirst = (k + 1 - w + 1) >> 1;
        if constexpr (sizeof(T2) == sizeof(float2)) {
            // single precision: packed FP32x2 arithmetic on (re, im)
            float2 nlr[R], lim[R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                nlr[r] = make_float2(-l[r].re, -l[r].re);
                lim[r] = make_float2(l[r].im, -l[r].im);
            }
            float2* A2f = reinterpret_cast<float2*>(A2);
            float2* colp = A2f + lane;
#pragma unroll 1
            for (int m0 = (mfirst / CB) * CB; m0 < MH; m0 += CB) {
                float2 u[CB], us[CB], a[R][CB];
#pragma unroll
                for (int c = 0; c < CB; ++c) {
                    const int j = 2 * (m0 + c) + w;
                    u[c] = (j > k) ? A2f[k + j * N] : make_float2(0.f, 0.f);
                    us[c] = make_float2(u[c].y, u[c].x);
                }
#pragma unroll
                for (int r = 0; r < R; ++r)
#pragma unroll
                    for (int c = 0; c < CB; ++c)
                        a[r][c] = act[r] ? colp[32 * r + (2 * (m0 + c) + w) * N] : make_float2(0.f, 0.f);
#pragma unroll
                for (int r = 0; r < R; ++r)
#pragma unroll
                    for (int c = 0; c < CB; ++c)
                        if (act[r]) colp[32 * r + (2 * (m0 + c) + w) * N] = cfnma2(nlr[r], lim[r], u[c], us[c], a[r][c]);
            }
        } else {
            T2* colp = A2 + lane;
#pragma unroll 1
            for (int m0 = (mfirst / CB) * CB; m0 < MH; m0 += CB) {
                T2 u[CB], a[R][CB];
#pragma unroll
                for (int c = 0; c < CB; ++c) {
                    const int j = 2 * (m0 + c) + w;
                    u[c] = (j > k) ? A2[k + j * N] : z2;
                }
#pragma unroll
                for (int r = 0; r < R; ++r)
#pragma unroll
                    for (int c = 0; c < CB; ++c)
                        a[r][c] = act[r] ? colp[32 * r + (2 * (m0 + c) + w) * N] : z2;
#pragma unroll
                for (int r = 0; r < R; ++r)
#pragma unroll
                    for (int c = 0; c < CB; ++c)
                        if (act[r]) colp[32 * r + (2 * (m0 + c) + w) * N] = efnma(l[r], u[c], a[r][c]);
            }
        }
        __syncthreads();
    }
    return make_int2(info1, info2);
}

// Solve (P^T L U) x = b in place on a shared-memory vector xb[N] (b in, x out):
// gather by perm, unit-lower forward and upper backward substitution with the
// reciprocal diagonal, x held in registers (in the factors' precision,
// SolveType), the next factor column loaded while the current one is applied.  (A zero entry of x is not skipped as
// dtrsm does; the update by an exact zero leaves finite values unchanged.)
template <int N, typename T>
__device__ __noinline__ void wsolve_real(const T* A, const T* dinv, const int* perm, double* xb)
{
    constexpr int R = (N + 31) / 32;
    const int lane = threadIdx.x & 31;
    using AT = typename SolveType<T>::type;
    AT x[R];
    T cur[R];
    double bv[R], m = 0.0;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int i = lane + 32 * r;
        bv[r] = i < N ? xb[perm[i]] : 0.0;
        m = fmax(m, fabs(bv[r]));
    }
    const double scale = sizeof(AT) == sizeof(float) ? warp_pow2_scale(m) : 1.0;
    const double iscale = 1.0 / scale;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int i = lane + 32 * r;
        x[r] = AT(bv[r] * iscale);
        cur[r] = (i > 0 && i < N) ? A[i] : T(0);
    }
    __syncwarp();
#pragma unroll 1
    for (int j = 0; j < N; ++j) {
        T nxt[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int i = lane + 32 * r;
            nxt[r] = (j + 1 < N && i > j + 1 && i < N) ? A[i + (j + 1) * N] : T(0);
        }
        const AT xj = __shfl_sync(0xffffffffu, vselt<R, AT>(x, j >> 5), j & 31);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            x[r] = fma(-xj, AT(cur[r]), x[r]);
            cur[r] = nxt[r];
        }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int i = lane + 32 * r;
        cur[r] = (i < N - 1) ? A[i + (N - 1) * N] : T(0);
    }
#pragma unroll 1
    for (int j = N - 1; j >= 0; --j) {
        T nxt[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int i = lane + 32 * r;
            nxt[r] = (j > 0 && i < j - 1) ? A[i + (j - 1) * N] : T(0);
        }
        const AT xv = vselt<R, AT>(x, j >> 5) * AT(dinv[j]);
        if (lane == (j & 31)) vputt<R, AT>(x, j >> 5, xv);
        const AT xj = __shfl_sync(0xffffffffu, xv, j & 31);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            x[r] = fma(-xj, AT(cur[r]), x[r]);
            cur[r] = nxt[r];
        }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int i = lane + 32 * r;
        if (i < N) xb[i] = double(x[r]) * scale;
    }
    __syncwarp();
}

template <int N, typename T>
__device__ __noinline__ void wsolve_cplx(const cx<T>* A, const cx<T>* dinv, const int* perm, double* xbr,
                                         double* xbi)
{
    constexpr int R = (N + 31) / 32;
    const int lane = threadIdx.x & 31;
    const cx<T> z{T(0), T(0)};
    using AT = typename SolveType<T>::type;
    AT xr[R], xi[R];
    cx<T> cur[R];
    double br0[R], bi0[R], m = 0.0;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int i = lane + 32 * r;
        br0[r] = i < N ? xbr[perm[i]] : 0.0;
        bi0[r] = i < N ? xbi[perm[i]] : 0.0;
        m = fmax(m, fmax(fabs(br0[r]), fabs(bi0[r])));
    }
    const double scale = sizeof(AT) == sizeof(float) ? warp_pow2_scale(m) : 1.0;
    const double iscale = 1.0 / scale;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int i = lane + 32 * r;
        xr[r] = AT(br0[r] * iscale);
        xi[r] = AT(bi0[r] * iscale);
        cur[r] = (i > 0 && i < N) ? A[i] : z;
    }
    __syncwarp();
#pragma unroll 1
    for (int j = 0; j < N; ++j) {
        cx<T> nxt[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int i = lane + 32 * r;
            nxt[r] = (j + 1 < N && i > j + 1 && i < N) ? A[i + (j + 1) * N] : z;
        }
        const AT br = __shfl_sync(0xffffffffu, vselt<R, AT>(xr, j >> 5), j & 31);
        const AT bi = __shfl_sync(0xffffffffu, vselt<R, AT>(xi, j >> 5), j & 31);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const AT lr = AT(cur[r].re), li = AT(cur[r].im);
            if constexpr (sizeof(AT) == sizeof(float)) {
                // (xr, xi) -= (br, bi) (lr, li) as two packed FP32x2 FMAs
                float2 v = __ffma2_rn(make_float2(-br, -br), make_float2(lr, li), make_float2(xr[r], xi[r]));
                v = __ffma2_rn(make_float2(bi, -bi), make_float2(li, lr), v);
                xr[r] = v.x;
                xi[r] = v.y;
            } else {
                xr[r] = fma(bi, li, fma(-br, lr, xr[r]));
                xi[r] = fma(-bi, lr, fma(-br, li, xi[r]));
            }
            cur[r] = nxt[r];
        }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int i = lane + 32 * r;
        cur[r] = (i < N - 1) ? A[i + (N - 1) * N] : z;
    }
#pragma unroll 1
    for (int j = N - 1; j >= 0; --j) {
        cx<T> nxt[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int i = lane + 32 * r;
            nxt[r] = (j > 0 && i < j - 1) ? A[i + (j - 1) * N] : z;
        }
        const cx<T> dv = dinv[j];
        const AT ar = vselt<R, AT>(xr, j >> 5), ai = vselt<R, AT>(xi, j >> 5);
        const AT nr = ar * AT(dv.re) - ai * AT(dv.im);
        const AT ni = ar * AT(dv.im) + ai * AT(dv.re);
        if (lane == (j & 31)) { vputt<R, AT>(xr, j >> 5, nr); vputt<R, AT>(xi, j >> 5, ni); }
        const AT br = __shfl_sync(0xffffffffu, nr, j & 31);
        const AT bi = __shfl_sync(0xffffffffu, ni, j & 31);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const AT ur = AT(cur[r].re), ui = AT(cur[r].im);
            if constexpr (sizeof(AT) == sizeof(float)) {
                float2 v = __ffma2_rn(make_float2(-br, -br), make_float2(ur, ui), make_float2(xr[r], xi[r]));
                v = __ffma2_rn(make_float2(bi, -bi), make_float2(ui, ur), v);
                xr[r] = v.x;
                xi[r] = v.y;
            } else {
                xr[r] = fma(bi, ui, fma(-br, ur, xr[r]));
                xi[r] = fma(-bi, ur, fma(-br, ui, xi[r]));
            }
            cur[r] = nxt[r];
        }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int i = lane + 32 * r;
        if (i < N) { xbr[i] = double(xr[r]) * scale; xbi[i] = double(xi[r]) * scale; }
    }
    __syncwarp();
}

}  // namespace aib
