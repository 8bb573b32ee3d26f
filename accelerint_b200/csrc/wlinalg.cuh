// Warp-level dense LU factorisation and solves for block teams: one warp per
// matrix (32 lanes, rows i = lane + 32 r), the matrix column-major in shared
// memory.  In a two-warp team warp 0 works on E1 while warp 1 works on E2.
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

// The same factorisation (xGETF2 semantics, as wlu_real / wlu_cplx) by the two
// warps of a 64-thread block team.  Both warps search the pivot of column k
// and form its multipliers in registers; the trailing update is split by
// column parity (warp w owns the columns j with j % 2 == w, 28 of the 56
// stored).  The owner of column k writes its multipliers at the start of step
// k + 1, after the block barrier that closes step k, so the other warp never
// reads a column that is being written and one barrier per step suffices.
template <int N, typename E>
__device__ __noinline__ int tlu(E* A, int* perm, E* dinv)
{
    constexpr int R = (N + 31) / 32;
    constexpr int CB = 4;
    constexpr int NC = lu_cols(N);
    constexpr int MH = NC / 2;
    static_assert(MH % CB == 0, "column padding");
    const int lane = threadIdx.x & 31;
    const int w = (threadIdx.x >> 5) & 1;
    const E zero = ezero_value<E>();
    int info = 0;
    if (w == 0)
        for (int i = lane; i < N; i += 32) perm[i] = i;
    __syncwarp();
    E lprev[R];
    E pivprev = zero;
#pragma unroll
    for (int r = 0; r < R; ++r) lprev[r] = zero;
#pragma unroll 1
    for (int k = 0; k < N; ++k) {
        // deferred multipliers (and pivot) of column k - 1 by its owner
        if (k > 0 && ((k - 1) & 1) == w) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int i = lane + 32 * r;
                if (i > k - 1 && i < N) A[i + (k - 1) * N] = lprev[r];
            }
            if (lane == 0) A[(k - 1) + (k - 1) * N] = pivprev;
            __syncwarp();
        }
        // pivot of column k, rows k..N-1 (both warps, same result)
        double best = -1.0;
        int bi = 0x7fffffff;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int i = lane + 32 * r;
            if (i >= k && i < N) {
                const double a = emag(A[i + k * N]);
                if (!(a <= best)) { best = a; bi = i; }
            }
        }
        int p = warp_pivot(best, bi);
        const E piv = A[p + k * N];
        const bool nz = !ezero(piv);
        E rc = zero;
        if (nz) {
            rc = erecip(piv);
        } else {
            if (info == 0) info = k + 1;
            p = k;   // no interchange without a pivot (xGETF2)
        }
        // multipliers of the rows below k after the interchange of rows k and p
        E l[R];
        bool act[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int i = lane + 32 * r;
            act[r] = i > k && i < N;
            const E a = act[r] ? ((i == p) ? A[k + k * N] : A[i + k * N]) : zero;
            l[r] = nz ? emul(a, rc) : a;
            lprev[r] = l[r];
        }
        pivprev = piv;
        if (w == 0 && lane == 0) {
            dinv[k] = nz ? rc : zero;
            if (p != k) { const int t = perm[k]; perm[k] = perm[p]; perm[p] = t; }
        }
        // interchange rows k and p in the owned columns other than k
        if (p != k) {
            const int j = 2 * lane + w;
            if (j < N && j != k) {
                const E t = A[k + j * N];
                A[k + j * N] = A[p + j * N];
                A[p + j * N] = t;
            }
            __syncwarp();
        }
        // trailing update of the owned columns j > k, CB owned columns at a time
        const int mfirst = (k + 1 - w + 1) >> 1;          // first owned m with 2m + w > k
        E* colp = A + lane;
#pragma unroll 1
        for (int m0 = (mfirst / CB) * CB; m0 < MH; m0 += CB) {
            E u[CB], a[R][CB];
#pragma unroll
            for (int c = 0; c < CB; ++c) {
                const int j = 2 * (m0 + c) + w;
                u[c] = (j > k) ? A[k + j * N] : zero;
            }
#pragma unroll
            for (int r = 0; r < R; ++r)
#pragma unroll
                for (int c = 0; c < CB; ++c)
                    a[r][c] = act[r] ? colp[32 * r + (2 * (m0 + c) + w) * N] : zero;
#pragma unroll
            for (int r = 0; r < R; ++r)
#pragma unroll
                for (int c = 0; c < CB; ++c)
                    if (act[r]) colp[32 * r + (2 * (m0 + c) + w) * N] = efnma(l[r], u[c], a[r][c]);
        }
        __syncthreads();
    }
    if (((N - 1) & 1) == w) {
        if (lane == 0) A[(N - 1) + (N - 1) * N] = pivprev;
    }
    __syncthreads();
    return info;
}

// Solve (P^T L U) x = b in place on a shared-memory vector xb[N] (b in, x out):
// gather by perm, unit-lower forward and upper backward substitution with the
// reciprocal diagonal, x held in registers, the next factor column loaded
// while the current one is applied.  (A zero entry of x is not skipped as
// dtrsm does; the update by an exact zero leaves finite values unchanged.)
template <int N, typename T>
__device__ __noinline__ void wsolve_real(const T* A, const T* dinv, const int* perm, double* xb)
{
    constexpr int R = (N + 31) / 32;
    const int lane = threadIdx.x & 31;
    double x[R];
    T cur[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int i = lane + 32 * r;
        x[r] = i < N ? xb[perm[i]] : 0.0;
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
        const double xj = __shfl_sync(0xffffffffu, vsel<R>(x, j >> 5), j & 31);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            x[r] = fma(-xj, dbl(cur[r]), x[r]);
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
        const double xv = vsel<R>(x, j >> 5) * dbl(dinv[j]);
        if (lane == (j & 31)) vput<R>(x, j >> 5, xv);
        const double xj = __shfl_sync(0xffffffffu, xv, j & 31);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            x[r] = fma(-xj, dbl(cur[r]), x[r]);
            cur[r] = nxt[r];
        }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int i = lane + 32 * r;
        if (i < N) xb[i] = x[r];
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
    double xr[R], xi[R];
    cx<T> cur[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int i = lane + 32 * r;
        xr[r] = i < N ? xbr[perm[i]] : 0.0;
        xi[r] = i < N ? xbi[perm[i]] : 0.0;
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
        const double br = __shfl_sync(0xffffffffu, vsel<R>(xr, j >> 5), j & 31);
        const double bi = __shfl_sync(0xffffffffu, vsel<R>(xi, j >> 5), j & 31);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const double lr = dbl(cur[r].re), li = dbl(cur[r].im);
            xr[r] = fma(bi, li, fma(-br, lr, xr[r]));
            xi[r] = fma(-bi, lr, fma(-br, li, xi[r]));
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
        const double ar = vsel<R>(xr, j >> 5), ai = vsel<R>(xi, j >> 5);
        const double nr = ar * dbl(dv.re) - ai * dbl(dv.im);
        const double ni = ar * dbl(dv.im) + ai * dbl(dv.re);
        if (lane == (j & 31)) { vput<R>(xr, j >> 5, nr); vput<R>(xi, j >> 5, ni); }
        const double br = __shfl_sync(0xffffffffu, nr, j & 31);
        const double bi = __shfl_sync(0xffffffffu, ni, j & 31);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const double ur = dbl(cur[r].re), ui = dbl(cur[r].im);
            xr[r] = fma(bi, ui, fma(-br, ur, xr[r]));
            xi[r] = fma(-bi, ur, fma(-br, ui, xi[r]));
            cur[r] = nxt[r];
        }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int i = lane + 32 * r;
        if (i < N) { xbr[i] = xr[r]; xbi[i] = xi[r]; }
    }
    __syncwarp();
}

}  // namespace aib
