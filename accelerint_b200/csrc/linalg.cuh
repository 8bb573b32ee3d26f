// Team-cooperative dense LU factorisation and solves for the Radau iteration
// matrices E1 = (gamma/h) I - J (real) and E2 = ((alpha + i beta)/h) I - J
// (complex), after radau2a/radau2a.c:256-278 (RK_Decomp) and :388-441
// (RK_Solve), which call LAPACK dgetrf/zgetrf/dgetrs/zgetrs.
//
// Semantics kept from LAPACK's unblocked xGETF2: partial pivoting on the first
// maximal |a| (real) or |Re a| + |Im a| (complex, izamax); the multiplier
// column is scaled by the reciprocal of the pivot; zero pivot -> info = k + 1
// and the factorisation continues.  Storage is column-major in shared memory
// (or registers when the team is one thread); lanes own rows.
//
// The storage type T (double or float) is the precision of the factorisation;
// the right-hand sides arrive and leave in double.
#pragma once
#include "common.cuh"

namespace aib {

// Real LU in place: A[N*N] column-major.  perm[i] receives the row of the
// original matrix that ends up in position i (the product of the LAPACK
// interchanges), dinv[i] = 1 / U(i,i).  Returns info.
template <int N, int TS, typename T>
__device__ int lu_real(T* A, int* perm, T* dinv)
{
    using TM = Team<TS>;
    const int lane = TM::lane();
    int info = 0;
    if (lane == 0)
        for (int i = 0; i < N; ++i) perm[i] = i;
    TM::sync();
#pragma unroll 1
    for (int k = 0; k < N; ++k) {
        double best = -1.0;
        int bi = 0x7fffffff;   // no candidate on this lane
        for (int i = k + lane; i < N; i += TS) {
            double a = fabs(double(A[i + k * N]));
            if (!(a <= best)) { best = a; bi = i; }   // NaN-safe: a row is always taken
        }
        const int p = TM::argmax(best, bi);
        const T piv = A[p + k * N];
        if (piv != T(0)) {
            if (p != k) {
                for (int j = lane; j < N; j += TS) {
                    T t = A[k + j * N];
                    A[k + j * N] = A[p + j * N];
                    A[p + j * N] = t;
                }
                if (lane == 0) { int t = perm[k]; perm[k] = perm[p]; perm[p] = t; }
            }
            TM::sync();
            const T r = T(1) / A[k + k * N];
            if (lane == 0) dinv[k] = r;
            for (int i = k + 1 + lane; i < N; i += TS) A[i + k * N] *= r;
        } else {
            if (info == 0) info = k + 1;
            if (lane == 0) dinv[k] = T(0);
        }
        TM::sync();
        // rank-1 update of the trailing block; lanes own rows, multipliers stay in
        // registers; columns go in chunks of CB so the shared-memory loads of a
        // chunk are in flight together.  (A zero pivot-row entry is not skipped as
        // LAPACK's dger does: the update by an exact zero leaves finite values unchanged.)
        constexpr int S = (N + TS - 1) / TS;
        constexpr int CB = 8;
        T l[S];
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int i = k + 1 + lane + TS * s;
            l[s] = i < N ? A[i + k * N] : T(0);
        }
        for (int j0 = k + 1; j0 < N; j0 += CB) {
            T u[CB];
            T a[S][CB];
#pragma unroll
            for (int c = 0; c < CB; ++c) u[c] = (j0 + c < N) ? A[k + (j0 + c) * N] : T(0);
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const int i = k + 1 + lane + TS * s;
#pragma unroll
                for (int c = 0; c < CB; ++c) a[s][c] = (i < N && j0 + c < N) ? A[i + (j0 + c) * N] : T(0);
            }
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const int i = k + 1 + lane + TS * s;
#pragma unroll
                for (int c = 0; c < CB; ++c)
                    if (i < N && j0 + c < N) A[i + (j0 + c) * N] = fma(l[s], -u[c], a[s][c]);
            }
        }
        TM::sync();
    }
    return info;
}

// Complex LU in place, same conventions; pivot by |Re| + |Im| (LAPACK izamax).
template <int N, int TS, typename T>
__device__ int lu_cplx(cx<T>* A, int* perm, cx<T>* dinv)
{
    using TM = Team<TS>;
    const int lane = TM::lane();
    int info = 0;
    if (lane == 0)
        for (int i = 0; i < N; ++i) perm[i] = i;
    TM::sync();
#pragma unroll 1
    for (int k = 0; k < N; ++k) {
        double best = -1.0;
        int bi = 0x7fffffff;   // no candidate on this lane
        for (int i = k + lane; i < N; i += TS) {
            double a = double(cabs1(A[i + k * N]));
            if (!(a <= best)) { best = a; bi = i; }   // NaN-safe: a row is always taken
        }
        const int p = TM::argmax(best, bi);
        const cx<T> piv = A[p + k * N];
        if (piv.re != T(0) || piv.im != T(0)) {
            if (p != k) {
                for (int j = lane; j < N; j += TS) {
                    cx<T> t = A[k + j * N];
                    A[k + j * N] = A[p + j * N];
                    A[p + j * N] = t;
                }
                if (lane == 0) { int t = perm[k]; perm[k] = perm[p]; perm[p] = t; }
            }
            TM::sync();
            const cx<T> r = crecip(A[k + k * N]);
            if (lane == 0) dinv[k] = r;
            for (int i = k + 1 + lane; i < N; i += TS) A[i + k * N] = cmul(A[i + k * N], r);
        } else {
            if (info == 0) info = k + 1;
            if (lane == 0) dinv[k] = cx<T>{T(0), T(0)};
        }
        TM::sync();
        constexpr int S = (N + TS - 1) / TS;
        constexpr int CB = 4;
        cx<T> l[S];
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int i = k + 1 + lane + TS * s;
            l[s] = i < N ? A[i + k * N] : cx<T>{T(0), T(0)};
        }
        for (int j0 = k + 1; j0 < N; j0 += CB) {
            cx<T> u[CB];
            cx<T> a[S][CB];
#pragma unroll
            for (int c = 0; c < CB; ++c) u[c] = (j0 + c < N) ? A[k + (j0 + c) * N] : cx<T>{T(0), T(0)};
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const int i = k + 1 + lane + TS * s;
#pragma unroll
                for (int c = 0; c < CB; ++c)
                    a[s][c] = (i < N && j0 + c < N) ? A[i + (j0 + c) * N] : cx<T>{T(0), T(0)};
            }
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const int i = k + 1 + lane + TS * s;
#pragma unroll
                for (int c = 0; c < CB; ++c)
                    if (i < N && j0 + c < N) A[i + (j0 + c) * N] = cfnma(l[s], u[c], a[s][c]);
            }
        }
        TM::sync();
    }
    return info;
}

// Gather a distributed vector through shared memory: out(i) = in(perm[i]).
template <int N, int TS>
__device__ __forceinline__ void permute(Vec<N, TS>& x, const int* perm, double* buf)
{
    using TM = Team<TS>;
#pragma unroll
    for (int s = 0; s < Vec<N, TS>::S; ++s)
        if (Vec<N, TS>::ok(s)) buf[Vec<N, TS>::idx(s)] = x[s];
    TM::sync();
#pragma unroll
    for (int s = 0; s < Vec<N, TS>::S; ++s)
        if (Vec<N, TS>::ok(s)) x[s] = buf[perm[Vec<N, TS>::idx(s)]];
    TM::sync();
}

// Solve (LU) x = P b for one real and one complex system at once, the
// pattern of RK_Solve (radau2a.c:404,417).  b arrives permuted; x stays
// distributed in registers; column j of L/U is read by all lanes (coalesced).
// Zero entries of the running solution skip their column as in dtrsm.
template <int N, int TS, typename T1, typename T>
__device__ void lu_solve_pair(const T1* A1, const T1* d1, Vec<N, TS>& x1,
                              const cx<T>* A2, const cx<T>* d2, Vec<N, TS>& x2r, Vec<N, TS>& x2i)
{
    using TM = Team<TS>;
    constexpr int S = Vec<N, TS>::S;
    const int lane = TM::lane();
    // forward: unit lower triangular
#pragma unroll
    for (int j = 0; j < N; ++j) {
        const int src = j % TS, sj = j / TS;
        const double a = TM::bcast(x1[sj], src);
        const double br = TM::bcast(x2r[sj], src);
        const double bi = TM::bcast(x2i[sj], src);
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int i = lane + TS * s;
            if (i > j && i < N) {
                if (a != 0.0) x1[s] = fma(-a, double(A1[i + j * N]), x1[s]);
                if (br != 0.0 || bi != 0.0) {
                    const cx<T> l = A2[i + j * N];
                    x2r[s] = x2r[s] - br * double(l.re) + bi * double(l.im);
                    x2i[s] = x2i[s] - br * double(l.im) - bi * double(l.re);
                }
            }
        }
    }
    // backward: upper triangular with precomputed reciprocal diagonal
#pragma unroll
    for (int j = N - 1; j >= 0; --j) {
        const int src = j % TS, sj = j / TS;
        if (lane == src) {
            x1[sj] = x1[sj] * double(d1[j]);
            const cx<T> dv = d2[j];
            const double xr = x2r[sj], xi = x2i[sj];
            x2r[sj] = xr * double(dv.re) - xi * double(dv.im);
            x2i[sj] = xr * double(dv.im) + xi * double(dv.re);
        }
        const double a = TM::bcast(x1[sj], src);
        const double br = TM::bcast(x2r[sj], src);
        const double bi = TM::bcast(x2i[sj], src);
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int i = lane + TS * s;
            if (i < j) {
                if (a != 0.0) x1[s] = fma(-a, double(A1[i + j * N]), x1[s]);
                if (br != 0.0 || bi != 0.0) {
                    const cx<T> u = A2[i + j * N];
                    x2r[s] = x2r[s] - br * double(u.re) + bi * double(u.im);
                    x2i[s] = x2i[s] - br * double(u.im) - bi * double(u.re);
                }
            }
        }
    }
}

// Real-only solve (RK_ErrorEstimate, radau2a.c:479,498).
template <int N, int TS, typename T>
__device__ void lu_solve_real(const T* A1, const T* d1, Vec<N, TS>& x1)
{
    using TM = Team<TS>;
    constexpr int S = Vec<N, TS>::S;
    const int lane = TM::lane();
#pragma unroll
    for (int j = 0; j < N; ++j) {
        const double a = TM::bcast(x1[j / TS], j % TS);
        if (a != 0.0) {
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const int i = lane + TS * s;
                if (i > j && i < N) x1[s] = fma(-a, double(A1[i + j * N]), x1[s]);
            }
        }
    }
#pragma unroll
    for (int j = N - 1; j >= 0; --j) {
        const int src = j % TS, sj = j / TS;
        if (lane == src) x1[sj] = x1[sj] * double(d1[j]);
        const double a = TM::bcast(x1[sj], src);
        if (a != 0.0) {
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const int i = lane + TS * s;
                if (i < j) x1[s] = fma(-a, double(A1[i + j * N]), x1[s]);
            }
        }
    }
}

}  // namespace aib
