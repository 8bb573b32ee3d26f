// Register-resident LU of the Radau iteration matrices in single precision,
// for block teams of TS = 32 or 64 threads and N <= TS: thread i owns row i of
// E1 = (gamma/h) I - J (real) or E2 = ((alpha + i beta)/h) I - J (complex) in
// registers, assembled straight from the Jacobian; E2 is factored first, then E1.
// Each elimination step k takes ONE barrier:
//
//   1. every thread takes its row's column-k entry; each warp finds its
//      candidate pivot (first maximal |a|, |Re a| + |Im a|) with two warp
//      reductions, and the candidate's owner writes the warp's slot: the key,
//      the position, 1/pivot and the row's entries right of column k;
//   2. barrier;
//   3. every thread reads the warp slots, picks the winner (larger key, then the
//      smaller position), and updates its own row with the winner's.
//
// Rows are never moved: each thread tracks its row's position in the row order
// that LAPACK's xGETF2 interchanges would produce (the pivot row takes position
// k, the row that held position k takes the pivot row's old one), and ties go to
// the smaller position, so pivots, multipliers and info are those of the
// unblocked xGETF2 the radau2a/radau2a.c:256-278 calls make (reciprocal scaling
// of the multipliers, info = k + 1 at the first zero pivot, NaN counted as a
// candidate).  The factors end in the column-major shared-memory layout the
// triangular solves read (wsolve_real / wsolve_cplx), with perm[position] =
// original row and dinv[k] = 1 / U(k,k).
//
// Register a[j] of a thread holds column k + j of its row at step k (the
// "shifting row"): column k is always a[0], and the update writes
// a[j - 1] = a[j] - l u[j], which moves the row one column left in the same
// instruction, so the step loop needs no unrolling.  The Radau team kernels use
// this form for one-warp teams; with two warps (N up to 64) the row's registers
// force spills in the integrator around the call, and the shared-memory LU
// (tlu_pair) is faster there.
#pragma once
#include "common.cuh"
#include "wlinalg.cuh"

namespace aib {

__device__ __forceinline__ unsigned rlu_key(float m, bool active) {
    // |.| >= 0 orders as its bit pattern; NaN (0x7fc00000) above every number; + 1
    // keeps a zero magnitude apart from "no candidate"
    return active ? __float_as_uint(m) + 1u : 0u;
}

__device__ __forceinline__ void rlu_sync(int W) {
    if (W > 1) __syncthreads();
    else __syncwarp();
}

// The update length is a compile-time bound per range of steps (NR ranges, each
// updating the most columns any of its steps needs), so the code is NR copies
// of one short step.  Multipliers go to shared memory as they are made, at the
// row's current position, and LAPACK's interchange of positions k and q is
// applied to the multiplier columns left of k in parallel (thread j moves column
// j); a row's U part stays in its registers from the step it becomes the pivot
// and is stored at the end.
template <bool CPLX> struct SluElem { using type = float; };
template <> struct SluElem<true> { using type = float2; };

template <bool CPLX, int N> struct SluSlot {
    using E = typename SluElem<CPLX>::type;
    static constexpr int NU = CPLX ? (N + 1) / 2 * 2 : (N + 3) / 4 * 4;
    unsigned key;     // ordered |pivot| bits + 1 (0: the warp has no candidate row)
    int pos;          // position of the candidate row
    int row;          // its thread (original row index)
    int pad;
    float2 rc;        // 1 / pivot (0 for a zero pivot; .y unused for a real matrix)
    float2 pad2;
    E u[NU];          // u[j] = column k + j of the candidate row
};

__host__ __device__ constexpr int slu_slot_bytes(int n, int ts, bool cplx) {
    return 2 * (ts / 32) * (32 + (cplx ? 8 * ((n + 1) / 2 * 2) : 4 * ((n + 3) / 4 * 4)));
}

template <int N, int TS, bool CPLX, int UL>
__device__ __forceinline__ void slu_steps(int k0, int k1, typename SluElem<CPLX>::type (&a)[N], int& pos,
                                          int& info, float* A, float* dinv, unsigned char* xbuf)
{
    using E = typename SluElem<CPLX>::type;
    using Slot = SluSlot<CPLX, N>;
    constexpr int W = TS / 32;
    static_assert(sizeof(Slot) % 16 == 0, "slot layout");
    Slot* slots = reinterpret_cast<Slot*>(xbuf);   // [parity][warp]
    const int tid = int(threadIdx.x) & (TS - 1);
    const int lane = tid & 31;
    const int w = tid >> 5;
    const bool own = tid < N;
#pragma unroll 1
    for (int k = k0; k < k1; ++k) {
        Slot* sl = slots + (k & 1) * W;
        const E v = a[0];
        float mag;
        if constexpr (CPLX) mag = fabsf(v.x) + fabsf(v.y);
        else mag = fabsf(v);
        const unsigned key = rlu_key(mag, own && pos >= k);
        const unsigned mx = __reduce_max_sync(0xffffffffu, key);
        const unsigned mp = __reduce_min_sync(0xffffffffu, (mx != 0u && key == mx) ? unsigned(pos) : 0xffffffffu);
        const bool win = mx != 0u && key == mx && unsigned(pos) == mp;
        if (mx == 0u ? lane == 0 : win) {
            Slot& my = sl[w];
            my.key = mx;
            my.pos = int(mp);
            my.row = tid;
            float2 rc = make_float2(0.0f, 0.0f);
            if (mx > 1u) {
                if constexpr (CPLX) {
                    const cx<float> r = crecip(cx<float>{v.x, v.y});
                    rc = make_float2(r.re, r.im);
                } else {
                    rc.x = 1.0f / v;
                }
            }
            my.rc = rc;
#pragma unroll
            for (int j = 1; j <= UL; ++j) my.u[j] = a[j];
        }
        rlu_sync(W);
        int s = 0;
        if (W > 1) {
            const unsigned ka = sl[0].key, kb = sl[1].key;
            s = (kb > ka || (kb == ka && sl[1].pos < sl[0].pos)) ? 1 : 0;
        }
        const Slot& ws = sl[s];
        const bool nz = ws.key > 1u;
        const int q = ws.pos, r = ws.row;
        const float2 rc = ws.rc;
        if (!nz && info == 0) info = k + 1;
        if (tid == 0) {
            if constexpr (CPLX) reinterpret_cast<float2*>(dinv)[k] = rc;
            else dinv[k] = rc.x;
        }
        // xGETF2's interchange of positions k and q on the multiplier columns j < k
        if (q != k && tid < k) {
            E* Ae = reinterpret_cast<E*>(A);
            const E x = Ae[k + tid * N], y = Ae[q + tid * N];
            Ae[k + tid * N] = y;
            Ae[q + tid * N] = x;
        }
        if (tid == r) pos = k;
        else if (pos == k) pos = q;
        if (own && pos > k) {
            if constexpr (CPLX) {
                cx<float> l = cx<float>{v.x, v.y};
                if (nz) l = cmul(l, cx<float>{rc.x, rc.y});
                reinterpret_cast<float2*>(A)[pos + k * N] = make_float2(l.re, l.im);
                const float2 nlr = make_float2(-l.re, -l.re), lim = make_float2(l.im, -l.im);
#pragma unroll
                for (int j = 1; j <= UL; ++j) {
                    const float2 u = ws.u[j];
                    a[j - 1] = cfnma2(nlr, lim, u, make_float2(u.y, u.x), a[j]);
                }
            } else {
                const float l = nz ? v * rc.x : v;
                A[pos + k * N] = l;
#pragma unroll
                for (int j = 1; j <= UL; ++j) a[j - 1] = fmaf(-l, ws.u[j], a[j]);
            }
        }
    }
}

// One single-precision factorisation of the N x N matrix s I - J (s = sr + i si
// for CPLX, sr for a real matrix) into A (column-major, leading dimension N),
// perm, dinv; returns info.  The exchange slots (xbuf, slu_slot_bytes) must not
// overlap A, which holds the multipliers while the factorisation runs.
template <int N, int TS, bool CPLX, int NR = 3>
__device__ __noinline__ int slu_factor(const double* __restrict__ J, double sr, double si, float* A, int* perm,
                                       float* dinv, unsigned char* xbuf)
{
    static_assert(TS == 32 || TS == 64, "block teams of one or two warps");
    static_assert(N <= TS, "one row per thread");
    using E = typename SluElem<CPLX>::type;
    constexpr int W = TS / 32;
    constexpr int KR = (N + NR - 1) / NR;   // steps per range
    const int tid = int(threadIdx.x) & (TS - 1);
    const bool own = tid < N;
    E a[N];
#pragma unroll
    for (int j0 = 0; j0 < N; j0 += 8) {
        double v[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) v[c] = (own && j0 + c < N) ? -__ldcg(J + tid + (j0 + c) * N) : 0.0;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const int j = j0 + c;
            if (j >= N) break;
            const bool d = own && tid == j;
            if constexpr (CPLX) a[j] = make_float2(float(d ? v[c] + sr : v[c]), float(d ? si : 0.0));
            else a[j] = float(d ? v[c] + sr : v[c]);
        }
    }
    int pos = tid, info = 0;
    // the update of step k needs columns k+1 .. N-1 of the pivot row: N - 1 - k of them
    slu_steps<N, TS, CPLX, N - 1>(0, KR < N ? KR : N, a, pos, info, A, dinv, xbuf);
    if constexpr (NR > 1 && KR < N)
        slu_steps<N, TS, CPLX, N - 1 - KR>(KR, 2 * KR < N ? 2 * KR : N, a, pos, info, A, dinv, xbuf);
    if constexpr (NR > 2 && 2 * KR < N)
        slu_steps<N, TS, CPLX, (N - 1 - 2 * KR > 0 ? N - 1 - 2 * KR : 0)>(2 * KR, 3 * KR < N ? 3 * KR : N, a, pos,
                                                                            info, A, dinv, xbuf);
    if constexpr (NR > 3 && 3 * KR < N)
        slu_steps<N, TS, CPLX, (N - 1 - 3 * KR > 0 ? N - 1 - 3 * KR : 0)>(3 * KR, N, a, pos, info, A, dinv, xbuf);
    static_assert(NR <= 4, "at most four ranges");
    // ---- U rows (held since each row became the pivot) at their positions
    rlu_sync(W);
    if (own) {
        E* Ae = reinterpret_cast<E*>(A);
#pragma unroll
        for (int j = 0; j < N; ++j)
            if (pos + j < N) Ae[pos + (pos + j) * N] = a[j];
        perm[pos] = tid;
    }
    rlu_sync(W);
    return info;
}

}  // namespace aib
