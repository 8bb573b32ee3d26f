// Mechanism callbacks on the device: the plugin slot of the reference's
// dydt / eval_jacob / sparse_multiplier (examples/van_der_pol/dydt.h:31,
// jacob.h:31, sparse_multiplier.h:22; pyJac's generated code in mechanism/).
//
// A mechanism is a struct with
//   static constexpr int N;                    state length
//   static constexpr int SMEM_RHS, SMEM_JAC;   team shared-memory doubles needed
//   dydt(t, var, y, dy, smem)                  dy = f(t, y)
//   jacob(t, var, y, J, smem)                  J[i + j*N] = d f_i / d y_j (column-major)
// evaluated cooperatively by a team (TS lanes) on distributed vectors.
#pragma once
#include "common.cuh"

namespace aib {

// ---------------------------------------------------------------- van der Pol
// examples/van_der_pol/dydt.c:88-95, jacob.c:129-141; thread-per-system only.
struct VanDerPol {
    static constexpr int N = 2;
    static constexpr int SMEM_RHS = 0;
    static constexpr int SMEM_JAC = 0;
    // TS = 1: the thread owns both elements.  TS > 1 (a team): lane 0 owns y1 and
    // lane 1 owns y2; the Jacobian is written by lane 0.
    template <int TS>
    __device__ __forceinline__ void dydt(double, double mu, const Vec<2, TS>& y, Vec<2, TS>& dy, double*) const {
        if constexpr (TS == 1) {
            dy[0] = y[1];
            dy[1] = mu * (1 - y[0] * y[0]) * y[1] - y[0];
        } else {
            const double y0 = Team<TS>::bcast(y[0], 0), y1 = Team<TS>::bcast(y[0], 1);
            const int l = Team<TS>::lane();
            dy[0] = l == 0 ? y1 : (l == 1 ? mu * (1 - y0 * y0) * y1 - y0 : 0.0);
        }
    }
    template <int TS>
    __device__ __forceinline__ void jacob(double, double mu, const Vec<2, TS>& y, double* jac, double*) const {
        double y0, y1;
        if constexpr (TS == 1) {
            y0 = y[0];
            y1 = y[1];
        } else {
            y0 = Team<TS>::bcast(y[0], 0);
            y1 = Team<TS>::bcast(y[0], 1);
        }
        if (Team<TS>::lane() == 0) {
            jac[0] = 0;
            jac[1] = -2 * mu * y0 * y1 - 1;
            jac[2] = 1;
            jac[3] = mu * (1 - y0 * y0);
        }
    }
};

// ---------------------------------------------------------------- mass action
// Device tables of the synthetic constant-pressure mechanism (model in
// accelerint_b200/mechanism.py).  Species-centred CSR lists give every species
// its reactions in reaction order, so wdot_k accumulates in the same order as
// a sequential loop over reactions.
struct MassActionTables {
    int K, R;
    const double* inv_mw;   // [K] 1/W_k
    const double* mw;       // [K]
    const double* cp;       // [K]
    const double* h_form;   // [K]
    const double* s_ref;    // [K]
    const int4* rsp;        // [R] reactant0, reactant1, product0, product1 (-1 = empty)
    const double* log_a;    // [R]
    const double* beta;     // [R]
    const double* ta;       // [R]
    const int* sp_ptr;      // [K+1]
    const int* sp_ent;      // [nnz] reaction * 4 + slot (slots 0,1 reactants; 2,3 products)
};

constexpr double R_U = 8.31446261815324;
constexpr double P_ATM = 101325.0;
constexpr double T_REF = 298.15;
// Rates and thermodynamics are evaluated at max(T, T_FLOOR) so that Newton
// iterates of an over-long step with unphysical temperatures stay finite.
constexpr double T_FLOOR = 100.0;


// Tables of the mechanism in use (pointers into global memory; one mechanism
// per process, as the reference compiles one into its library).
__constant__ MassActionTables c_ma;

// One state element per thread of a block team of TS threads (TS > K):
// thread t owns y_t (t = 0: temperature, t = 1 + k: mass fraction of k).
// Shared scratch sm: ys[N], C[K], h[K], grt[K], then per reaction q (dydt) or
// q, dqdT, dH, dqdC[4] (jacob).  Out of line: one copy serves every call site.
template <int K> struct MaPrep {
    double T, S, c0, cpm, logT, log_catm;
};

template <int K, int TS>
__device__ __forceinline__ MaPrep<K> ma_prepare(double P, double yi, double* ys, double* C, double* h, double* grt)
{
    constexpr int N = K + 1;
    using TM = Team<TS>;
    const int t = TM::lane();
    const MassActionTables& tb = c_ma;
    if (t < N) ys[t] = yi;
    TM::sync();
    MaPrep<K> p;
    p.T = fmax(ys[0], T_FLOOR);
    double S = 0.0, cpm = 0.0;
    if (t < K) {
        const double yk = ys[1 + t] * __ldg(tb.inv_mw + t);
        S = yk;
        cpm = yk * __ldg(tb.cp + t);
    }
    p.S = TM::sum(S);
    p.cpm = TM::sum(cpm);
    p.c0 = 1e-6 * P / (R_U * p.T);
    p.logT = log(p.T);
    p.log_catm = log(1e-6 * P_ATM / (R_U * p.T));
    if (t < K) {
        const double lnt = log(p.T / T_REF);
        C[t] = (p.c0 / p.S) * (ys[1 + t] * __ldg(tb.inv_mw + t));
        const double cpk = __ldg(tb.cp + t);
        const double hk = __ldg(tb.h_form + t) + cpk * (p.T - T_REF);
        h[t] = hk;
        grt[t] = hk / (R_U * p.T) - (__ldg(tb.s_ref + t) + cpk * lnt) * (1.0 / R_U);
    }
    TM::sync();
    return p;
}

template <int K>
__device__ __forceinline__ void ma_rates(int r, const MaPrep<K>& p, const double* grt, int4 sp, double& kf,
                                         double& kr, int& nre, int& npd)
{
    const MassActionTables& tb = c_ma;
    double g = grt[sp.z] - grt[sp.x];
    nre = 1;
    npd = 1;
    if (sp.y >= 0) { g -= grt[sp.y]; nre = 2; }
    if (sp.w >= 0) { g += grt[sp.w]; npd = 2; }
    const double lkf = __ldg(tb.log_a + r) + __ldg(tb.beta + r) * p.logT - __ldg(tb.ta + r) / p.T;
    kf = exp(lkf);
    kr = exp(lkf + g - double(npd - nre) * p.log_catm);
}

// f(y)_t for the calling thread's element t.
template <int K, int TS>
__device__ __noinline__ double ma_dydt(double P, double yi, double* sm)
{
    constexpr int N = K + 1;
    using TM = Team<TS>;
    const int t = TM::lane();
    const MassActionTables& tb = c_ma;
    double* ys = sm;
    double* C = ys + N;
    double* h = C + K;
    double* grt = h + K;
    double* q = grt + K;
    const int R = tb.R;
    const MaPrep<K> p = ma_prepare<K, TS>(P, yi, ys, C, h, grt);
    for (int r = t; r < R; r += TS) {
        const int4 sp = __ldg(tb.rsp + r);
        double kf, kr;
        int nre, npd;
        ma_rates<K>(r, p, grt, sp, kf, kr, nre, npd);
        double fwd = kf * C[sp.x];
        if (nre == 2) fwd *= C[sp.y];
        double rev = kr * C[sp.z];
        if (npd == 2) rev *= C[sp.w];
        q[r] = fwd - rev;
    }
    TM::sync();
    double Qp = 0.0, out = 0.0;
    if (t >= 1 && t < N) {
        const int k = t - 1;
        // net production of species k over its reactions, four entries at a time
        // (independent gathers, two partial sums)
        double w0 = 0.0, w1 = 0.0;
        const int e0 = __ldg(tb.sp_ptr + k), e1 = __ldg(tb.sp_ptr + k + 1);
        int e = e0;
        for (; e + 4 <= e1; e += 4) {
            const int a = __ldg(tb.sp_ent + e), b = __ldg(tb.sp_ent + e + 1);
            const int c = __ldg(tb.sp_ent + e + 2), d = __ldg(tb.sp_ent + e + 3);
            const double qa = q[a >> 2], qb = q[b >> 2], qc = q[c >> 2], qd = q[d >> 2];
            w0 += ((a & 3) < 2 ? -qa : qa) + ((b & 3) < 2 ? -qb : qb);
            w1 += ((c & 3) < 2 ? -qc : qc) + ((d & 3) < 2 ? -qd : qd);
        }
        for (; e < e1; ++e) {
            const int ent = __ldg(tb.sp_ent + e);
            const double qr = q[ent >> 2];
            w0 += (ent & 3) < 2 ? -qr : qr;
        }
        const double w = w0 + w1;
        Qp = h[k] * w;
        out = __ldg(tb.mw + k) * (p.S / p.c0) * w;
    }
    const double Q = TM::sum(Qp);
    if (t == 0) out = -p.S * Q / (p.c0 * p.cpm);
    TM::sync();
    return out;
}

// Analytic Jacobian into column-major J[N*N] (global memory); thread t writes row t.
template <int K, int TS>
__device__ __noinline__ void ma_jacob(double P, double yi, double* J, double* sm)
{
    constexpr int N = K + 1;
    using TM = Team<TS>;
    const int t = TM::lane();
    const MassActionTables& tb = c_ma;
    const int R = tb.R;
    double* ys = sm;
    double* C = ys + N;
    double* h = C + K;
    double* grt = h + K;
    double* q = grt + K;
    double* dqT = q + R;
    double* dH = dqT + R;
    double* dqC = dH + R;   // [R][4]
    const MaPrep<K> p = ma_prepare<K, TS>(P, yi, ys, C, h, grt);
    for (int r = t; r < R; r += TS) {
        const int4 sp = __ldg(tb.rsp + r);
        double kf, kr;
        int nre, npd;
        ma_rates<K>(r, p, grt, sp, kf, kr, nre, npd);
        const double c_r0 = C[sp.x], c_r1 = nre == 2 ? C[sp.y] : 1.0;
        const double c_p0 = C[sp.z], c_p1 = npd == 2 ? C[sp.w] : 1.0;
        const double fwd = kf * c_r0 * c_r1;
        const double rev = kr * c_p0 * c_p1;
        double dh = h[sp.z] - h[sp.x];
        if (npd == 2) dh += h[sp.w];
        if (nre == 2) dh -= h[sp.y];
        const double dlkf = (__ldg(tb.beta + r) + __ldg(tb.ta + r) / p.T) / p.T;
        const double dlkr = dlkf - dh / (R_U * p.T * p.T) + double(npd - nre) / p.T;
        q[r] = fwd - rev;
        dqT[r] = fwd * dlkf - rev * dlkr - (nre * fwd - npd * rev) / p.T;
        dH[r] = dh;
        dqC[4 * r + 0] = kf * c_r1;
        dqC[4 * r + 1] = nre == 2 ? kf * c_r0 : 0.0;
        dqC[4 * r + 2] = -kr * c_p1;
        dqC[4 * r + 3] = npd == 2 ? -kr * c_p0 : 0.0;
    }
    TM::sync();
    const double inv_c0 = 1.0 / p.c0;
    double hgp = 0.0, Qp = 0.0, dQTp = 0.0;
    if (t >= 1 && t < N) {
        const int k = t - 1;
        double w = 0.0, wT = 0.0, g = 0.0;
        const int e0 = __ldg(tb.sp_ptr + k), e1 = __ldg(tb.sp_ptr + k + 1);
        for (int e = e0; e < e1; ++e) {
            const int ent = __ldg(tb.sp_ent + e);
            const int r = ent >> 2;
            const double nu = (ent & 3) < 2 ? -1.0 : 1.0;
            const int4 sp = __ldg(tb.rsp + r);
            w += nu * q[r];
            wT += nu * dqT[r];
            double gr = dqC[4 * r + 0] * C[sp.x] + dqC[4 * r + 2] * C[sp.z];
            if (sp.y >= 0) gr += dqC[4 * r + 1] * C[sp.y];
            if (sp.w >= 0) gr += dqC[4 * r + 3] * C[sp.w];
            g += nu * gr * inv_c0;
        }
        hgp = h[k] * g;
        Qp = h[k] * w;
        dQTp = __ldg(tb.cp + k) * w + h[k] * wT;
        // dense part of row t, then the sparse G entries of the same row.  The
        // sparse additions are reductions without a returned value: the thread
        // does not wait for the scattered read-modify-writes (they are ordered
        // after its own stores to the same entries).  They are performed in L2,
        // so every reader of the Jacobian loads it with ld.global.cg (__ldcg):
        // an L1 line kept from an earlier read would miss them.
        const double a = w * inv_c0 - g;
        const double wmk = __ldg(tb.mw + k);
        for (int j = 0; j < K; ++j) J[t + N * (1 + j)] = wmk * __ldg(tb.inv_mw + j) * a;
        J[t] = (wmk * p.S * inv_c0) * (wT + w / p.T);
        for (int e = e0; e < e1; ++e) {
            const int ent = __ldg(tb.sp_ent + e);
            const int r = ent >> 2;
            const double nu = (ent & 3) < 2 ? -1.0 : 1.0;
            const int4 sp = __ldg(tb.rsp + r);
            atomicAdd(J + t + N * (1 + sp.x), wmk * __ldg(tb.inv_mw + sp.x) * nu * dqC[4 * r + 0]);
            if (sp.y >= 0) atomicAdd(J + t + N * (1 + sp.y), wmk * __ldg(tb.inv_mw + sp.y) * nu * dqC[4 * r + 1]);
            atomicAdd(J + t + N * (1 + sp.z), wmk * __ldg(tb.inv_mw + sp.z) * nu * dqC[4 * r + 2]);
            if (sp.w >= 0) atomicAdd(J + t + N * (1 + sp.w), wmk * __ldg(tb.inv_mw + sp.w) * nu * dqC[4 * r + 3]);
        }
    }
    const double hg = TM::sum(hgp);
    const double Q = TM::sum(Qp);
    const double dQT = TM::sum(dQTp);
    const double f = -1.0 / (p.c0 * p.cpm);
    if (t < K) {
        // temperature row, column 1 + t: sum_r dH_r dq_r/dC_t over the reactions of species t
        double hG = 0.0;
        const int e1 = __ldg(tb.sp_ptr + t + 1);
        for (int e = __ldg(tb.sp_ptr + t); e < e1; ++e) {
            const int ent = __ldg(tb.sp_ent + e);
            hG += dH[ent >> 2] * dqC[ent];
        }
        const double iw = __ldg(tb.inv_mw + t);
        J[N * (1 + t)] = f * (Q * iw - p.S * Q * __ldg(tb.cp + t) * iw / p.cpm + p.c0 * iw * (hG - hg));
    }
    if (t == 0) J[0] = f * p.S * (Q / p.T + dQT);
    TM::sync();
    // below the temperature floor f does not depend on T: zero column 0
    if (!(ys[0] > T_FLOOR) && t < N) J[t] = 0.0;
    TM::sync();
}

// Mechanism object used by the integrators: teams of TS >= N lanes (a block, a warp
// or part of a warp), one element per lane.
template <int KS>
struct MassAction {
    static constexpr int K = KS;
    static constexpr int N = K + 1;
    // dydt scratch doubles: ys[N], C[K], h[K], grt[K], q[R]
    static int smem_rhs(int R) { return N + 3 * K + R; }
    // jacob scratch doubles (may alias the complex Radau matrix): ys, C, h, grt, q, dqdT, dH, dqdC[4]
    static int smem_jac(int R) { return N + 3 * K + 7 * R; }

    template <int TS>
    __device__ __forceinline__ void dydt(double, double P, const Vec<N, TS>& y, Vec<N, TS>& dy, double* sm) const {
        static_assert(Vec<N, TS>::S == 1, "mass action runs on teams of at least N lanes, one element per lane");
        dy[0] = ma_dydt<K, TS>(P, y[0], sm);
    }
    template <int TS>
    __device__ __forceinline__ void jacob(double, double P, const Vec<N, TS>& y, double* J, double* sm) const {
        static_assert(Vec<N, TS>::S == 1, "mass action runs on teams of at least N lanes, one element per lane");
        ma_jacob<K, TS>(P, y[0], J, sm);
    }
};

// Finite-difference Jacobian over any mechanism's dydt (generic/fd_jacob.c with
// FD_ORD 1): forward differences with increment r_j = max(sqrt(eps) |y_j|,
// r0 / ewt_j), ewt = atol + rtol |y|, r0 = 1000 rtol eps N sqrt(sum (ewt dy)^2 / N)
// -- the reference's weighting, kept for parity.  N + 1 dydt calls per Jacobian;
// the owner of column j perturbs its element, every thread writes its rows.
template <class Mech>
struct FdJacobian : Mech {
    static constexpr int N = Mech::N;
    double atol, rtol;
    template <int TS>
    __device__ __noinline__ void jacob(double t, double P, const Vec<N, TS>& y, double* J, double* sm) const {
        using V = Vec<N, TS>;
        using TM = Team<TS>;
        V dy, yp, ft;
        Mech::template dydt<TS>(t, P, y, dy, sm);
        double ewt[V::S], sum = 0.0;
#pragma unroll
        for (int s = 0; s < V::S; ++s) {
            ewt[s] = atol + rtol * fabs(y[s]);
            if (V::ok(s)) sum += (ewt[s] * dy[s]) * (ewt[s] * dy[s]);
        }
        const double fac = sqrt(TM::sum(sum) / double(N));
        const double r0 = 1000.0 * rtol * DBL_EPSILON * double(N) * fac;
        const double srur = sqrt(DBL_EPSILON);
        for (int j = 0; j < N; ++j) {
            double rj = 0.0;
#pragma unroll
            for (int s = 0; s < V::S; ++s)
                if (V::idx(s) == j) rj = fmax(srur * fabs(y[s]), r0 / ewt[s]);
            const double r = TM::bcast(rj, j % TS);
#pragma unroll
            for (int s = 0; s < V::S; ++s) yp[s] = (V::idx(s) == j) ? y[s] + r : y[s];
            Mech::template dydt<TS>(t, P, yp, ft, sm);
#pragma unroll
            for (int s = 0; s < V::S; ++s)
                if (V::ok(s)) J[V::idx(s) + N * j] = (ft[s] - dy[s]) / r;
        }
        TM::sync();
    }
};

}  // namespace aib
