// Radau IIA (3-stage, order 5) for one system per team, after
// radau2a/radau2a.c:520-736 (CPU reference; the GPU reference radau2a.cu has
// the RK_ErrorEstimate bug of solving with the raw Jacobian, radau2a.cu:612,
// which is not reproduced).
//
// Same control logic, constants and operation sequence as the CPU reference:
// simplified Newton with the real E1 and complex E2 factorisations, Gustafsson
// step control, Jacobian / LU reuse (SkipJac / SkipLU), quadratic-interpolant
// starting values (by default including the reference's x2 factor in Z3,
// radau2a.c:312; RadauParams::stage_extrap selects the collocation polynomial).
// The matrices are factorised in precision LT (double, or float for the
// precision form where the Newton loop itself refines the solution and the
// error-estimate solve gets one FP64 refinement step against J).
#pragma once
#include "common.cuh"
#include "linalg.cuh"
#include "wlinalg.cuh"
#include "rlinalg.cuh"
#include "mlp.cuh"

namespace aib {

namespace radau {
// radau2a.c:38-65
constexpr int MAX_NO_STEPS = 200000;
constexpr int NEWTON_MAXIT = 8;
constexpr double ROUNDOFF = DBL_EPSILON;
constexpr double FAC_MIN = 0.2, FAC_MAX = 8, FAC_SAFE = 0.9, FAC_REJ = 0.1;
constexpr double THETA_MIN = 0.001, NEWTON_TOL = 0.03, Q_MIN = 1.0, Q_MAX = 1.2;
constexpr int MAX_CONSECUTIVE_ERRS = 5;
// radau2a.c:101-229
__host__ __device__ constexpr double A(int i, int j) {
    constexpr double v[3][3] = {
    {1.968154772236604258683861429918299e-1, -6.55354258501983881085227825696087e-2,
     2.377097434822015242040823210718965e-2},
    {3.944243147390872769974116714584975e-1, 2.920734116652284630205027458970589e-1,
     -4.154875212599793019818600988496743e-2},
    {3.764030627004672750500754423692808e-1, 5.124858261884216138388134465196080e-1,
     1.111111111111111111111111111111111e-1}};
    return v[i][j];
}
__host__ __device__ constexpr double C(int i) {
    constexpr double v[3] = {1.550510257216821901802715925294109e-1, 6.449489742783178098197284074705891e-1, 1.0};
    return v[i];
}
__host__ __device__ constexpr double E(int i) {
    constexpr double v[4] = {0.05, -10.04880939982741556246032950764708 * 0.05,
                         1.382142733160748895793662840980412 * 0.05, -0.3333333333333333333333333333333333 * 0.05};
    return v[i];
}
constexpr double GAMMA = 3.637834252744495732208418513577775;
constexpr double ALPHA = 2.681082873627752133895790743211112;
constexpr double BETA = 3.050430199247410569426377624787569;
__host__ __device__ constexpr double T(int i, int j) {
    constexpr double v[3][3] = {
    {9.443876248897524148749007950641664e-2, -1.412552950209542084279903838077973e-1,
     -3.00291941051474244918611170890539e-2},
    {2.502131229653333113765090675125018e-1, 2.041293522937999319959908102983381e-1,
     3.829421127572619377954382335998733e-1},
    {1.0, 1.0, 0.0e0}};
    return v[i][j];
}
__host__ __device__ constexpr double TIA(int i, int j) {
    constexpr double v[3][3] = {
    {1.520148562492775501049204957366528e+1, 1.192055789400527921212348994770778,
     1.903956760517560343018332287285119},
    {-9.669512977505946748632625374449567, -8.724028436822336183071773193986487,
     3.096043239482439656981667712714881},
    {-1.409513259499574544876303981551774e+1, 5.895975725255405108079130152868952,
     -1.441236197545344702389881889085515e-1}};
    return v[i][j];
}
constexpr double ELO = 4;
}  // namespace radau

// Matrix storage of one team: shared memory for teams of several lanes (J may
// live in global scratch), registers/local memory for a thread per system.
// L1 is the precision of E1 (the matrix of the error estimate), LT that of E2.
template <int N, typename LT, typename L1 = LT> struct RadauRegStore {
    using E1T = L1;
    static constexpr bool jac_global = false;   // J is the thread's own (local) array
    double J[N * N];
    L1 E1[N * N];
    cx<LT> E2[N * N];
    L1 d1[N];
    cx<LT> d2[N];
    int p1[N], p2[N];
    double buf[N];
    __device__ double* jac() { return J; }
    __device__ L1* e1() { return E1; }
    __device__ cx<LT>* e2() { return E2; }
    __device__ L1* dinv1() { return d1; }
    __device__ cx<LT>* dinv2() { return d2; }
    __device__ int* perm1() { return p1; }
    __device__ int* perm2() { return p2; }
    __device__ double* vbuf() { return buf; }
    __device__ double* scratch_rhs() { return nullptr; }
    __device__ double* scratch_jac() { return nullptr; }
};

// L1 is the precision of E1 (the matrix of the error estimate), LT that of E2.
template <int N, typename LT, typename L1 = LT> struct RadauTeamStore {
    using E1T = L1;
    static constexpr bool jac_global = true;    // J is global scratch
    double* J;        // N*N (global scratch)
    L1* E1;           // N*N
    cx<LT>* E2;       // N*N (also the Jacobian evaluation scratch)
    L1* d1;
    cx<LT>* d2;
    int* p1;
    int* p2;
    double* buf;      // 3N (right-hand sides of the block-team solves)
    double* rhs;      // mechanism dydt scratch
    int* inf;         // 2 (factorisation status of E1, E2)
    __device__ int* infos() { return inf; }
    __device__ double* jac() { return J; }
    __device__ L1* e1() { return E1; }
    __device__ cx<LT>* e2() { return E2; }
    __device__ L1* dinv1() { return d1; }
    __device__ cx<LT>* dinv2() { return d2; }
    __device__ int* perm1() { return p1; }
    __device__ int* perm2() { return p2; }
    __device__ double* vbuf() { return buf; }
    __device__ double* scratch_rhs() { return rhs; }
    __device__ double* scratch_jac() { return reinterpret_cast<double*>(E2); }
    // shared-memory bytes of one team (J excluded)
    static constexpr size_t bytes(int smem_rhs) {
        return sizeof(LT) * N * N + sizeof(cx<LT>) * N * N + sizeof(LT) * N + sizeof(cx<LT>) * N +
               2 * sizeof(int) * N + sizeof(double) * N + sizeof(double) * smem_rhs;
    }
};

struct RadauParams {
    double atol, rtol;
    // state length of the error norms (radau2a.c:446-453 divide by NSP): N, or the
    // caller's state length when the mechanism is padded to the next instantiated size
    // (the padding rows stay zero and add nothing to the sums)
    int n_eff = 0;
    // starting values of the Newton iteration after an accepted step: 0 the reference's
    // extrapolation (radau2a.c:312 evaluates Z3 with x2 in its outer factor), 1 the
    // collocation polynomial of the last step evaluated at all three new nodes (x3 in
    // both factors of Z3, as in Hairer and Wanner's RADAU5)
    int stage_extrap = 0;
};

// LEARN (block teams only): 0 off; 1 step-size proposals and step records; 2 also
// stage proposals (which hold three more state vectors per thread)
template <int N, int TS, class Mech, typename LT, class Store, int LEARN = 0>
struct Radau {
    // A Jacobian entry: from L2 (ld.global.cg) when J is global scratch, which a
    // mechanism may have written with reductions that an L1 line kept from an
    // earlier read would miss; a plain load when J is the thread's own local
    // array (ld.global is not valid on a local address).
    __device__ __forceinline__ static double jload(const double* p) {
        if constexpr (Store::jac_global) return __ldcg(p);
        else return *p;
    }
    using V = Vec<N, TS>;
    using TM = Team<TS>;
    static_assert(!LEARN || TM::block, "learned mode runs on block teams");
    using L1 = typename Store::E1T;
    static constexpr int S = V::S;

    const Mech& mech;
    Store& st;
    RadauParams prm;
    double pr;
    Stats& stats;
    const LearnArgs* learn = nullptr;   // block teams only: learned proposals / step records

    // MLP input features of the calling thread's element (raw; standardised in mlp_infer_team)
    __device__ __forceinline__ void mlp_features(const V& y, double Hprev, float* x) const {
        const int l = TM::lane();
        float f = 0.0f;
        if (l == 0) f = float(y[0]);
        else if (l < N) f = float(log10(fmax(y[0], 1e-20)));
        else if (l == N) f = float(log10(Hprev));
        else if (l == N + 1) f = float(log10(pr / 101325.0));
        for (int i = l; i < MLP_D0; i += TS) x[i] = (i == l) ? f : 0.0f;
    }

    // Append one step record (features at the step start, converged stages,
    // log10 of the accepted H over the previous accepted H).
    __device__ void record_step(const V& y, double Hprev, double H, const V& Z1, const V& Z2, const V& Z3) {
        int slot = 0;
        if (TM::lane() == 0) slot = atomicAdd(learn->rec_count, 1);
        slot = TM::bcast(slot, 0);
        if (slot >= learn->rec_cap) return;
        float* r = learn->rec + size_t(slot) * MLP_REC;
        mlp_features(y, Hprev, r);
        float* tg = r + MLP_D0;
        const int l = TM::lane();
        if (l < N) {
            const double si = prm.atol + prm.rtol * fabs(y[0]);
            tg[l] = float(symlog(Z1[0] / si));
            tg[N + l] = float(symlog(Z2[0] / si));
            tg[2 * N + l] = float(symlog(Z3[0] / si));
        }
        for (int i = 3 * N + l; i < MLP_D4; i += TS) tg[i] = (i == 3 * N) ? float(log10(H / Hprev)) : 0.0f;
    }

    __device__ __forceinline__ void rhs(double t, const V& y, V& f) {
        mech.template dydt<TS>(t, pr, y, f, st.scratch_rhs());
        stats.c[ST_RHS]++;
    }

    __device__ __forceinline__ double err_norm(const V& sc, const V& d) const {
        double sum = 0.0;
#pragma unroll
        for (int s = 0; s < S; ++s)
            if (V::ok(s)) sum += sc[s] * sc[s] * d[s] * d[s];
        sum = TM::sum(sum);
        return fmax(sqrt(sum / double(prm.n_eff > 0 ? prm.n_eff : N)), 1e-10);
    }

    // radau2a.c:256-278; returns info (0 on success)
    __device__ int decomp(double H) {
        const double* J = st.jac();
        L1* E1 = st.e1();
        cx<LT>* E2 = st.e2();
        const double g = radau::GAMMA / H, ar = radau::ALPHA / H, ai = radau::BETA / H;
        if constexpr (Team<TS>::block && TS == 32 && N <= TS && sizeof(LT) == 4 && sizeof(L1) == 4) {
            // single precision on a one-warp team: each matrix assembled and factored in
            // registers (slu_factor, rlinalg.cuh), E2 first, then E1.  The matrices hold
            // their multipliers while they are factored: E2's exchange slots go to E1's
            // region (factored afterwards), E1's to the dydt scratch.
            stats.c[ST_DECOMP]++;
            const int i2 = slu_factor<N, TS, true>(J, ar, ai, reinterpret_cast<float*>(E2), st.perm2(),
                                                   reinterpret_cast<float*>(st.dinv2()),
                                                   reinterpret_cast<unsigned char*>(E1));
            const int i1 = slu_factor<N, TS, false>(J, g, 0.0, reinterpret_cast<float*>(E1), st.perm1(),
                                                    reinterpret_cast<float*>(st.dinv1()),
                                                    reinterpret_cast<unsigned char*>(st.scratch_rhs()));
            return i1 != 0 ? i1 : i2;
        }
        const int lane = TM::lane();
        // block teams store lu_cols(N) columns, the ones past N zero (see wlinalg.cuh)
        constexpr int NC = Team<TS>::block ? lu_cols(N) : N;
        if constexpr (Team<TS>::block && TS >= N) {
            // thread i assembles row i; the Jacobian loads of 8 columns are in flight together
            if (lane < N) {
                const int i = lane;
#pragma unroll 1
                for (int j0 = 0; j0 < NC; j0 += 8) {
                    double v[8];
#pragma unroll
                    for (int c = 0; c < 8; ++c) v[c] = (j0 + c < N) ? -jload(J + i + (j0 + c) * N) : 0.0;
#pragma unroll
                    for (int c = 0; c < 8; ++c) {
                        const int j = j0 + c;
                        E1[i + j * N] = L1(i == j ? v[c] + g : v[c]);
                        E2[i + j * N] = cx<LT>{LT(i == j ? v[c] + ar : v[c]), LT(i == j ? ai : 0.0)};
                    }
                }
            }
        } else {
            for (int e = lane; e < N * NC; e += TS) {
                const int i = e % N, j = e / N;
                const double mj = j < N ? -jload(J + e) : 0.0;
                E1[e] = L1(i == j ? mj + g : mj);
                E2[e] = cx<LT>{LT(i == j ? mj + ar : mj), LT(i == j ? ai : 0.0)};
            }
        }
        TM::sync();
        stats.c[ST_DECOMP]++;
        if constexpr (Team<TS>::block) {
            // warp 0 factors E1 while warp 1 factors E2 (one warp does both in a 32-thread team)
            int* inf = st.infos();
            const int w = TM::warp();
            const bool l0 = (threadIdx.x & 31) == 0;
            if (TS == 64) {
                // E2 pivots on warp 1 overlapped with E1 on warp 0, E2 updates on both.  A
                // two-column panel form, 1.15-1.22x faster alone, ran the FP32_ALL integrator 6 %
                // slower on identical work, so this overlapped split serves every precision
                const int2 ii = tlu_pair<N, L1, cx<LT>>(E1, st.perm1(), st.dinv1(), E2, st.perm2(), st.dinv2(), inf);
                TM::sync();
                // E1's info is known on warp 0, E2's on warp 1 (which pivots it)
                if (l0) inf[w] = w == 0 ? ii.x : ii.y;
            } else if (TS > 64) {
                if (w == 0) {
                    const int i1 = wlu_real<N, L1>(E1, st.perm1(), st.dinv1());
                    if (l0) inf[0] = i1;
                } else if (w == 1) {
                    const int i2 = wlu_cplx<N, LT>(E2, st.perm2(), st.dinv2());
                    if (l0) inf[1] = i2;
                }
            } else {
                const int i1 = wlu_real<N, L1>(E1, st.perm1(), st.dinv1());
                const int i2 = wlu_cplx<N, LT>(E2, st.perm2(), st.dinv2());
                if (l0) { inf[0] = i1; inf[1] = i2; }
            }
            TM::sync();
            const int info = inf[0] != 0 ? inf[0] : inf[1];
            TM::sync();
            return info;
        } else {
            int info = lu_real<N, TS, L1>(E1, st.perm1(), st.dinv1());
            if (info != 0) return info;
            return lu_cplx<N, TS, LT>(E2, st.perm2(), st.dinv2());
        }
    }

    // Block teams: E1 x = b through the shared buffer, solved by warp 0.
    __device__ void block_solve_e1(V& x) {
        double* xb = st.vbuf();
        const int t = TM::lane();
        if (t < N) xb[t] = x[0];
        TM::sync();
        if (TM::warp() == 0) wsolve_real<N, L1>(st.e1(), st.dinv1(), st.perm1(), xb);
        TM::sync();
        if (t < N) x[0] = xb[t];
        TM::sync();
    }

    // radau2a.c:388-441: Z <- T (E^-1 ((1/h) T^-1 A^-1 Z))
    __device__ void solve(double H, V& R1, V& R2, V& R3) {
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const double x1 = R1[s] / H, x2 = R2[s] / H, x3 = R3[s] / H;
            R1[s] = radau::TIA(0, 0) * x1 + radau::TIA(0, 1) * x2 + radau::TIA(0, 2) * x3;
            R2[s] = radau::TIA(1, 0) * x1 + radau::TIA(1, 1) * x2 + radau::TIA(1, 2) * x3;
            R3[s] = radau::TIA(2, 0) * x1 + radau::TIA(2, 1) * x2 + radau::TIA(2, 2) * x3;
        }
        double* buf = st.vbuf();
        if constexpr (Team<TS>::block) {
            const int t = TM::lane();
            if (t < N) {
                buf[t] = R1[0];
                buf[N + t] = R2[0];
                buf[2 * N + t] = R3[0];
            }
            TM::sync();
            const int w = TM::warp();
            if (TS >= 64) {
                if (w == 0) wsolve_real<N, L1>(st.e1(), st.dinv1(), st.perm1(), buf);
                else if (w == 1) wsolve_cplx<N, LT>(st.e2(), st.dinv2(), st.perm2(), buf + N, buf + 2 * N);
            } else {
                wsolve_real<N, L1>(st.e1(), st.dinv1(), st.perm1(), buf);
                wsolve_cplx<N, LT>(st.e2(), st.dinv2(), st.perm2(), buf + N, buf + 2 * N);
            }
            TM::sync();
            if (t < N) {
                R1[0] = buf[t];
                R2[0] = buf[N + t];
                R3[0] = buf[2 * N + t];
            }
            TM::sync();
        } else {
            permute<N, TS>(R1, st.perm1(), buf);
            permute<N, TS>(R2, st.perm2(), buf);
            permute<N, TS>(R3, st.perm2(), buf);
            lu_solve_pair<N, TS, L1, LT>(st.e1(), st.dinv1(), R1, st.e2(), st.dinv2(), R2, R3);
        }
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const double x1 = R1[s], x2 = R2[s], x3 = R3[s];
            R1[s] = radau::T(0, 0) * x1 + radau::T(0, 1) * x2 + radau::T(0, 2) * x3;
            R2[s] = radau::T(1, 0) * x1 + radau::T(1, 1) * x2 + radau::T(1, 2) * x3;
            R3[s] = radau::T(2, 0) * x1 + radau::T(2, 1) * x2 + radau::T(2, 2) * x3;
        }
    }

    // E1 x = b with one FP64 refinement step when the factors are single precision.
    __device__ void solve_e1(double H, V& x) {
        double* buf = st.vbuf();
        if constexpr (Team<TS>::block) {
            if (sizeof(L1) == sizeof(double)) {
                block_solve_e1(x);
                return;
            }
            // single-precision factors: one refinement step r = b - ((gamma/h) x - J x) in FP64
            const V b = x;
            block_solve_e1(x);
            const int t = TM::lane();
            if (t < N) buf[t] = x[0];
            TM::sync();
            const double* J = st.jac();
            double jx = 0.0;
            if (t < N) {
                // four partial sums: the Jacobian loads are issued together
                double a[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
                for (int j = 0; j < N; ++j) a[j & 3] = fma(jload(J + t + N * j), buf[j], a[j & 3]);
                jx = (a[0] + a[1]) + (a[2] + a[3]);
            }
            V r;
            r[0] = t < N ? b[0] - ((radau::GAMMA / H) * x[0] - jx) : 0.0;
            TM::sync();
            block_solve_e1(r);
            x[0] += r[0];
            return;
        }
        if (sizeof(L1) == sizeof(double)) {
            permute<N, TS>(x, st.perm1(), buf);
            lu_solve_real<N, TS, L1>(st.e1(), st.dinv1(), x);
            return;
        }
        V b = x;
        permute<N, TS>(x, st.perm1(), buf);
        lu_solve_real<N, TS, L1>(st.e1(), st.dinv1(), x);
        // r = b - ((gamma/h) x - J x)
        const double g = radau::GAMMA / H;
#pragma unroll
        for (int s = 0; s < S; ++s)
            if (V::ok(s)) buf[V::idx(s)] = x[s];
        TM::sync();
        const double* J = st.jac();
        V r;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            r[s] = 0.0;
            if (V::ok(s)) {
                const int i = V::idx(s);
                double jx = 0.0;
                for (int j = 0; j < N; ++j) jx = fma(jload(J + i + N * j), buf[j], jx);
                r[s] = b[s] - (g * x[s] - jx);
            }
        }
        TM::sync();
        permute<N, TS>(r, st.perm1(), buf);
        lu_solve_real<N, TS, L1>(st.e1(), st.dinv1(), r);
#pragma unroll
        for (int s = 0; s < S; ++s) x[s] += r[s];
    }

    // radau2a.c:458-508
    __device__ double error_estimate(double H, double t, const V& Y, const V& F0, const V& Z1, const V& Z2,
                                     const V& Z3, const V& sc, bool FirstStep, bool Reject) {
        const double e1 = radau::E(1) / H, e2 = radau::E(2) / H, e3 = radau::E(3) / H;
        V F2, TMP;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            F2[s] = e1 * Z1[s] + e2 * Z2[s] + e3 * Z3[s];
            TMP[s] = radau::E(0) * F0[s] + F2[s];
        }
        solve_e1(H, TMP);
        stats.c[ST_AUX]++;
        double Err = err_norm(sc, TMP);
        if (Err >= 1.0 && (FirstStep || Reject)) {
#pragma unroll
            for (int s = 0; s < S; ++s) TMP[s] += Y[s];
            V F1;
            rhs(t, TMP, F1);
#pragma unroll
            for (int s = 0; s < S; ++s) TMP[s] = F1[s] + F2[s];
            solve_e1(H, TMP);
            stats.c[ST_AUX]++;
            Err = err_norm(sc, TMP);
        }
        return Err;
    }

    // radau2a.c:520-736
    __device__ int integrate(double t_start, double t_end, V& y) {
        const double ATOL = prm.atol, RTOL = prm.rtol;
        double Hmin = 0, Hold = 0, Hacc = 0, ErrOld = 0;
        double H = fmin(5e-7, t_end - t_start);
        double Hnew;
        double t = t_start;
        bool Reject = false, FirstStep = true, SkipJac = false, SkipLU = false;
        V sc, y0, F0, Z1, Z2, Z3, DZ1, DZ2, DZ3, CONT0, CONT1, CONT2;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            sc[s] = 1.0 / (ATOL + fabs(y[s]) * RTOL);
            y0[s] = y[s];
            Z1[s] = Z2[s] = Z3[s] = 0.0;
            CONT0[s] = CONT1[s] = CONT2[s] = 0.0;
        }
        int Nconsecutive = 0, Nsteps = 0;
        double NewtonRate = pow(2.0, 1.25);
        // learned mode (block teams): proposals for the stages (ZP*) and the step size
        int mlp_flags = 0;
        if constexpr (LEARN) {
            if (learn) mlp_flags = learn->mlp.flags;
        }
        double Hprev = H;   // last accepted step size (the model's h feature)
        bool have_zp = false;
        V ZP1, ZP2, ZP3;
        while (t + radau::ROUNDOFF < t_end) {
            if (!Reject) rhs(t, y, F0);
            if constexpr (LEARN) {
                // the step-size proposal can only bind when the controller grows the
                // step more than 2x; stage proposals are wanted on every step
                const double gf = learn ? learn->mlp.growth_floor : 2.0;
                if (mlp_flags && !Reject && ((mlp_flags & MLP_USE_Z) || H > gf * Hprev)) {
                    float* xb = reinterpret_cast<float*>(st.scratch_rhs());
                    mlp_features(y, Hprev, xb);
                    TM::sync();
                    // without stage proposals only the step-size output is needed
                    const float* o = mlp_infer_team<TS>(learn->mlp, xb, xb + MLP_D0, xb + MLP_D0 + MLP_D4,
                                                        (mlp_flags & MLP_USE_Z) ? -1 : 3 * N);
                    const double Hp = Hprev * exp10(double(o[3 * N]));
                    if constexpr (LEARN >= 2) {
                      if (mlp_flags & MLP_USE_Z) {
#pragma unroll
                        for (int s = 0; s < S; ++s) {
                            const int i = V::idx(s);
                            const double si = ATOL + RTOL * fabs(y[s]);
                            ZP1[s] = V::ok(s) ? symexp(double(o[i])) * si : 0.0;
                            ZP2[s] = V::ok(s) ? symexp(double(o[N + i])) * si : 0.0;
                            ZP3[s] = V::ok(s) ? symexp(double(o[2 * N + i])) * si : 0.0;
                        }
                        have_zp = true;
                      }
                    }
                    TM::sync();
                    if ((mlp_flags & MLP_USE_H) && Hp == Hp) {
                        // limits growth only: never above the controller's step, and
                        // never below growth_floor (> 1) x the last accepted one, so the
                        // proposal cannot hold the step size down
                        const double Hn = fmin(H, fmax(Hp, gf * Hprev));
                        if (Hn != H) {
                            H = Hn;
                            SkipLU = false;
                        }
                    }
                    stats.c[ST_KRYLOV]++;
                }
            }
            if (!SkipLU) {
                if (!SkipJac) {
                    mech.template jacob<TS>(t, pr, y, st.jac(), st.scratch_jac());
                    stats.c[ST_JAC]++;
                }
                const int info = decomp(H);
                if (info != 0) {
                    Nconsecutive += 1;
                    if (Nconsecutive >= radau::MAX_CONSECUTIVE_ERRS) return EC_consecutive_steps;
                    H *= 0.5;
                    Reject = true;
                    SkipJac = true;
                    SkipLU = false;
                    stats.c[ST_REJECT]++;
                    continue;
                }
                Nconsecutive = 0;
            }
            Nsteps += 1;
            stats.c[ST_STEPS]++;
            if (Nsteps >= radau::MAX_NO_STEPS) return EC_max_steps_exceeded;
            if (0.1 * fabs(H) <= fabs(t) * radau::ROUNDOFF) return EC_h_plus_t_equals_h;
            NewtonRate = pow(fmax(NewtonRate, DBL_EPSILON), 0.8);
            bool NewtonDone = false;
            double Fac = 0.5;
            int NewtonIter = 0;
            double Theta = 0;
            for (int attempt = 0; attempt < (LEARN >= 2 ? 2 : 1); ++attempt) {
            const bool use_zp = LEARN >= 2 && have_zp && attempt == 0;
            if (use_zp) {
#pragma unroll
                for (int s = 0; s < S; ++s) { Z1[s] = ZP1[s]; Z2[s] = ZP2[s]; Z3[s] = ZP3[s]; }
            } else if (FirstStep) {
#pragma unroll
                for (int s = 0; s < S; ++s) Z1[s] = Z2[s] = Z3[s] = 0.0;
            } else {
                const double r = H / Hold;
                const double x1 = 1.0 + radau::C(0) * r, x2 = 1.0 + radau::C(1) * r, x3 = 1.0 + radau::C(2) * r;
                const double x3o = prm.stage_extrap ? x3 : x2;   // outer factor of Z3
#pragma unroll
                for (int s = 0; s < S; ++s) {
                    Z1[s] = CONT0[s] + x1 * (CONT1[s] + x1 * CONT2[s]);
                    Z2[s] = CONT0[s] + x2 * (CONT1[s] + x2 * CONT2[s]);
                    Z3[s] = CONT0[s] + x3o * (CONT1[s] + x3 * CONT2[s]);
                }
            }
            NewtonDone = false;
            double NewtonIncrementOld = 0;
            Fac = 0.5;
            NewtonIter = 0;
            Theta = 0;
            for (; NewtonIter < radau::NEWTON_MAXIT; NewtonIter++) {
                stats.c[ST_NEWTON]++;
                // RK_PrepareRHS (radau2a.c:353-383)
#pragma unroll
                for (int s = 0; s < S; ++s) { DZ1[s] = Z1[s]; DZ2[s] = Z2[s]; DZ3[s] = Z3[s]; }
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    V TMP, F;
                    const V& Zc = c == 0 ? Z1 : (c == 1 ? Z2 : Z3);
#pragma unroll
                    for (int s = 0; s < S; ++s) TMP[s] = y[s] + Zc[s];
                    rhs(t + radau::C(c) * H, TMP, F);
                    const double a1 = -H * radau::A(0, c), a2 = -H * radau::A(1, c), a3 = -H * radau::A(2, c);
#pragma unroll
                    for (int s = 0; s < S; ++s) {
                        DZ1[s] += a1 * F[s];
                        DZ2[s] += a2 * F[s];
                        DZ3[s] += a3 * F[s];
                    }
                }
                solve(H, DZ1, DZ2, DZ3);
                const double d1 = err_norm(sc, DZ1), d2 = err_norm(sc, DZ2), d3 = err_norm(sc, DZ3);
                const double NewtonIncrement = sqrt((d1 * d1 + d2 * d2 + d3 * d3) / 3.0);
                Theta = radau::THETA_MIN;
                if (NewtonIter > 0) {
                    Theta = NewtonIncrement / NewtonIncrementOld;
                    if (Theta < 0.99) {
                        NewtonRate = Theta / (1.0 - Theta);
                    } else {
                        break;
                    }
                    const double NewtonPredictedErr =
                        (NewtonIncrement * pow(Theta, double(radau::NEWTON_MAXIT - NewtonIter - 1))) / (1.0 - Theta);
                    if (NewtonPredictedErr >= radau::NEWTON_TOL) {
                        const double Qnewton = fmin(10.0, NewtonPredictedErr / radau::NEWTON_TOL);
                        Fac = 0.8 * pow(Qnewton, -1.0 / double(radau::NEWTON_MAXIT - NewtonIter));
                        break;
                    }
                }
                NewtonIncrementOld = fmax(NewtonIncrement, radau::ROUNDOFF);
#pragma unroll
                for (int s = 0; s < S; ++s) {
                    Z1[s] -= DZ1[s];
                    Z2[s] -= DZ2[s];
                    Z3[s] -= DZ3[s];
                }
                NewtonDone = (NewtonRate * NewtonIncrement <= radau::NEWTON_TOL);
                if (NewtonDone) break;
                if (NewtonIter == radau::NEWTON_MAXIT - 1) {
                    if (use_zp) break;   // learned guess failed: fall back to the extrapolation
                    return EC_newton_max_iterations_exceeded;
                }
            }
            if (NewtonDone || !use_zp) break;
            stats.c[ST_ARNOLDI]++;   // fall-back to the extrapolated guess, same H and LU
            }
            have_zp = false;
            if (!NewtonDone) {
                H = Fac * H;
                Reject = true;
                SkipJac = true;
                SkipLU = false;
                stats.c[ST_REJECT]++;
                continue;
            }
            const double Err = error_estimate(H, t, y, F0, Z1, Z2, Z3, sc, FirstStep, Reject);
            Fac = pow(Err, (-1.0 / radau::ELO)) * (1.0 + 2 * radau::NEWTON_MAXIT) /
                  (NewtonIter + 1.0 + 2 * radau::NEWTON_MAXIT);
            Fac = fmin(radau::FAC_MAX, fmax(radau::FAC_MIN, Fac));
            Hnew = Fac * H;
            if (Err < 1.0) {
                if (!FirstStep) {
                    double FacGus = radau::FAC_SAFE * (H / Hacc) * pow(Err * Err / ErrOld, -0.25);
                    FacGus = fmin(radau::FAC_MAX, fmax(radau::FAC_MIN, FacGus));
                    Fac = fmin(Fac, FacGus);
                    Hnew = Fac * H;
                }
                if constexpr (LEARN) {
                    if (learn && learn->rec) record_step(y, Hprev, H, Z1, Z2, Z3);
                }
                Hprev = H;
                Hacc = H;
                ErrOld = fmax(1e-2, Err);
                FirstStep = false;
                Hold = H;
                t += H;
                stats.c[ST_ACCEPT]++;
                // y += Z3; interpolant (radau2a.c:283-297); new scale
                const double c0 = radau::C(0), c1 = radau::C(1), c2 = radau::C(2);
                const double den = (c2 - c1) * (c1 - c0) * (c0 - c2);
#pragma unroll
                for (int s = 0; s < S; ++s) {
                    y[s] += Z3[s];
                    CONT0[s] = ((-c2 * c2 * c1 * Z1[s] + Z3[s] * c1 * c0 * c0 + c1 * c1 * c2 * Z1[s] -
                                 c1 * c1 * c0 * Z3[s] + c2 * c2 * c0 * Z2[s] - Z2[s] * c2 * c0 * c0) /
                                den) - Z3[s];
                    CONT1[s] = -(c0 * c0 * (Z3[s] - Z2[s]) + c1 * c1 * (Z1[s] - Z3[s]) + c2 * c2 * (Z2[s] - Z1[s])) / den;
                    CONT2[s] = (c0 * (Z3[s] - Z2[s]) + c1 * (Z1[s] - Z3[s]) + c2 * (Z2[s] - Z1[s])) / den;
                    sc[s] = 1.0 / (ATOL + fmax(fabs(y[s]), fabs(y0[s])) * RTOL);
                    y0[s] = y[s];
                }
                Hnew = fmin(fmax(Hnew, Hmin), t_end - t);
                if (Reject) Hnew = fmin(Hnew, H);
                Reject = false;
                if (t + Hnew / radau::Q_MIN - t_end >= 0.0) {
                    H = t_end - t;
                } else {
                    const double Hratio = Hnew / H;
                    SkipLU = (Theta <= radau::THETA_MIN) && (Hratio >= radau::Q_MIN) && (Hratio <= radau::Q_MAX);
                    if (!SkipLU) H = Hnew;
                }
                SkipJac = NewtonIter == 1 || NewtonRate <= radau::THETA_MIN;
            } else {
                if (FirstStep || Reject) {
                    H = radau::FAC_REJ * H;
                } else {
                    H = Hnew;
                }
                Reject = true;
                SkipJac = true;
                SkipLU = false;
                stats.c[ST_REJECT]++;
            }
        }
        return EC_success;
    }
};

}  // namespace aib
