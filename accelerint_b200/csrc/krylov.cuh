// Exponential Krylov integrators EXPRB43 and EXP4 for one system per block
// team.  Thread i owns state element i (TS >= N); the Krylov basis, the
// Hessenberg matrix, phi(cH) and the complex work matrix live in shared
// memory, the Jacobian in the team's global scratch (read column-wise,
// coalesced, by the Jacobian-vector products).
//
// Semantics follow the reference CPU code:
//   arnoldi                  exponential_integrators/arnoldi.h:45-141 (CPU loop
//                            condition err > 1, Q8)
//   phiAc / expAc            exponential_integrators/phiAHessenberg.c:83-184
//   Hessenberg LU / inverse  generic/complexInverse.c:35-248
//   vector helpers           exponential_integrators/exponential_linear_algebra.h
//   EXPRB43                  exponential_integrators/exprb43/exprb43.c:47-309
//   EXP4                     exponential_integrators/exp4/exp4.c:46-320
// The basis Vm, Hm and phiHm start from zero on every integrate call: after a
// happy breakdown the reference's error estimate reads a basis column that
// the current Arnoldi call did not write (arnoldi.h:118).
#pragma once
#include "common.cuh"

namespace aib {

constexpr int CF_NRA = 10;   // N_RA, the (10, 10) CF approximant
struct CfTable {
    double pr[CF_NRA], pi[CF_NRA], rr[CF_NRA], ri[CF_NRA];   // poles, residues
};
__constant__ CfTable c_cf;

// Krylov dimensions at which the error estimate is checked (arnoldi.h:26)
__device__ __forceinline__ int krylov_index_list(int k) {
    constexpr int L[23] = {1, 2, 3, 4, 5, 6, 7, 9, 11, 14, 17, 21, 27, 34, 42, 53, 67, 84, 106, 133, 167, 211, 265};
    return L[k < 23 ? k : 22];
}

struct KrylovStore {
    double* J;       // [N*N] Jacobian, column-major (global)
    double* Vm;      // [N*STRIDE] basis, column j at Vm + j*N
    double* Hm;      // [STRIDE*STRIDE] Hessenberg matrix, column-major
    double* phiHm;   // [STRIDE*STRIDE]
    cxd* inv;        // [STRIDE*STRIDE] complex work matrix; mechanism scratch outside phi
    cxd* cw;         // [STRIDE]
    int* piv;        // [STRIDE]
    double* mv0;     // [STRIDE] m-vectors
    double* mv1;     // [STRIDE]
    double* nv;      // [N] an N-vector shared for a Jacobian-vector product
};

template <int N, int TS, class Mech, int P>
struct Krylov {
    using V = Vec<N, TS>;
    using TM = Team<TS>;
    static constexpr int STRIDE = N + P;
    static_assert(V::S == 1, "one state element per thread");

    const Mech& mech;
    KrylovStore s;
    double atol, rtol, pr;
    Stats& st;

    __device__ __forceinline__ static int lane() { return TM::lane(); }
    __device__ __forceinline__ static bool own() { return lane() < N; }
    __device__ __forceinline__ static double sum(double x) { return TM::sum(x); }
    __device__ __forceinline__ static void sync() { TM::sync(); }
    __device__ __forceinline__ double* mscratch() const { return reinterpret_cast<double*>(s.inv); }

    // exponential_linear_algebra.h: sc_norm
    __device__ __forceinline__ static double sc_norm(double v, double sc) {
        const double x = own() ? v * v * sc * sc : 0.0;
        return sqrt(sum(x) / N);
    }

    __device__ __forceinline__ void rhs(double t, double yi, double& f) {
        V y, dy;
        y[0] = own() ? yi : 0.0;
        mech.template dydt<TS>(t, pr, y, dy, mscratch());
        f = dy[0];
        st.c[ST_RHS]++;
        sync();
    }

    __device__ __forceinline__ void jac(double t, double yi) {
        V y;
        y[0] = own() ? yi : 0.0;
        mech.template jacob<TS>(t, pr, y, s.J, mscratch());
        st.c[ST_JAC]++;
        sync();
    }

    // sparse_multiplier: w_i = sum_k J[i + N k] v_k, v in shared memory.  The Jacobian
    // is read from L2 (ld.global.cg): a mechanism may write its entries with reductions,
    // which the L1 copy of an earlier read would not see.
    __device__ __forceinline__ double jacvec_smem(const double* v) const {
        if (!own()) return 0.0;
        const int i = lane();
        double acc = __ldcg(s.J + i) * v[0];
#pragma unroll 6
        for (int k = 1; k < N; ++k) acc += __ldcg(s.J + i + N * k) * v[k];
        return acc;
    }
    __device__ __forceinline__ double jacvec(double vi) {
        if (own()) s.nv[lane()] = vi;
        sync();
        const double w = jacvec_smem(s.nv);
        sync();
        return w;
    }

    // matvec_m_by_m (exponential_linear_algebra.h:28-70): out = A V (+ V)
    __device__ __forceinline__ static void matvec_mm(int m, const double* A, const double* Vv, double* out,
                                                     bool plus_eye) {
        for (int i = lane(); i < m; i += TS) {
            double acc = A[i] * Vv[0];
            for (int j = 1; j < m; ++j) acc += A[j * STRIDE + i] * Vv[j];
            if (plus_eye) acc += Vv[i];
            out[i] = acc;
        }
        sync();
    }

    // row i of Vm (first m columns) times an m-vector in shared memory
    __device__ __forceinline__ double matvec_nm(int m, const double* Vv) const {
        if (!own()) return 0.0;
        const int i = lane();
        double acc = s.Vm[i] * Vv[0];
        for (int j = 1; j < m; ++j) acc += s.Vm[j * N + i] * Vv[j];
        return acc;
    }

    // ------------------------------------------------ Hessenberg LU and inverse
    // cabs(z) > 0, the zero test of the inverse's inner products (complexInverse.c),
    // without the square root: true when a part is infinite, false when a part is NaN
    // (and none infinite), else true unless both parts are zero.
    __device__ __forceinline__ static bool cnonzero(cxd z) {
        if (isinf(z.re) || isinf(z.im)) return true;
        if (isnan(z.re) || isnan(z.im)) return false;
        return z.re != 0.0 || z.im != 0.0;
    }

    // complexInverse.c:35-74: LU with adjacent-row pivoting; thread per column.
    __device__ int hessenberg_lu(int n) {
        cxd* A = s.inv;
        int last_pivot = 0;
        for (int i = 0; i < n - 1; ++i) {
            const cxd a = A[i * STRIDE + i], b = A[i * STRIDE + i + 1];
            const bool swap = hypot(a.re, a.im) < hypot(b.re, b.im);
            const int lp = last_pivot;
            if (lane() == 0) s.piv[i] = swap ? i + 1 : i;
            if (!swap) last_pivot = i;
            const cxd d = swap ? b : a, e = swap ? a : b;
            if (!(hypot(d.re, d.im) > 0.0)) {
                sync();
                return i;
            }
            const cxd tau = cdiv(e, d);
            for (int k = lane(); k < n; k += TS) {
                cxd* col = A + k * STRIDE;
                cxd ri = col[i], rn = col[i + 1];
                if (swap && k >= lp) {
                    const cxd tmp = ri;
                    ri = rn;
                    rn = tmp;
                }
                if (k > i) rn = cfnma(tau, ri, rn);
                if (k == i) rn = tau;
                col[i] = ri;
                col[i + 1] = rn;
            }
            sync();
        }
        if (lane() == 0) s.piv[n - 1] = n - 1;
        sync();
        return 0;
    }

    // complexInverse.c:178-227: inv(U), then inv(A) L = inv(U), then column swaps.
    __device__ int hessenberg_inverse(int n) {
        cxd* A = s.inv;
        // inv(U), column by column; rows i < j of column j become
        // -inv(u_jj) * (Uinv[0:j, 0:j] x) (upper_mv, complexInverse.c:108-123)
        for (int j = 0; j < n; ++j) {
            const cxd ajj = A[j + STRIDE * j];
            if (hypot(ajj.re, ajj.im) == 0.0) {
                sync();
                return j;
            }
            const cxd rj = crecip(ajj);
            const cxd mAjj = cmake(-rj.re, -rj.im);
            cxd* x = A + STRIDE * j;
            cxd acc[(STRIDE + TS - 1) / TS];
#pragma unroll
            for (int r = 0; r < (STRIDE + TS - 1) / TS; ++r) {
                const int i = lane() + r * TS;
                if (i < j) {
                    const cxd xi = x[i];
                    cxd v = xi;
                    if (cnonzero(xi)) v = cmul(xi, A[i + STRIDE * i]);
                    for (int k = i + 1; k < j; ++k) {
                        const cxd xk = x[k];
                        if (cnonzero(xk)) v = cadd(v, cmul(xk, A[i + STRIDE * k]));
                    }
                    acc[r] = cmul(v, mAjj);
                }
            }
            sync();
#pragma unroll
            for (int r = 0; r < (STRIDE + TS - 1) / TS; ++r) {
                const int i = lane() + r * TS;
                if (i < j) x[i] = acc[r];
            }
            if (lane() == 0) x[j] = rj;
            sync();
        }
        // solve inv(A) L = inv(U) for inv(A), last column first (cgemv, complexInverse.c:146-164)
        for (int j = n - 1; j >= 0; --j) {
            for (int i = lane(); i < n; i += TS)
                if (i > j) s.cw[i] = A[i + STRIDE * j];
            sync();
            if (j < n - 1) {
                for (int i = lane(); i < n; i += TS) {
                    cxd v = (i > j) ? cmake(0.0, 0.0) : A[i + STRIDE * j];
                    for (int k = j + 1; k < n; ++k) {
                        const cxd w = s.cw[k];
                        if (cnonzero(w)) v = cadd(v, cmul(cmake(-w.re, -w.im), A[i + STRIDE * k]));
                    }
                    A[i + STRIDE * j] = v;
                }
            }
            sync();
        }
        // column interchanges, last pivot first; every thread owns its rows
        for (int i = lane(); i < n; i += TS) {
            for (int j = n - 2; j >= 0; --j) {
                const int pj = s.piv[j];
                if (pj != j) {
                    const cxd tmp = A[STRIDE * j + i];
                    A[STRIDE * j + i] = A[STRIDE * pj + i];
                    A[STRIDE * pj + i] = tmp;
                }
            }
        }
        sync();
        return 0;
    }

    // phiAHessenberg.c:83-184: phiHm = sum_{q even} 2 Re(c_q (cs H - theta_q I)^-1),
    // c_q = r_q (order 0) or r_q / theta_q (order 1); m x m leading block.
    __device__ int phi(int order, int m, double cs) {
        for (int r = lane(); r < m * m; r += TS) s.phiHm[(r / m) * STRIDE + (r % m)] = 0.0;
        for (int q = 0; q < CF_NRA; q += 2) {
            const cxd pole = cmake(c_cf.pr[q], c_cf.pi[q]);
            const cxd res = cmake(c_cf.rr[q], c_cf.ri[q]);
            sync();
            for (int r = lane(); r < m * m; r += TS) {
                const int i = r % m, j = r / m;
                const double h = cs * s.Hm[i + j * STRIDE];
                s.inv[i + j * STRIDE] = (i == j) ? cmake(h - pole.re, -pole.im) : cmake(h, 0.0);
            }
            sync();
            int info = hessenberg_lu(m);
            if (info != 0) return info;
            info = hessenberg_inverse(m);
            if (info != 0) return info;
            const cxd coef = order == 0 ? res : cdiv(res, pole);
            for (int r = lane(); r < m * m; r += TS) {
                const int i = r % m, j = r / m;
                const cxd a = s.inv[i + j * STRIDE];
                s.phiHm[i + j * STRIDE] += 2.0 * (coef.re * a.re - coef.im * a.im);
            }
        }
        sync();
        return 0;
    }

    // arnoldi.h:45-141.  v: this thread's element of the start vector.
    // Returns the Krylov dimension m, or -info when a phi evaluation failed.
    __device__ int arnoldi(int order, double scale, int p, double h, double v, double sc, double& beta) {
        const double vv = own() ? v : 0.0;
        double nrm = sqrt(sum(vv * vv));
        if (nrm == 0.0) nrm = 1.0;
        beta = nrm;
        const double mn = 1.0 / nrm;
        if (own()) s.Vm[lane()] = vv * mn;
        sync();
        double store = 0.0, err = 2.0;
        int index = 0, j = 0;
        while (err > 1.0) {
            for (; j < krylov_index_list(index) && j + p < STRIDE; ++j) {
                double w = jacvec_smem(s.Vm + j * N);
                for (int i = 0; i <= j; ++i) {
                    const double vij = own() ? s.Vm[i * N + lane()] : 0.0;
                    const double d = sum(w * vij);
                    if (lane() == 0) s.Hm[j * STRIDE + i] = d;
                    w -= d * vij;
                }
                const double hn = sqrt(sum(w * w));
                if (lane() == 0) s.Hm[j * STRIDE + j + 1] = hn;
                if (fabs(hn) < atol) {
                    ++j;
                    break;
                }
                const double hinv = 1.0 / hn;
                if (own()) s.Vm[(j + 1) * N + lane()] = w * hinv;
                sync();
            }
            sync();
            if (j + p >= STRIDE) return j;
            ++index;
            store = s.Hm[(j - 1) * STRIDE + j];
            sync();
            // augment Hm for the p-extended phi evaluation (arnoldi.h:103-111)
            for (int r = lane(); r < STRIDE; r += TS) {
                if (r <= j + 1) s.Hm[j * STRIDE + r] = (r == 0) ? 1.0 : 0.0;
                for (int i = 1; i < p; ++i)
                    if (r <= j + i + 1) s.Hm[(j + i) * STRIDE + r] = (r == j + i - 1) ? 1.0 : 0.0;
            }
            if (lane() == 0) s.Hm[(j - 1) * STRIDE + j] = 0.0;
            sync();
            const int info = phi(order, j + p, h * scale);
            if (info != 0) return -info;
            const double scn = sc_norm(own() ? s.Vm[j * N + lane()] : 0.0, sc);
            err = h * beta * fabs(store * s.phiHm[j * STRIDE + j - 1]) * scn;
            sync();
            if (lane() == 0) {
                s.Hm[(j - 1) * STRIDE + j] = store;
                s.Hm[j * STRIDE] = 0.0;
            }
            sync();
        }
        return j;
    }

    __device__ void clear_work() {
        for (int r = lane(); r < N * STRIDE; r += TS) s.Vm[r] = 0.0;
        for (int r = lane(); r < STRIDE * STRIDE; r += TS) {
            s.Hm[r] = 0.0;
            s.phiHm[r] = 0.0;
        }
        sync();
    }

    __device__ __forceinline__ void count_arnoldi(int m) {
        st.c[ST_ARNOLDI]++;
        st.c[ST_KRYLOV] += m > 0 ? m : 0;
    }

    // error control shared by both methods (exprb43.c:236-270, exp4.c:263-300)
    struct Control {
        double h, h_old, err_old;
        bool reject;
        int failures, steps;
    };

    __device__ __forceinline__ void finish(Control& c, double err, double& t, double t_end, double& y,
                                           double y1, double& sc, double scn) {
        constexpr double ORD = 3.0;
        double h_new = pow(err, -1.0 / ORD);
        c.failures = 0;
        if (err <= 1.0) {
            sc = scn;
            h_new = fmin(h_new, (c.h / c.h_old) * pow(c.err_old / (err * err), 1.0 / ORD));
            h_new = c.h * fmax(fmin(0.9 * h_new, 8.0), 0.2);
            y = y1;
            t += c.h;
            st.c[ST_ACCEPT]++;
            c.err_old = fmax(1.0e-2, err);
            c.h_old = c.h;
            if (c.reject) {
                c.reject = false;
                h_new = fmin(c.h, h_new);
            }
            c.h = fmin(h_new, t_end - t);
        } else {
            h_new = c.h * fmax(fmin(0.9 * h_new, 8.0), 0.2);
            h_new = fmin(h_new, t_end - t);
            c.reject = true;
            st.c[ST_REJECT]++;
            c.h = fmin(c.h, h_new);
        }
    }

    __device__ __forceinline__ bool krylov_failed(Control& c, int m, int p) {
        if (m + p >= STRIDE || m < 0) {
            c.h /= 5.0;
            c.failures++;
            c.reject = true;
            st.c[ST_REJECT]++;
            return true;
        }
        return false;
    }

    // exprb43.c:47-309 (P = 4)
    __device__ int integrate_exprb43(double t, double t_end, V& yv) {
        double y = own() ? yv[0] : 0.0;
        Control c{fmin(1.0e-8, t_end - t), 0.0, 1.0, false, 0, 0};
        c.h_old = c.h;
        double sc = 1.0 / (atol + fabs(y) * rtol);
        double beta = 0.0, fy = 0.0, gy = 0.0;
        clear_work();
        while (t < t_end && t + c.h > t) {
            if (c.failures >= 5) { yv[0] = y; return EC_consecutive_steps; }
            if (c.steps++ >= 100000) { yv[0] = y; return EC_max_steps_exceeded; }
            if (t + c.h <= t) { yv[0] = y; return EC_h_plus_t_equals_h; }
            st.c[ST_STEPS]++;
            const double h = c.h;
            if (!c.reject) {
                rhs(t, y, fy);
                jac(t, y);
                gy = fy - jacvec(y);
            }
            int m = arnoldi(0, 0.5, 1, h, fy, sc, beta);
            count_arnoldi(m);
            if (krylov_failed(c, m, 1)) continue;
            matvec_mm(m, s.phiHm, s.phiHm + m * STRIDE, s.mv0, true);
            const double sa0 = matvec_nm(m, s.mv0) * beta;
            double temp = matvec_nm(m, s.phiHm + m * STRIDE) * beta + y;
            double sa1 = 0.0;
            rhs(t, temp, sa1);
            temp = sa1 - jacvec(temp) - gy;
            const int m1 = arnoldi(0, 1.0, 4, h, temp, sc, beta);
            count_arnoldi(m1);
            if (krylov_failed(c, m1, 4)) continue;
            // matvec_n_by_m_scale_special (exponential_linear_algebra.h:118-139)
            double sa2;
            {
                const double a0 = matvec_nm(m1, s.phiHm + (m1 + 2) * STRIDE);
                const double a1 = matvec_nm(m1, s.phiHm + (m1 + 3) * STRIDE);
                const double a2 = matvec_nm(m1, s.phiHm + m1 * STRIDE);
                sa1 = a0 * (beta / (h * h));
                sa2 = a1 * (beta / (h * h * h));
                temp = a2 * beta + sa0 + y;
            }
            double sa3 = 0.0;
            rhs(t, temp, sa3);
            temp = sa3 - jacvec(temp) - gy;
            const int m2 = arnoldi(0, 1.0, 4, h, temp, sc, beta);
            count_arnoldi(m2);
            if (krylov_failed(c, m2, 4)) continue;
            // matvec_n_by_m_scale_special2 (:158-176)
            double sa4;
            {
                const double a0 = matvec_nm(m2, s.phiHm + (m2 + 2) * STRIDE);
                const double a1 = matvec_nm(m2, s.phiHm + (m2 + 3) * STRIDE);
                sa3 = a0 * (beta / (h * h));
                sa4 = a1 * (beta / (h * h * h));
            }
            double y1 = y + sa0 + 16.0 * sa1 - 48.0 * sa2 + -2.0 * sa3 + 12.0 * sa4;
            if (!own()) y1 = 0.0;
            const double e = 48.0 * sa2 - 12.0 * sa4;
            const double scn = 1.0 / (atol + fmax(fabs(y), fabs(y1)) * rtol);
            const double err = fmax(DBL_EPSILON, sc_norm(e, scn));
            finish(c, err, t, t_end, y, y1, sc, scn);
            sync();
        }
        yv[0] = y;
        return EC_success;
    }

    // exp4.c:46-320 (P = 1)
    __device__ int integrate_exp4(double t, double t_end, V& yv) {
        double y = own() ? yv[0] : 0.0;
        Control c{fmin(1.0e-8, t_end - t), 0.0, 1.0, false, 0, 0};
        c.h_old = c.h;
        double sc = 1.0 / (atol + fabs(y) * rtol);
        double beta = 0.0, fy = 0.0;
        clear_work();
        while (t < t_end && t + c.h > t) {
            if (c.failures >= 5) { yv[0] = y; return EC_consecutive_steps; }
            if (c.steps++ >= 100000) { yv[0] = y; return EC_max_steps_exceeded; }
            if (t + c.h <= t) { yv[0] = y; return EC_h_plus_t_equals_h; }
            st.c[ST_STEPS]++;
            const double h = c.h;
            if (!c.reject) {
                rhs(t, y, fy);
                jac(t, y);
            }
            const int m = arnoldi(1, 1.0 / 3.0, 1, h, fy, sc, beta);
            count_arnoldi(m);
            if (krylov_failed(c, m, 1)) continue;
            const double k1 = matvec_nm(m, s.phiHm) * beta;
            matvec_mm(m, s.phiHm, s.phiHm, s.mv0, false);
            matvec_mm(m, s.Hm, s.mv0, s.mv1, false);
            const double k2 = matvec_nm(m, s.mv1) * (beta * (h / 6.0)) + k1;
            matvec_mm(m, s.phiHm, s.mv1, s.mv0, false);
            matvec_mm(m, s.Hm, s.mv0, s.mv1, false);
            const double k3 = matvec_nm(m, s.mv1) * (beta * (h * h / 27.0)) + 2.0 * k2 - k1;
            double ft = h * ((-7.0 / 300.0) * k1 + (97.0 / 150.0) * k2 - (37.0 / 300.0) * k3);
            double temp = 0.0;
            rhs(t, y + ft, temp);
            double k4 = temp - fy - jacvec(ft);
            const int m1 = arnoldi(1, 1.0 / 3.0, 1, h, k4, sc, beta);
            count_arnoldi(m1);
            if (krylov_failed(c, m1, 1)) continue;
            k4 = matvec_nm(m1, s.phiHm) * beta;
            matvec_mm(m1, s.phiHm, s.phiHm, s.mv0, false);
            matvec_mm(m1, s.Hm, s.mv0, s.mv1, false);
            const double k5 = matvec_nm(m1, s.mv1) * (beta * (h / 6.0)) + k4;
            matvec_mm(m1, s.phiHm, s.mv1, s.mv0, false);
            matvec_mm(m1, s.Hm, s.mv0, s.mv1, false);
            const double k6 = matvec_nm(m1, s.mv1) * (beta * (h * h / 27.0)) + 2.0 * k5 - k4;
            ft = h * ((59.0 / 300.0) * k1 - (7.0 / 75.0) * k2 + (269.0 / 300.0) * k3 + (2.0 / 3.0) * (k4 + k5 + k6));
            rhs(t, y + ft, temp);
            double k7 = temp - fy - jacvec(ft);
            const int m2 = arnoldi(1, 1.0 / 3.0, 1, h, k7, sc, beta);
            count_arnoldi(m2);
            if (krylov_failed(c, m2, 1)) continue;
            k7 = matvec_nm(m2, s.phiHm + m2 * STRIDE) * (beta / (h / 3.0));
            double y1 = y + h * (k3 + k4 - (4.0 / 3.0) * k5 + k6 + (1.0 / 6.0) * k7);
            if (!own()) y1 = 0.0;
            const double scn = 1.0 / (atol + fmax(fabs(y), fabs(y1)) * rtol);
            double e = k3 - (2.0 / 3.0) * k5 + 0.5 * (k6 + k7 - k4) - (y1 - y) / h;
            double err = h * sc_norm(e, scn);
            e = -k1 + 2.0 * k2 - k4 + k7 - (y1 - y) / h;
            err = fmax(DBL_EPSILON, fmin(err, h * sc_norm(e, scn)));
            finish(c, err, t, t_end, y, y1, sc, scn);
            sync();
        }
        yv[0] = y;
        return EC_success;
    }
};

}  // namespace aib
