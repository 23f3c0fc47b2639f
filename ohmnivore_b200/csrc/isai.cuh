// ISAI(1) preconditioner on the device: ILU(0) factor by Chow-Patel sweeps,
// ISAI(1) columns by local triangular solves, and a BiCGSTAB whose
// preconditioner apply is z = M_U (M_L r) (src/solver/gpu.rs:159-162).
// Included by solver_kernel.cuh; the symbolic set-up is in isai_host.h.
#pragma once

namespace ohm {

// Number of Chow-Patel sweeps per factorisation (each one a grid phase).
constexpr int kChowPatelSweeps = 6;
// Largest local system of one ISAI column (the host caps the patterns to it).
constexpr int kIsaiLocal = 32;

// ILU(0) factor + ISAI(1) values for the current a.vals64.  Grid phases:
// fill (factor initial guess from A), kChowPatelSweeps fixed-point sweeps
// (Jacobi style, double-buffered, so the result is deterministic), then one
// thread per column of M_L and of M_U.  Returns false if a barrier gave up.
template <class Team>
__device__ __forceinline__ bool isai_setup(const KernelArgs &a, Team &g) {
    const int n = a.n;
    const int gtid = g.gtid, gstride = g.gstride;
    double *F = a.isai_f0, *Fn = a.isai_f1;
    // initial guess: U = upper part of A, L = strictly lower part scaled by 1/A_jj
    for (int i = gtid; i < n; i += gstride) {
        for (uint32_t s = a.aug_rp[i]; s < a.aug_rp[i + 1]; ++s) {
            const int32_t m = a.aug_map[s];
            const double av = m >= 0 ? a.vals64[m] : 0.0;
            const uint32_t j = a.aug_col[s];
            if ((int)j < i) {
                const int32_t dm = a.aug_map[a.aug_diag[j]];
                const double ajj = dm >= 0 ? a.vals64[dm] : 0.0;
                F[s] = fabs(ajj) > 1e-300 ? av / ajj : av;
            } else {
                F[s] = av;
            }
        }
    }
    if (!g.sync()) return false;
    for (int sweep = 0; sweep < kChowPatelSweeps; ++sweep) {
        for (int i = gtid; i < n; i += gstride) {
            for (uint32_t s = a.aug_rp[i]; s < a.aug_rp[i + 1]; ++s) {
                const int32_t m = a.aug_map[s];
                double acc = m >= 0 ? a.vals64[m] : 0.0;
                for (uint32_t q = a.cp_ptr[s]; q < a.cp_ptr[s + 1]; ++q)
                    acc -= F[a.cp_pair[2 * q]] * F[a.cp_pair[2 * q + 1]];
                const uint32_t j = a.aug_col[s];
                if ((int)j < i) {
                    const double ujj = F[a.aug_diag[j]];
                    acc = fabs(ujj) > 1e-300 ? acc / ujj : acc;
                }
                Fn[s] = acc;
            }
        }
        if (!g.sync()) return false;
        double *tmp = F; F = Fn; Fn = tmp;
    }
    // value of the factor at (r, c): L (strict lower, unit diagonal implied) or U
    auto fval = [&](uint32_t r, uint32_t c) -> double {
        for (uint32_t s = a.aug_rp[r]; s < a.aug_rp[r + 1]; ++s) {
            const uint32_t cc = a.aug_col[s];
            if (cc == c) return F[s];
            if (cc > c) break;
        }
        return 0.0;
    };
    double m[kIsaiLocal];
    for (int k = gtid; k < 2 * n; k += gstride) {
        if (k < n) {
            // column k of M_L: (L + I)[J, J] m = e_k, rows J ascending, J[0] = k
            const uint32_t b = a.ml_cp[k], e = a.ml_cp[k + 1];
            const int len = min((int)(e - b), kIsaiLocal);
            for (int x = 0; x < len; ++x) {
                const uint32_t rx = a.ml_row[b + x];
                double acc = (rx == (uint32_t)k) ? 1.0 : 0.0;
                for (int y = 0; y < x; ++y) acc -= fval(rx, a.ml_row[b + y]) * m[y];
                m[x] = acc;
                a.ml_val[a.ml_pos[b + x]] = acc;
            }
        } else {
            // column c of M_U: U[J, J] m = e_c, rows J ascending, J[last] = c
            const int c = k - n;
            const uint32_t b = a.mu_cp[c], e = a.mu_cp[c + 1];
            const int len = min((int)(e - b), kIsaiLocal);
            for (int x = len - 1; x >= 0; --x) {
                const uint32_t rx = a.mu_row[b + x];
                double acc = (rx == (uint32_t)c) ? 1.0 : 0.0;
                for (int y = x + 1; y < len; ++y) acc -= fval(rx, a.mu_row[b + y]) * m[y];
                const double uxx = fval(rx, rx);
                m[x] = fabs(uxx) > 1e-300 ? acc / uxx : 0.0;
                a.mu_val[a.mu_pos[b + x]] = m[x];
            }
        }
    }
    return g.sync();
}

// Right-preconditioned BiCGSTAB with the ISAI(1) apply, same operation order
// as krylov() (bicgstab.rs:104-183); seven grid synchronisations per
// iteration: y = M_L p (p formed on the fly), phat = M_U y, v = A phat,
// y = M_L s (s formed on the fly), shat = M_U y, t = A shat, update.
template <typename T, int LPR, class Team>
__device__ __forceinline__ int krylov_isai(const KernelArgs &a, Team &g, double tol_floor, double inner_rtol,
                                           int max_it, bool accept_partial, KrylovOut &out) {
    using Acc = T;
    const int r0 = g.r0, r1 = g.r1, n = a.n;
    // vectors carved from the record area (4n slots each)
    T *pin = (T *)a.rec0, *pout = (T *)a.rec0 + n, *v = (T *)a.rec0 + 2 * (size_t)n;
    T *r = (T *)a.rec0 + 3 * (size_t)n, *y = (T *)a.rec1;
    T *rhat = (T *)a.rhat, *s = (T *)a.s, *t = (T *)a.t;
    T *phat = (T *)a.phat, *shat = (T *)a.shat, *d = (T *)a.d;
    const T *A;
    if constexpr (sizeof(T) == 4) A = (const T *)a.vals32; else A = (const T *)a.vals64;
    out.iterations = 0;
    out.restarts = 0;

    // stopping norm: scaled residual W r for Newton solves, as in krylov()
    const bool wt = a.newton != 0;
    double *w = a.dx;
    double acc0[2] = {0.0, 0.0};
    for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
        const T rt = cvt<T>(a.r64[i]);
        r[i] = rt; rhat[i] = rt; pin[i] = T(0); v[i] = T(0); d[i] = T(0);
        double wi = 1.0;
        if (wt) {
            const uint32_t ds = a.diag_slot[i];
            const double aii = ds == kSentinel ? 0.0 : a.vals64[ds];
            if (fabs(aii) > 1e-30) wi = 1.0 / fabs(aii);
            w[i] = wi;
        }
        acc0[0] += (double)rt * (double)rt;
        acc0[1] += (wi * (double)rt) * (wi * (double)rt);
    }
    {
        if (!g.template allreduce<2>(acc0)) return kKrylovAbort;
    }
    const double r0norm = sqrt(acc0[1]);
    const double abs_tol = fmax(tol_floor, inner_rtol * r0norm);
    double rr_cur = acc0[0], rhat2 = acc0[0], rho_new = acc0[0];
    double rho = 1.0, alpha = 1.0, omega = 1.0;
    int code = kKrylovRunning;
    int it = 0;
#define OHM_RESTART_ISAI()                                                     \
    do {                                                                       \
        for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {              \
            rhat[i] = r[i]; pin[i] = T(0); v[i] = T(0);                        \
        }                                                                      \
        OHM_SYNC_OR(kKrylovAbort);                                             \
        rho = 1.0; alpha = 1.0; omega = 1.0;                                   \
        rho_new = rr_cur; rhat2 = rr_cur;                                      \
        ++out.restarts;                                                        \
    } while (0)
    if (!isfinite(r0norm)) {
        code = kKrylovNan;
    } else if (r0norm < abs_tol || r0norm == 0.0) {
        code = kKrylovConverged;
    } else {
        for (; it < max_it; ++it) {
            if (!(fabs(rho_new) >= kBreakdownRel * sqrt(rhat2 * rr_cur))) {
                if (out.restarts < a.max_restarts && rr_cur > 0.0) {
                    OHM_RESTART_ISAI();
                } else {
                    code = kKrylovBreakRho;
                    break;
                }
            }
            const double beta = (rho_new / rho) * (alpha / omega);
            rho = rho_new;
            const double om = omega;
            auto pnew = [&](int j, bool) -> T {
                return cvt<T>(((double)pin[j] + (-om) * (double)v[j]) * beta + (double)r[j]);
            };
            // y = M_L p ; p written for own rows
            spmv_rows<LPR, double>(a.ml_rp, a.ml_col, a.ml_val, (const uint8_t *)nullptr, r0, r1, pnew,
                                   [&](int i, double yy) { pout[i] = pnew(i, false); y[i] = cvt<T>(yy); });
            OHM_SYNC_OR(kKrylovAbort);
            { T *tmp = pin; pin = pout; pout = tmp; }
            auto y_at = [&](int j, bool) -> T { return y[j]; };
            // phat = M_U y
            spmv_rows<LPR, double>(a.mu_rp, a.mu_col, a.mu_val, (const uint8_t *)nullptr, r0, r1, y_at,
                                   [&](int i, double z) { phat[i] = cvt<T>(z); });
            OHM_SYNC_OR(kKrylovAbort);
            // v = A phat ; (r_hat, v), (v, v)
            auto ph_at = [&](int j, bool) -> T { return phat[j]; };
            double acc1[2] = {0.0, 0.0};
            spmv_rows<LPR, Acc>(a.row_ptr, a.col, A, (const uint8_t *)nullptr, r0, r1, ph_at, [&](int i, double yv) {
                const T vt = cvt<T>(yv);
                v[i] = vt;
                acc1[0] += (double)rhat[i] * (double)vt;
                acc1[1] += (double)vt * (double)vt;
            });
            {
                if (!g.template allreduce<2>(acc1)) return kKrylovAbort;
            }
            if (!(fabs(acc1[0]) >= kBreakdownRel * sqrt(rhat2 * acc1[1]))) {
                if (out.restarts < a.max_restarts && rr_cur > 0.0) {
                    OHM_RESTART_ISAI();
                    continue;
                }
                code = kKrylovBreakRv;
                break;
            }
            alpha = rho / acc1[0];
            const double al = alpha;
            auto s_of = [&](int j, bool) -> T { return cvt<T>((double)r[j] + (-al) * (double)v[j]); };
            // y = M_L s ; s written for own rows ; ||s||^2
            double acc2[1] = {0.0};
            spmv_rows<LPR, double>(a.ml_rp, a.ml_col, a.ml_val, (const uint8_t *)nullptr, r0, r1, s_of,
                                   [&](int i, double yy) {
                                       const T si = s_of(i, false);
                                       s[i] = si;
                                       y[i] = cvt<T>(yy);
                                       const double ws = wt ? w[i] * (double)si : (double)si;
                                       acc2[0] += ws * ws;
                                   });
            {
                if (!g.template allreduce<1>(acc2)) return kKrylovAbort;
            }
            if (sqrt(acc2[0]) < abs_tol) {          // early exit (bicgstab.rs:134-139)
                for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x)
                    d[i] = cvt<T>((double)d[i] + al * (double)phat[i]);
                code = kKrylovConverged;
                ++it;
                break;
            }
            // shat = M_U y
            spmv_rows<LPR, double>(a.mu_rp, a.mu_col, a.mu_val, (const uint8_t *)nullptr, r0, r1, y_at,
                                   [&](int i, double z) { shat[i] = cvt<T>(z); });
            OHM_SYNC_OR(kKrylovAbort);
            // t = A shat ; (t, s), (t, t)
            auto sh_at = [&](int j, bool) -> T { return shat[j]; };
            double acc3[2] = {0.0, 0.0};
            spmv_rows<LPR, Acc>(a.row_ptr, a.col, A, (const uint8_t *)nullptr, r0, r1, sh_at, [&](int i, double tv) {
                const T tt = cvt<T>(tv);
                t[i] = tt;
                acc3[0] += (double)tt * (double)s[i];
                acc3[1] += (double)tt * (double)tt;
            });
            {
                if (!g.template allreduce<2>(acc3)) return kKrylovAbort;
            }
            if (!(acc3[1] > 0.0)) { code = kKrylovBreakTt; break; }
            omega = acc3[0] / acc3[1];
            double acc4[3] = {0.0, 0.0, 0.0};
            for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
                d[i] = cvt<T>(((double)d[i] + al * (double)phat[i]) + omega * (double)shat[i]);
                const T rt = cvt<T>((double)s[i] + (-omega) * (double)t[i]);
                r[i] = rt;
                const double wr = wt ? w[i] * (double)rt : (double)rt;
                acc4[0] += (double)rhat[i] * (double)rt;
                acc4[1] += (double)rt * (double)rt;
                acc4[2] += wr * wr;
            }
            {
                if (!g.template allreduce<3>(acc4)) return kKrylovAbort;
            }
            rho_new = acc4[0];
            rr_cur = acc4[1];
            const double rnorm = sqrt(acc4[2]);
            if (!isfinite(rnorm)) { code = kKrylovNan; ++it; break; }
            if (rnorm < abs_tol) { code = kKrylovConverged; ++it; break; }
            if (fabs(omega) < 1e-30) { code = kKrylovBreakOmega; ++it; break; }
            if (accept_partial && it + 1 == max_it && rnorm <= 0.5 * r0norm) {
                code = kKrylovConverged;
                ++it;
                break;
            }
        }
        if (code == kKrylovRunning) code = kKrylovMaxIter;
    }
#undef OHM_RESTART_ISAI
    out.iterations = it;
    if (code == kKrylovConverged)
        for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) a.dx[i] = (double)d[i];
    return code;
}

}  // namespace ohm
