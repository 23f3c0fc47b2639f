// AC sweep: A(f) x(f) = b_ac with A(f) = G + j 2 pi f C for many frequency
// points in one launch (src/analysis/ac.rs:56-70 solves them one at a time).
//
// One thread block per frequency point, taken from a work queue; each runs a
// complex FP64 right-preconditioned BiCGSTAB with the reference's operation
// order (src/solver/gpu.rs:608-690: conjugated dots sum(conj(x) y), stop at
// ||r|| < tol ||b||).  A(f) is never stored: the SpMV reads the shared G and
// C values of one pattern and forms g + j w c per nonzero, so every
// frequency's matrix traffic hits the same L2-resident arrays.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "host_util.h"

using namespace ohm;

namespace {

constexpr int kAcBlock = 256;       // points >> SMs: several blocks per SM
constexpr int kAcWideBlock = 1024;  // points <= SMs on a large system: one wide block per point
constexpr int kAcVecs = 11;        // x r rhat p v s t phat shat m_self m_part

struct AcDev {
    int code, iterations, restarts, pad;
    double rnorm, bnorm;
};

struct AcArgs {
    int n, n_freq, precond, max_it, max_restarts;
    double tol;
    const uint32_t *rp, *col;
    const double *g, *c;               // c may be null
    const double2 *b;
    const double *omega;               // per frequency point of this launch
    const int32_t *partner;
    const uint32_t *diag_slot, *off_slot;
    double2 *work;                     // kAcVecs * n per frequency point
    AcDev *info;
    unsigned int *queue;
};

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// conj(a) * b
__device__ __forceinline__ double2 cdotc(double2 a, double2 b) {
    return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double cabs2(double2 a) { return a.x * a.x + a.y * a.y; }
__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
    const double d = cabs2(b);
    return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}
__device__ __forceinline__ double2 cval(const AcArgs &A, uint32_t k, double w) {
    return make_double2(A.g[k], A.c ? w * A.c[k] : 0.0);
}

// y_i = sum_k A(f)_ik x_k for every row, LPR lanes per row; f(i, y).
template <int LPR, typename F>
__device__ __forceinline__ void cspmv(const AcArgs &A, double w, const double2 *x, F f) {
    const int lane = threadIdx.x % LPR, group = threadIdx.x / LPR, ngroups = blockDim.x / LPR;
    for (int base = 0; base < A.n; base += ngroups) {
        const int i = base + group;
        const bool ok = i < A.n;
        const uint32_t b = ok ? A.rp[i] : 0u, e = ok ? A.rp[i + 1] : 0u;
        uint32_t len = e - b;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) len = max(len, __shfl_xor_sync(0xffffffffu, len, o));
        double2 acc = make_double2(0.0, 0.0);
        for (uint32_t off = lane; off < len; off += LPR) {
            const uint32_t k = b + off;
            if (k < e) acc = cadd(acc, cmul(cval(A, k, w), x[A.col[k]]));
        }
#pragma unroll
        for (int o = LPR / 2; o > 0; o >>= 1) {
            acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o, LPR);
            acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o, LPR);
        }
        if (ok && lane == 0) f(i, acc);
    }
}

template <int LPR, int BLOCK>
__global__ void __launch_bounds__(BLOCK) ac_sweep_kernel(AcArgs A) {
    __shared__ double smem[32 * 4];
    __shared__ int s_q;
    const int n = A.n;
    for (;;) {
        if (threadIdx.x == 0) s_q = (int)atomicAdd(A.queue, 1u);
        __syncthreads();
        const int q = s_q;
        __syncthreads();
        if (q >= A.n_freq) return;
        const double w = A.omega[q];
        double2 *W = A.work + (size_t)q * kAcVecs * n;
        double2 *x = W, *r = W + n, *rh = W + 2 * (size_t)n, *p = W + 3 * (size_t)n, *v = W + 4 * (size_t)n;
        double2 *s = W + 5 * (size_t)n, *t = W + 6 * (size_t)n, *ph = W + 7 * (size_t)n, *sh = W + 8 * (size_t)n;
        double2 *ms = W + 9 * (size_t)n, *mp = W + 10 * (size_t)n;

        // preconditioner coefficients for this frequency, and the start vectors
        double acc0[1] = {0.0};
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            double2 cs = make_double2(0.0, 0.0), cp = make_double2(0.0, 0.0);
            const uint32_t ds = A.diag_slot[i];
            const double2 aii = ds == kSentinel ? make_double2(0.0, 0.0) : cval(A, ds, w);
            const int pi = A.partner[i];
            if (A.precond == kPcNone) {
                cs = make_double2(1.0, 0.0);
            } else if (A.precond == kPcAuto && pi >= 0) {
                // [[a_ii a_ik] [a_ki a_kk]]^-1, the row-i half
                const uint32_t dk = A.diag_slot[pi];
                const double2 akk = dk == kSentinel ? make_double2(0.0, 0.0) : cval(A, dk, w);
                const double2 aik = cval(A, A.off_slot[i], w), aki = cval(A, A.off_slot[pi], w);
                const double2 det = csub(cmul(aii, akk), cmul(aik, aki));
                if (cabs2(det) > 1e-300) {
                    cs = cdiv(akk, det);
                    cp = cdiv(make_double2(-aik.x, -aik.y), det);
                }
            } else if (cabs2(aii) > 1e-30) {
                cs = cdiv(make_double2(1.0, 0.0), aii);        // gpu.rs:300-313
            } else if (A.precond == kPcAuto) {
                cs = make_double2(1.0, 0.0);
            }
            ms[i] = cs;
            mp[i] = cp;
            const double2 bi = A.b[i];
            x[i] = make_double2(0.0, 0.0);
            r[i] = bi;
            rh[i] = bi;
            p[i] = make_double2(0.0, 0.0);
            v[i] = make_double2(0.0, 0.0);
            acc0[0] += cabs2(bi);
        }
        block_sum<1>(acc0, smem);
        const double bnorm = sqrt(acc0[0]);
        int code = kKrylovRunning, it = 0, restarts = 0;
        double rnorm = bnorm;
        if (!(bnorm >= 1e-30)) {
            code = isfinite(bnorm) ? kKrylovConverged : kKrylovNan;    // b = 0: x = 0 (gpu.rs:618-621)
        } else {
            const double abs_tol = A.tol * bnorm;
            double2 rho = make_double2(1.0, 0.0), alpha = rho, omega = rho;
            double2 rho_new = make_double2(acc0[0], 0.0);
            double rr = acc0[0], rh2 = acc0[0];
            auto restart = [&]() {
                for (int i = threadIdx.x; i < n; i += blockDim.x) {
                    rh[i] = r[i];
                    p[i] = make_double2(0.0, 0.0);
                    v[i] = make_double2(0.0, 0.0);
                }
                __syncthreads();
                rho = make_double2(1.0, 0.0);
                alpha = rho;
                omega = rho;
                rho_new = make_double2(rr, 0.0);
                rh2 = rr;
                ++restarts;
            };
            for (; it < A.max_it; ++it) {
                if (!(sqrt(cabs2(rho_new)) >= kBreakdownRel * sqrt(rh2 * rr))) {
                    if (restarts < A.max_restarts && rr > 0.0) restart();
                    else { code = kKrylovBreakRho; break; }
                }
                const double2 beta = cmul(cdiv(rho_new, rho), cdiv(alpha, omega));
                rho = rho_new;
                for (int i = threadIdx.x; i < n; i += blockDim.x)
                    p[i] = cadd(cmul(csub(p[i], cmul(omega, v[i])), beta), r[i]);
                __syncthreads();
                for (int i = threadIdx.x; i < n; i += blockDim.x) {
                    double2 z = cmul(ms[i], p[i]);
                    const int pi = A.partner[i];
                    if (pi >= 0) z = cadd(z, cmul(mp[i], p[pi]));
                    ph[i] = z;
                }
                __syncthreads();
                double a1[4] = {0.0, 0.0, 0.0, 0.0};     // r_hat^H v, ||v||^2
                cspmv<LPR>(A, w, ph, [&](int i, double2 y) {
                    v[i] = y;
                    const double2 d = cdotc(rh[i], y);
                    a1[0] += d.x;
                    a1[1] += d.y;
                    a1[2] += cabs2(y);
                });
                block_sum<4>(a1, smem);
                const double2 rhv = make_double2(a1[0], a1[1]);
                if (!(sqrt(cabs2(rhv)) >= kBreakdownRel * sqrt(rh2 * a1[2]))) {
                    if (restarts < A.max_restarts && rr > 0.0) { restart(); continue; }
                    code = kKrylovBreakRv;
                    break;
                }
                alpha = cdiv(rho, rhv);
                double a2[1] = {0.0};
                for (int i = threadIdx.x; i < n; i += blockDim.x) {
                    const double2 si = csub(r[i], cmul(alpha, v[i]));
                    s[i] = si;
                    a2[0] += cabs2(si);
                }
                block_sum<1>(a2, smem);
                if (sqrt(a2[0]) < abs_tol) {                     // gpu.rs:646-650
                    for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] = cadd(x[i], cmul(alpha, ph[i]));
                    rnorm = sqrt(a2[0]);
                    code = kKrylovConverged;
                    ++it;
                    break;
                }
                for (int i = threadIdx.x; i < n; i += blockDim.x) {
                    double2 z = cmul(ms[i], s[i]);
                    const int pi = A.partner[i];
                    if (pi >= 0) z = cadd(z, cmul(mp[i], s[pi]));
                    sh[i] = z;
                }
                __syncthreads();
                double a3[3] = {0.0, 0.0, 0.0};          // t^H s, t^H t
                cspmv<LPR>(A, w, sh, [&](int i, double2 y) {
                    t[i] = y;
                    const double2 d = cdotc(y, s[i]);
                    a3[0] += d.x;
                    a3[1] += d.y;
                    a3[2] += cabs2(y);
                });
                block_sum<3>(a3, smem);
                if (!(a3[2] > 0.0)) { code = kKrylovBreakTt; break; }
                omega = cdiv(make_double2(a3[0], a3[1]), make_double2(a3[2], 0.0));
                double a4[3] = {0.0, 0.0, 0.0};          // r_hat^H r, ||r||^2
                for (int i = threadIdx.x; i < n; i += blockDim.x) {
                    x[i] = cadd(cadd(x[i], cmul(alpha, ph[i])), cmul(omega, sh[i]));
                    const double2 ri = csub(s[i], cmul(omega, t[i]));
                    r[i] = ri;
                    const double2 d = cdotc(rh[i], ri);
                    a4[0] += d.x;
                    a4[1] += d.y;
                    a4[2] += cabs2(ri);
                }
                block_sum<3>(a4, smem);
                rho_new = make_double2(a4[0], a4[1]);
                rr = a4[2];
                rnorm = sqrt(rr);
                if (!isfinite(rnorm)) { code = kKrylovNan; ++it; break; }
                if (rnorm < abs_tol) { code = kKrylovConverged; ++it; break; }
                if (!(cabs2(omega) > 1e-60)) { code = kKrylovBreakOmega; ++it; break; }
            }
            if (code == kKrylovRunning) code = kKrylovMaxIter;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            AcDev &d = A.info[q];
            d.code = code;
            d.iterations = it;
            d.restarts = restarts;
            d.rnorm = rnorm;
            d.bnorm = bnorm;
        }
        __syncthreads();
    }
}

using AcFn = void (*)(AcArgs);

AcFn pick_ac(double avg, bool wide) {
    if (wide) {
        if (avg <= 3.0) return ac_sweep_kernel<2, kAcWideBlock>;
        if (avg <= 12.0) return ac_sweep_kernel<4, kAcWideBlock>;
        return ac_sweep_kernel<8, kAcWideBlock>;
    }
    if (avg <= 3.0) return ac_sweep_kernel<2, kAcBlock>;
    if (avg <= 12.0) return ac_sweep_kernel<4, kAcBlock>;
    return ac_sweep_kernel<8, kAcBlock>;
}

}  // namespace

extern "C" ohm_status ohm_ac_sweep(ohm_ctx *c, int64_t n, int64_t nnz, const uint32_t *row_ptr, const uint32_t *col,
                                   const double *g_values, const double *c_values, const double *b_re_im,
                                   int64_t n_freq, const double *freqs_hz, const ohm_krylov_params *params,
                                   double *x_re_im, ohm_ac_point_info *points) {
    if (!c || !params || n_freq < 0) return ohm_fail(OHM_ERR_INVALID_ARG, "bad arguments");
    ohm_status st = ohm_check_krylov(params);
    if (st != OHM_OK) return st;
    if (params->precond == OHM_PRECOND_ISAI1)
        return ohm_fail(OHM_ERR_INVALID_ARG, "the AC sweep uses block Jacobi, Jacobi or no preconditioner");
    if (n_freq == 0 || n == 0) return OHM_OK;
    if (!b_re_im || !x_re_im || !freqs_hz || (nnz && !g_values))
        return ohm_fail(OHM_ERR_INVALID_ARG, "null array");
    st = check_csr(n, nnz, row_ptr, col);
    if (st != OHM_OK) return st;
    for (int64_t k = 0; k < n_freq; ++k)
        if (!std::isfinite(freqs_hz[k])) return ohm_fail(OHM_ERR_INVALID_ARG, "frequency %lld is not finite", (long long)k);
    CUDA_TRY(cudaSetDevice(c->device));
    // block-Jacobi pairing from the real part's structure
    std::vector<char> touched(nnz, 0);
    PcHost pc;
    build_precond(n, row_ptr, col, g_values, touched, params->precond == OHM_PRECOND_AUTO, pc);
    // frequency groups sized so the per-point workspace stays under ~4 GB
    const size_t per_point = (size_t)kAcVecs * n * sizeof(double2);
    const int64_t group = std::max<int64_t>(1, std::min<int64_t>(n_freq, ((size_t)4 << 30) / per_point));
    std::vector<void *> allocs;
    auto put = [&](auto **dst, const auto *src, size_t count) -> cudaError_t {
        cudaError_t e = dalloc(dst, count);
        if (e == cudaSuccess) allocs.push_back((void *)*dst);
        if (e == cudaSuccess && src && count)
            e = cudaMemcpyAsync(*dst, src, count * sizeof(**dst), cudaMemcpyHostToDevice, c->stream);
        return e;
    };
    AcArgs A{};
    uint32_t *d_rp = nullptr, *d_col = nullptr, *d_diag = nullptr, *d_off = nullptr;
    double *d_g = nullptr, *d_c = nullptr, *d_omega = nullptr;
    double2 *d_b = nullptr, *d_work = nullptr;
    int32_t *d_partner = nullptr;
    AcDev *d_info = nullptr;
    unsigned int *d_queue = nullptr;
    cudaError_t e = put(&d_rp, row_ptr, n + 1);
    if (e == cudaSuccess) e = put(&d_col, col, nnz);
    if (e == cudaSuccess) e = put(&d_g, g_values, nnz);
    if (e == cudaSuccess && c_values) e = put(&d_c, c_values, nnz);
    if (e == cudaSuccess) e = put(&d_b, (const double2 *)b_re_im, n);
    if (e == cudaSuccess) e = put(&d_partner, pc.partner.data(), n);
    if (e == cudaSuccess) e = put(&d_diag, pc.diag_slot.data(), n);
    if (e == cudaSuccess) e = put(&d_off, pc.off_slot.data(), n);
    if (e == cudaSuccess) e = put(&d_omega, (const double *)nullptr, group);
    if (e == cudaSuccess) e = put(&d_work, (const double2 *)nullptr, (size_t)group * kAcVecs * n);
    if (e == cudaSuccess) e = put(&d_info, (const AcDev *)nullptr, group);
    if (e == cudaSuccess) e = put(&d_queue, (const unsigned int *)nullptr, 1);
    A.n = (int)n;
    A.precond = params->precond == OHM_PRECOND_NONE ? kPcNone
              : (params->precond == OHM_PRECOND_JACOBI ? kPcJacobi : kPcAuto);
    A.max_it = params->max_iterations;
    A.max_restarts = std::max(0, params->max_restarts);
    A.tol = params->tolerance;
    A.rp = d_rp; A.col = d_col; A.g = d_g; A.c = d_c; A.b = d_b; A.omega = d_omega;
    A.partner = d_partner; A.diag_slot = d_diag; A.off_slot = d_off;
    A.work = d_work; A.info = d_info; A.queue = d_queue;
    // a point per SM at most: give each point a whole SM when the system is large
    const bool wide = n >= 2048 && n_freq <= c->num_sms;
    const int block = wide ? kAcWideBlock : kAcBlock;
    AcFn fn = pick_ac((double)nnz / (double)n, wide);
    int per_sm = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, block, 0);
    std::vector<double> omega(group);
    std::vector<AcDev> hinfo(group);
    int64_t failed = -1;
    AcDev fail_info{};
    for (int64_t f0 = 0; e == cudaSuccess && f0 < n_freq; f0 += group) {
        const int64_t m = std::min(group, n_freq - f0);
        for (int64_t k = 0; k < m; ++k) omega[k] = 2.0 * 3.14159265358979323846 * freqs_hz[f0 + k];   // ac.rs:57
        e = cudaMemcpyAsync(d_omega, omega.data(), m * sizeof(double), cudaMemcpyHostToDevice, c->stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(d_queue, 0, sizeof(unsigned int), c->stream);
        A.n_freq = (int)m;
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)std::max(per_sm, 1) * c->num_sms, m));
        if (e == cudaSuccess) {
            fn<<<grid, block, 0, c->stream>>>(A);
            e = cudaGetLastError();
        }
        // x of every point: the first of its kAcVecs vectors
        for (int64_t k = 0; e == cudaSuccess && k < m; ++k)
            e = cudaMemcpyAsync(x_re_im + 2 * (size_t)(f0 + k) * n, d_work + (size_t)k * kAcVecs * n,
                                n * sizeof(double2), cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(hinfo.data(), d_info, m * sizeof(AcDev), cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        for (int64_t k = 0; e == cudaSuccess && k < m; ++k) {
            const AcDev &d = hinfo[k];
            if (points) {
                ohm_ac_point_info &o = points[f0 + k];
                o.krylov_code = d.code;
                o.iterations = d.iterations;
                o.restarts = d.restarts;
                o.reserved = 0;
                o.residual_norm = d.rnorm;
                o.b_norm = d.bnorm;
            }
            if (d.code != kKrylovConverged && failed < 0) { failed = f0 + k; fail_info = d; }
        }
    }
    cudaStreamSynchronize(c->stream);
    for (void *q : allocs) ohm_pool_free(q);
    if (e != cudaSuccess) return ohm_fail(OHM_ERR_CUDA, "AC sweep: %s", cudaGetErrorString(e));
    if (failed >= 0)
        return ohm_fail(OHM_ERR_SOLVE, "BiCGSTAB did not converge at frequency point %lld (%.6e Hz, code %d)",
                        (long long)failed, freqs_hz[failed], fail_info.code);
    return OHM_OK;
}

// LinearSolver::solve_complex (src/solver/mod.rs:27-34, gpu.rs:210-735): one
// complex system A x = b as a one-point sweep with G = Re A, C = Im A and
// f = 1 / (2 pi), so that w = 2 pi f is exactly 1.0 and A(f) = A.
extern "C" ohm_status ohm_solve_complex(ohm_ctx *c, int64_t n, int64_t nnz, const uint32_t *row_ptr,
                                        const uint32_t *col, const double *values_re_im, const double *b_re_im,
                                        double *x_re_im, const ohm_krylov_params *params, ohm_ac_point_info *info) {
    if (!c || !params || n < 0 || nnz < 0) return ohm_fail(OHM_ERR_INVALID_ARG, "bad arguments");
    if (info) std::memset(info, 0, sizeof *info);
    if (n == 0) return OHM_OK;
    if (!row_ptr || !b_re_im || !x_re_im || (nnz && (!col || !values_re_im)))
        return ohm_fail(OHM_ERR_INVALID_ARG, "null array");
    std::vector<double> re((size_t)nnz), im((size_t)nnz);
    for (int64_t k = 0; k < nnz; ++k) {
        re[k] = values_re_im[2 * k];
        im[k] = values_re_im[2 * k + 1];
    }
    const double f = 1.0 / (2.0 * 3.14159265358979323846);
    ohm_ac_point_info pt{};
    const ohm_status st =
        ohm_ac_sweep(c, n, nnz, row_ptr, col, re.data(), im.data(), b_re_im, 1, &f, params, x_re_im, &pt);
    if (info) *info = pt;
    return st;
}
