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
#include <numeric>
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
    // Team mode (fewer points than resident blocks): block b works on point
    // blk_point[b] as member blk_member[b] of point_team[q] blocks, with a
    // per-point barrier counter and reduction partials [2][4][kAcMaxTeam].
    int team_mode;
    const int32_t *blk_point, *blk_member, *point_team;
    unsigned long long *team_count;
    double *team_part;
    int *team_error;
};

constexpr int kAcMaxTeam = 8;

// The blocks solving one frequency point.  A one-block team (TEAM false, the
// queue mode) synchronises and reduces within the block; a team of T blocks
// splits the rows evenly and meets at a bounded barrier on the point's
// arrival counter, its dot products summed from per-member partials in
// member order (identical in every member).
template <bool TEAM>
struct AcTeam {
    int T, m, r0, r1;
    unsigned long long *count;
    unsigned long long epoch;
    double *part;
    int red;
    int *error;
    double *smem;

    __device__ __forceinline__ bool sync() {
        if constexpr (!TEAM) { __syncthreads(); return true; }
        __shared__ int s_ok;
        epoch += (unsigned long long)T;
        __syncthreads();
        if (threadIdx.x == 0) {
            red_release_add_u64(count, 1ull);
            int ok = 1;
            uint32_t spins = 0;
            while (ld_acquire_u64(count) < epoch) {
                if (++spins > kBarrierSpinLimit || *(volatile int *)error != 0) {
                    atomicCAS(error, 0, kStatusTimeout);
                    ok = 0;
                    break;
                }
                if (spins > kTightSpins) __nanosleep(64);
            }
            s_ok = ok;
        }
        __syncthreads();
        return s_ok != 0;
    }
    template <int NV>
    __device__ __forceinline__ bool sum(double (&v)[NV]) {
        block_sum<NV>(v, smem);
        if constexpr (!TEAM) return true;
        double *p = part + (size_t)(red & 1) * 4 * kAcMaxTeam;
        ++red;
        if (threadIdx.x == 0)
            for (int k = 0; k < NV; ++k) p[k * kAcMaxTeam + m] = v[k];
        if (!sync()) return false;
        for (int k = 0; k < NV; ++k) {
            double x = 0.0;
            for (int j = 0; j < T; ++j) x += __ldcg(p + k * kAcMaxTeam + j);
            v[k] = x;
        }
        return true;
    }
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

// y_i = sum_k A(f)_ik x_k for rows [r0, r1), LPR lanes per row; f(i, y).
template <int LPR, typename F>
__device__ __forceinline__ void cspmv(const AcArgs &A, double w, const double2 *x, int r0, int r1, F f) {
    const int lane = threadIdx.x % LPR, group = threadIdx.x / LPR, ngroups = blockDim.x / LPR;
    for (int base = r0; base < r1; base += ngroups) {
        const int i = base + group;
        const bool ok = i < r1;
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

// One frequency point solved by team g (rows [g.r0, g.r1) of this block).
// Returns false when a team barrier gave up.
template <int LPR, bool TEAM>
__device__ bool ac_point(const AcArgs &A, int q, AcTeam<TEAM> &g) {
    const int n = A.n, r0 = g.r0, r1 = g.r1;
    {
        const double w = A.omega[q];
        double2 *W = A.work + (size_t)q * kAcVecs * n;
        double2 *x = W, *r = W + n, *rh = W + 2 * (size_t)n, *p = W + 3 * (size_t)n, *v = W + 4 * (size_t)n;
        double2 *s = W + 5 * (size_t)n, *t = W + 6 * (size_t)n, *ph = W + 7 * (size_t)n, *sh = W + 8 * (size_t)n;
        double2 *ms = W + 9 * (size_t)n, *mp = W + 10 * (size_t)n;

        // preconditioner coefficients for this frequency, and the start vectors
        double acc0[1] = {0.0};
        for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
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
        if (!g.sum<1>(acc0)) return false;
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
            auto restart = [&]() -> bool {
                for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
                    rh[i] = r[i];
                    p[i] = make_double2(0.0, 0.0);
                    v[i] = make_double2(0.0, 0.0);
                }
                if (!g.sync()) return false;
                rho = make_double2(1.0, 0.0);
                alpha = rho;
                omega = rho;
                rho_new = make_double2(rr, 0.0);
                rh2 = rr;
                ++restarts;
                return true;
            };
            for (; it < A.max_it; ++it) {
                if (!(sqrt(cabs2(rho_new)) >= kBreakdownRel * sqrt(rh2 * rr))) {
                    if (restarts < A.max_restarts && rr > 0.0) { if (!restart()) return false; }
                    else { code = kKrylovBreakRho; break; }
                }
                const double2 beta = cmul(cdiv(rho_new, rho), cdiv(alpha, omega));
                rho = rho_new;
                for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x)
                    p[i] = cadd(cmul(csub(p[i], cmul(omega, v[i])), beta), r[i]);
                if (!g.sync()) return false;
                for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
                    double2 z = cmul(ms[i], p[i]);
                    const int pi = A.partner[i];
                    if (pi >= 0) z = cadd(z, cmul(mp[i], p[pi]));
                    ph[i] = z;
                }
                if (!g.sync()) return false;
                double a1[4] = {0.0, 0.0, 0.0, 0.0};     // r_hat^H v, ||v||^2
                cspmv<LPR>(A, w, ph, r0, r1, [&](int i, double2 y) {
                    v[i] = y;
                    const double2 d = cdotc(rh[i], y);
                    a1[0] += d.x;
                    a1[1] += d.y;
                    a1[2] += cabs2(y);
                });
                if (!g.sum<4>(a1)) return false;
                const double2 rhv = make_double2(a1[0], a1[1]);
                if (!(sqrt(cabs2(rhv)) >= kBreakdownRel * sqrt(rh2 * a1[2]))) {
                    if (restarts < A.max_restarts && rr > 0.0) {
                        if (!restart()) return false;
                        continue;
                    }
                    code = kKrylovBreakRv;
                    break;
                }
                alpha = cdiv(rho, rhv);
                double a2[1] = {0.0};
                for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
                    const double2 si = csub(r[i], cmul(alpha, v[i]));
                    s[i] = si;
                    a2[0] += cabs2(si);
                }
                if (!g.sum<1>(a2)) return false;
                if (sqrt(a2[0]) < abs_tol) {                     // gpu.rs:646-650
                    for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) x[i] = cadd(x[i], cmul(alpha, ph[i]));
                    rnorm = sqrt(a2[0]);
                    code = kKrylovConverged;
                    ++it;
                    break;
                }
                for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
                    double2 z = cmul(ms[i], s[i]);
                    const int pi = A.partner[i];
                    if (pi >= 0) z = cadd(z, cmul(mp[i], s[pi]));
                    sh[i] = z;
                }
                if (!g.sync()) return false;
                double a3[3] = {0.0, 0.0, 0.0};          // t^H s, t^H t
                cspmv<LPR>(A, w, sh, r0, r1, [&](int i, double2 y) {
                    t[i] = y;
                    const double2 d = cdotc(y, s[i]);
                    a3[0] += d.x;
                    a3[1] += d.y;
                    a3[2] += cabs2(y);
                });
                if (!g.sum<3>(a3)) return false;
                if (!(a3[2] > 0.0)) { code = kKrylovBreakTt; break; }
                omega = cdiv(make_double2(a3[0], a3[1]), make_double2(a3[2], 0.0));
                double a4[3] = {0.0, 0.0, 0.0};          // r_hat^H r, ||r||^2
                for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
                    x[i] = cadd(cadd(x[i], cmul(alpha, ph[i])), cmul(omega, sh[i]));
                    const double2 ri = csub(s[i], cmul(omega, t[i]));
                    r[i] = ri;
                    const double2 d = cdotc(rh[i], ri);
                    a4[0] += d.x;
                    a4[1] += d.y;
                    a4[2] += cabs2(ri);
                }
                if (!g.sum<3>(a4)) return false;
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
        if (g.m == 0 && threadIdx.x == 0) {
            AcDev &d = A.info[q];
            d.code = code;
            d.iterations = it;
            d.restarts = restarts;
            d.rnorm = rnorm;
            d.bnorm = bnorm;
        }
        __syncthreads();
    }
    return true;
}

// Team mode (cooperative launch, fewer points than resident blocks): block
// b solves point blk_point[b] with the other members of its team.
template <int LPR>
__global__ void __launch_bounds__(kAcWideBlock) ac_team_kernel(AcArgs A) {
    __shared__ double smem[32 * 4];
    AcTeam<true> g;
    g.smem = smem;
    g.epoch = 0;
    g.red = 0;
    const int q = A.blk_point[blockIdx.x];
    g.T = A.point_team[q];
    g.m = A.blk_member[blockIdx.x];
    g.r0 = (int)(((long long)A.n * g.m) / g.T);
    g.r1 = (int)(((long long)A.n * (g.m + 1)) / g.T);
    g.count = A.team_count + q;
    g.part = A.team_part + (size_t)q * 8 * kAcMaxTeam;
    g.error = A.team_error;
    ac_point<LPR, true>(A, q, g);
}

// Queue mode: each block takes points from the queue and solves each alone.
template <int LPR, int BLOCK>
__global__ void __launch_bounds__(BLOCK) ac_sweep_kernel(AcArgs A) {
    __shared__ double smem[32 * 4];
    __shared__ int s_q;
    AcTeam<false> g;
    g.smem = smem;
    g.epoch = 0;
    g.red = 0;
    g.T = 1;
    g.m = 0;
    g.r0 = 0;
    g.r1 = A.n;
    g.count = nullptr;
    g.part = nullptr;
    g.error = nullptr;
    for (;;) {
        if (threadIdx.x == 0) s_q = (int)atomicAdd(A.queue, 1u);
        __syncthreads();
        const int q = s_q;
        __syncthreads();
        if (q >= A.n_freq) return;
        ac_point<LPR, false>(A, q, g);
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

AcFn pick_ac_team(double avg) {
    if (avg <= 3.0) return ac_team_kernel<2>;
    if (avg <= 12.0) return ac_team_kernel<4>;
    return ac_team_kernel<8>;
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
    // Team mode: with fewer points than resident blocks, the spare blocks
    // join the lowest-frequency points (the slowest: the conductances
    // dominate) as teams of up to kAcMaxTeam blocks of >= 1024 rows each.
    const int total_blocks = std::max(per_sm, 1) * c->num_sms;
    const int tmax = (int)std::min<int64_t>(kAcMaxTeam, std::max<int64_t>(1, n / 1024));
    const AcFn fn_team = pick_ac_team((double)nnz / (double)n);
    int team_per_sm = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&team_per_sm, fn_team, kAcWideBlock, 0);
    // the team kernel must be co-resident: no more teamed blocks than it can hold
    const bool team_capable = wide && tmax >= 2 && group < total_blocks && team_per_sm * c->num_sms >= total_blocks;
    int32_t *d_blk_point = nullptr, *d_blk_member = nullptr, *d_point_team = nullptr;
    unsigned long long *d_team_count = nullptr;
    double *d_team_part = nullptr;
    int *d_team_error = nullptr;
    std::vector<int32_t> h_blk_point, h_blk_member, h_point_team;
    if (team_capable) {
        if (e == cudaSuccess) e = put(&d_blk_point, (const int32_t *)nullptr, total_blocks);
        if (e == cudaSuccess) e = put(&d_blk_member, (const int32_t *)nullptr, total_blocks);
        if (e == cudaSuccess) e = put(&d_point_team, (const int32_t *)nullptr, group);
        if (e == cudaSuccess) e = put(&d_team_count, (const unsigned long long *)nullptr, group);
        if (e == cudaSuccess) e = put(&d_team_part, (const double *)nullptr, (size_t)group * 8 * kAcMaxTeam);
        if (e == cudaSuccess) e = put(&d_team_error, (const int *)nullptr, 1);
        A.blk_point = d_blk_point; A.blk_member = d_blk_member; A.point_team = d_point_team;
        A.team_count = d_team_count; A.team_part = d_team_part; A.team_error = d_team_error;
    }
    int team_err_host = 0;
    for (int64_t f0 = 0; e == cudaSuccess && f0 < n_freq; f0 += group) {
        const int64_t m = std::min(group, n_freq - f0);
        for (int64_t k = 0; k < m; ++k) omega[k] = 2.0 * 3.14159265358979323846 * freqs_hz[f0 + k];   // ac.rs:57
        e = cudaMemcpyAsync(d_omega, omega.data(), m * sizeof(double), cudaMemcpyHostToDevice, c->stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(d_queue, 0, sizeof(unsigned int), c->stream);
        A.n_freq = (int)m;
        // team sizes: the same base size for every point, one more block for
        // the lowest frequencies while blocks are left
        int teamed = 0;
        if (team_capable && m < total_blocks) {
            const int base = std::min<int>(tmax, (int)(total_blocks / m));
            int spare = base < tmax ? total_blocks - base * (int)m : 0;
            std::vector<int32_t> by_freq((size_t)m);
            std::iota(by_freq.begin(), by_freq.end(), 0);
            std::stable_sort(by_freq.begin(), by_freq.end(), [&](int32_t x, int32_t y) { return omega[x] < omega[y]; });
            h_point_team.assign((size_t)m, base);
            for (int32_t q : by_freq) {
                if (spare == 0) break;
                ++h_point_team[q];
                --spare;
            }
            h_blk_point.clear();
            h_blk_member.clear();
            for (int64_t q = 0; q < m; ++q)
                for (int j = 0; j < h_point_team[q]; ++j) {
                    h_blk_point.push_back((int32_t)q);
                    h_blk_member.push_back(j);
                }
            if (base > 1 || h_point_team[by_freq[0]] > 1) teamed = (int)h_blk_point.size();
        }
        if (teamed > 0) {
            A.team_mode = 1;
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(d_blk_point, h_blk_point.data(), teamed * sizeof(int32_t), cudaMemcpyHostToDevice,
                                    c->stream);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(d_blk_member, h_blk_member.data(), teamed * sizeof(int32_t),
                                    cudaMemcpyHostToDevice, c->stream);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(d_point_team, h_point_team.data(), m * sizeof(int32_t), cudaMemcpyHostToDevice,
                                    c->stream);
            if (e == cudaSuccess) e = cudaMemsetAsync(d_team_count, 0, m * sizeof(unsigned long long), c->stream);
            if (e == cudaSuccess) e = cudaMemsetAsync(d_team_error, 0, sizeof(int), c->stream);
            void *args[] = {&A};
            if (e == cudaSuccess)
                e = cudaLaunchCooperativeKernel((void *)fn_team, dim3(teamed), dim3(kAcWideBlock), args, 0, c->stream);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(&team_err_host, d_team_error, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
        } else {
            A.team_mode = 0;
            const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)total_blocks, m));
            if (e == cudaSuccess) {
                fn<<<grid, block, 0, c->stream>>>(A);
                e = cudaGetLastError();
            }
        }
        // x of every point: the first of its kAcVecs vectors
        for (int64_t k = 0; e == cudaSuccess && k < m; ++k)
            e = cudaMemcpyAsync(x_re_im + 2 * (size_t)(f0 + k) * n, d_work + (size_t)k * kAcVecs * n,
                                n * sizeof(double2), cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(hinfo.data(), d_info, m * sizeof(AcDev), cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e == cudaSuccess && team_err_host != 0) break;
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
    if (team_err_host != 0) return ohm_fail(OHM_ERR_TIMEOUT, "AC sweep: a team barrier wait gave up");
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
