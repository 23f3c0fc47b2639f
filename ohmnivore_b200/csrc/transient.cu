// Fixed-step backward-Euler transient with a Newton solve per step.
//
// One persistent cooperative kernel runs a chunk of steps; per step the grid
//   1. forms the BE right-hand side b_n = b(t_n) + (C/h) x_{n-1}
//      (transient.rs:326-333) with the sources evaluated on the device
//      (transient_source.rs:8-118), C in its own compact CSR,
//   2. runs the Newton loop (newton_run) on the companion system whose base
//      values A = G + C/h were formed once for the run (transient.rs:285-323),
//      starting from x_{n-1},
//   3. records the probe rows of x_n.
// The host launches ceil(n_steps / steps_per_launch) chunks, optionally
// recorded once as a CUDA graph and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "host_util.h"

using namespace ohm;

namespace {

// Device-side run record, accumulated by the grid leader.
struct TranDev {
    int status, steps_done, failed_step, kcode;
    long long newton_its, krylov_its;
    int fallbacks, pad;
    double max_residual;
};

struct TranArgs {
    int s0, s1;                        // steps [s0, s1) of this launch
    double t0, h;
    const uint32_t *c_rp, *c_col;
    const double *c_val;
    const int32_t *src_of_row;         // per row: index into srow_ptr, -1 none
    const uint32_t *srow_ptr, *srow_src;
    const double *srow_sign;
    const ohm_source *src;
    const double *pwl;
    const uint32_t *probe;
    int n_probes;
    double *wave;                      // n_steps x n_probes
    double *beff;                      // base rhs of the current step
    TranDev *st;
    double *states;                    // optional: x after step s at (s - state_base) * n
    int state_base;
    // Newton start of step s > 0: x_{n-1} (predict 0), the linear
    // extrapolation 2 x_{n-1} - x_{n-2} (predict 1; xpp holds x_{n-2}) or,
    // from step 2 on, the quadratic 3 x_{n-1} - 3 x_{n-2} + x_{n-3}
    // (predict 2; xppp holds x_{n-3})
    int predict;
    double *xpp, *xppp;
};

// Source waveforms, the formulas of transient_source.rs:39-118.
__device__ double source_value(const ohm_source &s, double t, const double *pwl) {
    const double *p = s.p;
    switch (s.kind) {
        case OHM_TRAN_PULSE: {
            const double v1 = p[0], v2 = p[1], td = p[2], tr = p[3], tf = p[4], pw = p[5], per = p[6];
            if (t < td) return v1;
            const double trel = (per > 0.0 && per < 1.7976931348623157e308) ? fmod(t - td, per) : t - td;
            if (trel < tr) return tr > 0.0 ? v1 + (v2 - v1) * trel / tr : v2;
            if (trel < tr + pw) return v2;
            if (trel < tr + pw + tf) return tf > 0.0 ? v2 + (v1 - v2) * (trel - tr - pw) / tf : v1;
            return v1;
        }
        case OHM_TRAN_SIN: {
            const double vo = p[0], va = p[1], freq = p[2], td = p[3], theta = p[4];
            if (t < td) return vo;
            const double dt = t - td;
            const double env = theta != 0.0 ? exp(-dt * theta) : 1.0;
            return vo + va * sin(2.0 * 3.14159265358979323846 * freq * dt) * env;
        }
        case OHM_TRAN_PWL: {
            const double *q = pwl + 2 * (size_t)s.pwl_offset;
            const int m = s.pwl_count;
            if (m <= 0) return 0.0;
            if (t <= q[0]) return q[1];
            if (t >= q[2 * (m - 1)]) return q[2 * (m - 1) + 1];
            for (int i = 1; i < m; ++i) {
                if (t <= q[2 * i]) {
                    const double t0 = q[2 * (i - 1)], v0 = q[2 * (i - 1) + 1], t1 = q[2 * i], v1 = q[2 * i + 1];
                    return v0 + (v1 - v0) * ((t - t0) / (t1 - t0));
                }
            }
            return q[2 * (m - 1) + 1];
        }
        case OHM_TRAN_EXP: {
            const double v1 = p[0], v2 = p[1], td1 = p[2], tau1 = p[3], td2 = p[4], tau2 = p[5];
            if (t < td1) return v1;
            const double rise = (v2 - v1) * (1.0 - exp(-(t - td1) / tau1));
            if (t < td2) return v1 + rise;
            const double fall = (v1 - v2) * (1.0 - exp(-(t - td2) / tau2));
            return v1 + rise + fall;
        }
        default:
            return s.dc;
    }
}

template <int LPR>
__global__ void __launch_bounds__(kSolverBlock, 1) transient_kernel(KernelArgs a, TranArgs T) {
    __shared__ double smem[32 * 4 + 4];   // GridTeam reductions: warp values + results
    GridTeam g;
    g.G = gridDim.x;
    g.bid = blockIdx.x;
    g.r0 = (int)(((long long)a.n * g.bid) / g.G);
    g.r1 = (int)(((long long)a.n * (g.bid + 1)) / g.G);
    g.gtid = g.bid * blockDim.x + threadIdx.x;
    g.gstride = g.G * blockDim.x;
    g.smem = smem;
    g.partials = a.partials;
    g.red = 0;
    g.epoch = 0;
    g.gs = a.gs;
    if (T.st->status != 0) return;     // an earlier chunk failed (uniform: written before this launch)
    const double inv_h = 1.0 / T.h;
    for (int s = T.s0; s < T.s1; ++s) {
        const double tn = T.t0 + (double)(s + 1) * T.h;
        // ---- b_n = b(t_n) + (C/h) x_{n-1} for the rows of this block ----
        for (int i = g.r0 + threadIdx.x; i < g.r1; i += blockDim.x) {
            double bs = 0.0;
            const int q = T.src_of_row[i];
            if (q >= 0)
                for (uint32_t e = T.srow_ptr[q]; e < T.srow_ptr[q + 1]; ++e)
                    bs += T.srow_sign[e] * source_value(T.src[T.srow_src[e]], tn, T.pwl);
            double cx = 0.0;
            for (uint32_t k = T.c_rp[i]; k < T.c_rp[i + 1]; ++k) cx += T.c_val[k] * a.x[T.c_col[k]];
            const double bb = bs + cx * inv_h;
            T.beff[i] = bb;
            a.b[i] = bb;
        }
        if (!g.sync()) return;
        if (T.predict) {
            // after every block's (C/h) x_{n-1}: own rows start from the
            // extrapolation (x_{n-2} is known from step 1 of the run on)
            for (int i = g.r0 + threadIdx.x; i < g.r1; i += blockDim.x) {
                const double xp = a.x[i];
                if (T.predict == 2 && s > 1) a.x[i] = 3.0 * (xp - T.xpp[i]) + T.xppp[i];
                else if (s > 0) a.x[i] = 2.0 * xp - T.xpp[i];
                if (T.predict == 2) T.xppp[i] = T.xpp[i];
                T.xpp[i] = xp;
            }
            if (!g.sync()) return;
        }
        // ---- Newton on the companion system, from x_{n-1} ----
        RunOut o;
        RunCfg c{0.0, 1.0, 0.0, a.max_outer, a.max_krylov, false};
        if (!newton_run<LPR>(a, g, c, o)) return;
        if (g.leader()) {
            TranDev &d = *T.st;
            d.newton_its += o.outer_done;
            d.krylov_its += o.kiters;
            d.fallbacks += o.fallbacks;
            d.kcode = o.kcode;
            if (o.status == kOk) {
                d.steps_done = s + 1;
            } else {
                d.status = o.status;
                d.failed_step = s;
                d.max_residual = o.last_dmax;
            }
        }
        if (o.status != kOk) return;
        for (int k = g.gtid; k < T.n_probes; k += g.gstride)
            T.wave[(size_t)s * T.n_probes + k] = a.x[T.probe[k]];
        if (T.states) {
            double *st = T.states + (size_t)(s - T.state_base) * a.n;
            for (int i = g.r0 + threadIdx.x; i < g.r1; i += blockDim.x) st[i] = a.x[i];
        }
    }
}

// Adaptive BE / TRAP step control of the reference (transient.rs:77-178):
// the first step and the step after a rejection are BE; every other step
// solves TRAP and BE from x_{n-1}, estimates LTE = (2/3) max|x_trap - x_be|
// (compute_lte, :355-362), rejects it when LTE > 1e-3 (h *= clamp(0.9
// sqrt(tol / LTE), 0.5, 2), at least h_min) and otherwise accepts x_trap and
// takes h = clamp(h * that factor, h_min, h_max); h_min = tstep / 10^4,
// h_max = tstep.  Companion matrices A = G + (alpha / h) C (:285-323) are
// formed on the device for every solve.  TRAP's rhs is
// b(t_n) + (2/h) C x_{n-1} - f(x_{n-1}) + b(t_{n-1}) (:336-352) with
// f(x) = G x + i(x): the reference's G x_{n-1} plus, for nonlinear devices,
// their currents, taken as J(x) x - b of the system stamped at x on the base
// (G, 0), so TRAP integrates the same device equations Newton solves.
constexpr int kAdTimestep = 20;   // consecutive rejections at h_min (OhmnivoreError::Timestep)

struct AdaptDev {
    int status, accepted, rejected, points;
    long long newton_its, krylov_its;
    int solves, fallbacks, kcode, failed_kind;
    double t, h, t_fail, max_residual;
};

struct AdaptArgs {
    double tstep, tstop, tstart;
    int max_points;
    long long nnz;
    const double *g_vals;      // G, the plan's base values
    const double *cg;          // C on G's pattern (0 off C)
    const double *zeros;       // n zeros: the rhs base of the f(x) evaluation
    double *aval;              // companion base values of the current solve
    double *xs, *xt, *fdev;    // x_{n-1}, x_trap, f(x_{n-1})
    double *times;             // output times (max_points)
    AdaptDev *st;
};

template <int LPR>
__global__ void __launch_bounds__(kSolverBlock, 1) adaptive_kernel(KernelArgs a, TranArgs T, AdaptArgs P) {
    __shared__ double smem[32 * 4 + 4];   // GridTeam reductions: warp values + results
    GridTeam g;
    g.G = gridDim.x;
    g.bid = blockIdx.x;
    g.r0 = (int)(((long long)a.n * g.bid) / g.G);
    g.r1 = (int)(((long long)a.n * (g.bid + 1)) / g.G);
    g.gtid = g.bid * blockDim.x + threadIdx.x;
    g.gstride = g.G * blockDim.x;
    g.smem = smem;
    g.partials = a.partials;
    g.red = 0;
    g.epoch = 0;
    g.gs = a.gs;
    const int r0 = g.r0, r1 = g.r1;
    const double h_min = P.tstep / 10000.0, h_max = P.tstep, lte_tol = 1e-3;
    constexpr int kMaxFailures = 10;
    // every thread holds the same control state: it changes only through
    // grid-wide results (Newton status, the all-reduced LTE)
    double t = 0.0, h = fmin(P.tstep, h_max), t_next = 0.0, h_next = 0.0;
    bool use_be = true;
    int stage = 0;               // 0: new step, 1: its TRAP solve, 2: its BE solve
    int fails = 0, points = 0, accepted = 0, rejected = 0, solves = 0, fallbacks = 0, kcode = 0;
    int status = kOk, failed_kind = 0;
    long long nits = 0, kits = 0;
    double t_fail = 0.0, max_res = 0.0;

    // output row `points` (kept only below max_points; the count continues)
    auto record = [&](double tr) {
        if (points < P.max_points) {
            for (int k = g.gtid; k < T.n_probes; k += g.gstride)
                T.wave[(size_t)points * T.n_probes + k] = a.x[T.probe[k]];
            if (g.leader()) P.times[points] = tr;
        }
        ++points;
    };
    if (P.tstart <= 0.0) record(0.0);
    while (true) {
        if (stage == 0) {
            if (!(t < P.tstop)) break;
            if (t + h > P.tstop) h = P.tstop - t;
            if (h < h_min * 0.5) break;
            t_next = t + h;
            for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) P.xs[i] = a.x[i];
            if (!use_be) {
                // f(x_{n-1}) = J x - b of the system stamped at x on (G, 0)
                for (long long k = g.gtid; k < P.nnz; k += g.gstride) {
                    a.vals64[k] = P.g_vals[k];
                    if (a.vals32) a.vals32[k] = (float)P.g_vals[k];
                }
                for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) a.b[i] = 0.0;
                if (!g.sync()) return;
                const RunCfg c0{0.0, 1.0, 0.0, 0, 0, false};
                if (!assemble(a, g, c0, P.g_vals, P.zeros)) return;
                const double *xv = a.x;
                auto x_at = [&](int j, bool) -> double { return xv[j]; };
                auto f_row = [&](int i, double ax) { P.fdev[i] = ax - a.b[i]; };
                spmv_rows<LPR, double>(a.row_ptr, a.col, a.vals64, (const uint8_t *)nullptr, r0, r1, x_at, f_row,
                                       a.longflag);
                if (!spmv_long<double>(a, g, a.col, a.vals64, (const uint8_t *)nullptr, x_at, f_row)) return;
                if (!g.sync()) return;
            }
            stage = use_be ? 2 : 1;
        }
        // companion base A = G + (alpha / h) C and the step's rhs
        const double fac = (stage == 1 ? 2.0 : 1.0) / h;
        for (long long k = g.gtid; k < P.nnz; k += g.gstride) {
            const double v = P.g_vals[k] + fac * P.cg[k];
            P.aval[k] = v;
            a.vals64[k] = v;
            if (a.vals32) a.vals32[k] = (float)v;
        }
        for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
            double bn = 0.0, bp = 0.0;
            const int q = T.src_of_row[i];
            if (q >= 0)
                for (uint32_t e = T.srow_ptr[q]; e < T.srow_ptr[q + 1]; ++e) {
                    const ohm_source &src = T.src[T.srow_src[e]];
                    bn += T.srow_sign[e] * source_value(src, t_next, T.pwl);
                    if (stage == 1) bp += T.srow_sign[e] * source_value(src, t, T.pwl);
                }
            double cx = 0.0;
            for (uint32_t k = T.c_rp[i]; k < T.c_rp[i + 1]; ++k) cx += T.c_val[k] * a.x[T.c_col[k]];
            const double bb = stage == 1 ? ((bn + fac * cx) - P.fdev[i]) + bp : bn + fac * cx;
            T.beff[i] = bb;
            a.b[i] = bb;
        }
        if (!g.sync()) return;
        RunOut o;
        const RunCfg c{0.0, 1.0, 0.0, a.max_outer, a.max_krylov, false};
        if (!newton_run<LPR>(a, g, c, o)) return;
        nits += o.outer_done;
        kits += o.kiters;
        fallbacks += o.fallbacks;
        kcode = o.kcode;
        ++solves;
        if (o.status != kOk) {
            status = o.status;
            failed_kind = stage;
            t_fail = t_next;
            max_res = o.last_dmax;
            break;
        }
        if (stage == 1) {            // keep x_trap, solve BE from x_{n-1}
            for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
                P.xt[i] = a.x[i];
                a.x[i] = P.xs[i];
            }
            if (!g.sync()) return;
            stage = 2;
            continue;
        }
        stage = 0;
        if (!use_be) {
            double mx[1] = {0.0};
            for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) mx[0] = fmax(mx[0], fabs(P.xt[i] - a.x[i]));
            if (!g.template allmax<1>(mx)) return;
            const double lte = (2.0 / 3.0) * mx[0];
            const double factor = fmin(fmax(0.9 * sqrt(lte_tol / lte), 0.5), 2.0);
            if (lte > lte_tol) {     // reject: smaller h, BE from x_{n-1}
                h = fmax(h * factor, h_min);
                ++fails;
                if (fails >= kMaxFailures && h <= h_min * 1.01) {
                    status = kAdTimestep;
                    t_fail = t;
                    break;
                }
                ++rejected;
                use_be = true;
                for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) a.x[i] = P.xs[i];
                if (!g.sync()) return;
                continue;
            }
            h_next = fmin(fmax(h * factor, h_min), h_max);
            for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) a.x[i] = P.xt[i];
            if (!g.sync()) return;
        } else {
            use_be = false;
            h_next = h;
        }
        fails = 0;
        ++accepted;
        t = t_next;
        h = h_next;
        if (t >= P.tstart) record(t);
    }
    if (g.leader()) {
        AdaptDev &d = *P.st;
        d.status = status;
        d.accepted = accepted;
        d.rejected = rejected;
        d.points = points;
        d.newton_its = nits;
        d.krylov_its = kits;
        d.solves = solves;
        d.fallbacks = fallbacks;
        d.kcode = kcode;
        d.failed_kind = failed_kind;
        d.t = t;
        d.h = h;
        d.t_fail = t_fail;
        d.max_residual = max_res;
    }
}

using AdaptFn = void (*)(KernelArgs, TranArgs, AdaptArgs);

AdaptFn pick_adaptive(int lpr) {
    switch (lpr) {
        case 1: return adaptive_kernel<1>;
        case 2: return adaptive_kernel<2>;
        case 4: return adaptive_kernel<4>;
        default: return adaptive_kernel<8>;
    }
}

using TranFn = void (*)(KernelArgs, TranArgs);

TranFn pick_tran(int lpr) {
    switch (lpr) {
        case 1: return transient_kernel<1>;
        case 2: return transient_kernel<2>;
        case 4: return transient_kernel<4>;
        default: return transient_kernel<8>;
    }
}

// A = G + C/h on the plan's pattern, copied to the assembled arrays.
__global__ void companion_kernel(const double *G, double *A, double *vals64, float *vals32, int64_t nnz,
                                 const uint32_t *c_slot, const double *c_val, int64_t c_nnz, double inv_h,
                                 int phase) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (phase == 0) {
        for (int64_t k = i0; k < nnz; k += stride) A[k] = G[k];
    } else if (phase == 1) {
        for (int64_t k = i0; k < c_nnz; k += stride) A[c_slot[k]] += c_val[k] * inv_h;   // C slots are distinct
    } else {
        for (int64_t k = i0; k < nnz; k += stride) {
            vals64[k] = A[k];
            if (vals32) vals32[k] = (float)A[k];
        }
    }
}

__global__ void restore_kernel(const double *G, double *vals64, float *vals32, int64_t nnz) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += stride) {
        vals64[k] = G[k];
        if (vals32) vals32[k] = (float)G[k];
    }
}

int steps_grid(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 4096)); }

int tran_lpr(int64_t n, int64_t nnz) {
    const double avg = n > 0 ? (double)nnz / (double)n : 1.0;
    return avg <= 5.5 ? 1 : (avg <= 12.0 ? 4 : 8);
}

}  // namespace

struct ohm_transient {
    ohm_plan *plan = nullptr;
    ohm_ctx *ctx = nullptr;
    int64_t n = 0, c_nnz = 0, nnz = 0;
    int n_probes = 0;
    std::vector<void *> allocs;
    uint32_t *c_rp = nullptr, *c_col = nullptr, *c_slot = nullptr;
    double *c_val = nullptr, *aval = nullptr, *beff = nullptr, *pwl = nullptr;
    int32_t *src_of_row = nullptr;
    uint32_t *srow_ptr = nullptr, *srow_src = nullptr, *probe = nullptr;
    double *srow_sign = nullptr;
    ohm_source *src = nullptr;
    TranDev *st = nullptr;
    double *wave = nullptr;
    int64_t wave_cap = 0;
    // adaptive runs
    double *cg = nullptr;                       // C on G's pattern (nnz)
    double *ad_xs = nullptr, *ad_xt = nullptr, *ad_fdev = nullptr, *ad_zeros = nullptr;
    AdaptDev *ad_st = nullptr;
    double *times = nullptr;
    int64_t times_cap = 0;
    int predict = 0;                            // ohm_transient_set_predictor
    double *xpp = nullptr;                      // x_{n-2} for the predictor
    double *xppp = nullptr;                     // x_{n-3} (quadratic predictor)

    template <typename T>
    cudaError_t put(T **dst, const T *h, size_t count) {
        cudaError_t e = dalloc(dst, count);
        if (e == cudaSuccess) allocs.push_back((void *)*dst);
        if (e == cudaSuccess && h && count)
            e = cudaMemcpyAsync(*dst, h, count * sizeof(T), cudaMemcpyHostToDevice, ctx->stream);
        return e;
    }
};

extern "C" ohm_status ohm_transient_create(ohm_plan *plan, int64_t c_nnz, const uint32_t *c_row_ptr,
                                           const uint32_t *c_col, const double *c_values, const ohm_source *sources,
                                           int32_t n_sources, const double *pwl_points, int32_t n_pwl_points,
                                           const uint32_t *probe_rows, int32_t n_probes, ohm_transient **out) {
    if (!plan || !out || !c_row_ptr || c_nnz < 0 || n_sources < 0 || n_probes < 0 || n_pwl_points < 0)
        return ohm_fail(OHM_ERR_INVALID_ARG, "bad transient arguments");
    *out = nullptr;
    if ((c_nnz && (!c_col || !c_values)) || (n_sources && !sources) || (n_probes && !probe_rows) ||
        (n_pwl_points && !pwl_points))
        return ohm_fail(OHM_ERR_INVALID_ARG, "null array");
    ohm_ctx *c = ohm_plan_context(plan);
    ohm_newton_params np;
    ohm_newton_params_default(&np);
    KernelArgs a;
    int64_t nnz = 0;
    ohm_status st = ohm_plan_kernel_args(plan, &np, nullptr, a, &nnz);
    if (st != OHM_OK) return st;
    const int64_t n = a.n;
    st = check_csr(n, c_nnz, c_row_ptr, c_col);
    if (st != OHM_OK) return ohm_fail(st, "capacitance matrix: %s", ohm_last_error());
    // host copy of the plan pattern to locate each C entry's slot
    std::vector<uint32_t> rp(n + 1), col(nnz);
    CUDA_TRY(cudaMemcpy(rp.data(), a.row_ptr, (n + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if (nnz) CUDA_TRY(cudaMemcpy(col.data(), a.col, nnz * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    std::vector<uint32_t> slot(c_nnz);
    for (int64_t i = 0; i < n; ++i) {
        for (uint32_t k = c_row_ptr[i]; k < c_row_ptr[i + 1]; ++k) {
            const auto b = col.begin() + rp[i], e = col.begin() + rp[i + 1];
            const auto it = std::lower_bound(b, e, c_col[k]);
            if (it == e || *it != c_col[k])
                return ohm_fail(OHM_ERR_COMPILE, "capacitance entry (%lld, %u) is not on the conductance pattern",
                                (long long)i, c_col[k]);
            slot[k] = (uint32_t)(it - col.begin());
        }
    }
    // sources per rhs row, in source order
    std::vector<std::vector<std::pair<uint32_t, double>>> per_row(n);
    for (int32_t k = 0; k < n_sources; ++k) {
        const ohm_source &s = sources[k];
        if (s.n_rows < 0 || s.n_rows > 2) return ohm_fail(OHM_ERR_INVALID_ARG, "source %d: n_rows must be 0-2", k);
        if (s.kind < OHM_TRAN_DC || s.kind > OHM_TRAN_EXP)
            return ohm_fail(OHM_ERR_INVALID_ARG, "source %d: unknown kind %d", k, s.kind);
        if (s.kind == OHM_TRAN_PWL && (s.pwl_offset < 0 || s.pwl_count < 0 ||
                                       (int64_t)s.pwl_offset + s.pwl_count > n_pwl_points))
            return ohm_fail(OHM_ERR_INVALID_ARG, "source %d: PWL points out of range", k);
        for (int j = 0; j < s.n_rows; ++j) {
            if ((int64_t)s.rows[j] >= n) return ohm_fail(OHM_ERR_INVALID_ARG, "source %d: row out of range", k);
            per_row[s.rows[j]].push_back({(uint32_t)k, s.sign[j]});
        }
    }
    std::vector<int32_t> src_of_row(n, -1);
    std::vector<uint32_t> srow_ptr(1, 0), srow_src;
    std::vector<double> srow_sign;
    for (int64_t i = 0; i < n; ++i) {
        if (per_row[i].empty()) continue;
        src_of_row[i] = (int32_t)(srow_ptr.size() - 1);
        for (auto &pr : per_row[i]) { srow_src.push_back(pr.first); srow_sign.push_back(pr.second); }
        srow_ptr.push_back((uint32_t)srow_src.size());
    }
    for (int32_t k = 0; k < n_probes; ++k)
        if ((int64_t)probe_rows[k] >= n) return ohm_fail(OHM_ERR_INVALID_ARG, "probe %d out of range", k);

    ohm_transient *t = new ohm_transient();
    t->plan = plan; t->ctx = c; t->n = n; t->c_nnz = c_nnz; t->nnz = nnz; t->n_probes = n_probes;
    cudaError_t e = t->put(&t->c_rp, c_row_ptr, n + 1);
    if (e == cudaSuccess) e = t->put(&t->c_col, c_col, c_nnz);
    if (e == cudaSuccess) e = t->put(&t->c_val, c_values, c_nnz);
    if (e == cudaSuccess) e = t->put(&t->c_slot, slot.data(), c_nnz);
    if (e == cudaSuccess) {
        std::vector<double> cg(nnz, 0.0);
        for (int64_t k = 0; k < c_nnz; ++k) cg[slot[k]] = c_values[k];
        e = t->put(&t->cg, cg.data(), nnz);
    }
    if (e == cudaSuccess) e = t->put(&t->aval, (const double *)nullptr, nnz);
    if (e == cudaSuccess) e = t->put(&t->beff, (const double *)nullptr, n);
    if (e == cudaSuccess) e = t->put(&t->pwl, pwl_points, 2 * (size_t)n_pwl_points);
    if (e == cudaSuccess) e = t->put(&t->src_of_row, src_of_row.data(), n);
    if (e == cudaSuccess) e = t->put(&t->srow_ptr, srow_ptr.data(), srow_ptr.size());
    if (e == cudaSuccess) e = t->put(&t->srow_src, srow_src.data(), srow_src.size());
    if (e == cudaSuccess) e = t->put(&t->srow_sign, srow_sign.data(), srow_sign.size());
    if (e == cudaSuccess) e = t->put(&t->src, sources, n_sources);
    if (e == cudaSuccess) e = t->put(&t->probe, probe_rows, n_probes);
    if (e == cudaSuccess) e = t->put(&t->st, (const TranDev *)nullptr, 1);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        for (void *q : t->allocs) ohm_pool_free(q);
        delete t;
        return ohm_fail(OHM_ERR_CUDA, "transient upload: %s", cudaGetErrorString(e));
    }
    ohm_ctx_retain(c);
    *out = t;
    return OHM_OK;
}

extern "C" ohm_status ohm_transient_destroy(ohm_transient *t) {
    if (!t) return OHM_OK;
    ohm_ctx *c = t->ctx;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    for (void *q : t->allocs) ohm_pool_free(q);
    ohm_pool_free(t->wave);
    ohm_pool_free(t->times);
    delete t;
    ohm_ctx_release(c);
    return OHM_OK;
}

// Kernel arguments of a run on x_dev: the plan's system with the companion
// base values t->aval and rhs base t->beff; G receives the plan's own base.
static ohm_status tran_args(ohm_transient *t, double *x_dev, const ohm_newton_params *np, KernelArgs &a,
                            TranArgs &T, const double *&G) {
    ohm_ctx *c = t->ctx;
    int64_t nnz = 0;
    ohm_status st = ohm_plan_kernel_args(t->plan, np, x_dev, a, &nnz);
    if (st != OHM_OK) return st;
    G = a.base_vals;
    a.base_vals = t->aval;
    a.base_b = t->beff;
    a.trace = nullptr;
    a.continuation = 0;
    a.gs.count = (unsigned long long *)c->sync_words;
    a.gs.error = (int *)(c->sync_words + 2);
    a.info = c->info_dev;
    T = TranArgs{};
    T.c_rp = t->c_rp; T.c_col = t->c_col; T.c_val = t->c_val;
    T.src_of_row = t->src_of_row; T.srow_ptr = t->srow_ptr; T.srow_src = t->srow_src; T.srow_sign = t->srow_sign;
    T.src = t->src; T.pwl = t->pwl; T.probe = t->probe; T.n_probes = t->n_probes; T.wave = t->wave;
    T.beff = t->beff; T.st = t->st;
    return OHM_OK;
}

// Cooperative grid of a transient kernel: up to two blocks per SM, no more
// blocks than rows or devices need; and the dynamic shared memory of its
// Krylov slices (a.smem_bytes, 0 when they do not fit).
static ohm_status tran_grid(ohm_transient *t, const void *fn, KernelArgs &a, int &grid) {
    int per_sm = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kSolverBlock, 0));
    if (per_sm < 1) return ohm_fail(OHM_ERR_CUDA, "transient kernel does not fit on an SM");
    per_sm = std::min(per_sm, 2);
    int64_t want = (t->n + kSolverBlock - 1) / kSolverBlock;
    want = std::max<int64_t>(want, ((int64_t)a.nd + a.nq + a.nm + kSolverBlock - 1) / kSolverBlock);
    grid = (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)per_sm * t->ctx->num_sms));
    a.smem_bytes = ohm_krylov_smem_bytes(fn, t->n, t->nnz - a.nnz_long, grid);
    if (a.smem_bytes > 0) {
        int fit = 0;
        CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, fn, kSolverBlock, a.smem_bytes));
        if (fit < 1) a.smem_bytes = 0;
        else grid = (int)std::min<int64_t>(grid, (int64_t)fit * t->ctx->num_sms);
    }
    return OHM_OK;
}

// Kernel arguments of a fixed-step run on x_dev with step h: the companion
// base A = G + C/h is formed (and copied to the assembled arrays), the run
// record zeroed.  Returns the kernel and grid to launch.
static ohm_status tran_prepare(ohm_transient *t, double *x_dev, double h, const ohm_newton_params *np,
                               KernelArgs &a, TranArgs &T, TranFn &fn, int &grid, const double *&G) {
    ohm_ctx *c = t->ctx;
    ohm_status st = tran_args(t, x_dev, np, a, T, G);
    if (st != OHM_OK) return st;
    const int64_t nnz = t->nnz;
    for (int phase = 0; phase < 3; ++phase) {
        companion_kernel<<<steps_grid(phase == 1 ? t->c_nnz : nnz), 256, 0, c->stream>>>(
            G, t->aval, a.vals64, a.vals32, nnz, t->c_slot, t->c_val, t->c_nnz, 1.0 / h, phase);
        CUDA_TRY(cudaGetLastError());
    }
    CUDA_TRY(cudaMemsetAsync(t->st, 0, sizeof(TranDev), c->stream));
    T.h = h;
    fn = pick_tran(tran_lpr(t->n, nnz));
    return tran_grid(t, (const void *)fn, a, grid);
}

// One cooperative launch of steps [s0, s1).
static cudaError_t tran_launch(ohm_ctx *c, TranFn fn, int grid, const KernelArgs &a, TranArgs T, int s0, int s1) {
    T.s0 = s0;
    T.s1 = s1;
    cudaError_t e = cudaMemsetAsync(c->sync_words, 0, 4 * sizeof(unsigned int), c->stream);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kSolverBlock);
    cfg.dynamicSmemBytes = (size_t)a.smem_bytes;
    cfg.stream = c->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, fn, a, T);
}

// Status of a run from the device record and the barrier error word.
static ohm_status tran_status(ohm_transient *t, double t0, double h, TranDev &d) {
    ohm_ctx *c = t->ctx;
    unsigned int words[4] = {0, 0, 0, 0};
    CUDA_TRY(cudaMemcpyAsync(&d, t->st, sizeof d, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaMemcpyAsync(words, c->sync_words, sizeof words, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (words[2] != 0) return ohm_fail(OHM_ERR_TIMEOUT, "a device barrier wait gave up (error word %u)", words[2]);
    if (d.status != 0)
        return ohm_fail(d.status == kErrSolve ? OHM_ERR_SOLVE
                        : (d.status == kErrNewtonNumerical ? OHM_ERR_NEWTON_NUMERICAL : OHM_ERR_NEWTON_NOT_CONVERGED),
                        "transient step %d at t = %.6e failed (status %d, krylov code %d)", d.failed_step,
                        t0 + (d.failed_step + 1) * h, d.status, d.kcode);
    return OHM_OK;
}

extern "C" ohm_status ohm_transient_set_predictor(ohm_transient *t, int32_t order) {
    if (!t || order < 0 || order > 2) return ohm_fail(OHM_ERR_INVALID_ARG, "predictor order must be 0, 1 or 2");
    if (order >= 1 && !t->xpp) {
        cudaError_t e = t->put(&t->xpp, (const double *)nullptr, (size_t)t->n);
        if (e != cudaSuccess) return ohm_fail(OHM_ERR_CUDA, "predictor buffer: %s", cudaGetErrorString(e));
    }
    if (order == 2 && !t->xppp) {
        cudaError_t e = t->put(&t->xppp, (const double *)nullptr, (size_t)t->n);
        if (e != cudaSuccess) return ohm_fail(OHM_ERR_CUDA, "predictor buffer: %s", cudaGetErrorString(e));
    }
    t->predict = order;
    return OHM_OK;
}

extern "C" ohm_status ohm_transient_run(ohm_transient *t, double *x_dev, double t0, double h, int32_t n_steps,
                                        int32_t steps_per_launch, const ohm_newton_params *np, int32_t use_graph,
                                        double *waveforms_host, ohm_transient_info *info) {
    if (!t || !x_dev || !np) return ohm_fail(OHM_ERR_INVALID_ARG, "null argument");
    if (!(h > 0.0) || n_steps < 0 || steps_per_launch <= 0)
        return ohm_fail(OHM_ERR_INVALID_ARG, "need h > 0, n_steps >= 0, steps_per_launch > 0");
    if (np->continuation) return ohm_fail(OHM_ERR_INVALID_ARG, "continuation is for DC solves, not transient steps");
    if (np->krylov.precond == OHM_PRECOND_ISAI1)
        return ohm_fail(OHM_ERR_INVALID_ARG, "transient steps use block Jacobi or Jacobi");
    ohm_ctx *c = t->ctx;
    CUDA_TRY(cudaSetDevice(c->device));
    if (np->initial_guess)
        CUDA_TRY(cudaMemcpyAsync(x_dev, np->initial_guess, t->n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    const int64_t need = (int64_t)n_steps * t->n_probes;
    if (need > t->wave_cap) {
        ohm_pool_free(t->wave);
        t->wave = nullptr;
        t->wave_cap = 0;
        CUDA_TRY(dalloc(&t->wave, (size_t)need));
        t->wave_cap = need;
    }
    KernelArgs a;
    TranArgs T;
    TranFn fn = nullptr;
    int grid = 0;
    const double *G = nullptr;
    ohm_status st = tran_prepare(t, x_dev, h, np, a, T, fn, grid, G);
    if (st != OHM_OK) return st;
    T.t0 = t0;
    T.predict = t->predict;
    T.xpp = t->xpp;
    T.xppp = t->xppp;
    const int64_t nnz = t->nnz;
    const int n_launch = (n_steps + steps_per_launch - 1) / steps_per_launch;
    auto enqueue = [&]() -> cudaError_t {
        for (int l = 0; l < n_launch; ++l) {
            const int s0 = l * steps_per_launch;
            cudaError_t e = tran_launch(c, fn, grid, a, T, s0, std::min(n_steps, s0 + steps_per_launch));
            if (e != cudaSuccess) return e;
        }
        if (waveforms_host && need)
            return cudaMemcpyAsync(waveforms_host, t->wave, (size_t)need * sizeof(double), cudaMemcpyDeviceToHost,
                                   c->stream);
        return cudaSuccess;
    };

    int graph_used = 0;
    if (use_graph && n_launch > 0) {
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        CUDA_TRY(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = enqueue();
        cudaError_t e2 = cudaStreamEndCapture(c->stream, &graph);
        if (e == cudaSuccess) e = e2;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
        if (e == cudaSuccess) e = cudaGraphLaunch(exec, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (e != cudaSuccess) return ohm_fail(OHM_ERR_CUDA, "transient graph: %s", cudaGetErrorString(e));
        graph_used = 1;
    } else {
        cudaError_t e = enqueue();
        if (e != cudaSuccess) return ohm_fail(OHM_ERR_CUDA, "transient launch: %s", cudaGetErrorString(e));
    }
    // restore the plan's assembled system to its conductance base
    restore_kernel<<<steps_grid(nnz), 256, 0, c->stream>>>(G, a.vals64, a.vals32, nnz);
    CUDA_TRY(ohm_plan_restore_rhs(t->plan));
    CUDA_TRY(cudaGetLastError());
    TranDev d{};
    const ohm_status rs = tran_status(t, t0, h, d);
    if (info) {
        std::memset(info, 0, sizeof *info);
        info->status = rs;
        info->steps_done = d.steps_done;
        info->failed_step = d.status != 0 ? d.failed_step : -1;
        info->krylov_code = d.kcode;
        info->newton_iterations = d.newton_its;
        info->krylov_iterations = d.krylov_its;
        info->fp64_fallbacks = d.fallbacks;
        info->launches = n_launch;
        info->graph = graph_used;
        info->max_residual = d.max_residual;
    }
    return rs;
}

// Output arrays of a run: `points` rows of n_probes doubles (and times).
static ohm_status ensure_wave(ohm_transient *t, int64_t points, bool times) {
    const int64_t need = points * t->n_probes;
    if (need > t->wave_cap) {
        ohm_pool_free(t->wave);
        t->wave = nullptr;
        t->wave_cap = 0;
        CUDA_TRY(dalloc(&t->wave, (size_t)need));
        t->wave_cap = need;
    }
    if (times && points > t->times_cap) {
        ohm_pool_free(t->times);
        t->times = nullptr;
        t->times_cap = 0;
        CUDA_TRY(dalloc(&t->times, (size_t)points));
        t->times_cap = points;
    }
    return OHM_OK;
}

extern "C" ohm_status ohm_transient_run_adaptive(ohm_transient *t, double *x_dev, double tstep, double tstop,
                                                 double tstart, const ohm_newton_params *np, int32_t max_points,
                                                 double *times_host, double *waveforms_host,
                                                 ohm_adaptive_info *info) {
    if (!t || !x_dev || !np) return ohm_fail(OHM_ERR_INVALID_ARG, "null argument");
    if (!(tstep > 0.0) || !(tstop >= 0.0) || !std::isfinite(tstop) || !std::isfinite(tstart) || max_points < 0)
        return ohm_fail(OHM_ERR_INVALID_ARG, "need tstep > 0, finite tstop >= 0 and tstart, max_points >= 0");
    if (np->continuation) return ohm_fail(OHM_ERR_INVALID_ARG, "continuation is for DC solves, not transient steps");
    if (np->krylov.precond == OHM_PRECOND_ISAI1)
        return ohm_fail(OHM_ERR_INVALID_ARG, "transient steps use block Jacobi or Jacobi");
    ohm_ctx *c = t->ctx;
    CUDA_TRY(cudaSetDevice(c->device));
    if (np->initial_guess)
        CUDA_TRY(cudaMemcpyAsync(x_dev, np->initial_guess, t->n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    if (!t->ad_st) {
        cudaError_t e = t->put(&t->ad_xs, (const double *)nullptr, t->n);
        if (e == cudaSuccess) e = t->put(&t->ad_xt, (const double *)nullptr, t->n);
        if (e == cudaSuccess) e = t->put(&t->ad_fdev, (const double *)nullptr, t->n);
        if (e == cudaSuccess) e = t->put(&t->ad_zeros, (const double *)nullptr, t->n);
        if (e == cudaSuccess && t->n) e = cudaMemsetAsync(t->ad_zeros, 0, t->n * sizeof(double), c->stream);
        if (e == cudaSuccess) e = t->put(&t->ad_st, (const AdaptDev *)nullptr, 1);
        if (e != cudaSuccess) return ohm_fail(OHM_ERR_CUDA, "adaptive transient buffers: %s", cudaGetErrorString(e));
    }
    ohm_status st = ensure_wave(t, std::max<int64_t>(1, max_points), true);
    if (st != OHM_OK) return st;
    KernelArgs a;
    TranArgs T;
    const double *G = nullptr;
    st = tran_args(t, x_dev, np, a, T, G);
    if (st != OHM_OK) return st;
    AdaptArgs P{};
    P.tstep = tstep;
    P.tstop = tstop;
    P.tstart = tstart;
    P.max_points = max_points;
    P.nnz = t->nnz;
    P.g_vals = G;
    P.cg = t->cg;
    P.zeros = t->ad_zeros;
    P.aval = t->aval;
    P.xs = t->ad_xs;
    P.xt = t->ad_xt;
    P.fdev = t->ad_fdev;
    P.times = t->times;
    P.st = t->ad_st;
    const AdaptFn fn = pick_adaptive(tran_lpr(t->n, t->nnz));
    int grid = 0;
    st = tran_grid(t, (const void *)fn, a, grid);
    if (st != OHM_OK) return st;
    CUDA_TRY(cudaMemsetAsync(t->ad_st, 0, sizeof(AdaptDev), c->stream));
    CUDA_TRY(cudaMemsetAsync(c->sync_words, 0, 4 * sizeof(unsigned int), c->stream));
    {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(grid);
        cfg.blockDim = dim3(kSolverBlock);
        cfg.dynamicSmemBytes = (size_t)a.smem_bytes;
        cfg.stream = c->stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        CUDA_TRY(cudaLaunchKernelEx(&cfg, fn, a, T, P));
    }
    // restore the plan's assembled system to its conductance base
    restore_kernel<<<steps_grid(t->nnz), 256, 0, c->stream>>>(G, a.vals64, a.vals32, t->nnz);
    CUDA_TRY(ohm_plan_restore_rhs(t->plan));
    CUDA_TRY(cudaGetLastError());
    AdaptDev d{};
    unsigned int words[4] = {0, 0, 0, 0};
    CUDA_TRY(cudaMemcpyAsync(&d, t->ad_st, sizeof d, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaMemcpyAsync(words, c->sync_words, sizeof words, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    const int64_t kept = std::min<int64_t>(d.points, max_points);
    if (kept > 0) {
        if (times_host)
            CUDA_TRY(cudaMemcpyAsync(times_host, t->times, kept * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        if (waveforms_host && t->n_probes)
            CUDA_TRY(cudaMemcpyAsync(waveforms_host, t->wave, kept * t->n_probes * sizeof(double),
                                     cudaMemcpyDeviceToHost, c->stream));
        CUDA_TRY(cudaStreamSynchronize(c->stream));
    }
    ohm_status rs = OHM_OK;
    if (words[2] != 0) {
        rs = ohm_fail(OHM_ERR_TIMEOUT, "a device barrier wait gave up (error word %u)", words[2]);
    } else if (d.status == kAdTimestep) {
        rs = ohm_fail(OHM_ERR_TIMESTEP, "simulation failed: %d consecutive failures at minimum timestep "
                      "h_min=%.2e near t=%.2e", 10, tstep / 10000.0, d.t_fail);
    } else if (d.status != 0) {
        rs = ohm_fail(d.status == kErrSolve ? OHM_ERR_SOLVE
                      : (d.status == kErrNewtonNumerical ? OHM_ERR_NEWTON_NUMERICAL : OHM_ERR_NEWTON_NOT_CONVERGED),
                      "%s solve of the step to t = %.6e failed (status %d, krylov code %d)",
                      d.failed_kind == 1 ? "TRAP" : "BE", d.t_fail, d.status, d.kcode);
    }
    if (info) {
        std::memset(info, 0, sizeof *info);
        info->status = rs;
        info->accepted = d.accepted;
        info->rejected = d.rejected;
        info->points = d.points;
        info->newton_iterations = d.newton_its;
        info->krylov_iterations = d.krylov_its;
        info->linear_solves = d.solves;
        info->fp64_fallbacks = d.fallbacks;
        info->krylov_code = d.kcode;
        info->failed_solve = d.status != 0 && d.status != kAdTimestep ? d.failed_kind : 0;
        info->t_end = d.t;
        info->h_last = d.h;
        info->t_failed = d.t_fail;
        info->max_residual = d.max_residual;
    }
    return rs;
}

// ================================================================= adjoint ==
namespace {

struct BackArgs {
    const double *x, *xprev, *lam;     // xprev null: DC (no capacitor term)
    double inv_h;
    int64_t nr, nc, nd, nm;
    const int32_t *ra, *rb, *ca, *cb;
    const double *rv, *cv;
    const DiodeDesc *dio;
    const MosfetDesc *mos;
    double *gr, *gc, *gd, *gvto, *gkp;
};

__device__ __forceinline__ double at(const double *v, int32_t i) { return i >= 0 ? v[i] : 0.0; }

// do/dp += -lambda^T dF/dp for every component, one thread per component
// (accumulation over steps in launch order: deterministic).  A device current
// i enters F at its first terminal and leaves at its second, so a parameter p
// of it contributes -(lambda_1 - lambda_2) di/dp: diode di/dIs = exp(v/nVt) - 1;
// MOSFET (drain, source) di/d|VTO| = -polarity g_m, di/dKP = i / KP.
__global__ void backstamp_kernel(BackArgs B) {
    const int64_t total = B.nr + (B.xprev ? B.nc : 0) + B.nd + B.nm;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
        if (k < B.nr) {
            const int32_t a = B.ra[k], b = B.rb[k];
            const double r = B.rv[k];
            B.gr[k] += (at(B.x, a) - at(B.x, b)) * (at(B.lam, a) - at(B.lam, b)) / (r * r);
            continue;
        }
        int64_t q = k - B.nr;
        if (B.xprev) {
            if (q < B.nc) {
                const int32_t a = B.ca[q], b = B.cb[q];
                const double dv = (at(B.x, a) - at(B.x, b)) - (at(B.xprev, a) - at(B.xprev, b));
                B.gc[q] -= dv * B.inv_h * (at(B.lam, a) - at(B.lam, b));
                continue;
            }
            q -= B.nc;
        }
        if (q < B.nd) {
            const DiodeDesc &d = B.dio[q];
            const double v = node_v(B.x, d.anode) - node_v(B.x, d.cathode);
            const double e = clamp_exp(v / (double)d.n_vt);
            B.gd[q] -= (node_v(B.lam, d.anode) - node_v(B.lam, d.cathode)) * (e - 1.0);
            continue;
        }
        q -= B.nd;
        const MosfetDesc &m = B.mos[q];
        const MosEval ev = mosfet_eval(m, B.x);
        const double dl = node_v(B.lam, m.drain) - node_v(B.lam, m.source);
        B.gvto[q] += dl * ((double)m.polarity * ev.gm);
        B.gkp[q] -= dl * ev.i_per_kp;
    }
}

__global__ void gather_kernel(double *dst, const double *src, const uint32_t *perm, int64_t m) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x)
        dst[k] = src[perm[k]];
}

// rhs = (C/h)^T lambda, C^T in CSR
__global__ void ct_rhs_kernel(double *rhs, const uint32_t *rp, const uint32_t *col, const double *val,
                              const double *lam, double inv_h, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (uint32_t k = rp[i]; k < rp[i + 1]; ++k) acc += val[k] * lam[col[k]];
        rhs[i] = acc * inv_h;
    }
}

// Transposed CSR of a pattern: t_rp, t_col and perm (t slot -> source slot).
void transpose_pattern(int64_t n, const std::vector<uint32_t> &rp, const std::vector<uint32_t> &col,
                       std::vector<uint32_t> &t_rp, std::vector<uint32_t> &t_col, std::vector<uint32_t> &perm) {
    const int64_t nnz = (int64_t)col.size();
    t_rp.assign(n + 1, 0);
    for (int64_t k = 0; k < nnz; ++k) ++t_rp[col[k] + 1];
    for (int64_t i = 0; i < n; ++i) t_rp[i + 1] += t_rp[i];
    t_col.assign(nnz, 0);
    perm.assign(nnz, 0);
    std::vector<uint32_t> fill(t_rp.begin(), t_rp.end() - 1);
    for (int64_t i = 0; i < n; ++i)
        for (uint32_t k = rp[i]; k < rp[i + 1]; ++k) {
            const uint32_t d = fill[col[k]]++;
            t_col[d] = (uint32_t)i;
            perm[d] = k;
        }
}

// Device state of one adjoint computation (freed on destruction).
struct AdjointCtx {
    ohm_ctx *c = nullptr;
    std::vector<void *> allocs;
    ohm_linsys *L = nullptr;
    int64_t n = 0, nnz = 0;
    uint32_t *perm = nullptr;
    double *J = nullptr, *JT = nullptr, *lam = nullptr, *rhs = nullptr;
    BackArgs B{};
    ~AdjointCtx() {
        if (c) cudaStreamSynchronize(c->stream);
        ohm_linsys_destroy(L);
        for (void *p : allocs) ohm_pool_free(p);
    }
    template <typename T>
    cudaError_t put(T **dst, const T *h, size_t count) {
        cudaError_t e = dalloc(dst, count);
        if (e == cudaSuccess) allocs.push_back((void *)*dst);
        if (e == cudaSuccess && count) {
            if (h) e = cudaMemcpyAsync(*dst, h, count * sizeof(T), cudaMemcpyHostToDevice, c->stream);
            else e = cudaMemsetAsync(*dst, 0, count * sizeof(T), c->stream);
        }
        return e;
    }

    // pattern transpose, J^T linear system, component arrays, accumulators
    ohm_status setup(ohm_plan *plan, const ohm_components *comps, const KernelArgs &a, int64_t nnz_) {
        c = ohm_plan_context(plan);
        n = a.n;
        nnz = nnz_;
        if (comps && ((comps->n_resistors && (!comps->r_a || !comps->r_b || !comps->r_ohms)) ||
                      (comps->n_capacitors && (!comps->c_a || !comps->c_b || !comps->c_farads))))
            return ohm_fail(OHM_ERR_INVALID_ARG, "null component array");
        const int64_t nr = comps ? comps->n_resistors : 0, nc = comps ? comps->n_capacitors : 0;
        for (int64_t k = 0; k < nr; ++k)
            if (comps->r_a[k] < -1 || comps->r_a[k] >= n || comps->r_b[k] < -1 || comps->r_b[k] >= n)
                return ohm_fail(OHM_ERR_INVALID_ARG, "resistor %lld: row out of range", (long long)k);
        for (int64_t k = 0; k < nc; ++k)
            if (comps->c_a[k] < -1 || comps->c_a[k] >= n || comps->c_b[k] < -1 || comps->c_b[k] >= n)
                return ohm_fail(OHM_ERR_INVALID_ARG, "capacitor %lld: row out of range", (long long)k);
        std::vector<uint32_t> rp(n + 1), col(nnz), t_rp, t_col, pm;
        std::vector<double> g(nnz), gt(nnz);
        CUDA_TRY(cudaMemcpy(rp.data(), a.row_ptr, (n + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost));
        if (nnz) CUDA_TRY(cudaMemcpy(col.data(), a.col, nnz * sizeof(uint32_t), cudaMemcpyDeviceToHost));
        if (nnz) CUDA_TRY(cudaMemcpy(g.data(), a.base_vals, nnz * sizeof(double), cudaMemcpyDeviceToHost));
        transpose_pattern(n, rp, col, t_rp, t_col, pm);
        for (int64_t k = 0; k < nnz; ++k) gt[k] = g[pm[k]];
        ohm_status st = ohm_linsys_create(c, n, nnz, t_rp.data(), t_col.data(), gt.data(), &L);
        if (st != OHM_OK) return st;
        cudaError_t e = put(&perm, pm.data(), nnz);
        if (e == cudaSuccess) e = put(&J, (const double *)nullptr, nnz);
        if (e == cudaSuccess) e = put(&JT, (const double *)nullptr, nnz);
        if (e == cudaSuccess) e = put(&lam, (const double *)nullptr, n);
        if (e == cudaSuccess) e = put(&rhs, (const double *)nullptr, n);
        int32_t *i32 = nullptr;
        double *f64 = nullptr;
        B = BackArgs{};
        B.nr = nr; B.nc = nc; B.nd = a.nd; B.dio = a.diodes; B.nm = a.nm; B.mos = a.mosfets;
        if (e == cudaSuccess && nr) { e = put(&i32, comps->r_a, nr); B.ra = i32; }
        if (e == cudaSuccess && nr) { e = put(&i32, comps->r_b, nr); B.rb = i32; }
        if (e == cudaSuccess && nr) { e = put(&f64, comps->r_ohms, nr); B.rv = f64; }
        if (e == cudaSuccess && nc) { e = put(&i32, comps->c_a, nc); B.ca = i32; }
        if (e == cudaSuccess && nc) { e = put(&i32, comps->c_b, nc); B.cb = i32; }
        if (e == cudaSuccess && nc) { e = put(&f64, comps->c_farads, nc); B.cv = f64; }
        if (e == cudaSuccess) { e = put(&f64, (const double *)nullptr, std::max<int64_t>(nr, 1)); B.gr = f64; }
        if (e == cudaSuccess) { e = put(&f64, (const double *)nullptr, std::max<int64_t>(nc, 1)); B.gc = f64; }
        if (e == cudaSuccess) { e = put(&f64, (const double *)nullptr, std::max<int64_t>(a.nd, 1)); B.gd = f64; }
        if (e == cudaSuccess) { e = put(&f64, (const double *)nullptr, std::max<int64_t>(a.nm, 1)); B.gvto = f64; }
        if (e == cudaSuccess) { e = put(&f64, (const double *)nullptr, std::max<int64_t>(a.nm, 1)); B.gkp = f64; }
        if (e != cudaSuccess) return ohm_fail(OHM_ERR_CUDA, "adjoint set-up: %s", cudaGetErrorString(e));
        B.lam = lam;
        return OHM_OK;
    }

    // J(x)^T lam = rhs on base values `base`, then the back-stamp at (x, xprev).
    ohm_status step(ohm_plan *plan, const double *x, const double *xprev, const double *base, double inv_h,
                    const ohm_krylov_params *kp, int64_t &kiters) {
        ohm_status st = ohm_plan_jacobian_device(plan, x, base, J);
        if (st != OHM_OK) return st;
        gather_kernel<<<steps_grid(nnz), 256, 0, c->stream>>>(JT, J, perm, nnz);
        CUDA_TRY(cudaGetLastError());
        ohm_solve_info si{};
        st = ohm_linsys_solve(L, JT, rhs, lam, kp, &si);
        kiters += si.krylov_iterations;
        if (st != OHM_OK) return st;
        BackArgs b = B;
        b.x = x;
        b.xprev = xprev;
        b.inv_h = inv_h;
        const int64_t total = b.nr + (xprev ? b.nc : 0) + b.nd + b.nm;
        if (total) backstamp_kernel<<<steps_grid(total), 256, 0, c->stream>>>(b);
        CUDA_TRY(cudaGetLastError());
        return OHM_OK;
    }

    ohm_status download(double *gr, double *gc, double *gd, double *gvto, double *gkp, double *lam_host) {
        if (gr && B.nr) CUDA_TRY(cudaMemcpyAsync(gr, B.gr, B.nr * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        if (gvto && B.nm) CUDA_TRY(cudaMemcpyAsync(gvto, B.gvto, B.nm * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        if (gkp && B.nm) CUDA_TRY(cudaMemcpyAsync(gkp, B.gkp, B.nm * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        if (gc && B.nc) CUDA_TRY(cudaMemcpyAsync(gc, B.gc, B.nc * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        if (gd && B.nd) CUDA_TRY(cudaMemcpyAsync(gd, B.gd, B.nd * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        if (lam_host) CUDA_TRY(cudaMemcpyAsync(lam_host, lam, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CUDA_TRY(cudaStreamSynchronize(c->stream));
        return OHM_OK;
    }
};

double host_dot(ohm_ctx *c, const double *w, const double *x_dev, int64_t n) {
    std::vector<double> x(n);
    if (cudaMemcpyAsync(x.data(), x_dev, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
        cudaStreamSynchronize(c->stream) != cudaSuccess)
        return NAN;
    double s = 0.0;
    for (int64_t i = 0; i < n; ++i) s += w[i] * x[i];
    return s;
}

}  // namespace

extern "C" ohm_status ohm_plan_adjoint_dc(ohm_plan *plan, const double *x_dev, const double *w_host,
                                          const ohm_components *comps, const ohm_krylov_params *kp, double *d_out_dr,
                                          double *d_out_dis, double *d_out_dvto, double *d_out_dkp,
                                          double *lambda_host, ohm_adjoint_info *info) {
    if (!plan || !x_dev || !w_host || !kp) return ohm_fail(OHM_ERR_INVALID_ARG, "null argument");
    ohm_newton_params np;
    ohm_newton_params_default(&np);
    KernelArgs a;
    int64_t nnz = 0;
    ohm_status st = ohm_plan_kernel_args(plan, &np, const_cast<double *>(x_dev), a, &nnz);
    if (st != OHM_OK) return st;
    AdjointCtx A;
    st = A.setup(plan, comps, a, nnz);
    if (st != OHM_OK) return st;
    ohm_ctx *c = A.c;
    CUDA_TRY(cudaMemcpyAsync(A.rhs, w_host, a.n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    int64_t kiters = 0;
    st = A.step(plan, x_dev, nullptr, nullptr, 0.0, kp, kiters);
    if (st == OHM_OK) st = A.download(d_out_dr, nullptr, d_out_dis, d_out_dvto, d_out_dkp, lambda_host);
    if (info) {
        std::memset(info, 0, sizeof *info);
        info->status = st;
        info->linear_solves = 1;
        info->krylov_iterations = kiters;
        info->output = host_dot(c, w_host, x_dev, a.n);
    }
    return st;
}

extern "C" ohm_status ohm_transient_adjoint(ohm_transient *t, const double *x0_dev, double t0, double h,
                                            int32_t n_steps, int32_t checkpoint_every, const ohm_newton_params *np,
                                            const double *w_host, const ohm_components *comps,
                                            const ohm_krylov_params *kp, double *d_out_dr, double *d_out_dc,
                                            double *d_out_dis, double *d_out_dvto, double *d_out_dkp,
                                            ohm_adjoint_info *info) {
    if (!t || !x0_dev || !np || !w_host || !kp) return ohm_fail(OHM_ERR_INVALID_ARG, "null argument");
    if (!(h > 0.0) || n_steps < 1 || checkpoint_every < 0)
        return ohm_fail(OHM_ERR_INVALID_ARG, "need h > 0, n_steps >= 1, checkpoint_every >= 0");
    if (np->continuation || np->krylov.precond == OHM_PRECOND_ISAI1)
        return ohm_fail(OHM_ERR_INVALID_ARG, "transient steps use block Jacobi or Jacobi, no continuation");
    ohm_ctx *c = t->ctx;
    CUDA_TRY(cudaSetDevice(c->device));
    const int64_t n = t->n;
    // checkpoint_every = 0: the forward pass keeps every state (n_steps x n
    // doubles) and the reverse sweep recomputes nothing
    const bool keep_all = checkpoint_every == 0;
    const int K = keep_all ? n_steps : checkpoint_every;
    const int nseg = (n_steps + K - 1) / K;
    AdjointCtx A;
    double *x = nullptr, *ck = nullptr, *S = nullptr;
    {
        KernelArgs a0;
        int64_t nnz = 0;
        ohm_newton_params dp;
        ohm_newton_params_default(&dp);
        ohm_status st = ohm_plan_kernel_args(t->plan, &dp, const_cast<double *>(x0_dev), a0, &nnz);
        if (st != OHM_OK) return st;
        st = A.setup(t->plan, comps, a0, nnz);
        if (st != OHM_OK) return st;
    }
    cudaError_t e = A.put(&x, (const double *)nullptr, n);
    if (e == cudaSuccess) e = A.put(&ck, (const double *)nullptr, (size_t)nseg * n);
    if (e == cudaSuccess) e = A.put(&S, (const double *)nullptr, (size_t)K * n);
    if (e != cudaSuccess) return ohm_fail(OHM_ERR_CUDA, "adjoint buffers: %s", cudaGetErrorString(e));
    // C^T for the adjoint recursion
    std::vector<uint32_t> crp(n + 1), ccol(t->c_nnz), ctrp, ctcol, cpm;
    std::vector<double> cval(t->c_nnz), ctval(t->c_nnz);
    CUDA_TRY(cudaMemcpy(crp.data(), t->c_rp, (n + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if (t->c_nnz) {
        CUDA_TRY(cudaMemcpy(ccol.data(), t->c_col, t->c_nnz * sizeof(uint32_t), cudaMemcpyDeviceToHost));
        CUDA_TRY(cudaMemcpy(cval.data(), t->c_val, t->c_nnz * sizeof(double), cudaMemcpyDeviceToHost));
    }
    transpose_pattern(n, crp, ccol, ctrp, ctcol, cpm);
    for (int64_t k = 0; k < t->c_nnz; ++k) ctval[k] = cval[cpm[k]];
    uint32_t *d_ctrp = nullptr, *d_ctcol = nullptr;
    double *d_ctval = nullptr;
    e = A.put(&d_ctrp, ctrp.data(), n + 1);
    if (e == cudaSuccess) e = A.put(&d_ctcol, ctcol.data(), t->c_nnz);
    if (e == cudaSuccess) e = A.put(&d_ctval, ctval.data(), t->c_nnz);
    if (e != cudaSuccess) return ohm_fail(OHM_ERR_CUDA, "adjoint buffers: %s", cudaGetErrorString(e));

    // ---- forward, checkpoint at the start of every segment ----
    KernelArgs a;
    TranArgs T;
    TranFn fn = nullptr;
    int grid = 0;
    const double *G = nullptr;
    CUDA_TRY(cudaMemcpyAsync(x, x0_dev, n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    ohm_status st = tran_prepare(t, x, h, np, a, T, fn, grid, G);
    if (st != OHM_OK) return st;
    T.t0 = t0;
    T.n_probes = 0;
    int launches = 0;
    if (keep_all) {
        T.states = S;
        T.state_base = 0;
    }
    for (int sg = 0; sg < nseg; ++sg) {
        CUDA_TRY(cudaMemcpyAsync(ck + (size_t)sg * n, x, n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
        CUDA_TRY(tran_launch(c, fn, grid, a, T, sg * K, std::min(n_steps, (sg + 1) * K)));
    }
    TranDev d{};
    st = tran_status(t, t0, h, d);
    double output = NAN;
    if (st == OHM_OK) output = host_dot(c, w_host, x, n);
    // ---- reverse sweep ----
    int64_t kiters = 0;
    int solves = 0;
    if (st == OHM_OK) CUDA_TRY(cudaMemcpyAsync(A.rhs, w_host, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    const double inv_h = 1.0 / h;
    for (int sg = nseg - 1; st == OHM_OK && sg >= 0; --sg) {
        const int s0 = sg * K, s1 = std::min(n_steps, (sg + 1) * K);
        if (!keep_all) {
            // recompute x_{s0+1} .. x_{s1} from the checkpoint x_{s0}
            CUDA_TRY(cudaMemcpyAsync(x, ck + (size_t)sg * n, n * sizeof(double), cudaMemcpyDeviceToDevice,
                                     c->stream));
            T.states = S;
            T.state_base = s0;
            CUDA_TRY(tran_launch(c, fn, grid, a, T, s0, s1));
            ++launches;
            st = tran_status(t, t0, h, d);
        }
        for (int s = s1 - 1; st == OHM_OK && s >= s0; --s) {
            // step s maps x_s (state index s, or the checkpoint) to x_{s+1}
            const double *xn = S + (size_t)(s - s0) * n;
            const double *xp = s == s0 ? ck + (size_t)sg * n : S + (size_t)(s - s0 - 1) * n;
            st = A.step(t->plan, xn, xp, t->aval, inv_h, kp, kiters);
            ++solves;
            if (st != OHM_OK) {
                st = ohm_fail(st, "adjoint solve of step %d: %s", s, ohm_last_error());
                break;
            }
            ct_rhs_kernel<<<steps_grid(n), 256, 0, c->stream>>>(A.rhs, d_ctrp, d_ctcol, d_ctval, A.lam, inv_h, n);
            CUDA_TRY(cudaGetLastError());
        }
    }
    // ---- the DC start: J_0^T lambda_0 = (C/h)^T lambda_1 ----
    // Every DC back-stamp term carries a terminal voltage difference or
    // exp(v/nVt) - 1 at x_0, so when x_0 is zero the whole term is zero and
    // the solve is skipped.
    bool x0_zero = false;
    if (st == OHM_OK) {
        std::vector<double> hx(n);
        CUDA_TRY(cudaMemcpyAsync(hx.data(), ck, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CUDA_TRY(cudaStreamSynchronize(c->stream));
        x0_zero = std::all_of(hx.begin(), hx.end(), [](double v) { return v == 0.0; });
    }
    if (st == OHM_OK && !x0_zero) {
        st = A.step(t->plan, ck, nullptr, nullptr, 0.0, kp, kiters);
        ++solves;
        if (st != OHM_OK) st = ohm_fail(st, "adjoint solve of the DC start: %s", ohm_last_error());
    }
    restore_kernel<<<steps_grid(t->nnz), 256, 0, c->stream>>>(G, a.vals64, a.vals32, t->nnz);
    CUDA_TRY(ohm_plan_restore_rhs(t->plan));
    if (st == OHM_OK) st = A.download(d_out_dr, d_out_dc, d_out_dis, d_out_dvto, d_out_dkp, nullptr);
    if (info) {
        std::memset(info, 0, sizeof *info);
        info->status = st;
        info->steps = n_steps;
        info->linear_solves = solves;
        info->recompute_launches = launches;
        info->krylov_iterations = kiters;
        info->output = output;
    }
    return st;
}
