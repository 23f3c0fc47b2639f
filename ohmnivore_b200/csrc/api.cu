// C ABI of libohm_b200: contexts, device buffers (SolverBackend), the linear
// solve (LinearSolver::solve_real) and the device-resident Newton plan
// (newton_solve).  Host-side work here is validation, the stamp map and the
// preconditioner structure; all arithmetic runs in the persistent kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "internal.cuh"
#include "isai_host.h"
#include "host_util.h"

using namespace ohm;

static_assert(sizeof(ohm_diode_desc) == sizeof(DiodeDesc), "diode layout");
static_assert(sizeof(ohm_bjt_desc) == sizeof(BjtDesc), "bjt layout");
static_assert(sizeof(ohm_mosfet_desc) == sizeof(MosfetDesc), "mosfet layout");

// ----------------------------------------------------------------- errors --
static thread_local std::string g_last_error;

ohm_status ohm_fail(ohm_status st, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return st;
}
#define fail ohm_fail

extern "C" const char *ohm_last_error(void) { return g_last_error.c_str(); }
extern "C" const char *ohm_version(void) { return "ohm_b200 0.1 (sm_100a)"; }

extern "C" void ohm_krylov_params_default(ohm_krylov_params *p) {
    if (!p) return;
    p->max_iterations = 10000;        // bicgstab.rs:10
    p->tolerance = 1e-5;              // bicgstab.rs:11
    p->precision = OHM_PREC_FP64;
    p->precond = OHM_PRECOND_AUTO;
    p->inner_rtol = 0.0;
    p->max_refinements = 1;
    p->max_restarts = 50;
    p->fp32_max_iterations = 600;
    p->fp32_min_eta_exp = 0;
}

extern "C" void ohm_newton_params_default(ohm_newton_params *p) {
    if (!p) return;
    p->max_iterations = 50;           // newton.rs:48
    p->abs_tol = 1e-4;                // newton.rs:49
    p->rel_tol = 0.0;
    ohm_krylov_params_default(&p->krylov);
    p->initial_guess = nullptr;
    p->forcing = OHM_FORCING_CONSTANT;
    p->eta_max = 0.5;
    p->continuation = 0;
    p->n_nodes = 0;
}

// ---------------------------------------------------------------- context --
static void ctx_free(ohm_ctx *c);

extern "C" ohm_status ohm_ctx_create(int device, ohm_ctx **out) {
    if (!out) return fail(OHM_ERR_INVALID_ARG, "out is null");
    *out = nullptr;
    int ndev = 0;
    CUDA_TRY(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return fail(OHM_ERR_INVALID_ARG, "device %d out of range (%d)", device, ndev);
    CUDA_TRY(cudaSetDevice(device));
    int coop = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device));
    if (!coop) return fail(OHM_ERR_CUDA, "device %d lacks cooperative launch", device);
    ohm_ctx *c = new (std::nothrow) ohm_ctx();
    if (!c) return fail(OHM_ERR_INVALID_ARG, "out of host memory");
    c->device = device;
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = dalloc(&c->sync_words, 4);
    if (e == cudaSuccess) e = dalloc(&c->info_dev, 1);
    if (e == cudaSuccess) e = cudaMallocHost((void **)&c->info_host, sizeof(DeviceInfo));
    if (e == cudaSuccess) e = dalloc(&c->dot_scratch, 2048);
    if (e != cudaSuccess) {
        ctx_free(c);
        return fail(OHM_ERR_CUDA, "context setup failed: %s", cudaGetErrorString(e));
    }
    *out = c;
    return OHM_OK;
}

static void ctx_free(ohm_ctx *c) {
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    ohm_pool_free(c->sync_words);
    ohm_pool_free(c->info_dev);
    cudaFreeHost(c->info_host);
    ohm_pool_free(c->dot_scratch);
    if (c->stream) cudaStreamDestroy(c->stream);
    const int dev = c->device;
    delete c;
    ohm_pool_trim(dev);            // cached blocks of this device go back to CUDA
}

extern "C" ohm_status ohm_ctx_destroy(ohm_ctx *c) {
    if (!c) return OHM_OK;
    if (c->live_objects > 0) {
        c->destroy_pending = true;    // released when the last object goes
        return OHM_OK;
    }
    ctx_free(c);
    return OHM_OK;
}

void ohm_ctx_retain(ohm_ctx *c) { ++c->live_objects; }

void ohm_ctx_release(ohm_ctx *c) {
    if (--c->live_objects == 0 && c->destroy_pending) ctx_free(c);
}

extern "C" ohm_status ohm_ctx_synchronize(ohm_ctx *c) {
    if (!c) return fail(OHM_ERR_INVALID_ARG, "ctx is null");
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return OHM_OK;
}

extern "C" void *ohm_ctx_stream(ohm_ctx *c) { return c ? (void *)c->stream : nullptr; }

extern "C" ohm_status ohm_ctx_set_krylov_layout(ohm_ctx *c, int32_t layout) {
    if (!c) return fail(OHM_ERR_INVALID_ARG, "context is null");
    if (layout != OHM_KRYLOV_LAYOUT_AUTO && layout != OHM_KRYLOV_LAYOUT_GLOBAL)
        return fail(OHM_ERR_INVALID_ARG, "unknown Krylov layout %d", (int)layout);
    c->krylov_layout = layout;
    return OHM_OK;
}

// ------------------------------------------------------------ launch logic --
using KernelFn = void (*)(KernelArgs);

static KernelFn pick_kernel(int lpr) {
    switch (lpr) {
        case 1: return persistent_solver<1>;
        case 2: return persistent_solver<2>;
        case 4: return persistent_solver<4>;
        case 8: return persistent_solver<8>;
        case 16: return persistent_solver<16>;
        default: return persistent_solver<32>;
    }
}

static int choose_lpr(int64_t n, int64_t nnz) {
    const double avg = n > 0 ? (double)nnz / (double)n : 1.0;
    if (avg <= 5.5) return 1;     // measured: 29.0 us vs 31.8 us per BiCGSTAB iteration at 5 nnz/row
    if (avg <= 12.0) return 4;
    if (avg <= 24.0) return 8;
    if (avg <= 48.0) return 16;
    return 32;
}

static constexpr int kBlock = kSolverBlock;

// Dynamic shared memory for the Krylov slice of a block that owns `rows`
// rows: records, r_hat, t, d, weights (FP64, the larger of the two Krylov
// precisions), row pointers and pair flags per row, column + value per
// nonzero outside long rows (an estimate with a 3 % margin; a block whose
// slice is larger works from global memory), or 0 when it cannot fit.
int ohm_krylov_smem_bytes(const void *fn, int64_t n, int64_t nnz_short, int grid) {
    if (n <= 0 || grid <= 0) return 0;
    int dev = 0, optin = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return 0;
    cudaFuncAttributes fa{};
    if (cudaFuncGetAttributes(&fa, fn) != cudaSuccess) return 0;
    const int64_t avail = (int64_t)optin - (int64_t)fa.sharedSizeBytes - 1024;
    const int64_t rows = (n + grid - 1) / grid + 1;
    const int64_t nnz_blk = (int64_t)((double)std::max<int64_t>(nnz_short, 0) * (double)rows / (double)n * 1.03) + 256;
    const int64_t need = rows * (32 + 8 + 8 + 8 + 8 + 4 + 1) + nnz_blk * (8 + 4) + 16 * 16;
    if (need > avail) return 0;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need) != cudaSuccess)
        return 0;
    return (int)need;
}

ohm_status ohm_launch_persistent(const LaunchTarget &t, KernelArgs &a, int64_t nnz, int *launches) {
    const int lpr = choose_lpr(a.n, nnz);
    KernelFn fn = pick_kernel(lpr);
    int per_sm = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kBlock, 0));
    if (per_sm < 1) return fail(OHM_ERR_CUDA, "solver kernel does not fit on an SM");
    per_sm = std::min(per_sm, 2);
    int64_t want = (a.n + kBlock - 1) / kBlock;
    const int64_t ndev = (int64_t)a.nd + a.nq + a.nm;
    want = std::max<int64_t>(want, (ndev + kBlock - 1) / kBlock);
    int64_t cap = (int64_t)per_sm * t.num_sms;
    if (t.max_grid > 0) cap = std::min<int64_t>(cap, t.max_grid);
    int grid = (int)std::max<int64_t>(1, std::min<int64_t>(want, cap));
    // one block per SM either way: a block is 1024 threads at the register cap
    a.smem_bytes = t.krylov_layout != OHM_KRYLOV_LAYOUT_GLOBAL
                       ? ohm_krylov_smem_bytes((const void *)fn, a.n, nnz - a.nnz_long, grid) : 0;
    if (a.smem_bytes > 0) {
        int fit = 0;
        CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, fn, kBlock, a.smem_bytes));
        if (fit < 1) a.smem_bytes = 0;
        else grid = std::min<int64_t>(grid, (int64_t)fit * t.num_sms);
    }
    a.gs.count = (unsigned long long *)t.sync_words;     // words 0-1
    a.gs.error = (int *)(t.sync_words + 2);              // word 2
    a.info = t.info_dev;
    CUDA_TRY(cudaMemsetAsync(t.sync_words, 0, 4 * sizeof(unsigned int), t.stream));
    CUDA_TRY(cudaMemsetAsync(t.info_dev, 0, sizeof(DeviceInfo), t.stream));
    void *args[] = {&a};
    CUDA_TRY(cudaLaunchCooperativeKernel((void *)fn, dim3(grid), dim3(kBlock), args, (size_t)a.smem_bytes,
                                         t.stream));
    if (launches) *launches += 1;
    return OHM_OK;
}

static LaunchTarget ctx_target(ohm_ctx *c) {
    return LaunchTarget{c->num_sms, c->stream, c->sync_words, c->info_dev, c->info_host, 0, c->krylov_layout};
}

static ohm_status launch_solver(ohm_ctx *c, KernelArgs &a, int64_t nnz, int *launches) {
    return ohm_launch_persistent(ctx_target(c), a, nnz, launches);
}

static ohm_status finish_solver(ohm_ctx *c, ohm_solve_info *info, int launches) {
    return ohm_finish_persistent(ctx_target(c), info, launches);
}

ohm_status ohm_finish_persistent(const LaunchTarget &t, ohm_solve_info *info, int launches) {
    unsigned int words[4] = {0, 0, 0, 0};
    CUDA_TRY(cudaMemcpyAsync(t.info_host, t.info_dev, sizeof(DeviceInfo), cudaMemcpyDeviceToHost, t.stream));
    CUDA_TRY(cudaMemcpyAsync(words, t.sync_words, sizeof words, cudaMemcpyDeviceToHost, t.stream));
    CUDA_TRY(cudaStreamSynchronize(t.stream));
    const DeviceInfo &di = *t.info_host;
    ohm_status st = OHM_OK;
    if (words[2] != 0) {
        st = fail(OHM_ERR_TIMEOUT, "a device barrier wait gave up (error word %u)", words[2]);
    } else {
        switch (di.status) {
            case kOk: st = OHM_OK; break;
            case kErrSolve: {
                static const char *why[] = {"running", "converged", "did not converge within the iteration limit",
                                            "breakdown: rho ~ 0", "breakdown: r_hat.v ~ 0",
                                            "breakdown: ||t|| ~ 0", "breakdown: omega ~ 0",
                                            "diverged: NaN/Inf in residual"};
                const int k = (di.krylov_code >= 0 && di.krylov_code <= 7) ? di.krylov_code : 0;
                st = fail(OHM_ERR_SOLVE, "BiCGSTAB %s", why[k]);
                break;
            }
            case kErrNewtonNotConverged:
                st = fail(OHM_ERR_NEWTON_NOT_CONVERGED,
                          "Newton solver did not converge after %d iterations (max residual: %.2e)",
                          di.iterations, di.max_residual);
                break;
            case kErrNewtonNumerical:
                st = fail(OHM_ERR_NEWTON_NUMERICAL, "Newton solver encountered numerical error at iteration %d",
                          di.error_iteration);
                break;
            default: st = fail(OHM_ERR_CUDA, "unknown device status %d", di.status);
        }
    }
    if (info) {
        info->status = st;
        info->krylov_code = di.krylov_code;
        info->iterations = di.iterations;
        info->error_iteration = di.error_iteration;
        info->krylov_iterations = di.krylov_iterations;
        info->fp64_fallbacks = di.fp64_fallbacks;
        info->krylov_restarts = di.krylov_restarts;
        info->max_residual = di.max_residual;
        info->final_residual_norm = di.final_residual;
        info->b_norm = di.b_norm;
        info->kernel_launches = launches;
        info->continuation_steps = di.continuation_steps;
        info->continuation_kind = di.continuation_kind;
    }
    return st;
}

// Krylov workspace shared by the linear solve and the Newton plan: two
// record arrays (4 values per row, 8-byte slots so either precision fits),
// seven length-n vectors, the FP64 residual and correction, the
// preconditioner structure and the reduction partials.
struct Workspace {
    int64_t n = 0;
    double *vec = nullptr;       // 15 * n doubles
    double *r64 = nullptr;
    double *dx = nullptr;
    double *partials = nullptr;  // 8 * max grid
    int32_t *partner = nullptr;
    uint32_t *diag_slot = nullptr, *off_slot = nullptr;
    uint8_t *rowflag = nullptr;
    bool any_pair = false;
    void release() {
        ohm_pool_free(vec); ohm_pool_free(r64); ohm_pool_free(dx); ohm_pool_free(partials);
        ohm_pool_free(partner); ohm_pool_free(diag_slot); ohm_pool_free(off_slot); ohm_pool_free(rowflag);
        vec = r64 = dx = partials = nullptr; partner = nullptr; diag_slot = off_slot = nullptr;
        rowflag = nullptr;
    }
    cudaError_t alloc(int64_t n_, int num_sms) {
        n = n_;
        cudaError_t e = dalloc(&vec, 15 * (size_t)n);
        if (e == cudaSuccess) e = dalloc(&r64, n);
        if (e == cudaSuccess) e = dalloc(&dx, n);
        if (e == cudaSuccess) e = dalloc(&partials, 8 * (size_t)num_sms * 8);
        if (e == cudaSuccess) e = dalloc(&partner, n);
        if (e == cudaSuccess) e = dalloc(&diag_slot, n);
        if (e == cudaSuccess) e = dalloc(&off_slot, n);
        if (e == cudaSuccess) e = dalloc(&rowflag, n);
        return e;
    }
    void bind(KernelArgs &a) const {
        a.rec0 = (void *)vec;
        a.rec1 = (void *)(vec + 4 * (size_t)n);
        void **slots[] = {&a.rhat, &a.s, &a.t, &a.phat, &a.shat, &a.d, &a.pc_part};
        for (int k = 0; k < 7; ++k) *slots[k] = (void *)(vec + (8 + (size_t)k) * n);
        a.r64 = r64;
        a.dx = dx;
        a.partials = partials;
        a.partner = partner;
        a.diag_slot = diag_slot;
        a.off_slot = off_slot;
        a.rowflag = any_pair ? rowflag : nullptr;
    }
    cudaError_t upload_pc(const PcHost &pc, cudaStream_t s) {
        cudaError_t e = cudaMemcpyAsync(partner, pc.partner.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(diag_slot, pc.diag_slot.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(off_slot, pc.off_slot.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(rowflag, pc.rowflag.data(), n * sizeof(uint8_t), cudaMemcpyHostToDevice, s);
        // the host vectors must outlive the copies: callers synchronise before releasing them
        any_pair = pc.any_pair;
        return e;
    }
};

// Device copy of the ISAI(1) structure (isai_host.h) plus its value arrays.
struct IsaiDev {
    bool ready = false;
    uint32_t *aug_rp = nullptr, *aug_col = nullptr, *aug_diag = nullptr, *cp_ptr = nullptr, *cp_pair = nullptr;
    int32_t *aug_map = nullptr;
    double *f0 = nullptr, *f1 = nullptr, *ml_val = nullptr, *mu_val = nullptr;
    uint32_t *ml_rp = nullptr, *ml_col = nullptr, *ml_cp = nullptr, *ml_row = nullptr, *ml_pos = nullptr;
    uint32_t *mu_rp = nullptr, *mu_col = nullptr, *mu_cp = nullptr, *mu_row = nullptr, *mu_pos = nullptr;

    void release() {
        void *ptrs[] = {aug_rp, aug_col, aug_diag, cp_ptr, cp_pair, aug_map, f0, f1, ml_val, mu_val,
                        ml_rp, ml_col, ml_cp, ml_row, ml_pos, mu_rp, mu_col, mu_cp, mu_row, mu_pos};
        for (void *p : ptrs) ohm_pool_free(p);
        *this = IsaiDev{};
    }
    template <typename T>
    static cudaError_t put(T **dst, const std::vector<T> &v, cudaStream_t s) {
        cudaError_t e = dalloc(dst, v.size());
        if (e == cudaSuccess && !v.empty()) e = cudaMemcpyAsync(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s);
        return e;
    }
    cudaError_t build(int64_t n, const uint32_t *rp, const uint32_t *col, cudaStream_t s) {
        IsaiHost h;
        h.build(n, rp, col);
        cudaError_t e = put(&aug_rp, h.arp, s);
        if (e == cudaSuccess) e = put(&aug_col, h.acol, s);
        if (e == cudaSuccess) e = put(&aug_diag, h.adiag, s);
        if (e == cudaSuccess) e = put(&aug_map, h.amap, s);
        if (e == cudaSuccess) e = put(&cp_ptr, h.cptr, s);
        if (e == cudaSuccess) e = put(&cp_pair, h.cpair, s);
        if (e == cudaSuccess) e = put(&ml_rp, h.mlrp, s);
        if (e == cudaSuccess) e = put(&ml_col, h.mlcol, s);
        if (e == cudaSuccess) e = put(&ml_cp, h.mlcp, s);
        if (e == cudaSuccess) e = put(&ml_row, h.mlrow, s);
        if (e == cudaSuccess) e = put(&ml_pos, h.mlpos, s);
        if (e == cudaSuccess) e = put(&mu_rp, h.murp, s);
        if (e == cudaSuccess) e = put(&mu_col, h.mucol, s);
        if (e == cudaSuccess) e = put(&mu_cp, h.mucp, s);
        if (e == cudaSuccess) e = put(&mu_row, h.murow, s);
        if (e == cudaSuccess) e = put(&mu_pos, h.mupos, s);
        if (e == cudaSuccess) e = dalloc(&f0, h.nnz_aug);
        if (e == cudaSuccess) e = dalloc(&f1, h.nnz_aug);
        if (e == cudaSuccess) e = dalloc(&ml_val, h.mlcol.size());
        if (e == cudaSuccess) e = dalloc(&mu_val, h.mucol.size());
        // positions a column system leaves out stay zero
        if (e == cudaSuccess) e = cudaMemsetAsync(ml_val, 0, std::max<size_t>(1, h.mlcol.size()) * sizeof(double), s);
        if (e == cudaSuccess) e = cudaMemsetAsync(mu_val, 0, std::max<size_t>(1, h.mucol.size()) * sizeof(double), s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);   // host vectors go out of scope
        ready = e == cudaSuccess;
        return e;
    }
    void bind(KernelArgs &a) const {
        a.aug_rp = aug_rp; a.aug_col = aug_col; a.aug_diag = aug_diag; a.aug_map = aug_map;
        a.cp_ptr = cp_ptr; a.cp_pair = cp_pair; a.isai_f0 = f0; a.isai_f1 = f1;
        a.ml_rp = ml_rp; a.ml_col = ml_col; a.ml_cp = ml_cp; a.ml_row = ml_row; a.ml_pos = ml_pos; a.ml_val = ml_val;
        a.mu_rp = mu_rp; a.mu_col = mu_col; a.mu_cp = mu_cp; a.mu_row = mu_row; a.mu_pos = mu_pos; a.mu_val = mu_val;
    }
};

static int precond_kind(int p) {
    switch (p) {
        case OHM_PRECOND_NONE: return kPcNone;
        case OHM_PRECOND_JACOBI: return kPcJacobi;
        case OHM_PRECOND_ISAI1: return kPcIsai;
        default: return kPcAuto;
    }
}

ohm_status ohm_check_krylov(const ohm_krylov_params *p) {
    if (!p) return fail(OHM_ERR_INVALID_ARG, "params is null");
    if (p->max_iterations <= 0) return fail(OHM_ERR_SOLVE, "BiCGSTAB max_iterations must be > 0");
    if (!(p->tolerance > 0.0) || !std::isfinite(p->tolerance))
        return fail(OHM_ERR_SOLVE, "BiCGSTAB tolerance must be finite and > 0");
    if (p->precision != OHM_PREC_FP64 && p->precision != OHM_PREC_MIXED)
        return fail(OHM_ERR_INVALID_ARG, "unknown precision %d", p->precision);
    if (p->precond < 0 || p->precond > OHM_PRECOND_NONE)
        return fail(OHM_ERR_INVALID_ARG, "unknown preconditioner %d", p->precond);
    return OHM_OK;
}

__global__ void f64_to_f32_kernel(const double *in, float *out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (float)in[i];
}

cudaError_t ohm_f64_to_f32(const double *in, float *out, int64_t n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    f64_to_f32_kernel<<<std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 4096)), 256, 0, s>>>(in, out, n);
    return cudaGetLastError();
}

// -------------------------------------------------------- linear solves --
static ohm_status solve_real_impl(ohm_ctx *c, int64_t n, int64_t nnz, const uint32_t *d_rp, const uint32_t *d_col,
                                  double *d_val, const uint32_t *h_rp, const uint32_t *h_col, const double *h_val,
                                  double *d_b, double *d_x, const ohm_krylov_params *p, ohm_solve_info *info) {
    const bool mixed = p->precision == OHM_PREC_MIXED;
    Workspace ws;
    float *v32 = nullptr;
    int launches = 0;
    ohm_status st = OHM_OK;
    cudaError_t e = ws.alloc(n, c->num_sms);
    if (e == cudaSuccess && mixed) e = dalloc(&v32, nnz);
    if (e != cudaSuccess) { ws.release(); ohm_pool_free(v32); return fail(OHM_ERR_CUDA, "workspace: %s", cudaGetErrorString(e)); }
    PcHost pc;
    build_precond(n, h_rp, h_col, h_val, {}, p->precond == OHM_PRECOND_AUTO, pc);
    e = ws.upload_pc(pc, c->stream);
    IsaiDev isai;
    if (e == cudaSuccess && p->precond == OHM_PRECOND_ISAI1) e = isai.build(n, h_rp, h_col, c->stream);
    if (e == cudaSuccess && mixed && nnz > 0) {
        f64_to_f32_kernel<<<std::max<int64_t>(1, std::min<int64_t>((nnz + 255) / 256, 4096)), 256, 0, c->stream>>>(d_val, v32, nnz);
        e = cudaGetLastError();
        ++launches;
    }
    if (e != cudaSuccess) { ws.release(); ohm_pool_free(v32); return fail(OHM_ERR_CUDA, "setup: %s", cudaGetErrorString(e)); }
    KernelArgs a{};
    a.n = (int)n; a.nnz = (int)nnz;
    a.row_ptr = d_rp; a.col = d_col; a.vals64 = d_val; a.vals32 = v32;
    a.b = d_b; a.x = d_x;
    a.precond = precond_kind(p->precond);
    ws.bind(a);
    if (isai.ready) isai.bind(a);
    a.newton = 0;
    a.mixed = mixed ? 1 : 0;
    a.max_outer = std::max(1, p->max_refinements);
    a.max_krylov = p->max_iterations;
    a.krylov_tol = p->tolerance;
    a.inner_rtol = mixed ? (p->inner_rtol > 0.0 ? p->inner_rtol : 1e-4) : p->inner_rtol;
    a.require_true_residual = p->max_refinements > 1 ? 1 : 0;
    a.max_restarts = std::max(0, p->max_restarts);
    a.fp32_max_iterations = p->fp32_max_iterations > 0 ? p->fp32_max_iterations : p->max_iterations;
    a.eta_max = 0.5;
    st = launch_solver(c, a, nnz, &launches);
    if (st == OHM_OK) st = finish_solver(c, info, launches);
    cudaStreamSynchronize(c->stream);
    ws.release();
    isai.release();
    ohm_pool_free(v32);
    return st;
}

extern "C" ohm_status ohm_solve_real(ohm_ctx *c, int64_t n, int64_t nnz, const uint32_t *row_ptr, const uint32_t *col,
                                     const double *values, const double *b, double *x, const ohm_krylov_params *params,
                                     ohm_solve_info *info) {
    if (!c) return fail(OHM_ERR_INVALID_ARG, "ctx is null");
    ohm_status st = ohm_check_krylov(params);
    if (st != OHM_OK) return st;
    if (n == 0) return OHM_OK;                       // cpu.rs:39-41, gpu.rs:118-120
    if (!b || !x || (nnz && !values)) return fail(OHM_ERR_INVALID_ARG, "null array");
    st = check_csr(n, nnz, row_ptr, col);
    if (st != OHM_OK) return st;
    CUDA_TRY(cudaSetDevice(c->device));
    uint32_t *d_rp = nullptr, *d_col = nullptr;
    double *d_val = nullptr, *d_b = nullptr, *d_x = nullptr;
    cudaError_t e = dalloc(&d_rp, n + 1);
    if (e == cudaSuccess) e = dalloc(&d_col, nnz);
    if (e == cudaSuccess) e = dalloc(&d_val, nnz);
    if (e == cudaSuccess) e = dalloc(&d_b, n);
    if (e == cudaSuccess) e = dalloc(&d_x, n);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_rp, row_ptr, (n + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess && nnz) e = cudaMemcpyAsync(d_col, col, nnz * sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess && nnz) e = cudaMemcpyAsync(d_val, values, nnz * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_b, b, n * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_x, 0, n * sizeof(double), c->stream);
    if (e != cudaSuccess) st = fail(OHM_ERR_CUDA, "upload: %s", cudaGetErrorString(e));
    if (st == OHM_OK) st = solve_real_impl(c, n, nnz, d_rp, d_col, d_val, row_ptr, col, values, d_b, d_x, params, info);
    if (st == OHM_OK) {
        e = cudaMemcpyAsync(x, d_x, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) st = fail(OHM_ERR_CUDA, "download: %s", cudaGetErrorString(e));
    }
    cudaStreamSynchronize(c->stream);
    ohm_pool_free(d_rp); ohm_pool_free(d_col); ohm_pool_free(d_val); ohm_pool_free(d_b); ohm_pool_free(d_x);
    return st;
}

// ------------------------------------------------------------ Newton plan --
static constexpr int kTraceRows = 256;
struct ohm_plan {
    ohm_ctx *ctx = nullptr;
    int64_t n = 0, nnz = 0, nd = 0, nq = 0, nm = 0;
    uint32_t *rp = nullptr, *col = nullptr;
    double *base_vals = nullptr, *vals64 = nullptr, *base_b = nullptr, *b = nullptr;
    float *vals32 = nullptr;
    double *x_prev = nullptr, *x_scratch = nullptr;
    DiodeDesc *diodes = nullptr;
    BjtDesc *bjts = nullptr;
    MosfetDesc *mosfets = nullptr;
    double *vaf = nullptr;
    double *mstamp = nullptr, *rstamp = nullptr;
    int n_mslots = 0, n_rrows = 0;
    uint32_t *mslot = nullptr, *mslot_ptr = nullptr, *mslot_ids = nullptr;
    uint32_t *rrow = nullptr, *rrow_ptr = nullptr, *rrow_ids = nullptr;
    unsigned long long *node_scale = nullptr;
    uint8_t *stampflag = nullptr;      // per row: diagonal / rhs written by the stamp map
    // long rows and long stamp segments (team-cooperative)
    int n_long = 0, n_long_chunks = 0, n_lseg = 0, n_lseg_chunks = 0;
    int64_t nnz_long = 0;              // nonzeros in long rows
    uint8_t *longflag = nullptr, *lseg_flag = nullptr;
    uint32_t *long_row = nullptr, *long_chunk_ptr = nullptr, *long_chunk_owner = nullptr, *long_chunk_beg = nullptr,
             *long_chunk_end = nullptr;
    uint32_t *lseg = nullptr, *lseg_chunk_ptr = nullptr, *lseg_chunk_owner = nullptr, *lseg_chunk_beg = nullptr,
             *lseg_chunk_end = nullptr;
    double *long_part = nullptr, *lseg_part = nullptr;
    double *x_good = nullptr;          // DC continuation: last converged point
    double *trace = nullptr;           // kTraceRows x kTraceCols
    Workspace ws;
    IsaiDev isai;                      // built on the first ISAI(1) solve
    // Host copy of the CSR pattern (ISAI(1) set-up, preconditioner rebuilds
    // when the base changes), downloaded on first use (ensure_host_pattern);
    // the plain Jacobi structure is derived from pc_pairs on first use.
    std::vector<uint32_t> h_rp, h_col;
    std::vector<char> touched;
    PcHost pc_pairs, pc_plain;
    int pc_loaded = -1;     // which structure is on the device
};

static void plan_free(ohm_plan *p) {
    if (!p) return;
    ohm_pool_free(p->rp); ohm_pool_free(p->col); ohm_pool_free(p->base_vals); ohm_pool_free(p->vals64); ohm_pool_free(p->base_b);
    ohm_pool_free(p->b); ohm_pool_free(p->vals32); ohm_pool_free(p->x_prev); ohm_pool_free(p->x_scratch);
    ohm_pool_free(p->diodes); ohm_pool_free(p->bjts); ohm_pool_free(p->mosfets); ohm_pool_free(p->vaf);
    ohm_pool_free(p->mstamp); ohm_pool_free(p->rstamp);
    ohm_pool_free(p->mslot); ohm_pool_free(p->mslot_ptr); ohm_pool_free(p->mslot_ids);
    ohm_pool_free(p->rrow); ohm_pool_free(p->rrow_ptr); ohm_pool_free(p->rrow_ids);
    ohm_pool_free(p->node_scale);
    ohm_pool_free(p->stampflag); ohm_pool_free(p->x_good);
    void *lp[] = {p->longflag, p->lseg_flag, p->long_row, p->long_chunk_ptr, p->long_chunk_owner, p->long_chunk_beg,
                  p->long_chunk_end, p->lseg, p->lseg_chunk_ptr, p->lseg_chunk_owner, p->lseg_chunk_beg,
                  p->lseg_chunk_end, p->long_part, p->lseg_part};
    for (void *q : lp) ohm_pool_free(q);
    ohm_pool_free(p->trace);
    p->ws.release();
    p->isai.release();
    delete p;
}

template <typename T>
static cudaError_t up(T **dst, const T *src, size_t count, cudaStream_t s) {
    cudaError_t e = dalloc(dst, count);
    if (e == cudaSuccess && count && src) e = cudaMemcpyAsync(*dst, src, count * sizeof(T), cudaMemcpyHostToDevice, s);
    return e;
}

static cudaError_t ensure_host_pattern(ohm_plan *p) {
    if (!p->h_rp.empty()) return cudaSuccess;
    cudaStream_t s = p->ctx->stream;
    p->h_rp.resize(p->n + 1);
    p->h_col.resize(p->nnz);
    cudaError_t e = cudaMemcpyAsync(p->h_rp.data(), p->rp, (p->n + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && p->nnz)
        e = cudaMemcpyAsync(p->h_col.data(), p->col, p->nnz * sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { p->h_rp.clear(); p->h_col.clear(); }
    return e;
}

// The point-Jacobi structure: build_precond without pairs, whose diagonal
// slots are the paired structure's.
static void plain_from_pairs(const PcHost &pairs, PcHost &plain) {
    const size_t n = pairs.diag_slot.size();
    plain.partner.assign(n, -1);
    plain.diag_slot = pairs.diag_slot;
    plain.off_slot.assign(n, kSentinel);
    plain.rowflag.assign(n, 0);
    plain.any_pair = false;
}

extern "C" ohm_status ohm_plan_create(ohm_ctx *c, const double *base_g_values, const uint32_t *col_indices,
                                      const uint32_t *row_ptrs, const double *base_b,
                                      const ohm_diode_desc *diodes, int64_t n_diodes, const ohm_bjt_desc *bjts,
                                      int64_t n_bjts, const ohm_mosfet_desc *mosfets, int64_t n_mosfets,
                                      const double *bjt_vaf, int64_t size, int64_t nnz, ohm_plan **out) {
    if (!c || !out) return fail(OHM_ERR_INVALID_ARG, "null ctx or out");
    *out = nullptr;
    if (size <= 0) return fail(OHM_ERR_INVALID_ARG, "system size must be > 0");
    if (!base_g_values || !base_b) return fail(OHM_ERR_INVALID_ARG, "null base values / rhs");
    ohm_status st = check_csr(size, nnz, row_ptrs, col_indices);
    if (st != OHM_OK) return st;
    st = check_devices(diodes, n_diodes, bjts, n_bjts, mosfets, n_mosfets, size, nnz);
    if (st != OHM_OK) return st;
    CUDA_TRY(cudaSetDevice(c->device));
    ohm_plan *p = new (std::nothrow) ohm_plan();
    if (!p) return fail(OHM_ERR_INVALID_ARG, "out of host memory");
    p->ctx = c; p->n = size; p->nnz = nnz; p->nd = n_diodes; p->nq = n_bjts; p->nm = n_mosfets;
    cudaStream_t s = c->stream;

    // the caller's arrays go up first (asynchronous from pinned memory, so
    // the copies overlap the host work below)
    cudaError_t e = up(&p->rp, row_ptrs, size + 1, s);
    if (e == cudaSuccess) e = up(&p->col, col_indices, nnz, s);
    if (e == cudaSuccess) e = up(&p->base_vals, base_g_values, nnz, s);
    if (e == cudaSuccess) e = up(&p->vals64, base_g_values, nnz, s);
    if (e == cudaSuccess) e = dalloc(&p->vals32, nnz);
    if (e == cudaSuccess) e = up(&p->base_b, base_b, size, s);
    if (e == cudaSuccess) e = up(&p->b, base_b, size, s);
    if (e == cudaSuccess) e = up(&p->diodes, (const DiodeDesc *)diodes, n_diodes, s);
    if (e == cudaSuccess) e = up(&p->bjts, (const BjtDesc *)bjts, n_bjts, s);
    if (e == cudaSuccess) e = up(&p->mosfets, (const MosfetDesc *)mosfets, n_mosfets, s);
    if (e == cudaSuccess && bjt_vaf && n_bjts) e = up(&p->vaf, bjt_vaf, n_bjts, s);
    if (e == cudaSuccess && nnz) {
        f64_to_f32_kernel<<<std::max<int64_t>(1, std::min<int64_t>((nnz + 255) / 256, 4096)), 256, 0, s>>>(p->vals64, p->vals32, nnz);
        e = cudaGetLastError();
    }

    // stamp map
    std::vector<std::pair<uint32_t, uint32_t>> mp, rp_;
    const uint32_t base_q = 4u * (uint32_t)n_diodes, base_m = base_q + 9u * (uint32_t)n_bjts;
    const uint32_t rbase_q = 2u * (uint32_t)n_diodes, rbase_m = rbase_q + 3u * (uint32_t)n_bjts;
    for (int64_t k = 0; k < n_diodes; ++k) {
        for (int j = 0; j < 4; ++j) if (diodes[k].g_row_col[j] != kSentinel) mp.push_back({diodes[k].g_row_col[j], (uint32_t)(4 * k + j)});
        for (int j = 0; j < 2; ++j) if (diodes[k].b_idx[j] != kSentinel) rp_.push_back({diodes[k].b_idx[j], (uint32_t)(2 * k + j)});
    }
    for (int64_t k = 0; k < n_bjts; ++k) {
        for (int j = 0; j < 9; ++j) if (bjts[k].g_row_col[j] != kSentinel) mp.push_back({bjts[k].g_row_col[j], base_q + (uint32_t)(9 * k + j)});
        for (int j = 0; j < 3; ++j) if (bjts[k].b_idx[j] != kSentinel) rp_.push_back({bjts[k].b_idx[j], rbase_q + (uint32_t)(3 * k + j)});
    }
    for (int64_t k = 0; k < n_mosfets; ++k) {
        for (int j = 0; j < 6; ++j) if (mosfets[k].g_row_col[j] != kSentinel) mp.push_back({mosfets[k].g_row_col[j], base_m + (uint32_t)(6 * k + j)});
        for (int j = 0; j < 2; ++j) if (mosfets[k].b_idx[j] != kSentinel) rp_.push_back({mosfets[k].b_idx[j], rbase_m + (uint32_t)(2 * k + j)});
    }
    std::vector<uint32_t> ms, mptr, mids, rs, rptr, rids;
    build_stamp_map(mp, ms, mptr, mids);
    build_stamp_map(rp_, rs, rptr, rids);
    p->n_mslots = (int)ms.size();
    p->n_rrows = (int)rs.size();
    p->touched.assign(nnz, 0);
    for (uint32_t sl : ms) p->touched[sl] = 1;
    // the block-Jacobi pairing on a second thread, the flags and splits here
    bool pc_ok = true;
    std::thread pc_thread([&]() {
        try {
            build_precond(size, row_ptrs, col_indices, base_g_values, p->touched, true, p->pc_pairs);
        } catch (...) {
            pc_ok = false;
        }
    });
    std::vector<uint8_t> sflag;
    LongSplit lrows, lsegs;
    bool host_ok = true;
    try {
        sflag = stamp_flags(size, row_ptrs, col_indices, p->touched, rs);
        split_long(size, row_ptrs, kLongRowMin, kLongRowChunk, 0, lrows);
        split_long((int64_t)ms.size(), mptr.data(), kLongSegMin, kLongSegChunk, 0, lsegs);
        split_long((int64_t)rs.size(), rptr.data(), kLongSegMin, kLongSegChunk, (int64_t)ms.size(), lsegs);
    } catch (...) {
        host_ok = false;
    }
    pc_thread.join();
    if (!pc_ok || !host_ok) {
        cudaStreamSynchronize(s);
        plan_free(p);
        return fail(OHM_ERR_INVALID_ARG, "out of host memory");
    }
    p->n_long = (int)lrows.item.size();
    p->n_long_chunks = (int)lrows.chunk_beg.size();
    for (uint32_t r : lrows.item) p->nnz_long += row_ptrs[r + 1] - row_ptrs[r];
    p->n_lseg = (int)lsegs.item.size();
    p->n_lseg_chunks = (int)lsegs.chunk_beg.size();

    if (e == cudaSuccess) e = dalloc(&p->x_prev, size);
    if (e == cudaSuccess) e = dalloc(&p->x_scratch, size);
    if (e == cudaSuccess) e = dalloc(&p->mstamp, 4 * n_diodes + 9 * n_bjts + 6 * n_mosfets);
    if (e == cudaSuccess) e = dalloc(&p->rstamp, 2 * n_diodes + 3 * n_bjts + 2 * n_mosfets);
    if (e == cudaSuccess) e = up(&p->mslot, ms.data(), ms.size(), s);
    if (e == cudaSuccess) e = up(&p->mslot_ptr, mptr.data(), mptr.size(), s);
    if (e == cudaSuccess) e = up(&p->mslot_ids, mids.data(), mids.size(), s);
    if (e == cudaSuccess) e = up(&p->rrow, rs.data(), rs.size(), s);
    if (e == cudaSuccess) e = up(&p->rrow_ptr, rptr.data(), rptr.size(), s);
    if (e == cudaSuccess) e = up(&p->rrow_ids, rids.data(), rids.size(), s);
    if (e == cudaSuccess) e = dalloc(&p->node_scale, size);
    if (e == cudaSuccess) e = up(&p->stampflag, sflag.data(), size, s);
    if (e == cudaSuccess) e = dalloc(&p->x_good, size);
    if (e == cudaSuccess && p->n_long) {
        e = up(&p->longflag, lrows.flag.data(), lrows.flag.size(), s);
        if (e == cudaSuccess) e = up(&p->long_row, lrows.item.data(), lrows.item.size(), s);
        if (e == cudaSuccess) e = up(&p->long_chunk_ptr, lrows.chunk_ptr.data(), lrows.chunk_ptr.size(), s);
        if (e == cudaSuccess) e = up(&p->long_chunk_owner, lrows.chunk_owner.data(), lrows.chunk_owner.size(), s);
        if (e == cudaSuccess) e = up(&p->long_chunk_beg, lrows.chunk_beg.data(), lrows.chunk_beg.size(), s);
        if (e == cudaSuccess) e = up(&p->long_chunk_end, lrows.chunk_end.data(), lrows.chunk_end.size(), s);
        if (e == cudaSuccess) e = dalloc(&p->long_part, lrows.chunk_beg.size());
    }
    if (e == cudaSuccess && p->n_lseg) {
        e = up(&p->lseg_flag, lsegs.flag.data(), lsegs.flag.size(), s);
        if (e == cudaSuccess) e = up(&p->lseg, lsegs.item.data(), lsegs.item.size(), s);
        if (e == cudaSuccess) e = up(&p->lseg_chunk_ptr, lsegs.chunk_ptr.data(), lsegs.chunk_ptr.size(), s);
        if (e == cudaSuccess) e = up(&p->lseg_chunk_owner, lsegs.chunk_owner.data(), lsegs.chunk_owner.size(), s);
        if (e == cudaSuccess) e = up(&p->lseg_chunk_beg, lsegs.chunk_beg.data(), lsegs.chunk_beg.size(), s);
        if (e == cudaSuccess) e = up(&p->lseg_chunk_end, lsegs.chunk_end.data(), lsegs.chunk_end.size(), s);
        if (e == cudaSuccess) e = dalloc(&p->lseg_part, lsegs.chunk_beg.size());
    }
    if (e == cudaSuccess) e = dalloc(&p->trace, (size_t)kTraceRows * kTraceCols);
    if (e == cudaSuccess) e = p->ws.alloc(size, c->num_sms);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        cudaStreamSynchronize(s);
        plan_free(p);
        return fail(OHM_ERR_CUDA, "plan upload: %s", cudaGetErrorString(e));
    }
    ohm_ctx_retain(c);
    *out = p;
    return OHM_OK;
}

extern "C" ohm_status ohm_plan_destroy(ohm_plan *p) {
    if (!p) return OHM_OK;
    ohm_ctx *c = p->ctx;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    plan_free(p);
    ohm_ctx_release(c);
    return OHM_OK;
}

extern "C" ohm_status ohm_plan_set_base(ohm_plan *p, const double *base_g_values, const double *base_b) {
    if (!p) return fail(OHM_ERR_INVALID_ARG, "plan is null");
    cudaStream_t s = p->ctx->stream;
    CUDA_TRY(cudaSetDevice(p->ctx->device));
    if (base_g_values && p->nnz) {
        CUDA_TRY(cudaMemcpyAsync(p->base_vals, base_g_values, p->nnz * sizeof(double), cudaMemcpyHostToDevice, s));
        CUDA_TRY(cudaMemcpyAsync(p->vals64, base_g_values, p->nnz * sizeof(double), cudaMemcpyHostToDevice, s));
        f64_to_f32_kernel<<<std::max<int64_t>(1, std::min<int64_t>((p->nnz + 255) / 256, 4096)), 256, 0, s>>>(p->vals64, p->vals32, p->nnz);
        CUDA_TRY(cudaGetLastError());
        const cudaError_t he = ensure_host_pattern(p);
        if (he != cudaSuccess) return fail(OHM_ERR_CUDA, "pattern download: %s", cudaGetErrorString(he));
        build_precond(p->n, p->h_rp.data(), p->h_col.data(), base_g_values, p->touched, true, p->pc_pairs);
        p->pc_loaded = -1;
    }
    if (base_b) {
        CUDA_TRY(cudaMemcpyAsync(p->base_b, base_b, p->n * sizeof(double), cudaMemcpyHostToDevice, s));
        CUDA_TRY(cudaMemcpyAsync(p->b, base_b, p->n * sizeof(double), cudaMemcpyHostToDevice, s));
    }
    CUDA_TRY(cudaStreamSynchronize(s));
    return OHM_OK;
}

static ohm_status plan_args(ohm_plan *p, const ohm_newton_params *np, double *x_dev, KernelArgs &a);

extern "C" ohm_status ohm_plan_trace(ohm_plan *p, double *out, int32_t max_rows, int32_t *rows) {
    if (!p || !out || max_rows < 0) return fail(OHM_ERR_INVALID_ARG, "bad trace arguments");
    const int r = std::min<int>(max_rows, kTraceRows);
    if (r > 0)
        CUDA_TRY(cudaMemcpyAsync(out, p->trace, (size_t)r * kTraceCols * sizeof(double), cudaMemcpyDeviceToHost,
                                 p->ctx->stream));
    CUDA_TRY(cudaStreamSynchronize(p->ctx->stream));
    if (rows) *rows = r;
    return OHM_OK;
}

static ohm_status plan_args(ohm_plan *p, const ohm_newton_params *np, double *x_dev, KernelArgs &a) {
    const ohm_krylov_params &kp = np->krylov;
    const int want_pc = kp.precond == OHM_PRECOND_AUTO ? 1 : 0;
    if (p->pc_loaded != want_pc) {
        if (!want_pc && p->pc_plain.diag_slot.empty()) plain_from_pairs(p->pc_pairs, p->pc_plain);
        cudaError_t e = p->ws.upload_pc(want_pc ? p->pc_pairs : p->pc_plain, p->ctx->stream);
        if (e != cudaSuccess) return fail(OHM_ERR_CUDA, "preconditioner upload: %s", cudaGetErrorString(e));
        p->pc_loaded = want_pc;
    }
    a = KernelArgs{};
    a.n = (int)p->n; a.nnz = (int)p->nnz;
    a.row_ptr = p->rp; a.col = p->col;
    a.vals64 = p->vals64; a.vals32 = p->vals32;
    a.base_vals = p->base_vals; a.base_b = p->base_b; a.b = p->b;
    a.x = x_dev; a.x_prev = p->x_prev;
    a.precond = precond_kind(kp.precond);
    p->ws.bind(a);
    if (kp.precond == OHM_PRECOND_ISAI1) {
        if (!p->isai.ready) {
            cudaError_t e = ensure_host_pattern(p);
            if (e == cudaSuccess) e = p->isai.build(p->n, p->h_rp.data(), p->h_col.data(), p->ctx->stream);
            if (e != cudaSuccess) return fail(OHM_ERR_CUDA, "ISAI set-up: %s", cudaGetErrorString(e));
        }
        p->isai.bind(a);
    }
    a.nd = (int)p->nd; a.nq = (int)p->nq; a.nm = (int)p->nm;
    a.diodes = p->diodes; a.bjts = p->bjts; a.mosfets = p->mosfets; a.bjt_vaf = p->vaf;
    a.mstamp = p->mstamp; a.rstamp = p->rstamp;
    a.n_mslots = p->n_mslots; a.mslot = p->mslot; a.mslot_ptr = p->mslot_ptr; a.mslot_ids = p->mslot_ids;
    a.n_rrows = p->n_rrows; a.rrow = p->rrow; a.rrow_ptr = p->rrow_ptr; a.rrow_ids = p->rrow_ids;
    a.node_scale = p->node_scale;
    a.newton = 1;
    a.max_outer = np->max_iterations;
    a.abs_tol = np->abs_tol;
    a.rel_tol = np->rel_tol;
    a.max_krylov = kp.max_iterations;
    a.krylov_tol = kp.tolerance;
    const bool mixed = kp.precision == OHM_PREC_MIXED;
    a.mixed = mixed ? 1 : 0;
    a.inner_rtol = mixed ? (kp.inner_rtol > 0.0 ? kp.inner_rtol : 1e-4) : kp.inner_rtol;
    a.max_restarts = std::max(0, kp.max_restarts);
    a.fp32_max_iterations = kp.fp32_max_iterations > 0 ? kp.fp32_max_iterations : kp.max_iterations;
    a.fp32_min_eta = kp.fp32_min_eta_exp > 0 ? std::pow(10.0, -(double)kp.fp32_min_eta_exp) : 0.0;
    a.forcing = np->forcing;
    a.eta_max = np->eta_max > 0.0 ? np->eta_max : 0.5;
    a.trace = p->trace;
    a.trace_cap = kTraceRows;
    a.continuation = np->continuation ? (1 | (np->continuation & OHM_CONT_TEST_PSEUDO)) : 0;
    a.n_nodes = (int)std::min<int64_t>(np->n_nodes, p->n);
    a.stampflag = p->stampflag;
    a.x_good = p->x_good;
    a.n_long = p->n_long; a.n_long_chunks = p->n_long_chunks; a.longflag = p->longflag; a.nnz_long = p->nnz_long;
    a.long_row = p->long_row; a.long_chunk_ptr = p->long_chunk_ptr; a.long_chunk_owner = p->long_chunk_owner;
    a.long_chunk_beg = p->long_chunk_beg; a.long_chunk_end = p->long_chunk_end; a.long_part = p->long_part;
    a.n_lseg = p->n_lseg; a.n_lseg_chunks = p->n_lseg_chunks; a.lseg_flag = p->lseg_flag; a.lseg = p->lseg;
    a.lseg_chunk_ptr = p->lseg_chunk_ptr; a.lseg_chunk_owner = p->lseg_chunk_owner;
    a.lseg_chunk_beg = p->lseg_chunk_beg; a.lseg_chunk_end = p->lseg_chunk_end; a.lseg_part = p->lseg_part;
    return OHM_OK;
}

static ohm_status check_newton(const ohm_newton_params *np) {
    if (!np) return fail(OHM_ERR_INVALID_ARG, "params is null");
    if (np->max_iterations <= 0)
        return fail(OHM_ERR_NEWTON_NOT_CONVERGED, "Newton solver did not converge after 0 iterations");
    if (!(np->abs_tol >= 0.0) || !(np->rel_tol >= 0.0)) return fail(OHM_ERR_INVALID_ARG, "negative tolerance");
    if (np->continuation && np->n_nodes <= 0)
        return fail(OHM_ERR_INVALID_ARG, "continuation needs n_nodes (the node rows of the MNA system)");
    return ohm_check_krylov(&np->krylov);
}

ohm_status ohm_plan_kernel_args(ohm_plan *p, const ohm_newton_params *np, double *x_dev, KernelArgs &a,
                                int64_t *nnz) {
    if (!p) return fail(OHM_ERR_INVALID_ARG, "plan is null");
    ohm_status st = check_newton(np);
    if (st != OHM_OK) return st;
    CUDA_TRY(cudaSetDevice(p->ctx->device));
    st = plan_args(p, np, x_dev, a);
    if (nnz) *nnz = p->nnz;
    return st;
}

ohm_ctx *ohm_plan_context(ohm_plan *p) { return p ? p->ctx : nullptr; }

cudaError_t ohm_plan_restore_rhs(ohm_plan *p) {
    if (!p || p->n == 0) return cudaSuccess;
    return cudaMemcpyAsync(p->b, p->base_b, p->n * sizeof(double), cudaMemcpyDeviceToDevice, p->ctx->stream);
}

extern "C" ohm_status ohm_plan_newton_device(ohm_plan *p, double *x_dev, const ohm_newton_params *np,
                                             ohm_solve_info *info) {
    if (!p || !x_dev) return fail(OHM_ERR_INVALID_ARG, "null plan or x");
    ohm_status st = check_newton(np);
    if (st != OHM_OK) return st;
    ohm_ctx *c = p->ctx;
    CUDA_TRY(cudaSetDevice(c->device));
    if (np->initial_guess)
        CUDA_TRY(cudaMemcpyAsync(x_dev, np->initial_guess, p->n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    KernelArgs a;
    st = plan_args(p, np, x_dev, a);
    if (st != OHM_OK) return st;
    CUDA_TRY(cudaMemsetAsync(p->trace, 0xFF, (size_t)kTraceRows * kTraceCols * sizeof(double), c->stream));
    int launches = 0;
    st = launch_solver(c, a, p->nnz, &launches);
    if (st != OHM_OK) return st;
    return finish_solver(c, info, launches);
}

extern "C" ohm_status ohm_newton_solve(ohm_ctx *c, const double *base_g_values, const uint32_t *col_indices,
                                       const uint32_t *row_ptrs, const double *base_b, const ohm_diode_desc *diodes,
                                       int64_t n_diodes, const ohm_bjt_desc *bjts, int64_t n_bjts,
                                       const ohm_mosfet_desc *mosfets, int64_t n_mosfets, int64_t size, int64_t nnz,
                                       const ohm_newton_params *params, double *x_out, ohm_solve_info *info) {
    if (!x_out) return fail(OHM_ERR_INVALID_ARG, "x_out is null");
    ohm_status st = check_newton(params);
    if (st != OHM_OK) return st;
    ohm_plan *p = nullptr;
    st = ohm_plan_create(c, base_g_values, col_indices, row_ptrs, base_b, diodes, n_diodes, bjts, n_bjts, mosfets,
                         n_mosfets, nullptr, size, nnz, &p);
    if (st != OHM_OK) return st;
    cudaError_t e = cudaMemsetAsync(p->x_scratch, 0, size * sizeof(double), c->stream);
    if (e != cudaSuccess) { plan_free(p); return fail(OHM_ERR_CUDA, "x init: %s", cudaGetErrorString(e)); }
    st = ohm_plan_newton_device(p, p->x_scratch, params, info);
    // The iterate is returned on success; on NewtonNotConverged the caller
    // still gets the last iterate (the reference downloads it, newton.rs:491-512).
    if (st == OHM_OK || st == OHM_ERR_NEWTON_NOT_CONVERGED) {
        e = cudaMemcpyAsync(x_out, p->x_scratch, size * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) st = fail(OHM_ERR_CUDA, "download: %s", cudaGetErrorString(e));
    }
    ohm_plan_destroy(p);
    return st;
}

// ---------------------------------------------------------- ISAI(1) hook --
// One block builds the ILU(0) factor and the ISAI(1) columns (the same
// isai_setup the solver runs) and applies z = M_U (M_L r) to each vector.
__global__ void __launch_bounds__(1024) isai_apply_kernel(KernelArgs a, const double *R, double *Z, double *Y,
                                                          int n_vec) {
    __shared__ double smem[32 * 4];
    BlockTeam g;
    g.r0 = 0; g.r1 = a.n; g.gtid = threadIdx.x; g.gstride = blockDim.x; g.smem = smem;
    if (!isai_setup(a, g)) return;
    const int n = a.n;
    for (int v = 0; v < n_vec; ++v) {
        const double *r = R + (size_t)v * n;
        double *z = Z + (size_t)v * n;
        spmv_rows<1, double>(a.ml_rp, a.ml_col, a.ml_val, (const uint8_t *)nullptr, 0, n,
                             [&](int j, bool) { return r[j]; }, [&](int i, double y) { Y[i] = y; });
        __syncthreads();
        spmv_rows<1, double>(a.mu_rp, a.mu_col, a.mu_val, (const uint8_t *)nullptr, 0, n,
                             [&](int j, bool) { return Y[j]; }, [&](int i, double y) { z[i] = y; });
        __syncthreads();
    }
}

extern "C" ohm_status ohm_isai_apply(ohm_ctx *c, int64_t n, int64_t nnz, const uint32_t *row_ptr, const uint32_t *col,
                                     const double *values, const double *r, double *z, int64_t n_vectors) {
    if (!c) return fail(OHM_ERR_INVALID_ARG, "ctx is null");
    if (n <= 0 || n_vectors < 0 || !r || !z || (nnz && !values)) return fail(OHM_ERR_INVALID_ARG, "bad arguments");
    if (n * std::max<int64_t>(n_vectors, 1) > (int64_t)1 << 28) return fail(OHM_ERR_INVALID_ARG, "too many vectors");
    ohm_status st = check_csr(n, nnz, row_ptr, col);
    if (st != OHM_OK) return st;
    CUDA_TRY(cudaSetDevice(c->device));
    IsaiDev isai;
    uint32_t *d_rp = nullptr, *d_col = nullptr;
    double *d_val = nullptr, *d_r = nullptr, *d_z = nullptr, *d_y = nullptr;
    const size_t nv = (size_t)n * (size_t)n_vectors;
    cudaError_t e = isai.build(n, row_ptr, col, c->stream);
    if (e == cudaSuccess) e = dalloc(&d_rp, n + 1);
    if (e == cudaSuccess) e = dalloc(&d_col, nnz);
    if (e == cudaSuccess) e = dalloc(&d_val, nnz);
    if (e == cudaSuccess) e = dalloc(&d_r, nv);
    if (e == cudaSuccess) e = dalloc(&d_z, nv);
    if (e == cudaSuccess) e = dalloc(&d_y, n);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_rp, row_ptr, (n + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess && nnz) e = cudaMemcpyAsync(d_col, col, nnz * sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess && nnz) e = cudaMemcpyAsync(d_val, values, nnz * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess && nv) e = cudaMemcpyAsync(d_r, r, nv * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) {
        KernelArgs a{};
        a.n = (int)n;
        a.nnz = (int)nnz;
        a.row_ptr = d_rp;
        a.col = d_col;
        a.vals64 = d_val;
        isai.bind(a);
        isai_apply_kernel<<<1, 1024, 0, c->stream>>>(a, d_r, d_z, d_y, (int)n_vectors);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && nv) e = cudaMemcpyAsync(z, d_z, nv * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) st = fail(OHM_ERR_CUDA, "isai apply: %s", cudaGetErrorString(e));
    cudaStreamSynchronize(c->stream);
    ohm_pool_free(d_rp); ohm_pool_free(d_col); ohm_pool_free(d_val); ohm_pool_free(d_r); ohm_pool_free(d_z); ohm_pool_free(d_y);
    isai.release();
    return st;
}

extern "C" ohm_status ohm_solve_real_device(ohm_ctx *c, const ohm_csr *a, const ohm_buf *b, ohm_buf *x,
                                            const ohm_krylov_params *params, ohm_solve_info *info) {
    if (!c || !a || !b || !x) return fail(OHM_ERR_INVALID_ARG, "null argument");
    ohm_status st = ohm_check_krylov(params);
    if (st != OHM_OK) return st;
    if (b->n != a->n || x->n != a->n) return fail(OHM_ERR_INVALID_ARG, "dimension mismatch");
    if (a->n == 0) return OHM_OK;
    CUDA_TRY(cudaSetDevice(c->device));
    // the preconditioner structure is built on the host from the pattern
    std::vector<uint32_t> rp(a->n + 1), col(a->nnz);
    std::vector<double> val(a->nnz);
    CUDA_TRY(cudaMemcpyAsync(rp.data(), a->rp, rp.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
    if (a->nnz) {
        CUDA_TRY(cudaMemcpyAsync(col.data(), a->col, col.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
        CUDA_TRY(cudaMemcpyAsync(val.data(), a->val, val.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    }
    CUDA_TRY(cudaMemsetAsync(x->d, 0, a->n * sizeof(double), c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return solve_real_impl(c, a->n, a->nnz, a->rp, a->col, a->val, rp.data(), col.data(), val.data(), b->d, x->d,
                           params, info);
}

// ------------------------------------------- single steps (NonlinearBackend) --
// evaluate_* + assemble_* (nonlinear.rs:31-150) as stand-alone launches, for
// callers that drive the Newton loop themselves and for the tests.
namespace {

__global__ void eval_devices_kernel(KernelArgs a) {
    const int ndev = a.nd + a.nq + a.nm;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < ndev; k += gridDim.x * blockDim.x) {
        if (k < a.nd) {
            diode_stamps(a.diodes[k], a.x, a.mstamp + 4 * (size_t)k, a.rstamp + 2 * (size_t)k);
        } else if (k < a.nd + a.nq) {
            const int q = k - a.nd;
            const double vaf = a.bjt_vaf ? a.bjt_vaf[q] : __longlong_as_double(0x7ff0000000000000LL);
            bjt_stamps(a.bjts[q], vaf, a.x, a.mstamp + 4 * (size_t)a.nd + 9 * (size_t)q,
                       a.rstamp + 2 * (size_t)a.nd + 3 * (size_t)q);
        } else {
            const int m = k - a.nd - a.nq;
            mosfet_stamps(a.mosfets[m], a.x, a.mstamp + 4 * (size_t)a.nd + 9 * (size_t)a.nq + 6 * (size_t)m,
                          a.rstamp + 2 * (size_t)a.nd + 3 * (size_t)a.nq + 2 * (size_t)m);
        }
    }
}

__global__ void assemble_kernel(KernelArgs a) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < a.n_mslots + a.n_rrows; k += gridDim.x * blockDim.x) {
        if (k < a.n_mslots) {
            const uint32_t slot = a.mslot[k];
            double acc = a.base_vals[slot];
            for (uint32_t j = a.mslot_ptr[k]; j < a.mslot_ptr[k + 1]; ++j) acc += a.mstamp[a.mslot_ids[j]];
            a.vals64[slot] = acc;
            if (a.vals32) a.vals32[slot] = (float)acc;
        } else {
            const int q = k - a.n_mslots;
            const uint32_t row = a.rrow[q];
            double acc = a.base_b[row];
            for (uint32_t j = a.rrow_ptr[q]; j < a.rrow_ptr[q + 1]; ++j) acc += a.rstamp[a.rrow_ids[j]];
            a.b[row] = acc;
        }
    }
}

__global__ void limit_reset_kernel(int n, unsigned long long *scale) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        scale[i] = 0x3FF0000000000000ULL;
}

__global__ void limit_propose_kernel(KernelArgs a) {
    const int ndev = a.nd + a.nq + a.nm;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < ndev; k += gridDim.x * blockDim.x) {
        if (k < a.nd) diode_limit(a.diodes[k], a.x_prev, a.x, a.node_scale);
        else if (k < a.nd + a.nq) bjt_limit(a.bjts[k - a.nd], a.x_prev, a.x, a.node_scale);
        else mosfet_limit(a.mosfets[k - a.nd - a.nq], a.x_prev, a.x, a.node_scale);
    }
}

__global__ void limit_apply_kernel(int n, const double *xo, double *xn, const unsigned long long *scale) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double sc = __longlong_as_double((long long)scale[i]);
        if (sc < 1.0) xn[i] = xo[i] + (xn[i] - xo[i]) * sc;
    }
}

int steps_grid(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 8)); }

}  // namespace

extern "C" ohm_status ohm_plan_assemble(ohm_plan *p, const double *x_host, double *values_out, double *rhs_out) {
    if (!p || !x_host) return fail(OHM_ERR_INVALID_ARG, "null argument");
    ohm_ctx *c = p->ctx;
    cudaStream_t s = c->stream;
    CUDA_TRY(cudaSetDevice(c->device));
    CUDA_TRY(cudaMemcpyAsync(p->x_scratch, x_host, p->n * sizeof(double), cudaMemcpyHostToDevice, s));
    ohm_newton_params np;
    ohm_newton_params_default(&np);
    KernelArgs a;
    ohm_status st = plan_args(p, &np, p->x_scratch, a);
    if (st != OHM_OK) return st;
    const int64_t ndev = p->nd + p->nq + p->nm;
    if (ndev) eval_devices_kernel<<<steps_grid(ndev), 256, 0, s>>>(a);
    if (p->n_mslots + p->n_rrows) assemble_kernel<<<steps_grid(p->n_mslots + p->n_rrows), 256, 0, s>>>(a);
    CUDA_TRY(cudaGetLastError());
    return ohm_plan_download_system(p, values_out, rhs_out);
}

// ------------------------------------------------ internal: adjoint support --
ohm_status ohm_plan_jacobian_device(ohm_plan *p, const double *x_dev, const double *base_vals_dev, double *J_out) {
    if (!p || !x_dev || !J_out) return fail(OHM_ERR_INVALID_ARG, "null argument");
    ohm_ctx *c = p->ctx;
    cudaStream_t s = c->stream;
    ohm_newton_params np;
    ohm_newton_params_default(&np);
    KernelArgs a;
    ohm_status st = plan_args(p, &np, const_cast<double *>(x_dev), a);
    if (st != OHM_OK) return st;
    a.base_vals = base_vals_dev ? base_vals_dev : p->base_vals;
    a.vals64 = J_out;
    a.vals32 = nullptr;
    if (p->nnz) CUDA_TRY(cudaMemcpyAsync(J_out, a.base_vals, p->nnz * sizeof(double), cudaMemcpyDeviceToDevice, s));
    const int64_t ndev = p->nd + p->nq + p->nm;
    if (ndev) eval_devices_kernel<<<steps_grid(ndev), 256, 0, s>>>(a);
    if (p->n_mslots + p->n_rrows) assemble_kernel<<<steps_grid(p->n_mslots + p->n_rrows), 256, 0, s>>>(a);
    CUDA_TRY(cudaGetLastError());
    return OHM_OK;
}

struct ohm_linsys {
    ohm_ctx *ctx = nullptr;
    int64_t n = 0, nnz = 0;
    uint32_t *rp = nullptr, *col = nullptr;
    Workspace ws;
};

ohm_status ohm_linsys_create(ohm_ctx *c, int64_t n, int64_t nnz, const uint32_t *h_rp, const uint32_t *h_col,
                             const double *h_val, ohm_linsys **out) {
    if (!c || !out) return fail(OHM_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    ohm_status st = check_csr(n, nnz, h_rp, h_col);
    if (st != OHM_OK) return st;
    ohm_linsys *L = new ohm_linsys();
    L->ctx = c; L->n = n; L->nnz = nnz;
    PcHost pc;
    build_precond(n, h_rp, h_col, h_val, {}, true, pc);
    cudaError_t e = dalloc(&L->rp, n + 1);
    if (e == cudaSuccess) e = dalloc(&L->col, nnz);
    if (e == cudaSuccess) e = cudaMemcpyAsync(L->rp, h_rp, (n + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess && nnz) e = cudaMemcpyAsync(L->col, h_col, nnz * sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = L->ws.alloc(n, c->num_sms);
    if (e == cudaSuccess) e = L->ws.upload_pc(pc, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        ohm_linsys_destroy(L);
        return fail(OHM_ERR_CUDA, "linear system set-up: %s", cudaGetErrorString(e));
    }
    *out = L;
    return OHM_OK;
}

ohm_status ohm_linsys_solve(ohm_linsys *L, double *d_vals, double *d_b, double *d_x, const ohm_krylov_params *p,
                            ohm_solve_info *info) {
    ohm_status st = ohm_check_krylov(p);
    if (st != OHM_OK) return st;
    if (p->precision != OHM_PREC_FP64 || p->precond == OHM_PRECOND_ISAI1)
        return fail(OHM_ERR_INVALID_ARG, "adjoint solves run in FP64 with block Jacobi, Jacobi or none");
    ohm_ctx *c = L->ctx;
    CUDA_TRY(cudaMemsetAsync(d_x, 0, L->n * sizeof(double), c->stream));
    KernelArgs a{};
    a.n = (int)L->n; a.nnz = (int)L->nnz;
    a.row_ptr = L->rp; a.col = L->col; a.vals64 = d_vals; a.vals32 = nullptr;
    a.b = d_b; a.x = d_x;
    a.precond = precond_kind(p->precond);
    L->ws.bind(a);
    a.newton = 0;
    a.mixed = 0;
    a.max_outer = 1;
    a.max_krylov = p->max_iterations;
    a.krylov_tol = p->tolerance;
    a.inner_rtol = p->inner_rtol;
    a.max_restarts = std::max(0, p->max_restarts);
    a.fp32_max_iterations = p->max_iterations;
    a.eta_max = 0.5;
    int launches = 0;
    st = launch_solver(c, a, L->nnz, &launches);
    if (st == OHM_OK) st = finish_solver(c, info, launches);
    return st;
}

void ohm_linsys_destroy(ohm_linsys *L) {
    if (!L) return;
    cudaStreamSynchronize(L->ctx->stream);
    ohm_pool_free(L->rp);
    ohm_pool_free(L->col);
    L->ws.release();
    delete L;
}

extern "C" ohm_status ohm_plan_download_system(ohm_plan *p, double *values, double *rhs) {
    if (!p) return fail(OHM_ERR_INVALID_ARG, "plan is null");
    cudaStream_t s = p->ctx->stream;
    if (values && p->nnz) CUDA_TRY(cudaMemcpyAsync(values, p->vals64, p->nnz * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (rhs) CUDA_TRY(cudaMemcpyAsync(rhs, p->b, p->n * sizeof(double), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    return OHM_OK;
}

extern "C" ohm_status ohm_plan_limit(ohm_plan *p, const double *x_old_host, double *x_new_inout) {
    if (!p || !x_old_host || !x_new_inout) return fail(OHM_ERR_INVALID_ARG, "null argument");
    ohm_ctx *c = p->ctx;
    cudaStream_t s = c->stream;
    CUDA_TRY(cudaSetDevice(c->device));
    CUDA_TRY(cudaMemcpyAsync(p->x_prev, x_old_host, p->n * sizeof(double), cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaMemcpyAsync(p->x_scratch, x_new_inout, p->n * sizeof(double), cudaMemcpyHostToDevice, s));
    ohm_newton_params np;
    ohm_newton_params_default(&np);
    KernelArgs a;
    ohm_status st = plan_args(p, &np, p->x_scratch, a);
    if (st != OHM_OK) return st;
    limit_reset_kernel<<<steps_grid(p->n), 256, 0, s>>>((int)p->n, p->node_scale);
    const int64_t ndev = p->nd + p->nq + p->nm;
    if (ndev) limit_propose_kernel<<<steps_grid(ndev), 256, 0, s>>>(a);
    limit_apply_kernel<<<steps_grid(p->n), 256, 0, s>>>((int)p->n, p->x_prev, p->x_scratch, p->node_scale);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(x_new_inout, p->x_scratch, p->n * sizeof(double), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    return OHM_OK;
}
