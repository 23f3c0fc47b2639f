// Internal declarations shared by the C-ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <string>

#include "../../include/ohm.h"
#include "solver_kernel.cuh"

using ohm::DeviceInfo;

// Records the message for ohm_last_error() and returns `st`.
ohm_status ohm_fail(ohm_status st, const char *fmt, ...);

#define CUDA_TRY(expr)                                                                      \
    do {                                                                                    \
        cudaError_t e_ = (expr);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return ohm_fail(OHM_ERR_CUDA, "%s failed: %s", #expr, cudaGetErrorString(e_));  \
    } while (0)

// ---------------------------------------------------------------- context --
struct ohm_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    int num_sms = 0;
    // barrier words + info block
    unsigned int *sync_words = nullptr;   // [count, gen, error(int)]
    DeviceInfo *info_dev = nullptr;
    DeviceInfo *info_host = nullptr;      // pinned
    double *dot_scratch = nullptr;        // for ohm_dot
    int krylov_layout = 0;                    // OHM_KRYLOV_LAYOUT_*
    // Objects created on this context (plans, buffers, matrices).  Destroying
    // the context while some are alive defers the release to the last one.
    int live_objects = 0;
    bool destroy_pending = false;
};

// Where a persistent-solver launch puts its barrier words and status block.
struct LaunchTarget {
    int num_sms;
    cudaStream_t stream;
    unsigned int *sync_words;        // 4 words: count, generation, error, spare
    ohm::DeviceInfo *info_dev;
    ohm::DeviceInfo *info_host;      // host copy target (pinned or not)
    int max_grid;                    // 0: no cap beyond the co-residency limit
    int krylov_layout;               // OHM_KRYLOV_LAYOUT_* (0 when not given)
};
ohm_status ohm_launch_persistent(const LaunchTarget &t, ohm::KernelArgs &a, int64_t nnz, int *launches);
ohm_status ohm_finish_persistent(const LaunchTarget &t, ohm_solve_info *info, int launches);
ohm_status ohm_check_krylov(const ohm_krylov_params *p);
// Dynamic shared memory that lets a grid-team kernel `fn` of `grid` blocks
// keep its Krylov slices in shared memory (sets the kernel's limit), or 0.
int ohm_krylov_smem_bytes(const void *fn, int64_t n, int64_t nnz_short, int grid);
// Kernel arguments of a Newton solve on a plan (validated params), its
// context, and the launch of a plan-sized persistent kernel (api.cu).
ohm_status ohm_plan_kernel_args(ohm_plan *p, const ohm_newton_params *np, double *x_dev, ohm::KernelArgs &a,
                                int64_t *nnz);
ohm_ctx *ohm_plan_context(ohm_plan *p);
// Copies the plan's base rhs back into its assembled rhs (a Newton solve
// re-stamps only the rows that devices touch, so a run that assembled
// another rhs into the plan, such as a transient step, must restore it).
cudaError_t ohm_plan_restore_rhs(ohm_plan *p);
// J(x) values of a plan's system at a device x, on base values base_vals_dev
// (the plan's conductance base when null), written to J_out (nnz doubles).
ohm_status ohm_plan_jacobian_device(ohm_plan *p, const double *x_dev, const double *base_vals_dev, double *J_out);
// A device linear system of fixed pattern (uploaded once, with its
// preconditioner structure and Krylov workspace) solved for new values and
// right-hand sides; FP64.  x starts from zero.
struct ohm_linsys;
ohm_status ohm_linsys_create(ohm_ctx *c, int64_t n, int64_t nnz, const uint32_t *h_rp, const uint32_t *h_col,
                             const double *h_val, ohm_linsys **out);
ohm_status ohm_linsys_solve(ohm_linsys *L, double *d_vals, double *d_b, double *d_x, const ohm_krylov_params *p,
                            ohm_solve_info *info);
void ohm_linsys_destroy(ohm_linsys *L);
cudaError_t ohm_f64_to_f32(const double *in, float *out, int64_t n, cudaStream_t s);

// Child-object bookkeeping (see ohm_ctx::live_objects).
void ohm_ctx_retain(ohm_ctx *c);
void ohm_ctx_release(ohm_ctx *c);

struct ohm_buf {
    ohm_ctx *ctx;
    double *d;
    int64_t n;
};

struct ohm_csr {
    ohm_ctx *ctx;
    int64_t n, nnz;
    uint32_t *rp, *col;
    double *val;
};

// Device memory of the library's buffers comes from a per-device cache
// (pool.cu).  Every buffer is released with ohm_pool_free after the work on
// it has completed (the owner synchronises its stream first).
cudaError_t ohm_pool_alloc(void **p, size_t bytes);
void ohm_pool_free(void *p);
void ohm_pool_trim(int device);

template <typename T>
inline cudaError_t dalloc(T **p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    return ohm_pool_alloc((void **)p, count * sizeof(T));
}

