/*
 * ohm.h - C ABI of the B200-native Ohmnivore hot path (libohm_b200.so).
 *
 * This library replaces the reference's per-Newton-iteration solver layer
 * (the src/solver/ Rust modules of winstanley-industries/ohmnivore): device evaluation and
 * MNA stamping, CSR SpMV, and BiCGSTAB with Jacobi or ISAI(1)
 * preconditioning, run as persistent sm_100a kernels.  Every entry point
 * takes plain pointers and sizes; host arrays are caller-owned, device
 * objects are owned by the context that created them.
 *
 * Threading: a context is single-threaded, like the reference's backends
 * (src/solver/backend.rs:205-209 hold Cell counters and are not Sync).
 * Errors: every call returns an ohm_status; ohm_last_error() gives the text
 * of the last failure on the calling thread.  No call aborts the process.
 */
#ifndef OHM_H
#define OHM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes: OhmnivoreError (src/error.rs:4-33) ------------------ */
typedef enum {
    OHM_OK = 0,
    OHM_ERR_SOLVE = 1,                 /* OhmnivoreError::Solve (breakdown, no convergence, singular) */
    OHM_ERR_NEWTON_NOT_CONVERGED = 2,  /* OhmnivoreError::NewtonNotConverged{iterations, max_residual} */
    OHM_ERR_NEWTON_NUMERICAL = 3,      /* OhmnivoreError::NewtonNumericalError{iteration} */
    OHM_ERR_COMPILE = 4,               /* OhmnivoreError::Compile (descriptor / CSR validation) */
    OHM_ERR_TIMEOUT = 5,               /* a bounded device wait gave up (no OhmnivoreError twin) */
    OHM_ERR_INVALID_ARG = 6,           /* bad pointer, size or parameter */
    OHM_ERR_CUDA = 7,                  /* CUDA runtime failure */
    OHM_ERR_TIMESTEP = 8               /* OhmnivoreError::Timestep */
} ohm_status;

/* Detail code of an OHM_ERR_SOLVE from the Krylov solver; the status words of
 * the reference's fused kernel (src/solver/ds_backend.rs:71-76) plus the
 * breakdown kinds of src/solver/bicgstab.rs:107-182. */
typedef enum {
    OHM_KRYLOV_RUNNING = 0,
    OHM_KRYLOV_CONVERGED = 1,
    OHM_KRYLOV_MAXITER = 2,            /* "did not converge within N iterations" */
    OHM_KRYLOV_BREAKDOWN_RHO = 3,      /* "breakdown: rho ~ 0" */
    OHM_KRYLOV_BREAKDOWN_RV = 4,       /* "breakdown: r_hat.v ~ 0" */
    OHM_KRYLOV_BREAKDOWN_TT = 5,       /* "breakdown: ||t|| ~ 0" */
    OHM_KRYLOV_BREAKDOWN_OMEGA = 6,    /* "breakdown: omega ~ 0" */
    OHM_KRYLOV_NAN = 7                 /* "diverged: NaN/Inf in residual" */
} ohm_krylov_code;

typedef enum {
    OHM_PREC_FP64 = 0,   /* FP64 Krylov (the plain path) */
    OHM_PREC_MIXED = 1   /* FP32 Krylov bulk, FP64 dots, FP64 residual / Newton update */
} ohm_precision;

typedef enum {
    OHM_PRECOND_AUTO = 0,    /* block Jacobi: 1x1, 2x2 for zero-diagonal branch rows paired with
                                their node row, identity for unpaired zero-diagonal rows */
    OHM_PRECOND_JACOBI = 1,  /* reference Jacobi: 1/a_ii, 0 where |a_ii| <= 1e-30 (gpu.rs:177-190) */
    OHM_PRECOND_ISAI1 = 2,   /* ISAI(1) from ILU(0) factors, z = M_U (M_L r) (gpu.rs:139-168) */
    OHM_PRECOND_NONE = 3
} ohm_precond;

/* ---- device descriptors: byte-identical to src/compiler.rs:46-149 ------- */
typedef struct {                 /* GpuDiodeDescriptor, 48 bytes */
    uint32_t anode_idx, cathode_idx;
    float is_val, n_vt;
    uint32_t g_row_col[4];       /* [aa, cc, ac, ca] CSR value indices, UINT32_MAX = ground */
    uint32_t b_idx[2];           /* [anode, cathode] */
    uint32_t padding[2];
} ohm_diode_desc;

typedef struct {                 /* GpuBjtDescriptor, 96 bytes */
    uint32_t collector_idx, base_idx, emitter_idx;
    float polarity, is_val, bf, br, nf_vt, nr_vt;
    uint32_t node_fixed[3];
    uint32_t g_row_col[9];       /* [CC, CB, CE, BC, BB, BE, EC, EB, EE] */
    uint32_t b_idx[3];           /* [C, B, E] */
} ohm_bjt_desc;

typedef struct {                 /* GpuMosfetDescriptor, 64 bytes */
    uint32_t drain_idx, gate_idx, source_idx;
    float polarity, vto, kp, lambda;
    uint32_t node_fixed_packed;  /* bit0 drain, bit1 gate, bit2 source */
    uint32_t g_row_col[6];       /* [DD, DG, DS, SD, SG, SS] */
    uint32_t b_idx[2];           /* [D, S] */
} ohm_mosfet_desc;

/* ---- parameters --------------------------------------------------------- */
typedef struct {                 /* BiCgStabParams (src/solver/bicgstab.rs:14-27) + extensions */
    int32_t max_iterations;      /* default 10000 (bicgstab.rs:10) */
    double tolerance;            /* ||r|| < tolerance * ||b||, default 1e-5 (bicgstab.rs:11) */
    int32_t precision;           /* ohm_precision */
    int32_t precond;             /* ohm_precond */
    double inner_rtol;           /* mixed: inner FP32 solve also stops at inner_rtol*||r0||; 0 = off */
    int32_t max_refinements;     /* linear solves: FP64 iterative-refinement sweeps (>= 1);
                                    > 1 also requires the FP64 residual to meet the tolerance */
    int32_t max_restarts;        /* restarts with r_hat = r after a rho or r_hat.v breakdown;
                                    0 = the reference's breakdown error; default 50 */
    int32_t fp32_max_iterations; /* mixed: iterations of an FP32 attempt before the solve is
                                    redone in FP64 (unless it reduced ||r|| by 2x); default 600 */
    int32_t fp32_min_eta_exp;    /* mixed Newton: a linear solve whose inner tolerance is below
                                    10^-fp32_min_eta_exp goes straight to FP64 (FP32 BiCGSTAB
                                    stagnates short of tight tolerances on ill-conditioned
                                    systems); 0 = always try FP32 first (default) */
} ohm_krylov_params;

typedef enum {
    OHM_FORCING_CONSTANT = 0,    /* inner tolerance = krylov.inner_rtol */
    OHM_FORCING_EW = 1           /* Eisenstat-Walker (choice 2), floor krylov.inner_rtol */
} ohm_forcing;

/* ohm_newton_params.continuation flag for tests of the pseudo-transient stage */
#define OHM_CONT_TEST_PSEUDO 2

typedef struct {                 /* NewtonParams (src/solver/newton.rs:34-55) + extensions */
    int32_t max_iterations;      /* default 50 */
    double abs_tol;              /* converged when max|x - x_old| < abs_tol (+ rel_tol*max|x|); default 1e-4 */
    double rel_tol;              /* extension, default 0 */
    ohm_krylov_params krylov;    /* linear sub-solve; reference default tolerance 1e-5 */
    const double *initial_guess; /* NewtonParams::initial_guess, host pointer, may be NULL */
    int32_t forcing;             /* ohm_forcing, default constant */
    double eta_max;              /* Eisenstat-Walker upper bound, default 0.5 */
    int32_t continuation;        /* 1: when the direct solve fails, run the reference's DC strategy on
                                    the device (src/analysis/dc.rs:60-290): source stepping (MOSFET
                                    circuits), GMIN stepping, pseudo-transient continuation; default 0.
                                    | OHM_CONT_TEST_PSEUDO (testing): the true-GMIN solve that ends GMIN
                                    stepping counts as failed, so pseudo-transient continuation runs */
    int32_t n_nodes;             /* node rows (the first rows of the MNA system); required with
                                    continuation, which adds GMIN to their diagonals */
} ohm_newton_params;

typedef struct {
    int32_t status;              /* ohm_status of the solve */
    int32_t krylov_code;         /* ohm_krylov_code of the last linear solve */
    int32_t iterations;          /* Newton iterations (or Krylov iterations for linear solves) */
    int32_t error_iteration;     /* NewtonNumericalError{iteration} */
    int64_t krylov_iterations;   /* total BiCGSTAB iterations */
    int32_t fp64_fallbacks;      /* mixed: FP32 Krylov solves redone in FP64 */
    int32_t krylov_restarts;     /* BiCGSTAB restarts after a breakdown */
    double max_residual;         /* last max|x - x_old| (NewtonNotConverged{max_residual}) */
    double final_residual_norm;  /* ||b - A x||_2 at exit (FP64), when computed */
    double b_norm;               /* ||b||_2 of the last linear system */
    int64_t kernel_launches;     /* kernels this call launched */
    int32_t continuation_steps;  /* Newton runs of the DC continuation after the direct attempt */
    int32_t continuation_kind;   /* last continuation stage: 0 none, 1 source, 2 GMIN, 3 pseudo-transient */
} ohm_solve_info;

/* Reference defaults; fill before changing fields. */
void ohm_krylov_params_default(ohm_krylov_params *p);
void ohm_newton_params_default(ohm_newton_params *p);

/* ---- context ------------------------------------------------------------ */
typedef struct ohm_ctx ohm_ctx;
typedef struct ohm_buf ohm_buf;      /* SolverBackend::Buffer: FP64 device vector */
typedef struct ohm_csr ohm_csr;      /* GpuCsrMatrix: device CSR (u32 indices, FP64 values) */
typedef struct ohm_plan ohm_plan;    /* device-resident nonlinear system (Newton plan) */

const char *ohm_last_error(void);
const char *ohm_version(void);

/* One context = one CUDA device + one stream (WgpuDsBackend::new, ds_backend.rs).
 * Destroying a context while plans, buffers or matrices created on it are
 * alive is allowed: the context is released when the last of them is. */
ohm_status ohm_ctx_create(int device, ohm_ctx **out);
ohm_status ohm_ctx_destroy(ohm_ctx *ctx);
ohm_status ohm_ctx_synchronize(ohm_ctx *ctx);
/* The CUDA stream (cudaStream_t) the context launches on. */
void *ohm_ctx_stream(ohm_ctx *ctx);
/* Where the Krylov solves of this context's single-system solver keep their
 * working set (no counterpart in the reference, whose BiCGSTAB is a sequence
 * of dispatches; a tuning and testing switch):
 *   OHM_KRYLOV_LAYOUT_AUTO     each block's CSR slice and Krylov state in
 *                              shared memory where the slice fits, else in
 *                              global memory (default)
 *   OHM_KRYLOV_LAYOUT_GLOBAL   global memory for every block: the path of
 *                              systems too large for the slices, at any size
 * The two give the same iterates bit for bit.  Batches, transients and the
 * allocation-free solve keep their own choice. */
#define OHM_KRYLOV_LAYOUT_AUTO 0
#define OHM_KRYLOV_LAYOUT_GLOBAL 1
ohm_status ohm_ctx_set_krylov_layout(ohm_ctx *ctx, int32_t layout);

/* ---- SolverBackend (src/solver/backend.rs:51-96) ------------------------ */
ohm_status ohm_buf_create(ohm_ctx *ctx, int64_t n, ohm_buf **out);            /* new_buffer (zeroed) */
ohm_status ohm_buf_destroy(ohm_buf *buf);
ohm_status ohm_buf_upload(ohm_ctx *ctx, ohm_buf *buf, const double *host, int64_t n);   /* upload_vec */
ohm_status ohm_buf_download(ohm_ctx *ctx, const ohm_buf *buf, double *host, int64_t n); /* download_vec */
double *ohm_buf_device_ptr(ohm_buf *buf);
ohm_status ohm_csr_upload(ohm_ctx *ctx, int64_t n, int64_t nnz, const uint32_t *row_ptr,
                          const uint32_t *col, const double *values, ohm_csr **out); /* upload_matrix */
ohm_status ohm_csr_update_values(ohm_ctx *ctx, ohm_csr *m, const double *values, int64_t nnz);
ohm_status ohm_csr_destroy(ohm_csr *m);
ohm_status ohm_spmv(ohm_ctx *ctx, const ohm_csr *a, const ohm_buf *x, ohm_buf *y);       /* spmv */
ohm_status ohm_dot(ohm_ctx *ctx, const ohm_buf *a, const ohm_buf *b, double *out);      /* dot -> f64 */
/* dot_n (backend.rs:60-68): x . y over the first n entries only (the owned
 * rows of a buffer that also holds halo entries); n <= both lengths. */
ohm_status ohm_dot_n(ohm_ctx *ctx, const ohm_buf *a, const ohm_buf *b, int64_t n, double *out);
ohm_status ohm_axpy(ohm_ctx *ctx, double alpha, const ohm_buf *x, ohm_buf *y);          /* y += a x */
ohm_status ohm_copy(ohm_ctx *ctx, const ohm_buf *src, ohm_buf *dst);                    /* copy */
ohm_status ohm_scale(ohm_ctx *ctx, double alpha, ohm_buf *x);                            /* scale */

/* ---- LinearSolver::solve_real (src/solver/mod.rs:27-34, gpu.rs:107-208) --
 * Host CSR (u32 indices as uploaded by gpu.rs:124-125) and host b / x.
 * x is written on success.  Runs right-preconditioned BiCGSTAB
 * (bicgstab.rs:56-189) as one persistent kernel. */
ohm_status ohm_solve_real(ohm_ctx *ctx, int64_t n, int64_t nnz, const uint32_t *row_ptr,
                          const uint32_t *col, const double *values, const double *b,
                          double *x, const ohm_krylov_params *params, ohm_solve_info *info);

/* ISAI(1) preconditioner of A (host CSR) built on the device, applied to
 * n_vectors host vectors r (n doubles each): z = M_U (M_L r).  M_L, M_U are
 * the level-1 incomplete sparse approximate inverses of the ILU(0) factors
 * (reference: compute_isai, src/solver/preconditioner.rs:239-277, and the
 * apply of src/solver/gpu.rs:159-162).  For testing the set-up; one block. */
ohm_status ohm_isai_apply(ohm_ctx *ctx, int64_t n, int64_t nnz, const uint32_t *row_ptr, const uint32_t *col,
                          const double *values, const double *r, double *z, int64_t n_vectors);

/* Same on device-resident operands (no host copies). */
ohm_status ohm_solve_real_device(ohm_ctx *ctx, const ohm_csr *a, const ohm_buf *b, ohm_buf *x,
                                 const ohm_krylov_params *params, ohm_solve_info *info);

/* The solve of ohm_solve_real for callers that cannot allocate device memory
 * (no counterpart in the reference).  Some callers run inside another
 * program's device-memory budget, or on a path where cudaMalloc/cudaFree would
 * synchronise the device or fail under memory pressure; this entry point
 * calls neither.  The caller passes device pointers for the CSR, b and the
 * output x, and the stream to run on (NULL = the default stream), on the
 * current device.  All other working memory is one fixed file-scope device
 * array of about 6.2 MB, held by every GPU that loads the library until the
 * process exits; systems above 32768 rows or 262144 nonzeros are rejected
 * with OHM_ERR_INVALID_ARG.  The first call on a device looks up that
 * device's address of the array: make it before any stream capture.  Every
 * call shares the array, so calls that overlap on the GPU race; x and all
 * state that must start at zero are cleared by each call.  Each call
 * synchronises the stream (it reads the CSR check back before the solve and
 * the status after it) and returns when the solve has finished. */
ohm_status ohm_solve_real_noalloc(void *stream, int64_t n, int64_t nnz, const uint32_t *d_row_ptr,
                                  const uint32_t *d_col, const double *d_values, const double *d_b,
                                  double *d_x, const ohm_krylov_params *params, ohm_solve_info *info);

/* ---- newton_solve (src/solver/newton.rs:65-78) ---------------------------
 * Argument order follows the reference.  x_out receives the solution
 * (size entries).  The whole Newton loop (evaluate, stamp, solve, limit,
 * converge) runs on the device as one persistent kernel. */
ohm_status ohm_newton_solve(ohm_ctx *ctx, const double *base_g_values, const uint32_t *col_indices,
                            const uint32_t *row_ptrs, const double *base_b,
                            const ohm_diode_desc *diodes, int64_t n_diodes,
                            const ohm_bjt_desc *bjts, int64_t n_bjts,
                            const ohm_mosfet_desc *mosfets, int64_t n_mosfets,
                            int64_t size, int64_t nnz, const ohm_newton_params *params,
                            double *x_out, ohm_solve_info *info);

/* Device-resident Newton plan: uploads the system once, runs many solves.
 * bjt_vaf: optional per-BJT Early voltage (extension, NULL or +inf = none). */
ohm_status ohm_plan_create(ohm_ctx *ctx, const double *base_g_values, const uint32_t *col_indices,
                           const uint32_t *row_ptrs, const double *base_b,
                           const ohm_diode_desc *diodes, int64_t n_diodes,
                           const ohm_bjt_desc *bjts, int64_t n_bjts,
                           const ohm_mosfet_desc *mosfets, int64_t n_mosfets,
                           const double *bjt_vaf, int64_t size, int64_t nnz, ohm_plan **out);
ohm_status ohm_plan_destroy(ohm_plan *plan);
/* Replace base values / base rhs (e.g. GMIN stepping, a new timestep). NULL keeps. */
ohm_status ohm_plan_set_base(ohm_plan *plan, const double *base_g_values, const double *base_b);
/* Run Newton.  x_inout: device pointer (size doubles) holding the initial
 * guess (if params->initial_guess is NULL the device x is used as is) and
 * receiving the solution. */
ohm_status ohm_plan_newton_device(ohm_plan *plan, double *x_inout_device,
                                  const ohm_newton_params *params, ohm_solve_info *info);
/* Per-Newton-iteration record of the last ohm_plan_newton_device call, 6
 * doubles per iteration: FP32 Krylov iterations, FP64 Krylov iterations,
 * ||b - J x|| before the solve, inner tolerance, max|x - x_old|, restarts
 * (rows after the last iteration are NaN).  Stats::bicgstab_iters_per_newton
 * (src/stats.rs) is the reference counterpart. */
ohm_status ohm_plan_trace(ohm_plan *plan, double *out, int32_t max_rows, int32_t *rows);
/* Device-side system matrix / rhs of the last assembly (for tests). */
ohm_status ohm_plan_download_system(ohm_plan *plan, double *values, double *rhs);
/* Evaluate + stamp at x (host), return J values and b_eq (host): one assembly. */
ohm_status ohm_plan_assemble(ohm_plan *plan, const double *x_host, double *values_out, double *rhs_out);
/* One limiting step: x_new_inout (host) is damped against x_old (host). */
ohm_status ohm_plan_limit(ohm_plan *plan, const double *x_old_host, double *x_new_inout);

/* --------------------------------------------------------------------- AC --
 * AC sweep (src/analysis/ac.rs:25-78): for every frequency f solve
 * (G + j 2 pi f C) x = b_ac (sparse.rs:149-178 forms the matrix; gpu.rs:210-700
 * is the reference's complex Jacobi BiCGSTAB, one frequency at a time).  Here
 * all points are solved by one launch, one thread block per point, in FP64
 * complex arithmetic.  c_values lie on the pattern of g_values (NULL: no C);
 * b and x are interleaved (re, im); x_re_im holds n_freq x n complex values.
 * Like the reference, the devices are not linearised: pass the Jacobian
 * values of a DC operating point as g_values for a small-signal analysis.
 * params: tolerance / iteration limit / restarts / preconditioner (AUTO:
 * complex block Jacobi with 2x2 blocks for branch rows; JACOBI: the
 * reference's inverse diagonal).  Returns OHM_ERR_SOLVE naming the first
 * point that did not converge (the reference returns its last iterate). */
typedef struct {
    int32_t krylov_code;         /* ohm_krylov_code */
    int32_t iterations;
    int32_t restarts;
    int32_t reserved;
    double residual_norm;        /* ||r|| of the recurrence at exit */
    double b_norm;
} ohm_ac_point_info;

ohm_status ohm_ac_sweep(ohm_ctx *ctx, int64_t n, int64_t nnz, const uint32_t *row_ptr, const uint32_t *col,
                        const double *g_values, const double *c_values, const double *b_re_im, int64_t n_freq,
                        const double *freqs_hz, const ohm_krylov_params *params, double *x_re_im,
                        ohm_ac_point_info *points);

/* LinearSolver::solve_complex (src/solver/mod.rs:27-34, gpu.rs:210-735):
 * A x = b for a complex CSR matrix (values and vectors as interleaved re, im
 * doubles), the AC sweep's complex BiCGSTAB on one point (G = Re A,
 * C = Im A, w = 1).  Stops when ||b - A x|| < tolerance ||b||; an
 * unconverged solve is OHM_ERR_SOLVE with info->krylov_code.  info may be
 * NULL. */
ohm_status ohm_solve_complex(ohm_ctx *ctx, int64_t n, int64_t nnz, const uint32_t *row_ptr, const uint32_t *col,
                             const double *values_re_im, const double *b_re_im, double *x_re_im,
                             const ohm_krylov_params *params, ohm_ac_point_info *info);

/* -------------------------------------------------------------- transient --
 * Fixed-step backward-Euler transient with a Newton solve per step, run on
 * the device.  The reference's transient (src/analysis/transient.rs:25-210)
 * is linear only: it forms A = G + C/h and b = b(t_n) + (C/h) x_{n-1} per BE
 * step (:285-333) and ignores nonlinear devices; this engine uses the same
 * companion system as the base of a Newton solve (device evaluation and
 * stamping on top of it) at every step.  ohm_transient_run takes fixed BE
 * steps; ohm_transient_run_adaptive below is the reference's adaptive BE/TRAP
 * step control (:84-178).
 *
 * Time-dependent sources (collect_source_info / evaluate_b_at_time,
 * transient.rs:212-280, and transient_source.rs:8-118): b(t) is the sum over
 * sources of sign * value(t) at their rhs rows; a source without a transient
 * function contributes its DC value. */
typedef enum {
    OHM_TRAN_DC = -1,
    OHM_TRAN_PULSE = 0,   /* p = v1, v2, td, tr, tf, pw, per */
    OHM_TRAN_SIN = 1,     /* p = vo, va, freq, td, theta */
    OHM_TRAN_PWL = 2,     /* (t, v) pairs at pwl_points[2*pwl_offset ...] */
    OHM_TRAN_EXP = 3      /* p = v1, v2, td1, tau1, td2, tau2 */
} ohm_tran_kind;

typedef struct {
    int32_t kind;                /* ohm_tran_kind */
    int32_t n_rows;              /* rhs entries: 1 (voltage source branch) or 1-2 (current source) */
    uint32_t rows[2];
    double sign[2];
    double dc;                   /* value of an OHM_TRAN_DC source */
    double p[7];
    int32_t pwl_offset, pwl_count;
} ohm_source;

typedef struct {
    int32_t status;              /* ohm_status of the run */
    int32_t steps_done;          /* accepted steps */
    int32_t failed_step;         /* step whose Newton solve failed, -1 if none */
    int32_t krylov_code;
    int64_t newton_iterations;   /* over all steps */
    int64_t krylov_iterations;
    int32_t fp64_fallbacks;
    int32_t launches;            /* kernel launches (one per steps_per_launch steps) */
    int32_t graph;               /* 1: the launches ran as one CUDA graph */
    int32_t reserved;
    double max_residual;         /* max|dx| of the last Newton iteration of a failed step */
} ohm_transient_info;

typedef struct ohm_transient ohm_transient;
/* C: capacitance / inductance matrix in its own CSR (n rows, the plan's size);
 * each of its entries must lie on the plan's conductance pattern.  probes:
 * rows of x recorded after every step. */
ohm_status ohm_transient_create(ohm_plan *plan, int64_t c_nnz, const uint32_t *c_row_ptr, const uint32_t *c_col,
                                const double *c_values, const ohm_source *sources, int32_t n_sources,
                                const double *pwl_points, int32_t n_pwl_points, const uint32_t *probe_rows,
                                int32_t n_probes, ohm_transient **out);
ohm_status ohm_transient_destroy(ohm_transient *tr);
/* n_steps BE steps of size h from t0: x_inout_device holds x(t0) (e.g. the DC
 * operating point) and receives x(t0 + n_steps h).  Each launch runs
 * steps_per_launch steps in one persistent kernel; use_graph = 1 records
 * the launches (and the waveform download) as one CUDA graph and replays it.
 * waveforms_host (may be NULL): n_steps x n_probes doubles, row-major.  The
 * plan's assembled system is restored to its base afterwards. */
ohm_status ohm_transient_run(ohm_transient *tr, double *x_inout_device, double t0, double h, int32_t n_steps,
                             int32_t steps_per_launch, const ohm_newton_params *params, int32_t use_graph,
                             double *waveforms_host, ohm_transient_info *info);
/* Newton start of each step of ohm_transient_run after the first: order 0
 * (default) x_{n-1}; order 1 the linear extrapolation 2 x_{n-1} - x_{n-2};
 * order 2 the quadratic 3 x_{n-1} - 3 x_{n-2} + x_{n-3} from the third step
 * on (linear on the second).  All converge to the same backward-Euler
 * solution; an extrapolation usually needs fewer Newton iterations.  (The transient adjoint always
 * starts from x_{n-1}, so its checkpointed recomputation is exact.) */
ohm_status ohm_transient_set_predictor(ohm_transient *tr, int32_t order);

/* Adaptive BE / TRAP run of the reference's transient::run
 * (src/analysis/transient.rs:77-178) from t = 0 to tstop: the first step and
 * the step after a rejection are backward Euler; every other step solves
 * the trapezoidal companion system (A = G + 2C/h, b = b(t_n) + (2C/h) x -
 * f(x) + b(t_{n-1}), :336-352) and the BE one from the same x, estimates
 * LTE = (2/3) max|x_trap - x_be| (:355-362) and accepts x_trap when
 * LTE <= 1e-3, else retries with a smaller h; h_min = tstep / 10^4,
 * h_max = tstep.  f(x) = G x + i(x): G x in the reference (linear
 * circuits), plus the device currents here, where every solve is a Newton
 * solve on the companion base.  x_inout_device holds x(0) and receives the
 * last accepted x.  Output points: (0, x(0)) when tstart <= 0, then every
 * accepted step with t >= tstart; the first max_points are written to
 * times_host (max_points doubles) and waveforms_host (max_points x n_probes,
 * row-major), either may be NULL; info->points counts them all, so a run
 * with info->points > max_points was truncated and can be repeated with a
 * larger capacity.  The whole run is one cooperative launch.  Errors:
 * OHM_ERR_TIMESTEP as transient.rs:128-133, a failed Newton solve as in
 * ohm_transient_run (info->failed_solve 1 = TRAP, 2 = BE). */
typedef struct {
    int32_t status;
    int32_t accepted;            /* Stats::timesteps_accepted */
    int32_t rejected;            /* Stats::timesteps_rejected */
    int32_t points;              /* output points produced (kept: min(points, max_points)) */
    int64_t newton_iterations;
    int64_t krylov_iterations;
    int32_t linear_solves;       /* companion solves: 1 per BE step, 2 per TRAP step (Stats::linear_solves) */
    int32_t fp64_fallbacks;
    int32_t krylov_code;
    int32_t failed_solve;        /* 0 none, 1 TRAP, 2 BE */
    double t_end;                /* time reached */
    double h_last;               /* step size at the end */
    double t_failed;             /* time of a failed solve (target) or of the timestep failure */
    double max_residual;         /* max|dx| of the last Newton iteration of a failed solve */
} ohm_adaptive_info;

ohm_status ohm_transient_run_adaptive(ohm_transient *tr, double *x_inout_device, double tstep, double tstop,
                                      double tstart, const ohm_newton_params *params, int32_t max_points,
                                      double *times_host, double *waveforms_host, ohm_adaptive_info *info);

/* ---------------------------------------------------------------- adjoint --
 * Sensitivities of one output o = w . x (w = do/dx, host, size n) with
 * respect to every resistance, capacitance, diode saturation current and
 * MOSFET threshold |VTO| and transconductance KP, by the adjoint method; no
 * counterpart in the reference.
 *
 * DC: J(x)^T lambda = w at the operating point x (the BiCGSTAB of this
 * library on the transposed CSR), then do/dp = -lambda^T dF/dp, back-stamped
 * per component: resistor (a, b, R): (v_a - v_b)(lambda_a - lambda_b) / R^2;
 * diode: -(lambda_anode - lambda_cathode)(exp(v / nVt) - 1); MOSFET (drain
 * current i_d at x, g_m = di_d/dV_GS): d/d|VTO| = (lambda_D - lambda_S) pol g_m,
 * d/dKP = -(lambda_D - lambda_S) i_d / KP.
 *
 * Transient (backward Euler, F_n = (G + C/h) x_n - (C/h) x_{n-1} + i(x_n)
 * - b(t_n), o = w . x_N): J_N^T lambda_N = w, J_n^T lambda_n = (C/h)^T
 * lambda_{n+1}, then the DC start J_0^T lambda_0 = (C/h)^T lambda_1; each
 * step back-stamps as above plus capacitor (a, b, C):
 * -(lambda_a - lambda_b)((v_a - v_b)_n - (v_a - v_b)_{n-1}) / h.  The forward
 * states are recomputed segment by segment from checkpoints taken every
 * `checkpoint_every` steps, or, with checkpoint_every = 0, every state is
 * kept (n_steps x n doubles of device memory) and nothing is recomputed.
 * Gradients accumulate in FP64 on the device.
 * When x_0 is identically zero (all sources off at t0) every DC term is zero
 * and the DC start solve is skipped (info->linear_solves = n_steps). */
typedef struct {
    int64_t n_resistors;
    const int32_t *r_a, *r_b;    /* system rows of the terminals, -1 = ground */
    const double *r_ohms;
    int64_t n_capacitors;
    const int32_t *c_a, *c_b;
    const double *c_farads;
} ohm_components;

typedef struct {
    int32_t status;
    int32_t steps;               /* transient steps differentiated */
    int32_t linear_solves;       /* adjoint solves J^T lambda = rhs */
    int32_t recompute_launches;  /* forward launches of the checkpoint recomputation */
    int64_t krylov_iterations;   /* over the adjoint solves */
    double output;               /* o = w . x (x_N for a transient) */
} ohm_adjoint_info;

/* DC adjoint at the operating point x_dev (device).  Gradient outputs (host,
 * may be NULL): d_out_dr[n_resistors], d_out_dis[plan's diodes],
 * d_out_dvto[plan's MOSFETs] (with respect to the descriptor's |VTO|, the
 * threshold magnitude the model uses), d_out_dkp[plan's MOSFETs] (with
 * respect to the descriptor's KP, i.e. KP W/L where W/L is folded in);
 * lambda_host (may be NULL) receives lambda.  kp: FP64 Krylov settings. */
ohm_status ohm_plan_adjoint_dc(ohm_plan *plan, const double *x_dev, const double *w_host,
                               const ohm_components *comps, const ohm_krylov_params *kp, double *d_out_dr,
                               double *d_out_dis, double *d_out_dvto, double *d_out_dkp, double *lambda_host,
                               ohm_adjoint_info *info);
/* Transient adjoint: forward n_steps BE steps from x0_dev (the DC operating
 * point at t0, left unchanged) with Newton params np, then the reverse
 * sweep.  Outputs (host, may be NULL): d_out_dr, d_out_dc[n_capacitors],
 * d_out_dis, d_out_dvto, d_out_dkp (as for the DC adjoint).  Includes the
 * dependence of x0 on the parameters (the DC adjoint at the start). */
ohm_status ohm_transient_adjoint(ohm_transient *tr, const double *x0_dev, double t0, double h, int32_t n_steps,
                                 int32_t checkpoint_every, const ohm_newton_params *np, const double *w_host,
                                 const ohm_components *comps, const ohm_krylov_params *kp, double *d_out_dr,
                                 double *d_out_dc, double *d_out_dis, double *d_out_dvto, double *d_out_dkp,
                                 ohm_adjoint_info *info);

/* ---------------------------------------------------------------- batches --
 * Many independent nonlinear circuits solved by one launch (Monte Carlo
 * corners, parameter sweeps).  No counterpart in the reference, which runs
 * one circuit per call of newton_solve (src/solver/newton.rs:62-430); each
 * instance here follows that same Newton loop.
 *
 * Packed layout, instance i owning:
 *   rows       [row_off[i], row_off[i+1])            (its local size n_i)
 *   nonzeros   [nnz_off[i], nnz_off[i+1])
 *   row_ptrs   entries [row_off[i] + i, row_off[i+1] + i] (n_i + 1 local row
 *              pointers starting at 0; local column indices)
 *   devices    [diode_off[i], diode_off[i+1]) etc., with local node / value
 *              indices in their descriptors.
 * base_b and the solution vector are packed by rows.  Each instance is solved
 * by one thread block with the block-Jacobi preconditioner (ISAI(1) is
 * rejected), largest instances first.  n_nodes (per instance, may be NULL)
 * enables params->continuation; params->n_nodes is ignored for batches. */
typedef struct ohm_batch ohm_batch;
ohm_status ohm_batch_create(ohm_ctx *ctx, int64_t n_instances, const int64_t *row_off, const int64_t *nnz_off,
                            const uint32_t *row_ptrs, const uint32_t *col_indices,
                            const double *base_g_values, const double *base_b,
                            const int64_t *diode_off, const ohm_diode_desc *diodes,
                            const int64_t *bjt_off, const ohm_bjt_desc *bjts, const double *bjt_vaf,
                            const int64_t *mosfet_off, const ohm_mosfet_desc *mosfets,
                            const int32_t *n_nodes, ohm_batch **out);
ohm_status ohm_batch_destroy(ohm_batch *batch);
/* Newton on every instance.  x_inout_device: row_off[n] doubles.  `summary`
 * gets totals (iterations = the largest Newton count, error_iteration = the
 * first failed instance, -1 when all converged).  Returns the status
 * of the first failed instance, if any. */
ohm_status ohm_batch_newton_device(ohm_batch *batch, double *x_inout_device, const ohm_newton_params *params,
                                   ohm_solve_info *summary);
/* Per-instance results of the last ohm_batch_newton_device call. */
ohm_status ohm_batch_instance_info(ohm_batch *batch, ohm_solve_info *infos, int64_t n_instances);
/* Autotuner: times the batch kernel variants (lanes per row around the
 * density heuristic x launch shapes (256 threads, 2 blocks/SM), (256, 4),
 * (128, 8)) on `sample_size` instances (<= 0: 512) spread over the size
 * distribution, three Newton iterations with `params` from zero (no
 * continuation), and keeps the fastest for later ohm_batch_newton_device
 * calls.  Outputs may be NULL. */
ohm_status ohm_batch_autotune(ohm_batch *batch, const ohm_newton_params *params, int32_t sample_size,
                              int32_t *lanes_per_row, int32_t *threads_per_block, int32_t *blocks_per_sm,
                              double *sample_ms);
/* Choose the kernel variant directly (same choices as the autotuner). */
ohm_status ohm_batch_set_kernel(ohm_batch *batch, int32_t lanes_per_row, int32_t threads_per_block,
                                int32_t blocks_per_sm);
/* Split of each ohm_batch_newton_device call (on = 1, the default; 0 = every
 * instance in the batch kernel).  With few instances of mixed sizes one block
 * on the largest circuit would set the call's time while the other SMs idle,
 * so a circuit whose one-block solve is estimated (rows^1.5) to outlast the
 * rest of the batch spread over the resident blocks, and that has at least
 * 2,048 rows (below that one block beats the whole grid), is solved first,
 * alone, by the single-system persistent solver on the whole GPU; the batch
 * kernel then takes the rest.  summary's
 * kernel_launches counts both.  Large batches of similar sizes split nothing.
 * No counterpart in the reference (its batch is many newton_solve calls). */
ohm_status ohm_batch_set_split(ohm_batch *batch, int32_t on);

/* ---------------------------------------------------------------- compile --
 * Device-side MNA compile of compile (src/compiler.rs:194-754): node
 * numbering by first appearance, branch rows for V sources and inductors,
 * the stamps as CSR triplets summed in triplet order (CsrMatrix::from_triplets,
 * src/sparse.rs:51-104), GMIN and C's pattern zero-filled into G, the DC
 * right-hand side and the device descriptors (slots by value_index), all on
 * the GPU.  The result equals the reference's compile output bit for bit.
 *
 * Components in column form: kind[m] (0 R, 1 C, 2 L, 3 V, 4 I, 5 D, 6 Q,
 * 7 M, the order of the reference's Component enum); nodes[m x 3] labels,
 * <= 0 meaning ground, the third used only by BJTs (emitter) and MOSFETs
 * (source); value[m] (R ohms, C farads, L henries, V/I DC value, NaN = no
 * DC value); params[m x 7] (D: is, n; Q: is, bf, br, nf, nr, npn != 0;
 * M: vto, kp, lambda, nmos != 0).  OHM_ERR_COMPILE names the first
 * zero resistance, negative capacitance or device without a model
 * (compiler.rs:310-316, 336-340), in that order of checks. */
typedef struct {
    int64_t n_nodes, size, n_branches, g_nnz, c_nnz, n_diodes, n_bjts, n_mosfets;
} ohm_netlist_sizes;

typedef struct ohm_netlist ohm_netlist;
ohm_status ohm_compile(ohm_ctx *ctx, int64_t m, const int32_t *kind, const int64_t *nodes, const double *value,
                       const double *params, ohm_netlist **out);
ohm_status ohm_netlist_get_sizes(const ohm_netlist *netlist, ohm_netlist_sizes *out);
/* Copies the compiled system to host arrays (any may be NULL): G and C in
 * CSR (size + 1 row pointers, nnz columns and values), b_dc (size), the
 * node labels in matrix order (n_nodes), the component index of each branch
 * row (n_branches) and the descriptors. */
ohm_status ohm_netlist_download(const ohm_netlist *netlist, uint32_t *g_row_ptr, uint32_t *g_col, double *g_val,
                                uint32_t *c_row_ptr, uint32_t *c_col, double *c_val, double *b_dc,
                                int64_t *node_labels, int64_t *branch_components, ohm_diode_desc *diodes,
                                ohm_bjt_desc *bjts, ohm_mosfet_desc *mosfets);
ohm_status ohm_netlist_destroy(ohm_netlist *netlist);

#ifdef __cplusplus
}
#endif
#endif /* OHM_H */
