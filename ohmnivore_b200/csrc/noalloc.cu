// ohm_solve_real_noalloc: the linear solve of ohm_solve_real for callers that
// cannot allocate device memory.
//
// Who needs it: code that runs inside another program's device-memory budget
// (a simulator plugin or service whose host owns every byte through its own
// pool), and code on a latency-critical path where cudaMalloc / cudaFree
// would synchronise the device or fail under memory pressure.  The caller
// passes device-resident inputs and the output vector; every other byte the
// solve needs comes from one file-scope __device__ array of fixed size.
//
// Limits: at most kMaxRows rows and kMaxNnz nonzeros (about 6.2 MB of device
// memory, held by every GPU that loads this library until the process exits).
// Set-up: the first call on a device looks up that device's address of the
// array (cudaGetSymbolAddress, with the device current); make that first call
// before any stream capture.  Every call shares the array and leaves its
// contents behind; everything that must start at zero is cleared per call.
// Calls that overlap on the GPU (two streams, two threads) race on the array.
// Each call blocks the host: it reads the CSR check flag back before the solve
// and the solve's status after it, synchronising the stream both times.
#include <cuda_runtime.h>

#include <climits>
#include <cstring>
#include <mutex>

#include "internal.cuh"

using namespace ohm;

namespace {

constexpr int64_t kMaxRows = 32768;
constexpr int64_t kMaxNnz = 262144;
constexpr int kMaxGrid = 256;
constexpr int kMaxDevices = 64;

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Scratch layout (byte offsets), each region 256-byte aligned.
constexpr size_t kOffVec = 0;                                               // 15 x rows x 8
constexpr size_t kOffR64 = kOffVec + align256(15 * kMaxRows * 8);
constexpr size_t kOffDx = kOffR64 + align256(kMaxRows * 8);
constexpr size_t kOffPartials = kOffDx + align256(kMaxRows * 8);            // 8 x grid doubles
constexpr size_t kOffPartner = kOffPartials + align256(8 * kMaxGrid * 8);
constexpr size_t kOffDiag = kOffPartner + align256(kMaxRows * 4);
constexpr size_t kOffOff = kOffDiag + align256(kMaxRows * 4);
constexpr size_t kOffCand = kOffOff + align256(kMaxRows * 4);
constexpr size_t kOffChoice = kOffCand + align256(kMaxRows * 4);
constexpr size_t kOffFlag = kOffChoice + align256(kMaxRows * 4);
constexpr size_t kOffVals32 = kOffFlag + align256(kMaxRows);
constexpr size_t kOffSync = kOffVals32 + align256(kMaxNnz * 4);            // 4 words + check flag
constexpr size_t kOffInfo = kOffSync + 256;
constexpr size_t kScratchBytes = kOffInfo + align256(sizeof(DeviceInfo));

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_setup_mutex;
unsigned char *g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch array for the current device (looked up once).
ohm_status scratch_for_current_device(unsigned char **out) {
    int dev = -1;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return ohm_fail(OHM_ERR_INVALID_ARG, "device %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return ohm_fail(OHM_ERR_CUDA, "cudaGetSymbolAddress(scratch) failed: %s", cudaGetErrorString(e));
        g_scratch_addr[dev] = (unsigned char *)p;
    }
    *out = g_scratch_addr[dev];
    return OHM_OK;
}

// CSR sanity on the device (inputs are device pointers): row_ptr[0] == 0,
// non-decreasing, row_ptr[n] == nnz, every column < n.  Sets *bad on failure.
__global__ void check_csr_kernel(int n, int nnz, const uint32_t *rp, const uint32_t *col, unsigned int *bad) {
    const int stride = gridDim.x * blockDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += stride) {
        if (i == 0 && rp[0] != 0u) atomicOr(bad, 1u);
        if (i == n && rp[n] != (uint32_t)nnz) atomicOr(bad, 2u);
        if (i < n && rp[i + 1] < rp[i]) atomicOr(bad, 4u);
    }
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += stride)
        if (col[k] >= (uint32_t)n) atomicOr(bad, 8u);
}

// Block-Jacobi structure on the device (the same rule as the host builder
// for the allocating entry points; when two zero-diagonal rows want the same
// partner row, the lower row index gets it and the other stays unpaired).
__global__ void pc_diag_kernel(int n, const uint32_t *rp, const uint32_t *col, uint32_t *diag, int32_t *partner,
                               uint32_t *off, uint32_t *cand, int32_t *choice) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t d = kSentinel;
        for (uint32_t k = rp[i]; k < rp[i + 1]; ++k)
            if (col[k] == (uint32_t)i) { d = k; break; }
        diag[i] = d;
        partner[i] = -1;
        off[i] = kSentinel;
        cand[i] = 0xFFFFFFFFu;
        choice[i] = -1;
    }
}

__device__ __forceinline__ bool zero_diag(const uint32_t *diag, const double *val, int i) {
    return diag[i] == kSentinel || fabs(val[diag[i]]) <= 1e-30;
}

__device__ __forceinline__ uint32_t slot_of(const uint32_t *rp, const uint32_t *col, int r, int c) {
    for (uint32_t k = rp[r]; k < rp[r + 1]; ++k)
        if (col[k] == (uint32_t)c) return k;
    return kSentinel;
}

__global__ void pc_choose_kernel(int n, const uint32_t *rp, const uint32_t *col, const double *val,
                                 const uint32_t *diag, uint32_t *cand, int32_t *choice) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        if (!zero_diag(diag, val, k)) continue;
        int best = -1;
        double best_mag = 0.0;
        for (uint32_t e = rp[k]; e < rp[k + 1]; ++e) {
            const int j = (int)col[e];
            if (j == k || zero_diag(diag, val, j)) continue;
            const double mag = fabs(val[e]);
            if (!(mag > 0.0)) continue;
            const uint32_t jk = slot_of(rp, col, j, k);
            if (jk == kSentinel || !(fabs(val[jk]) > 0.0)) continue;
            if (mag > best_mag) { best_mag = mag; best = j; }
        }
        choice[k] = best;
        if (best >= 0) atomicMin(&cand[best], (uint32_t)k);
    }
}

__global__ void pc_pair_kernel(int n, const uint32_t *rp, const uint32_t *col, const uint32_t *cand,
                               const int32_t *choice, int32_t *partner, uint32_t *off) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int j = choice[k];
        if (j < 0 || cand[j] != (uint32_t)k) continue;
        partner[k] = j;
        partner[j] = k;
        off[k] = slot_of(rp, col, k, j);
        off[j] = slot_of(rp, col, j, k);
    }
}

// rowflag[i] = 1 when row i or one of its columns is paired.
__global__ void pc_flag_kernel(int n, const uint32_t *rp, const uint32_t *col, const int32_t *partner,
                               uint8_t *flag) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        bool f = partner[i] >= 0;
        for (uint32_t k = rp[i]; k < rp[i + 1] && !f; ++k) f = partner[col[k]] >= 0;
        flag[i] = f ? 1 : 0;
    }
}

int small_grid(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 1024)); }

}  // namespace

extern "C" ohm_status ohm_solve_real_noalloc(void *stream, int64_t n, int64_t nnz, const uint32_t *d_row_ptr,
                                             const uint32_t *d_col, const double *d_values, const double *d_b,
                                             double *d_x, const ohm_krylov_params *params, ohm_solve_info *info) {
    ohm_status st = ohm_check_krylov(params);
    if (st != OHM_OK) return st;
    if (params->precond == OHM_PRECOND_ISAI1)
        return ohm_fail(OHM_ERR_INVALID_ARG, "ohm_solve_real_noalloc: ISAI(1) needs allocated set-up; "
                                             "use block Jacobi or ohm_solve_real");
    if (n < 0 || nnz < 0) return ohm_fail(OHM_ERR_INVALID_ARG, "negative size");
    if (n > kMaxRows || nnz > kMaxNnz)
        return ohm_fail(OHM_ERR_INVALID_ARG,
                        "ohm_solve_real_noalloc: system of %lld rows / %lld nonzeros exceeds the fixed scratch "
                        "limit of %lld rows / %lld nonzeros; use ohm_solve_real",
                        (long long)n, (long long)nnz, (long long)kMaxRows, (long long)kMaxNnz);
    if (n == 0) return OHM_OK;
    if (!d_row_ptr || !d_b || !d_x || (nnz && (!d_col || !d_values)))
        return ohm_fail(OHM_ERR_INVALID_ARG, "null device pointer");
    cudaStream_t s = (cudaStream_t)stream;
    unsigned char *base = nullptr;
    st = scratch_for_current_device(&base);
    if (st != OHM_OK) return st;
    int dev = 0, num_sms = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    CUDA_TRY(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev));

    unsigned int *sync = (unsigned int *)(base + kOffSync);     // [count, gen, error, spare, check]
    DeviceInfo *info_dev = (DeviceInfo *)(base + kOffInfo);
    uint32_t *diag = (uint32_t *)(base + kOffDiag);
    int32_t *partner = (int32_t *)(base + kOffPartner);
    uint32_t *off = (uint32_t *)(base + kOffOff);
    uint32_t *cand = (uint32_t *)(base + kOffCand);
    int32_t *choice = (int32_t *)(base + kOffChoice);
    float *vals32 = (float *)(base + kOffVals32);
    uint8_t *rowflag = (uint8_t *)(base + kOffFlag);

    // validate the caller's CSR before any kernel indexes with it
    unsigned int bad = 0;
    CUDA_TRY(cudaMemsetAsync(sync + 4, 0, sizeof(unsigned int), s));
    check_csr_kernel<<<small_grid(std::max(n + 1, nnz)), 256, 0, s>>>((int)n, (int)nnz, d_row_ptr, d_col, sync + 4);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(&bad, sync + 4, sizeof bad, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    if (bad) return ohm_fail(OHM_ERR_COMPILE, "ohm_solve_real_noalloc: invalid CSR (check flags 0x%x)", bad);

    const bool mixed = params->precision == OHM_PREC_MIXED;
    int launches = 1;
    // The diagonal-slot table is rebuilt on every call, whatever the
    // preconditioner: the solver reads it for every row (the Jacobi
    // coefficient, or nothing but the sentinel check), and a table left by an
    // earlier, larger system would index past this call's values.  It also
    // resets partner to -1 (unpaired).
    pc_diag_kernel<<<small_grid(n), 256, 0, s>>>((int)n, d_row_ptr, d_col, diag, partner, off, cand, choice);
    launches += 1;
    if (params->precond == OHM_PRECOND_AUTO) {
        pc_choose_kernel<<<small_grid(n), 256, 0, s>>>((int)n, d_row_ptr, d_col, d_values, diag, cand, choice);
        pc_pair_kernel<<<small_grid(n), 256, 0, s>>>((int)n, d_row_ptr, d_col, cand, choice, partner, off);
        pc_flag_kernel<<<small_grid(n), 256, 0, s>>>((int)n, d_row_ptr, d_col, partner, rowflag);
        launches += 3;
    }
    CUDA_TRY(cudaGetLastError());
    if (mixed) {
        CUDA_TRY(ohm_f64_to_f32(d_values, vals32, nnz, s));
        launches += 1;
    }
    CUDA_TRY(cudaMemsetAsync(d_x, 0, n * sizeof(double), s));

    KernelArgs a{};
    a.n = (int)n;
    a.nnz = (int)nnz;
    a.row_ptr = d_row_ptr;
    a.col = d_col;
    a.vals64 = const_cast<double *>(d_values);   // read-only in a linear solve
    a.vals32 = vals32;
    a.b = const_cast<double *>(d_b);             // read-only in a linear solve
    a.x = d_x;
    a.precond = params->precond == OHM_PRECOND_NONE ? kPcNone
              : (params->precond == OHM_PRECOND_JACOBI ? kPcJacobi : kPcAuto);
    a.partner = partner;
    a.diag_slot = diag;
    a.off_slot = off;
    a.rowflag = params->precond == OHM_PRECOND_AUTO ? rowflag : nullptr;
    double *vec = (double *)(base + kOffVec);
    a.rec0 = (void *)vec;
    a.rec1 = (void *)(vec + 4 * (size_t)n);
    void **slots[] = {&a.rhat, &a.s, &a.t, &a.phat, &a.shat, &a.d, &a.pc_part};
    for (int k = 0; k < 7; ++k) *slots[k] = (void *)(vec + (8 + (size_t)k) * n);
    a.r64 = (double *)(base + kOffR64);
    a.dx = (double *)(base + kOffDx);
    a.partials = (double *)(base + kOffPartials);
    a.newton = 0;
    a.mixed = mixed ? 1 : 0;
    a.max_outer = std::max(1, params->max_refinements);
    a.max_krylov = params->max_iterations;
    a.krylov_tol = params->tolerance;
    a.inner_rtol = mixed ? (params->inner_rtol > 0.0 ? params->inner_rtol : 1e-4) : params->inner_rtol;
    a.require_true_residual = params->max_refinements > 1 ? 1 : 0;
    a.max_restarts = std::max(0, params->max_restarts);
    // the same FP32 attempt cap and forcing bound as ohm_solve_real
    a.fp32_max_iterations = params->fp32_max_iterations > 0 ? params->fp32_max_iterations : params->max_iterations;
    a.eta_max = 0.5;

    DeviceInfo host_info;
    std::memset(&host_info, 0, sizeof host_info);
    const LaunchTarget t{num_sms, s, sync, info_dev, &host_info, kMaxGrid};
    int kernel_launches = 0;
    st = ohm_launch_persistent(t, a, nnz, &kernel_launches);
    if (st != OHM_OK) return st;
    return ohm_finish_persistent(t, info, launches);
}
