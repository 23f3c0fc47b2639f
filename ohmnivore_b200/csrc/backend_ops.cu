// SolverBackend operations (src/solver/backend.rs:51-96) on FP64 device
// buffers: new_buffer, upload/download, upload_matrix, spmv, dot, axpy, copy,
// scale.  These are the step-by-step primitives a host-driven BiCGSTAB
// (bicgstab.rs:56-189) calls; the fused persistent solver does not use them.
// dot reduces on the device in FP64 with a fixed tree (no host partial sums,
// unlike backend.rs:385-447).
#include <cuda_runtime.h>

#include <algorithm>

#include "internal.cuh"

using namespace ohm;

namespace {

constexpr int kOpsBlock = 256;

int grid_for(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + kOpsBlock - 1) / kOpsBlock, 148 * 8)); }

// CSR SpMV, one thread per row: lane i of a warp sums row base + i in CSR
// order (the order of a sequential CSR product).  Consecutive lanes read
// consecutive rows, so a warp's column / value loads cover one contiguous
// stretch of the arrays and every fetched sector is used through L1; with
// 8 blocks of 256 threads per SM this streams at the HBM copy rate on short
// rows.  Rows longer than kLongRow would stall their warp, so they are found
// by a ballot and summed by the whole warp (lane-strided, xor tree); on a
// matrix of long rows this is a warp per row.
constexpr uint32_t kLongRow = 32;
constexpr int kStreamBlock = 256;

__global__ void __launch_bounds__(kStreamBlock) spmv_row_kernel(int n, const uint32_t *__restrict__ rp,
                                                                const uint32_t *__restrict__ col,
                                                                const double *__restrict__ val,
                                                                const double *__restrict__ x,
                                                                double *__restrict__ y) {
    const int lane = threadIdx.x & 31;
    const int threads = gridDim.x * blockDim.x;
    // warp-uniform loop bound: the warp's first row
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x + threadIdx.x - lane; base < n; base += threads) {
        const int64_t row = base + lane;
        uint32_t b = 0, e = 0;
        if (row < n) {
            b = rp[row];
            e = rp[row + 1];
        }
        const bool is_long = e - b > kLongRow;
        double acc = 0.0;
        if (!is_long)   // product and sum rounded separately, as a sequential CSR product does (no FMA)
            for (uint32_t k = b; k < e; ++k) acc = __dadd_rn(acc, __dmul_rn(val[k], x[col[k]]));
        for (unsigned pending = __ballot_sync(0xffffffffu, is_long); pending; pending &= pending - 1) {
            const int src = __ffs(pending) - 1;
            const uint32_t lb = __shfl_sync(0xffffffffu, b, src), le = __shfl_sync(0xffffffffu, e, src);
            double part = 0.0;
            for (uint32_t k = lb + lane; k < le; k += 32) part += val[k] * x[col[k]];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
            if (lane == src) acc = part;
        }
        if (row < n) y[row] = acc;
    }
}

// Block partial sums, then a single-block pass; fixed order -> deterministic.
__global__ void dot_partial_kernel(int64_t n, const double *__restrict__ a, const double *__restrict__ b,
                                   double *__restrict__ partial) {
    __shared__ double smem[32];
    double acc[1] = {0.0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        acc[0] += a[i] * b[i];
    block_sum<1>(acc, smem);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc[0];
}

__global__ void dot_final_kernel(int m, const double *__restrict__ partial, double *__restrict__ out) {
    __shared__ double smem[32];
    double acc[1] = {0.0};
    for (int i = threadIdx.x; i < m; i += blockDim.x) acc[0] += partial[i];
    block_sum<1>(acc, smem);
    if (threadIdx.x == 0) *out = acc[0];
}

__global__ void axpy_kernel(int64_t n, double alpha, const double *__restrict__ x, double *__restrict__ y) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] = y[i] + alpha * x[i];
}

__global__ void scale_kernel(int64_t n, double alpha, double *__restrict__ x) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] = x[i] * alpha;
}

}  // namespace

extern "C" ohm_status ohm_buf_create(ohm_ctx *c, int64_t n, ohm_buf **out) {
    if (!c || !out || n < 0) return ohm_fail(OHM_ERR_INVALID_ARG, "bad buffer arguments");
    *out = nullptr;
    CUDA_TRY(cudaSetDevice(c->device));
    ohm_buf *b = new ohm_buf{c, nullptr, n};
    cudaError_t e = dalloc(&b->d, n);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->d, 0, std::max<int64_t>(n, 1) * sizeof(double), c->stream);
    if (e != cudaSuccess) {
        ohm_pool_free(b->d);
        delete b;
        return ohm_fail(OHM_ERR_CUDA, "buffer allocation: %s", cudaGetErrorString(e));
    }
    ohm_ctx_retain(c);
    *out = b;
    return OHM_OK;
}

extern "C" ohm_status ohm_buf_destroy(ohm_buf *b) {
    if (!b) return OHM_OK;
    ohm_ctx *c = b->ctx;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    ohm_pool_free(b->d);
    delete b;
    ohm_ctx_release(c);
    return OHM_OK;
}

extern "C" double *ohm_buf_device_ptr(ohm_buf *b) { return b ? b->d : nullptr; }

extern "C" ohm_status ohm_buf_upload(ohm_ctx *c, ohm_buf *b, const double *host, int64_t n) {
    if (!c || !b || (n && !host)) return ohm_fail(OHM_ERR_INVALID_ARG, "null argument");
    if (n != b->n) return ohm_fail(OHM_ERR_INVALID_ARG, "length %lld != buffer length %lld", (long long)n, (long long)b->n);
    if (n) CUDA_TRY(cudaMemcpyAsync(b->d, host, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return OHM_OK;
}

extern "C" ohm_status ohm_buf_download(ohm_ctx *c, const ohm_buf *b, double *host, int64_t n) {
    if (!c || !b || (n && !host)) return ohm_fail(OHM_ERR_INVALID_ARG, "null argument");
    if (n != b->n) return ohm_fail(OHM_ERR_INVALID_ARG, "length %lld != buffer length %lld", (long long)n, (long long)b->n);
    if (n) CUDA_TRY(cudaMemcpyAsync(host, b->d, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return OHM_OK;
}

extern "C" ohm_status ohm_csr_upload(ohm_ctx *c, int64_t n, int64_t nnz, const uint32_t *row_ptr,
                                     const uint32_t *col, const double *values, ohm_csr **out) {
    if (!c || !out || !row_ptr || (nnz && (!col || !values)) || n < 0 || nnz < 0)
        return ohm_fail(OHM_ERR_INVALID_ARG, "bad CSR arguments");
    *out = nullptr;
    if (row_ptr[0] != 0 || (int64_t)row_ptr[n] != nnz) return ohm_fail(OHM_ERR_COMPILE, "row_ptr inconsistent with nnz");
    for (int64_t i = 0; i < n; ++i)
        if (row_ptr[i + 1] < row_ptr[i]) return ohm_fail(OHM_ERR_COMPILE, "row_ptr decreases at row %lld", (long long)i);
    for (int64_t k = 0; k < nnz; ++k)
        if ((int64_t)col[k] >= n) return ohm_fail(OHM_ERR_COMPILE, "column index out of range at %lld", (long long)k);
    CUDA_TRY(cudaSetDevice(c->device));
    ohm_csr *m = new ohm_csr{c, n, nnz, nullptr, nullptr, nullptr};
    cudaError_t e = dalloc(&m->rp, n + 1);
    if (e == cudaSuccess) e = dalloc(&m->col, nnz);
    if (e == cudaSuccess) e = dalloc(&m->val, nnz);
    if (e == cudaSuccess) e = cudaMemcpyAsync(m->rp, row_ptr, (n + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess && nnz) e = cudaMemcpyAsync(m->col, col, nnz * sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess && nnz) e = cudaMemcpyAsync(m->val, values, nnz * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        ohm_pool_free(m->rp); ohm_pool_free(m->col); ohm_pool_free(m->val);
        delete m;
        return ohm_fail(OHM_ERR_CUDA, "CSR upload: %s", cudaGetErrorString(e));
    }
    ohm_ctx_retain(c);
    *out = m;
    return OHM_OK;
}

extern "C" ohm_status ohm_csr_update_values(ohm_ctx *c, ohm_csr *m, const double *values, int64_t nnz) {
    if (!c || !m || (nnz && !values)) return ohm_fail(OHM_ERR_INVALID_ARG, "null argument");
    if (nnz != m->nnz) return ohm_fail(OHM_ERR_INVALID_ARG, "nnz mismatch");
    if (nnz) CUDA_TRY(cudaMemcpyAsync(m->val, values, nnz * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return OHM_OK;
}

extern "C" ohm_status ohm_csr_destroy(ohm_csr *m) {
    if (!m) return OHM_OK;
    ohm_ctx *c = m->ctx;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    ohm_pool_free(m->rp); ohm_pool_free(m->col); ohm_pool_free(m->val);
    delete m;
    ohm_ctx_release(c);
    return OHM_OK;
}

extern "C" ohm_status ohm_spmv(ohm_ctx *c, const ohm_csr *a, const ohm_buf *x, ohm_buf *y) {
    if (!c || !a || !x || !y) return ohm_fail(OHM_ERR_INVALID_ARG, "null argument");
    if (x->n != a->n || y->n != a->n) return ohm_fail(OHM_ERR_INVALID_ARG, "spmv dimension mismatch");
    if (a->n == 0) return OHM_OK;
    // 8 resident blocks of 256 threads per SM, grid-stride over the rows
    const int grid = (int)std::min<int64_t>((a->n + kStreamBlock - 1) / kStreamBlock, 148 * 8);
    spmv_row_kernel<<<grid, kStreamBlock, 0, c->stream>>>((int)a->n, a->rp, a->col, a->val, x->d, y->d);
    CUDA_TRY(cudaGetLastError());
    return OHM_OK;
}

// x . y over the first n entries: per-block partials, then one block sums
// them in a fixed order (the same result for the same inputs every call).
static ohm_status dot_first(ohm_ctx *c, const ohm_buf *a, const ohm_buf *b, int64_t n, double *out) {
    const int grid = std::min(grid_for(n), 1024);
    dot_partial_kernel<<<grid, kOpsBlock, 0, c->stream>>>(n, a->d, b->d, c->dot_scratch);
    dot_final_kernel<<<1, 1024, 0, c->stream>>>(grid, c->dot_scratch, c->dot_scratch + 2040);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(out, c->dot_scratch + 2040, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return OHM_OK;
}

extern "C" ohm_status ohm_dot(ohm_ctx *c, const ohm_buf *a, const ohm_buf *b, double *out) {
    if (!c || !a || !b || !out) return ohm_fail(OHM_ERR_INVALID_ARG, "null argument");
    if (a->n != b->n) return ohm_fail(OHM_ERR_INVALID_ARG, "dot length mismatch");
    return dot_first(c, a, b, a->n, out);
}

extern "C" ohm_status ohm_dot_n(ohm_ctx *c, const ohm_buf *a, const ohm_buf *b, int64_t n, double *out) {
    if (!c || !a || !b || !out) return ohm_fail(OHM_ERR_INVALID_ARG, "null argument");
    if (n < 0 || n > a->n || n > b->n)
        return ohm_fail(OHM_ERR_INVALID_ARG, "dot_n: n = %lld outside the buffers (%lld, %lld)", (long long)n,
                        (long long)a->n, (long long)b->n);
    return dot_first(c, a, b, n, out);
}

extern "C" ohm_status ohm_axpy(ohm_ctx *c, double alpha, const ohm_buf *x, ohm_buf *y) {
    if (!c || !x || !y) return ohm_fail(OHM_ERR_INVALID_ARG, "null argument");
    if (x->n != y->n) return ohm_fail(OHM_ERR_INVALID_ARG, "axpy length mismatch");
    if (x->n) axpy_kernel<<<grid_for(x->n), kOpsBlock, 0, c->stream>>>(x->n, alpha, x->d, y->d);
    CUDA_TRY(cudaGetLastError());
    return OHM_OK;
}

extern "C" ohm_status ohm_copy(ohm_ctx *c, const ohm_buf *src, ohm_buf *dst) {
    if (!c || !src || !dst) return ohm_fail(OHM_ERR_INVALID_ARG, "null argument");
    if (src->n != dst->n) return ohm_fail(OHM_ERR_INVALID_ARG, "copy length mismatch");
    if (src->n) CUDA_TRY(cudaMemcpyAsync(dst->d, src->d, src->n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    return OHM_OK;
}

extern "C" ohm_status ohm_scale(ohm_ctx *c, double alpha, ohm_buf *x) {
    if (!c || !x) return ohm_fail(OHM_ERR_INVALID_ARG, "null argument");
    if (x->n) scale_kernel<<<grid_for(x->n), kOpsBlock, 0, c->stream>>>(x->n, alpha, x->d);
    CUDA_TRY(cudaGetLastError());
    return OHM_OK;
}
