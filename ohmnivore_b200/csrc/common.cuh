// Shared device helpers for the persistent solver kernels: bounded grid
// barrier, deterministic block / grid reductions, small numeric helpers.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ohm {

constexpr uint32_t kSentinel = 0xFFFFFFFFu;   // u32::MAX, ground / absent slot

// Device status words shared by all kernels (ohm_status values).
constexpr int kStatusOk = 0;
constexpr int kStatusTimeout = 5;

// Upper bound on one barrier wait: iterations of a __nanosleep(128) loop
// (about 2^24 * 128 ns = 2 s).  A wait that runs out records kStatusTimeout
// and the kernel returns; with a cooperative launch every block is resident,
// so a healthy barrier never comes near the bound.
constexpr uint32_t kBarrierSpinLimit = 1u << 24;

struct GridSync {
    unsigned int *count;   // arrivals in the current generation
    unsigned int *gen;     // generation counter
    int *error;            // first error recorded by any block (0 = none)
};

// Grid-wide barrier for co-resident (cooperatively launched) blocks.
// Returns false when the wait gave up or another block recorded an error;
// the caller must then leave the kernel.
__device__ __forceinline__ bool grid_barrier(const GridSync &gs) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned int *vgen = gs.gen;
        const unsigned int my_gen = *vgen;
        __threadfence();
        const unsigned int arrived = atomicAdd(gs.count, 1u);
        int ok = 1;
        if (arrived == gridDim.x - 1) {
            atomicExch(gs.count, 0u);
            __threadfence();
            atomicAdd(gs.gen, 1u);
        } else {
            uint32_t spins = 0;
            while (*vgen == my_gen) {
                if (++spins > kBarrierSpinLimit) {
                    atomicCAS(gs.error, 0, kStatusTimeout);
                    ok = 0;
                    break;
                }
                __nanosleep(128);
            }
        }
        __threadfence();
        if (*((volatile int *)gs.error) != 0) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Sum NV doubles over the block; result valid in every thread.  Fixed
// reduction tree, so identical inputs give identical outputs.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *smem /* >= 32*NV */) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double x = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        v[k] = x;
    }
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) smem[k * 32 + warp] = v[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double x = (lane < nwarps) ? smem[k * 32 + lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        v[k] = x;
    }
    __syncthreads();
}

template <int NV>
__device__ __forceinline__ void block_max(double (&v)[NV], double *smem) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double x = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
        v[k] = x;
    }
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) smem[k * 32 + warp] = v[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double x = (lane < nwarps) ? smem[k * 32 + lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
        v[k] = x;
    }
    __syncthreads();
}

// Grid reduction, step 1: every block publishes its block sum to
// partials[k * gridDim.x + blockIdx.x].
template <int NV>
__device__ __forceinline__ void publish_partials(double (&v)[NV], double *partials, double *smem) {
    block_sum<NV>(v, smem);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) partials[k * gridDim.x + blockIdx.x] = v[k];
    }
}

// Grid reduction, step 2 (after a barrier): every block sums all partials in
// the same fixed order, so every block holds bit-identical results.
template <int NV>
__device__ __forceinline__ void gather_partials(const double *partials, double (&out)[NV],
                                                double *smem) {
    const int G = gridDim.x;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double s = 0.0;
        for (int j = threadIdx.x; j < G; j += blockDim.x) s += __ldcg(&partials[k * G + j]);
        out[k] = s;
    }
    block_sum<NV>(out, smem);
}

template <int NV>
__device__ __forceinline__ void publish_max(double (&v)[NV], double *partials, double *smem) {
    block_max<NV>(v, smem);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) partials[k * gridDim.x + blockIdx.x] = v[k];
    }
}

template <int NV>
__device__ __forceinline__ void gather_max(const double *partials, double (&out)[NV],
                                           double *smem) {
    const int G = gridDim.x;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double s = 0.0;
        for (int j = threadIdx.x; j < G; j += blockDim.x) s = fmax(s, __ldcg(&partials[k * G + j]));
        out[k] = s;
    }
    block_max<NV>(out, smem);
}

__device__ __forceinline__ bool is_finite_d(double x) { return isfinite(x); }

}  // namespace ohm
