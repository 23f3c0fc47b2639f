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

// Upper bound on one barrier wait: spin iterations (tight for the first
// kTightSpins, then __nanosleep(64)); about 2-3 s in total.  A wait that runs
// out records kStatusTimeout and the kernel returns; with a cooperative launch
// every block is resident, so a healthy barrier never comes near the bound.
constexpr uint32_t kBarrierSpinLimit = 1u << 22;
constexpr uint32_t kTightSpins = 2048;

struct GridSync {
    unsigned long long *count;   // arrivals since launch (monotone, zeroed per launch)
    int *error;                  // first error recorded by any block (0 = none)
};

__device__ __forceinline__ void red_release_add_u64(unsigned long long *p, unsigned long long v) {
    asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Grid-wide barrier for co-resident (cooperatively launched) blocks on a
// monotone arrival counter: barrier number k completes when the counter
// reaches k * gridDim.x, so nothing is reset and a block never waits on a
// generation flag.  `epoch` is the caller's barrier count (identical in every
// block).  The release add publishes this block's writes (bar.sync orders the
// other threads' writes before it); the acquire load orders everything after.
// Returns false when the wait gave up; the caller must then leave the kernel.
__device__ __forceinline__ bool grid_barrier(const GridSync &gs, unsigned long long &epoch) {
    __shared__ int s_ok;
    epoch += gridDim.x;
    __syncthreads();
    if (threadIdx.x == 0) {
        red_release_add_u64(gs.count, 1ull);
        int ok = 1;
        uint32_t spins = 0;
        while (ld_acquire_u64(gs.count) < epoch) {
            if (++spins > kBarrierSpinLimit) {
                atomicCAS(gs.error, 0, kStatusTimeout);
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

// Grid all-reduce (sum, or max when MAX) of NV <= 4 values in one grid
// barrier and three block synchronisations: warps reduce to shared memory;
// warp 0 forms the block value (the same fixed tree as block_sum /
// block_max) and its lane 0 publishes it to partials[k * G + block],
// arrives on the barrier counter (release) and waits for every block
// (acquire, bounded); then warp k sums the G partials of value k, lane-
// strided in block order and then by a fixed shuffle tree, and every thread
// reads the results.  The order is fixed, so every block holds bit-identical
// results and repeated runs agree; `smem` holds >= 32 * 4 + 4 doubles.
// Returns false when the barrier wait gave up.
template <int NV, bool MAX>
__device__ __forceinline__ bool grid_allreduce(double (&v)[NV], double *partials, const GridSync &gs,
                                               unsigned long long &epoch, double *smem) {
    __shared__ int s_ok;
    const int G = gridDim.x, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = (blockDim.x + 31) >> 5;
    double *res = smem + 32 * 4;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double x = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double y = __shfl_xor_sync(0xffffffffu, x, o);
            x = MAX ? fmax(x, y) : x + y;
        }
        if (lane == 0) smem[k * 32 + warp] = x;
    }
    epoch += gridDim.x;
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double x = (lane < nwarps) ? smem[k * 32 + lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double y = __shfl_xor_sync(0xffffffffu, x, o);
                x = MAX ? fmax(x, y) : x + y;
            }
            if (lane == 0) partials[k * G + blockIdx.x] = x;
        }
        if (lane == 0) {
            red_release_add_u64(gs.count, 1ull);
            int ok = 1;
            uint32_t spins = 0;
            while (ld_acquire_u64(gs.count) < epoch) {
                if (++spins > kBarrierSpinLimit) {
                    atomicCAS(gs.error, 0, kStatusTimeout);
                    ok = 0;
                    break;
                }
                if (spins > kTightSpins) __nanosleep(64);
            }
            s_ok = ok;
        }
    }
    __syncthreads();
    if (!s_ok) return false;
    if (warp < NV) {
        const double *p = partials + (size_t)warp * G;
        double x = 0.0;
#pragma unroll 4
        for (int j = lane; j < G; j += 32) x = MAX ? fmax(x, __ldcg(p + j)) : x + __ldcg(p + j);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double y = __shfl_xor_sync(0xffffffffu, x, o);
            x = MAX ? fmax(x, y) : x + y;
        }
        if (lane == 0) res[warp] = x;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = res[k];
    return true;
}

}  // namespace ohm
