// Device memory cache for the library's own buffers.  Plans, batches,
// transients and solves allocate tens of buffers per call; returning them to
// CUDA and asking again costs a device-wide synchronisation and an unmap per
// buffer.  Freed blocks are kept per (device, rounded size) and handed out
// again; the cache holds at most kPoolCap bytes per device (beyond that
// blocks go back to CUDA) and is emptied by ohm_pool_trim (context destroy).
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <unordered_map>
#include <utility>
#include <vector>

#include "internal.cuh"

namespace {

constexpr size_t kPoolCap = (size_t)16 << 30;

struct Block {
    int device;
    size_t bytes;
};

std::mutex g_mu;
std::unordered_map<void *, Block> g_live;                       // handed out
std::map<std::pair<int, size_t>, std::vector<void *>> g_free;   // cached
std::unordered_map<int, size_t> g_cached;                        // cached bytes per device

size_t round_size(size_t b) {
    if (b <= ((size_t)1 << 20)) return (b + 511) & ~(size_t)511;
    return (b + ((size_t)2 << 20) - 1) & ~(((size_t)2 << 20) - 1);
}

}  // namespace

cudaError_t ohm_pool_alloc(void **p, size_t bytes) {
    *p = nullptr;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const size_t b = round_size(bytes == 0 ? 1 : bytes);
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_free.find({dev, b});
        if (it != g_free.end() && !it->second.empty()) {
            *p = it->second.back();
            it->second.pop_back();
            g_cached[dev] -= b;
            g_live[*p] = Block{dev, b};
            return cudaSuccess;
        }
    }
    e = cudaMalloc(p, b);
    if (e != cudaSuccess) {
        // give the cache back to CUDA and try once more
        ohm_pool_trim(dev);
        cudaGetLastError();
        e = cudaMalloc(p, b);
        if (e != cudaSuccess) { *p = nullptr; return e; }
    }
    std::lock_guard<std::mutex> lk(g_mu);
    g_live[*p] = Block{dev, b};
    return cudaSuccess;
}

void ohm_pool_free(void *p) {
    if (!p) return;
    Block blk{};
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_live.find(p);
        if (it == g_live.end()) {
            cudaFree(p);                   // not from the cache
            return;
        }
        blk = it->second;
        g_live.erase(it);
        if (g_cached[blk.device] + blk.bytes <= kPoolCap) {
            // like cudaFree, wait for work that may still use the block
            int cur = 0;
            cudaGetDevice(&cur);
            if (cur != blk.device) cudaSetDevice(blk.device);
            cudaDeviceSynchronize();
            if (cur != blk.device) cudaSetDevice(cur);
            g_free[{blk.device, blk.bytes}].push_back(p);
            g_cached[blk.device] += blk.bytes;
            return;
        }
    }
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(blk.device);
    cudaFree(p);
    cudaSetDevice(cur);
}

void ohm_pool_trim(int device) {
    std::vector<void *> out;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        for (auto it = g_free.begin(); it != g_free.end();) {
            if (it->first.first == device) {
                out.insert(out.end(), it->second.begin(), it->second.end());
                it = g_free.erase(it);
            } else {
                ++it;
            }
        }
        g_cached[device] = 0;
    }
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(device);
    for (void *q : out) cudaFree(q);
    cudaSetDevice(cur);
}
