// Device-side MNA compile: components -> CSR conductance and capacitance
// matrices, the DC right-hand side and the device descriptors, on the GPU.
//
// Follows compile (src/compiler.rs:194-754), as the host compiler of this
// package restates it, bit for bit:
//   node index   order of first appearance over (component, terminal); the
//                third terminal only for BJTs and MOSFETs; labels <= 0 are
//                ground (compiler.rs:196-235)
//   branch rows  V sources and inductors in component order, after the nodes
//                (compiler.rs:237-252)
//   triplets     the stamps of compiler.rs:310-542 in component order (a
//                fixed sub-order per component), then GMIN on every node
//                diagonal and C's pattern zero-filled into G (:571-579)
//   CSR          CsrMatrix::from_triplets (sparse.rs:51-104): the pattern is
//                the unique (row, col) in row-major order; each value is the
//                sum of its nonzero triplets, left to right in triplet order
//   rhs          V sources at their branch rows; current sources -I at the
//                + node and +I at the - node, accumulated in component order
//                (compiler.rs:391-398, 440-468)
//   descriptors  compiler.rs:597-740, slots by value_index (sparse.rs:27-31)
//
// GPU design: labels are numbered with an open-addressing hash table (each
// label's first position by atomicMin) and a prefix scan over the
// first-appearance flags, so the labels are never sorted.  Triplets are
// written in triplet order at scanned offsets and ordered by a stable LSD
// radix sort on the key row * size + col (8-bit digits; a tile's items are
// ranked per warp with __match_any_sync, then across warps), which keeps
// the triplets of one entry in triplet order for the sums.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "internal.cuh"

using namespace ohm;

namespace {

constexpr int kT = 256;                       // threads per block, every kernel here
constexpr int kItems = 8;                     // items per thread in scans and sorts
constexpr int kTile = kT * kItems;            // 2048
constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr double kGmin = 1e-12;               // compiler.rs:44
constexpr double kVt300 = 0.02585;            // compiler.rs:40
enum : int32_t { kR = 0, kC, kL, kV, kI, kD, kQ, kM };

int blocks_for(int64_t n, int per_block = kT) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((n + per_block - 1) / per_block, 148 * 64));
}

// Temporary device buffers of one compile, released together at the end
// (after the stream has been synchronised).
struct Arena {
    std::vector<void *> bufs;
    template <typename T>
    cudaError_t get(T **p, size_t count) {
        cudaError_t e = dalloc(p, count);
        if (e == cudaSuccess) bufs.push_back((void *)*p);
        return e;
    }
    ~Arena() {
        for (void *q : bufs) ohm_pool_free(q);
    }
};

#define ARENA_TRY(expr)                                                                         \
    do {                                                                                        \
        cudaError_t e_ = (expr);                                                                \
        if (e_ != cudaSuccess) return ohm_fail(OHM_ERR_CUDA, "compile: %s", cudaGetErrorString(e_)); \
    } while (0)

// ------------------------------------------------------------------ scan --
// Exclusive scan of one value per thread over the block; *total receives the
// block sum.  Uses (and leaves reusable) a shared array of warp sums.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t *warp_sums, uint32_t &total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kT / 32 ? warp_sums[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kT / 32) warp_sums[lane] = w;
    }
    __syncthreads();
    const uint32_t base = warp == 0 ? 0u : warp_sums[warp - 1];
    total = warp_sums[kT / 32 - 1];
    __syncthreads();
    return base + x - v;
}

// Sum of each tile of kTile items.
__global__ void __launch_bounds__(kT) tile_sums_kernel(const uint32_t *__restrict__ in, int64_t n,
                                                       uint32_t *__restrict__ sums) {
    __shared__ uint32_t ws[kT / 32];
    const int64_t base = (int64_t)blockIdx.x * kTile + (int64_t)threadIdx.x * kItems;
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < kItems; ++i)
        if (base + i < n) s += in[base + i];
    uint32_t total = 0;
    block_exclusive_scan(s, ws, total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// out[i] = tile_base[tile] + sum of the tile's items before i; the last
// block also writes the grand total to *total_out when tile_base holds the
// scanned tile sums (or there is one tile).
__global__ void __launch_bounds__(kT) tile_scan_kernel(const uint32_t *__restrict__ in, uint32_t *__restrict__ out,
                                                       int64_t n, const uint32_t *__restrict__ tile_base,
                                                       uint32_t *__restrict__ total_out) {
    __shared__ uint32_t ws[kT / 32];
    const int64_t base = (int64_t)blockIdx.x * kTile + (int64_t)threadIdx.x * kItems;
    uint32_t v[kItems];
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        v[i] = base + i < n ? in[base + i] : 0u;
        s += v[i];
    }
    uint32_t total = 0;
    uint32_t run = block_exclusive_scan(s, ws, total) + (tile_base ? tile_base[blockIdx.x] : 0u);
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        if (base + i < n) out[base + i] = run;
        run += v[i];
    }
    if (total_out && blockIdx.x == gridDim.x - 1 && threadIdx.x == kT - 1) *total_out = run;
}

// out = exclusive scan of in (n items, u32); *total_dev = the sum.  Tiles
// of 2048, recursing on the tile sums.
cudaError_t scan_u32(const uint32_t *in, uint32_t *out, int64_t n, uint32_t *total_dev, cudaStream_t s, Arena &ar) {
    if (n <= 0) return cudaMemsetAsync(total_dev, 0, sizeof(uint32_t), s);
    const int64_t tiles = (n + kTile - 1) / kTile;
    if (tiles == 1) {
        tile_scan_kernel<<<1, kT, 0, s>>>(in, out, n, nullptr, total_dev);
        return cudaGetLastError();
    }
    uint32_t *sums = nullptr, *sums_scan = nullptr;
    cudaError_t e = ar.get(&sums, tiles);
    if (e == cudaSuccess) e = ar.get(&sums_scan, tiles);
    if (e != cudaSuccess) return e;
    tile_sums_kernel<<<(unsigned)tiles, kT, 0, s>>>(in, n, sums);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = scan_u32(sums, sums_scan, tiles, total_dev, s, ar)) != cudaSuccess) return e;
    tile_scan_kernel<<<(unsigned)tiles, kT, 0, s>>>(in, out, n, sums_scan, nullptr);
    return cudaGetLastError();
}

// ------------------------------------------------------------ radix sort --
// Histogram of one 8-bit digit per tile: counts[digit * tiles + tile].
__global__ void __launch_bounds__(kT) radix_hist_kernel(const uint64_t *__restrict__ keys, int64_t n, int shift,
                                                        uint32_t *__restrict__ counts, int64_t tiles) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kTile;
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const int64_t i = base + j * kT + threadIdx.x;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    counts[(int64_t)threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter by one digit.  Warp w of a tile holds items
// base + w * 256 + j * 32 + lane (j = 0..7), i.e. the tile's items in order;
// equal digits are ranked within the warp by __match_any_sync, across warps
// by a per-digit exclusive scan, and across tiles by `offsets`.
__global__ void __launch_bounds__(kT) radix_scatter_kernel(const uint64_t *__restrict__ kin,
                                                           const uint32_t *__restrict__ vin,
                                                           uint64_t *__restrict__ kout, uint32_t *__restrict__ vout,
                                                           int64_t n, int shift, const uint32_t *__restrict__ offsets,
                                                           int64_t tiles) {
    __shared__ uint32_t wbase[kT / 32][256];
    __shared__ uint32_t goff[256];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int d = threadIdx.x; d < (kT / 32) * 256; d += kT) (&wbase[0][0])[d] = 0;
    goff[threadIdx.x] = offsets[(int64_t)threadIdx.x * tiles + blockIdx.x];
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kTile + warp * (kTile / (kT / 32));
    uint64_t k[kItems];
    uint32_t v[kItems], dg[kItems];
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const int64_t i = base + j * 32 + lane;
        const bool ok = i < n;
        k[j] = ok ? kin[i] : 0ull;
        v[j] = ok ? vin[i] : 0u;
        dg[j] = ok ? (uint32_t)((k[j] >> shift) & 255u) : 256u;
    }
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const unsigned peers = __match_any_sync(0xffffffffu, dg[j]);
        if (dg[j] < 256u && lane == __ffs(peers) - 1) wbase[warp][dg[j]] += __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    {
        uint32_t run = 0;
        for (int w = 0; w < kT / 32; ++w) {
            const uint32_t c = wbase[w][threadIdx.x];
            wbase[w][threadIdx.x] = run;
            run += c;
        }
    }
    __syncthreads();
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const unsigned peers = __match_any_sync(0xffffffffu, dg[j]);
        if (dg[j] < 256u) {
            const uint32_t pos = goff[dg[j]] + wbase[warp][dg[j]] + __popc(peers & lt);
            kout[pos] = k[j];
            vout[pos] = v[j];
        }
        __syncwarp();
        if (dg[j] < 256u && lane == __ffs(peers) - 1) wbase[warp][dg[j]] += __popc(peers);
        __syncwarp();
    }
}

// Stable sort of (keys, vals) by the low `bits` bits of the keys; the result
// is in (keys, vals) on return (the buffers may have been swapped with the
// scratch pair).
cudaError_t radix_sort(uint64_t *&keys, uint32_t *&vals, uint64_t *&kt, uint32_t *&vt, int64_t n, int bits,
                       cudaStream_t s, Arena &ar) {
    if (n <= 1) return cudaSuccess;
    const int64_t tiles = (n + kTile - 1) / kTile;
    uint32_t *counts = nullptr, *offsets = nullptr, *total = nullptr;
    cudaError_t e = ar.get(&counts, 256 * tiles);
    if (e == cudaSuccess) e = ar.get(&offsets, 256 * tiles);
    if (e == cudaSuccess) e = ar.get(&total, 1);
    if (e != cudaSuccess) return e;
    for (int shift = 0; shift < bits; shift += 8) {
        radix_hist_kernel<<<(unsigned)tiles, kT, 0, s>>>(keys, n, shift, counts, tiles);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if ((e = scan_u32(counts, offsets, 256 * tiles, total, s, ar)) != cudaSuccess) return e;
        radix_scatter_kernel<<<(unsigned)tiles, kT, 0, s>>>(keys, vals, kt, vt, n, shift, offsets, tiles);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        std::swap(keys, kt);
        std::swap(vals, vt);
    }
    return cudaSuccess;
}

// ------------------------------------------------------- node numbering --
// MurmurHash3's 64-bit finaliser (a published bit mixer).
__device__ __forceinline__ uint64_t mix64(uint64_t k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return k;
}

__device__ __forceinline__ bool terminal_label(const int32_t *kind, const int64_t *nodes, int64_t f, uint64_t &L) {
    const int64_t c = f / 3;
    const int t = (int)(f - 3 * c);
    if (t == 2 && kind[c] != kQ && kind[c] != kM) return false;
    const int64_t lab = nodes[f];
    if (lab <= 0) return false;
    L = (uint64_t)lab;
    return true;
}

__device__ __forceinline__ uint64_t find_slot(const uint64_t *hkeys, uint64_t mask, uint64_t L) {
    uint64_t slot = mix64(L) & mask;
    for (uint64_t probe = 0; probe <= mask && hkeys[slot] != L; ++probe) slot = (slot + 1) & mask;
    return slot;
}

__global__ void label_insert_kernel(const int32_t *kind, const int64_t *nodes, int64_t nt, uint64_t *hkeys,
                                    uint32_t *hfirst, uint64_t mask) {
    for (int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; f < nt; f += (int64_t)gridDim.x * blockDim.x) {
        uint64_t L;
        if (!terminal_label(kind, nodes, f, L)) continue;
        uint64_t slot = mix64(L) & mask;
        for (uint64_t probe = 0; probe <= mask; ++probe) {
            const unsigned long long prev =
                atomicCAS((unsigned long long *)&hkeys[slot], 0ull, (unsigned long long)L);
            if (prev == 0ull || prev == L) {
                atomicMin(&hfirst[slot], (uint32_t)f);
                break;
            }
            slot = (slot + 1) & mask;
        }
    }
}

__global__ void first_flag_kernel(const int32_t *kind, const int64_t *nodes, int64_t nt, const uint64_t *hkeys,
                                  const uint32_t *hfirst, uint64_t mask, uint32_t *flag) {
    for (int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; f < nt; f += (int64_t)gridDim.x * blockDim.x) {
        uint64_t L;
        uint32_t fl = 0;
        if (terminal_label(kind, nodes, f, L)) fl = hfirst[find_slot(hkeys, mask, L)] == (uint32_t)f ? 1u : 0u;
        flag[f] = fl;
    }
}

__global__ void assign_nodes_kernel(const int32_t *kind, const int64_t *nodes, int64_t nt, const uint64_t *hkeys,
                                    const uint32_t *hfirst, uint64_t mask, const uint32_t *rank, int32_t *nidx,
                                    int64_t *labels) {
    for (int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; f < nt; f += (int64_t)gridDim.x * blockDim.x) {
        uint64_t L;
        int32_t idx = -1;
        if (terminal_label(kind, nodes, f, L)) {
            const uint32_t first = hfirst[find_slot(hkeys, mask, L)];
            idx = (int32_t)rank[first];
            if (first == (uint32_t)f) labels[idx] = (int64_t)L;
        }
        nidx[f] = idx;
    }
}

// ---------------------------------------------------- validation, branches --
// First offending component per check (compiler.rs:310-316, 336-340 and the
// model lookups): 0 zero resistance, 1 negative capacitance, 2-4 diode /
// BJT / MOSFET without a model (NaN first parameter).
__global__ void validate_kernel(const int32_t *kind, const double *value, const double *params, int64_t m,
                                unsigned long long *bad) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < m; c += (int64_t)gridDim.x * blockDim.x) {
        const int32_t k = kind[c];
        int check = -1;
        if (k == kR && value[c] == 0.0) check = 0;
        else if (k == kC && value[c] < 0.0) check = 1;
        else if (k == kD && isnan(params[c * 7])) check = 2;
        else if (k == kQ && isnan(params[c * 7])) check = 3;
        else if (k == kM && isnan(params[c * 7])) check = 4;
        if (check >= 0) atomicMin(&bad[check], (unsigned long long)c);
    }
}

__global__ void kind_flag_kernel(const int32_t *kind, int64_t m, int32_t k0, int32_t k1, uint32_t *flag) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < m; c += (int64_t)gridDim.x * blockDim.x)
        flag[c] = (kind[c] == k0 || kind[c] == k1) ? 1u : 0u;
}

__global__ void branch_kernel(const int32_t *kind, int64_t m, const uint32_t *bscan, int64_t n_nodes,
                              int32_t *bk, int64_t *branch_comp) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < m; c += (int64_t)gridDim.x * blockDim.x) {
        const bool br = kind[c] == kV || kind[c] == kL;
        bk[c] = br ? (int32_t)(n_nodes + bscan[c]) : -1;
        if (br) branch_comp[bscan[c]] = c;
    }
}

// ------------------------------------------------------------- triplets --
// The stamps of component c in triplet order.  emit(row, col, value) is
// called for G (g = true) or C entries; rows / columns are never negative.
template <typename Emit>
__device__ __forceinline__ void stamps(int32_t k, int32_t i, int32_t j, int32_t t3, int32_t b, double value,
                                       Emit &&emit) {
    const bool both = i >= 0 && j >= 0;
    switch (k) {
        case kR: {   // compiler.rs:310-330
            const double g = 1.0 / value;
            if (i >= 0) emit(true, i, i, g);
            if (j >= 0) emit(true, j, j, g);
            if (both) { emit(true, i, j, -g); emit(true, j, i, -g); }
            break;
        }
        case kC:     // compiler.rs:332-355
            if (i >= 0) emit(false, i, i, value);
            if (j >= 0) emit(false, j, j, value);
            if (both) { emit(false, i, j, -value); emit(false, j, i, -value); }
            break;
        case kL:
        case kV:     // compiler.rs:357-408
            if (i >= 0) { emit(true, i, b, 1.0); emit(true, b, i, 1.0); }
            if (j >= 0) { emit(true, j, b, -1.0); emit(true, b, j, -1.0); }
            if (k == kL) emit(false, b, b, -value);
            break;
        case kD:     // compiler.rs:427-437
            if (i >= 0) emit(true, i, i, 0.0);
            if (j >= 0) emit(true, j, j, 0.0);
            if (both) { emit(true, i, j, 0.0); emit(true, j, i, 0.0); }
            break;
        case kQ: {   // compiler.rs:489-497, (C, B, E) x (C, B, E)
            const int32_t t[3] = {i, j, t3};
            for (int a = 0; a < 3; ++a)
                for (int c2 = 0; c2 < 3; ++c2)
                    if (t[a] >= 0 && t[c2] >= 0) emit(true, t[a], t[c2], 0.0);
            break;
        }
        case kM: {   // compiler.rs:533-542, rows (D, S) x columns (D, G, S)
            const int32_t r[2] = {i, t3}, cc[3] = {i, j, t3};
            for (int a = 0; a < 2; ++a)
                for (int c2 = 0; c2 < 3; ++c2)
                    if (r[a] >= 0 && cc[c2] >= 0) emit(true, r[a], cc[c2], 0.0);
            break;
        }
        default:
            break;
    }
}

__global__ void stamp_count_kernel(const int32_t *kind, const int32_t *nidx, const int32_t *bk, const double *value,
                                   int64_t m, uint32_t *gcnt, uint32_t *ccnt) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < m; c += (int64_t)gridDim.x * blockDim.x) {
        uint32_t ng = 0, nc = 0;
        stamps(kind[c], nidx[3 * c], nidx[3 * c + 1], nidx[3 * c + 2], bk[c], value[c],
               [&](bool g, int32_t, int32_t, double) { (g ? ng : nc) += 1; });
        gcnt[c] = ng;
        ccnt[c] = nc;
    }
}

__global__ void stamp_write_kernel(const int32_t *kind, const int32_t *nidx, const int32_t *bk, const double *value,
                                   int64_t m, const uint32_t *goff, const uint32_t *coff, uint64_t size,
                                   uint64_t *gkey, double *gval, uint64_t *ckey, double *cval) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < m; c += (int64_t)gridDim.x * blockDim.x) {
        uint32_t pg = goff[c], pc = coff[c];
        stamps(kind[c], nidx[3 * c], nidx[3 * c + 1], nidx[3 * c + 2], bk[c], value[c],
               [&](bool g, int32_t r, int32_t cl, double v) {
                   const uint64_t key = (uint64_t)r * size + (uint64_t)cl;
                   if (g) { gkey[pg] = key; gval[pg] = v; ++pg; }
                   else { ckey[pc] = key; cval[pc] = v; ++pc; }
               });
    }
}

// G's tail: GMIN on the node diagonals, then C's entries as explicit zeros.
__global__ void g_tail_kernel(int64_t n_nodes, uint64_t size, const uint64_t *ckey, int64_t c_trip, uint64_t *gkey,
                              double *gval) {
    const int64_t total = n_nodes + c_trip;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        if (t < n_nodes) {
            gkey[t] = (uint64_t)t * size + (uint64_t)t;
            gval[t] = kGmin;
        } else {
            gkey[t] = ckey[t - n_nodes];
            gval[t] = 0.0;
        }
    }
}

__global__ void iota_kernel(uint32_t *v, int64_t n) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        v[t] = (uint32_t)t;
}

// ------------------------------------------------------------------- CSR --
__global__ void head_flag_kernel(const uint64_t *skey, int64_t n, uint32_t *flag) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        flag[t] = (t == 0 || skey[t] != skey[t - 1]) ? 1u : 0u;
}

__global__ void pattern_kernel(const uint64_t *skey, int64_t n, const uint32_t *flag, const uint32_t *pidx,
                               uint64_t size, uint32_t *col, uint32_t *row_cnt, uint32_t *head) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        if (!flag[t]) continue;
        const uint32_t p = pidx[t];
        col[p] = (uint32_t)(skey[t] % size);
        atomicAdd(&row_cnt[skey[t] / size], 1u);
        head[p] = (uint32_t)t;
    }
}

// Each entry's value: its triplets (sorted, in triplet order) summed left to
// right; skip_zero leaves zero-valued triplets out (CsrMatrix values), else
// every triplet is added (the current-source rhs, accumulated in place).
__global__ void entry_sum_kernel(const uint32_t *sidx, const double *val, const uint32_t *head, int64_t nnz,
                                 int64_t n, bool skip_zero, double *out) {
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < nnz; p += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = p + 1 < nnz ? (int64_t)head[p + 1] : n;
        double acc = 0.0;
        for (int64_t t = head[p]; t < e; ++t) {
            const double v = val[sidx[t]];
            if (!skip_zero || v != 0.0) acc = acc + v;
        }
        out[p] = acc;
    }
}

// ----------------------------------------------------------- rhs, fixed --
__global__ void isrc_count_kernel(const int32_t *kind, const int32_t *nidx, const double *value, int64_t m,
                                  uint32_t *cnt) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < m; c += (int64_t)gridDim.x * blockDim.x) {
        uint32_t k = 0;
        if (kind[c] == kI && !isnan(value[c])) k = (nidx[3 * c] >= 0 ? 1u : 0u) + (nidx[3 * c + 1] >= 0 ? 1u : 0u);
        cnt[c] = k;
    }
}

__global__ void isrc_write_kernel(const int32_t *kind, const int32_t *nidx, const double *value, int64_t m,
                                  const uint32_t *off, uint64_t *key, double *val) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < m; c += (int64_t)gridDim.x * blockDim.x) {
        if (kind[c] != kI || isnan(value[c])) continue;
        uint32_t p = off[c];
        if (nidx[3 * c] >= 0) { key[p] = (uint64_t)nidx[3 * c]; val[p] = -value[c]; ++p; }
        if (nidx[3 * c + 1] >= 0) { key[p] = (uint64_t)nidx[3 * c + 1]; val[p] = value[c]; }
    }
}

__global__ void scatter_rows_kernel(const uint64_t *skey, const uint32_t *flag, const uint32_t *pidx, int64_t n,
                                    const double *sums, double *b) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        if (flag[t]) b[skey[t]] = sums[pidx[t]];
}

__global__ void vsrc_kernel(const int32_t *kind, const int32_t *nidx, const int32_t *bk, const double *value,
                            int64_t m, double *b, uint8_t *fixed) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < m; c += (int64_t)gridDim.x * blockDim.x) {
        if (kind[c] != kV) continue;
        if (!isnan(value[c])) b[bk[c]] = value[c];
        if (nidx[3 * c] >= 0) fixed[nidx[3 * c]] = 1;          // compiler.rs:582-595
        if (nidx[3 * c + 1] >= 0) fixed[nidx[3 * c + 1]] = 1;
    }
}

// ----------------------------------------------------------- descriptors --
__device__ __forceinline__ uint32_t value_index(const uint32_t *rp, const uint32_t *col, int32_t r, int32_t c) {
    if (r < 0 || c < 0) return kNone;
    uint32_t lo = rp[r], hi = rp[r + 1];
    while (lo < hi) {
        const uint32_t mid = lo + (hi - lo) / 2;
        if (col[mid] < (uint32_t)c) lo = mid + 1;
        else hi = mid;
    }
    return (lo < rp[r + 1] && col[lo] == (uint32_t)c) ? lo : kNone;
}

__device__ __forceinline__ uint32_t u32n(int32_t a) { return a >= 0 ? (uint32_t)a : kNone; }

__global__ void descriptor_kernel(const int32_t *kind, const int32_t *nidx, const double *params, int64_t m,
                                  const uint32_t *dpos, const uint32_t *qpos, const uint32_t *mpos,
                                  const uint32_t *rp, const uint32_t *col, const uint8_t *fixed, DiodeDesc *dd,
                                  BjtDesc *qd, MosfetDesc *md) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < m; c += (int64_t)gridDim.x * blockDim.x) {
        const int32_t k = kind[c];
        const int32_t a = nidx[3 * c], b = nidx[3 * c + 1], e = nidx[3 * c + 2];
        const double *p = params + c * 7;
        auto fx = [&](int32_t n) -> uint32_t { return n >= 0 ? (uint32_t)fixed[n] : 0u; };
        if (k == kD) {                 // compiler.rs:597-640
            DiodeDesc d{};
            d.anode = u32n(a);
            d.cathode = u32n(b);
            d.is_val = (float)p[0];
            d.n_vt = (float)(p[1] * kVt300);
            d.g_row_col[0] = value_index(rp, col, a, a);
            d.g_row_col[1] = value_index(rp, col, b, b);
            d.g_row_col[2] = value_index(rp, col, a, b);
            d.g_row_col[3] = value_index(rp, col, b, a);
            d.b_idx[0] = u32n(a);
            d.b_idx[1] = u32n(b);
            dd[dpos[c]] = d;
        } else if (k == kQ) {          // compiler.rs:642-690
            BjtDesc q{};
            q.collector = u32n(a);
            q.base = u32n(b);
            q.emitter = u32n(e);
            q.polarity = p[5] != 0.0 ? 1.0f : -1.0f;
            q.is_val = (float)p[0];
            q.bf = (float)p[1];
            q.br = (float)p[2];
            q.nf_vt = (float)(p[3] * kVt300);
            q.nr_vt = (float)(p[4] * kVt300);
            const int32_t t[3] = {a, b, e};
            for (int x = 0; x < 3; ++x) {
                q.node_fixed[x] = fx(t[x]);
                q.b_idx[x] = u32n(t[x]);
                for (int y = 0; y < 3; ++y) q.g_row_col[3 * x + y] = value_index(rp, col, t[x], t[y]);
            }
            qd[qpos[c]] = q;
        } else if (k == kM) {          // compiler.rs:692-740
            MosfetDesc mo{};
            mo.drain = u32n(a);
            mo.gate = u32n(b);
            mo.source = u32n(e);
            mo.polarity = p[3] != 0.0 ? 1.0f : -1.0f;
            mo.vto = (float)fabs(p[0]);
            mo.kp = (float)p[1];
            mo.lambda = (float)p[2];
            mo.node_fixed_packed = fx(a) | (fx(b) << 1) | (fx(e) << 2);
            const int32_t r[2] = {a, e}, cc[3] = {a, b, e};
            for (int x = 0; x < 2; ++x)
                for (int y = 0; y < 3; ++y) mo.g_row_col[3 * x + y] = value_index(rp, col, r[x], cc[y]);
            mo.b_idx[0] = u32n(a);
            mo.b_idx[1] = u32n(e);
            md[mpos[c]] = mo;
        }
    }
}

}  // namespace

struct ohm_netlist {
    ohm_ctx *ctx = nullptr;
    ohm_netlist_sizes sz{};
    std::vector<void *> allocs;
    uint32_t *g_rp = nullptr, *g_col = nullptr, *c_rp = nullptr, *c_col = nullptr;
    double *g_val = nullptr, *c_val = nullptr, *b_dc = nullptr;
    int64_t *labels = nullptr, *branch_comp = nullptr;
    DiodeDesc *dd = nullptr;
    BjtDesc *qd = nullptr;
    MosfetDesc *md = nullptr;

    template <typename T>
    cudaError_t get(T **p, size_t count) {
        cudaError_t e = dalloc(p, count);
        if (e == cudaSuccess) allocs.push_back((void *)*p);
        return e;
    }
    ~ohm_netlist() {
        for (void *q : allocs) ohm_pool_free(q);
    }
};

namespace {

// Sorts n (key, value) triplets and builds the CSR of `rows` rows on them:
// row_ptr (rows + 1), col (nnz) and the entry sums into *val_out; returns nnz.
ohm_status build_csr(ohm_netlist *nl, uint64_t *key, double *val, int64_t n, int64_t rows, uint32_t **rp_out,
                     uint32_t **col_out, double **val_out, int64_t *nnz_out, cudaStream_t s, Arena &ar) {
    uint32_t *idx = nullptr, *vt = nullptr, *flag = nullptr, *pidx = nullptr, *tot = nullptr, *cnt = nullptr;
    uint64_t *kt = nullptr;
    ARENA_TRY(ar.get(&idx, n));
    ARENA_TRY(ar.get(&vt, n));
    ARENA_TRY(ar.get(&kt, n));
    ARENA_TRY(ar.get(&flag, n));
    ARENA_TRY(ar.get(&pidx, n));
    ARENA_TRY(ar.get(&tot, 1));
    ARENA_TRY(ar.get(&cnt, rows + 1));
    iota_kernel<<<blocks_for(n), kT, 0, s>>>(idx, n);
    ARENA_TRY(cudaGetLastError());
    const uint64_t maxkey = (uint64_t)rows * (uint64_t)rows;
    int bits = 0;
    while (bits < 64 && (maxkey >> bits) != 0) ++bits;
    ARENA_TRY(radix_sort(key, idx, kt, vt, n, bits, s, ar));
    head_flag_kernel<<<blocks_for(n), kT, 0, s>>>(key, n, flag);
    ARENA_TRY(cudaGetLastError());
    ARENA_TRY(scan_u32(flag, pidx, n, tot, s, ar));
    uint32_t nnz32 = 0;
    ARENA_TRY(cudaMemcpyAsync(&nnz32, tot, sizeof nnz32, cudaMemcpyDeviceToHost, s));
    ARENA_TRY(cudaStreamSynchronize(s));
    const int64_t nnz = n > 0 ? (int64_t)nnz32 : 0;
    uint32_t *col = nullptr, *head = nullptr, *rp = nullptr;
    double *vals = nullptr;
    ARENA_TRY(nl->get(&col, nnz));
    ARENA_TRY(nl->get(&vals, nnz));
    ARENA_TRY(nl->get(&rp, rows + 1));
    ARENA_TRY(ar.get(&head, nnz));
    ARENA_TRY(cudaMemsetAsync(cnt, 0, (rows + 1) * sizeof(uint32_t), s));
    if (n > 0) {
        pattern_kernel<<<blocks_for(n), kT, 0, s>>>(key, n, flag, pidx, (uint64_t)std::max<int64_t>(rows, 1), col, cnt,
                                                    head);
        ARENA_TRY(cudaGetLastError());
        entry_sum_kernel<<<blocks_for(nnz), kT, 0, s>>>(idx, val, head, nnz, n, true, vals);
        ARENA_TRY(cudaGetLastError());
    }
    ARENA_TRY(scan_u32(cnt, rp, rows + 1, tot, s, ar));
    *rp_out = rp;
    *col_out = col;
    *val_out = vals;
    *nnz_out = nnz;
    return OHM_OK;
}

}  // namespace

extern "C" ohm_status ohm_compile(ohm_ctx *c, int64_t m, const int32_t *kind, const int64_t *nodes,
                                  const double *value, const double *params, ohm_netlist **out) {
    if (!c || !out || m < 0 || (m > 0 && (!kind || !nodes || !value || !params)))
        return ohm_fail(OHM_ERR_INVALID_ARG, "bad compile arguments");
    *out = nullptr;
    if (3 * m >= (int64_t)0x7FFFFFFF) return ohm_fail(OHM_ERR_INVALID_ARG, "too many components");
    for (int64_t i = 0; i < m; ++i)
        if (kind[i] < kR || kind[i] > kM) return ohm_fail(OHM_ERR_INVALID_ARG, "component %lld: unknown kind %d",
                                                          (long long)i, kind[i]);
    CUDA_TRY(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    Arena ar;
    ohm_netlist *nl = new ohm_netlist();
    nl->ctx = c;
    auto fail = [&](ohm_status st) {
        cudaStreamSynchronize(s);
        delete nl;
        return st;
    };
#define NL_TRY(expr)                                                                              \
    do {                                                                                          \
        cudaError_t e_ = (expr);                                                                  \
        if (e_ != cudaSuccess) return fail(ohm_fail(OHM_ERR_CUDA, "compile: %s", cudaGetErrorString(e_))); \
    } while (0)
#define ST_TRY(expr)                            \
    do {                                        \
        ohm_status st_ = (expr);                \
        if (st_ != OHM_OK) return fail(st_);    \
    } while (0)

    // ---- inputs ----
    int32_t *d_kind = nullptr;
    int64_t *d_nodes = nullptr;
    double *d_value = nullptr, *d_params = nullptr;
    NL_TRY(ar.get(&d_kind, m));
    NL_TRY(ar.get(&d_nodes, 3 * m));
    NL_TRY(ar.get(&d_value, m));
    NL_TRY(ar.get(&d_params, 7 * m));
    if (m) {
        NL_TRY(cudaMemcpyAsync(d_kind, kind, m * sizeof(int32_t), cudaMemcpyHostToDevice, s));
        NL_TRY(cudaMemcpyAsync(d_nodes, nodes, 3 * m * sizeof(int64_t), cudaMemcpyHostToDevice, s));
        NL_TRY(cudaMemcpyAsync(d_value, value, m * sizeof(double), cudaMemcpyHostToDevice, s));
        NL_TRY(cudaMemcpyAsync(d_params, params, 7 * m * sizeof(double), cudaMemcpyHostToDevice, s));
    }
    // ---- validation ----
    unsigned long long *d_bad = nullptr;
    NL_TRY(ar.get(&d_bad, 5));
    NL_TRY(cudaMemsetAsync(d_bad, 0xFF, 5 * sizeof(unsigned long long), s));
    if (m) validate_kernel<<<blocks_for(m), kT, 0, s>>>(d_kind, d_value, d_params, m, d_bad);
    NL_TRY(cudaGetLastError());
    unsigned long long bad[5];
    NL_TRY(cudaMemcpyAsync(bad, d_bad, sizeof bad, cudaMemcpyDeviceToHost, s));
    NL_TRY(cudaStreamSynchronize(s));
    static const char *what[5] = {"Resistor component %lld has zero resistance",
                                  "Capacitor component %lld has negative capacitance",
                                  "Diode component %lld references undefined model",
                                  "BJT component %lld references undefined model",
                                  "MOSFET component %lld references undefined model"};
    for (int k = 0; k < 5; ++k)
        if (bad[k] != ~0ull) return fail(ohm_fail(OHM_ERR_COMPILE, what[k], (long long)bad[k]));

    // ---- node numbering by first appearance ----
    const int64_t nt = 3 * m;
    uint64_t cap = 64;
    while (cap < 2 * (uint64_t)nt) cap <<= 1;
    uint64_t *hkeys = nullptr;
    uint32_t *hfirst = nullptr, *flag = nullptr, *rank = nullptr, *d_tot = nullptr;
    int32_t *nidx = nullptr;
    NL_TRY(ar.get(&hkeys, cap));
    NL_TRY(ar.get(&hfirst, cap));
    NL_TRY(ar.get(&flag, nt));
    NL_TRY(ar.get(&rank, nt));
    NL_TRY(ar.get(&nidx, nt));
    NL_TRY(ar.get(&d_tot, 1));
    NL_TRY(cudaMemsetAsync(hkeys, 0, cap * sizeof(uint64_t), s));
    NL_TRY(cudaMemsetAsync(hfirst, 0xFF, cap * sizeof(uint32_t), s));
    if (nt) {
        label_insert_kernel<<<blocks_for(nt), kT, 0, s>>>(d_kind, d_nodes, nt, hkeys, hfirst, cap - 1);
        first_flag_kernel<<<blocks_for(nt), kT, 0, s>>>(d_kind, d_nodes, nt, hkeys, hfirst, cap - 1, flag);
        NL_TRY(cudaGetLastError());
    }
    NL_TRY(scan_u32(flag, rank, nt, d_tot, s, ar));
    uint32_t n_nodes32 = 0;
    NL_TRY(cudaMemcpyAsync(&n_nodes32, d_tot, sizeof n_nodes32, cudaMemcpyDeviceToHost, s));
    NL_TRY(cudaStreamSynchronize(s));
    const int64_t n_nodes = nt ? (int64_t)n_nodes32 : 0;
    NL_TRY(nl->get(&nl->labels, n_nodes));
    if (nt) {
        assign_nodes_kernel<<<blocks_for(nt), kT, 0, s>>>(d_kind, d_nodes, nt, hkeys, hfirst, cap - 1, rank, nidx,
                                                          nl->labels);
        NL_TRY(cudaGetLastError());
    }

    // ---- branches (V sources and inductors, component order) ----
    uint32_t *cflag = nullptr, *cscan = nullptr;
    int32_t *bk = nullptr;
    NL_TRY(ar.get(&cflag, m));
    NL_TRY(ar.get(&cscan, m));
    NL_TRY(ar.get(&bk, m));
    if (m) kind_flag_kernel<<<blocks_for(m), kT, 0, s>>>(d_kind, m, kV, kL, cflag);
    NL_TRY(cudaGetLastError());
    NL_TRY(scan_u32(cflag, cscan, m, d_tot, s, ar));
    uint32_t n_br32 = 0;
    NL_TRY(cudaMemcpyAsync(&n_br32, d_tot, sizeof n_br32, cudaMemcpyDeviceToHost, s));
    NL_TRY(cudaStreamSynchronize(s));
    const int64_t n_br = m ? (int64_t)n_br32 : 0;
    const int64_t size = n_nodes + n_br;
    if (size >= (int64_t)0xFFFFFFFF) return fail(ohm_fail(OHM_ERR_INVALID_ARG, "system too large"));
    NL_TRY(nl->get(&nl->branch_comp, n_br));
    if (m) branch_kernel<<<blocks_for(m), kT, 0, s>>>(d_kind, m, cscan, n_nodes, bk, nl->branch_comp);
    NL_TRY(cudaGetLastError());

    // ---- triplets in triplet order ----
    uint32_t *gcnt = nullptr, *ccnt = nullptr, *goff = nullptr, *coff = nullptr, *gtot = nullptr, *ctot = nullptr;
    NL_TRY(ar.get(&gcnt, m));
    NL_TRY(ar.get(&ccnt, m));
    NL_TRY(ar.get(&goff, m));
    NL_TRY(ar.get(&coff, m));
    NL_TRY(ar.get(&gtot, 1));
    NL_TRY(ar.get(&ctot, 1));
    if (m) stamp_count_kernel<<<blocks_for(m), kT, 0, s>>>(d_kind, nidx, bk, d_value, m, gcnt, ccnt);
    NL_TRY(cudaGetLastError());
    NL_TRY(scan_u32(gcnt, goff, m, gtot, s, ar));
    NL_TRY(scan_u32(ccnt, coff, m, ctot, s, ar));
    uint32_t tots[2] = {0, 0};
    NL_TRY(cudaMemcpyAsync(&tots[0], gtot, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    NL_TRY(cudaMemcpyAsync(&tots[1], ctot, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    NL_TRY(cudaStreamSynchronize(s));
    const int64_t g_comp = m ? tots[0] : 0, c_trip = m ? tots[1] : 0;
    const int64_t g_trip = g_comp + n_nodes + c_trip;
    uint64_t *gkey = nullptr, *ckey = nullptr, *ckey_copy = nullptr;
    double *gval = nullptr, *cval = nullptr;
    NL_TRY(ar.get(&gkey, g_trip));
    NL_TRY(ar.get(&gval, g_trip));
    NL_TRY(ar.get(&ckey, c_trip));
    NL_TRY(ar.get(&ckey_copy, c_trip));
    NL_TRY(ar.get(&cval, c_trip));
    const uint64_t usize = (uint64_t)std::max<int64_t>(size, 1);
    if (m)
        stamp_write_kernel<<<blocks_for(m), kT, 0, s>>>(d_kind, nidx, bk, d_value, m, goff, coff, usize, gkey, gval,
                                                        ckey, cval);
    NL_TRY(cudaGetLastError());
    if (n_nodes + c_trip)
        g_tail_kernel<<<blocks_for(n_nodes + c_trip), kT, 0, s>>>(n_nodes, usize, ckey, c_trip, gkey + g_comp,
                                                                  gval + g_comp);
    NL_TRY(cudaGetLastError());
    if (c_trip) NL_TRY(cudaMemcpyAsync(ckey_copy, ckey, c_trip * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));

    // ---- CSR of G and C ----
    int64_t g_nnz = 0, c_nnz = 0;
    ST_TRY(build_csr(nl, gkey, gval, g_trip, size, &nl->g_rp, &nl->g_col, &nl->g_val, &g_nnz, s, ar));
    ST_TRY(build_csr(nl, ckey_copy, cval, c_trip, size, &nl->c_rp, &nl->c_col, &nl->c_val, &c_nnz, s, ar));

    // ---- rhs: V sources at their branch rows, current sources in order ----
    uint8_t *fixed = nullptr;
    NL_TRY(nl->get(&nl->b_dc, size));
    NL_TRY(ar.get(&fixed, std::max<int64_t>(n_nodes, 1)));
    NL_TRY(cudaMemsetAsync(nl->b_dc, 0, std::max<int64_t>(size, 1) * sizeof(double), s));
    NL_TRY(cudaMemsetAsync(fixed, 0, std::max<int64_t>(n_nodes, 1), s));
    if (m) vsrc_kernel<<<blocks_for(m), kT, 0, s>>>(d_kind, nidx, bk, d_value, m, nl->b_dc, fixed);
    NL_TRY(cudaGetLastError());
    {
        uint32_t *icnt = nullptr, *ioff = nullptr;
        NL_TRY(ar.get(&icnt, m));
        NL_TRY(ar.get(&ioff, m));
        if (m) isrc_count_kernel<<<blocks_for(m), kT, 0, s>>>(d_kind, nidx, d_value, m, icnt);
        NL_TRY(cudaGetLastError());
        NL_TRY(scan_u32(icnt, ioff, m, d_tot, s, ar));
        uint32_t ni32 = 0;
        NL_TRY(cudaMemcpyAsync(&ni32, d_tot, sizeof ni32, cudaMemcpyDeviceToHost, s));
        NL_TRY(cudaStreamSynchronize(s));
        const int64_t ni = m ? (int64_t)ni32 : 0;
        if (ni) {
            uint64_t *ikey = nullptr, *ikt = nullptr;
            double *ival = nullptr, *isum = nullptr;
            uint32_t *iidx = nullptr, *ivt = nullptr, *iflag = nullptr, *ipidx = nullptr, *ihead = nullptr;
            NL_TRY(ar.get(&ikey, ni));
            NL_TRY(ar.get(&ikt, ni));
            NL_TRY(ar.get(&ival, ni));
            NL_TRY(ar.get(&iidx, ni));
            NL_TRY(ar.get(&ivt, ni));
            NL_TRY(ar.get(&iflag, ni));
            NL_TRY(ar.get(&ipidx, ni));
            isrc_write_kernel<<<blocks_for(m), kT, 0, s>>>(d_kind, nidx, d_value, m, ioff, ikey, ival);
            iota_kernel<<<blocks_for(ni), kT, 0, s>>>(iidx, ni);
            NL_TRY(cudaGetLastError());
            int bits = 0;
            while (bits < 64 && ((uint64_t)size >> bits) != 0) ++bits;
            NL_TRY(radix_sort(ikey, iidx, ikt, ivt, ni, bits, s, ar));
            head_flag_kernel<<<blocks_for(ni), kT, 0, s>>>(ikey, ni, iflag);
            NL_TRY(cudaGetLastError());
            NL_TRY(scan_u32(iflag, ipidx, ni, d_tot, s, ar));
            uint32_t nr32 = 0;
            NL_TRY(cudaMemcpyAsync(&nr32, d_tot, sizeof nr32, cudaMemcpyDeviceToHost, s));
            NL_TRY(cudaStreamSynchronize(s));
            NL_TRY(ar.get(&ihead, nr32));
            NL_TRY(ar.get(&isum, nr32));
            uint32_t *dummy_cnt = nullptr, *dummy_col = nullptr;
            NL_TRY(ar.get(&dummy_cnt, size + 1));
            NL_TRY(ar.get(&dummy_col, nr32));
            NL_TRY(cudaMemsetAsync(dummy_cnt, 0, (size + 1) * sizeof(uint32_t), s));
            pattern_kernel<<<blocks_for(ni), kT, 0, s>>>(ikey, ni, iflag, ipidx, usize, dummy_col, dummy_cnt, ihead);
            entry_sum_kernel<<<blocks_for(nr32), kT, 0, s>>>(iidx, ival, ihead, nr32, ni, false, isum);
            scatter_rows_kernel<<<blocks_for(ni), kT, 0, s>>>(ikey, iflag, ipidx, ni, isum, nl->b_dc);
            NL_TRY(cudaGetLastError());
        }
    }

    // ---- descriptors ----
    uint32_t *dpos = nullptr, *qpos = nullptr, *mpos = nullptr;
    NL_TRY(ar.get(&dpos, m));
    NL_TRY(ar.get(&qpos, m));
    NL_TRY(ar.get(&mpos, m));
    uint32_t counts3[3] = {0, 0, 0};
    const int32_t dev_kinds[3] = {kD, kQ, kM};
    uint32_t *pos3[3] = {dpos, qpos, mpos};
    for (int k = 0; k < 3; ++k) {
        if (m) kind_flag_kernel<<<blocks_for(m), kT, 0, s>>>(d_kind, m, dev_kinds[k], dev_kinds[k], cflag);
        NL_TRY(cudaGetLastError());
        NL_TRY(scan_u32(cflag, pos3[k], m, d_tot, s, ar));
        NL_TRY(cudaMemcpyAsync(&counts3[k], d_tot, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        NL_TRY(cudaStreamSynchronize(s));
        if (!m) counts3[k] = 0;
    }
    NL_TRY(nl->get(&nl->dd, counts3[0]));
    NL_TRY(nl->get(&nl->qd, counts3[1]));
    NL_TRY(nl->get(&nl->md, counts3[2]));
    if (m)
        descriptor_kernel<<<blocks_for(m), kT, 0, s>>>(d_kind, nidx, d_params, m, dpos, qpos, mpos, nl->g_rp,
                                                       nl->g_col, fixed, nl->dd, nl->qd, nl->md);
    NL_TRY(cudaGetLastError());
    NL_TRY(cudaStreamSynchronize(s));
#undef NL_TRY
#undef ST_TRY

    nl->sz.n_nodes = n_nodes;
    nl->sz.size = size;
    nl->sz.n_branches = n_br;
    nl->sz.g_nnz = g_nnz;
    nl->sz.c_nnz = c_nnz;
    nl->sz.n_diodes = counts3[0];
    nl->sz.n_bjts = counts3[1];
    nl->sz.n_mosfets = counts3[2];
    ohm_ctx_retain(c);
    *out = nl;
    return OHM_OK;
}

extern "C" ohm_status ohm_netlist_get_sizes(const ohm_netlist *nl, ohm_netlist_sizes *out) {
    if (!nl || !out) return ohm_fail(OHM_ERR_INVALID_ARG, "null argument");
    *out = nl->sz;
    return OHM_OK;
}

extern "C" ohm_status ohm_netlist_download(const ohm_netlist *nl, uint32_t *g_row_ptr, uint32_t *g_col,
                                           double *g_val, uint32_t *c_row_ptr, uint32_t *c_col, double *c_val,
                                           double *b_dc, int64_t *node_labels, int64_t *branch_components,
                                           ohm_diode_desc *diodes, ohm_bjt_desc *bjts, ohm_mosfet_desc *mosfets) {
    if (!nl) return ohm_fail(OHM_ERR_INVALID_ARG, "null netlist");
    ohm_ctx *c = nl->ctx;
    CUDA_TRY(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    const ohm_netlist_sizes &z = nl->sz;
    auto get = [&](void *dst, const void *src, size_t bytes) -> cudaError_t {
        if (!dst || bytes == 0) return cudaSuccess;
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s);
    };
    CUDA_TRY(get(g_row_ptr, nl->g_rp, (z.size + 1) * sizeof(uint32_t)));
    CUDA_TRY(get(g_col, nl->g_col, z.g_nnz * sizeof(uint32_t)));
    CUDA_TRY(get(g_val, nl->g_val, z.g_nnz * sizeof(double)));
    CUDA_TRY(get(c_row_ptr, nl->c_rp, (z.size + 1) * sizeof(uint32_t)));
    CUDA_TRY(get(c_col, nl->c_col, z.c_nnz * sizeof(uint32_t)));
    CUDA_TRY(get(c_val, nl->c_val, z.c_nnz * sizeof(double)));
    CUDA_TRY(get(b_dc, nl->b_dc, z.size * sizeof(double)));
    CUDA_TRY(get(node_labels, nl->labels, z.n_nodes * sizeof(int64_t)));
    CUDA_TRY(get(branch_components, nl->branch_comp, z.n_branches * sizeof(int64_t)));
    CUDA_TRY(get(diodes, nl->dd, z.n_diodes * sizeof(DiodeDesc)));
    CUDA_TRY(get(bjts, nl->qd, z.n_bjts * sizeof(BjtDesc)));
    CUDA_TRY(get(mosfets, nl->md, z.n_mosfets * sizeof(MosfetDesc)));
    CUDA_TRY(cudaStreamSynchronize(s));
    return OHM_OK;
}

extern "C" ohm_status ohm_netlist_destroy(ohm_netlist *nl) {
    if (!nl) return OHM_OK;
    ohm_ctx *c = nl->ctx;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    delete nl;
    ohm_ctx_release(c);
    return OHM_OK;
}
