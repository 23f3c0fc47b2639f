// Batch kernel: one thread block per circuit of a packed block-diagonal
// batch, instances taken from a work queue in decreasing order of nonzeros.
// Instantiated per (lanes per row, block size, blocks per SM) in the
// batch_k*.cu units so the autotuner can choose among them.
#pragma once

#include "solver_kernel.cuh"

namespace ohm {

struct BatchArgs {
    KernelArgs base;                // pointers to the packed arrays, shared scalars
    int n_inst;
    const int64_t *row_off, *nnz_off;
    const int64_t *d_off, *q_off, *m_off;      // device descriptor offsets
    const int64_t *ms_off, *mid_off, *rs_off, *rid_off;   // stamp-map offsets
    const int32_t *order;           // instances by decreasing nnz
    unsigned int *queue;            // next position in `order`
    DeviceInfo *infos;              // per instance
    double *node_scale_base;        // per row (8 bytes)
    const int32_t *n_nodes;         // per instance (continuation), may be null
    const uint8_t *stampflag;       // per row
    double *x_good;                 // per row
};

template <typename P>
__device__ __forceinline__ P *offset(P *p, int64_t k) { return p ? p + k : p; }

template <int LPR, int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) batch_solver(BatchArgs B) {
    __shared__ double smem[32 * 4];
    __shared__ int s_q;
    for (;;) {
        if (threadIdx.x == 0) s_q = (int)atomicAdd(B.queue, 1u);
        __syncthreads();
        const int q = s_q;
        __syncthreads();
        if (q >= B.n_inst) return;
        const int i = B.order[q];
        const int64_t ro = B.row_off[i], no = B.nnz_off[i];
        const int64_t dq = B.d_off[i], qq = B.q_off[i], mq = B.m_off[i];
        KernelArgs a = B.base;
        a.n = (int)(B.row_off[i + 1] - ro);
        a.nnz = (int)(B.nnz_off[i + 1] - no);
        a.row_ptr = B.base.row_ptr + ro + i;               // n_i + 1 local row pointers
        a.col = B.base.col + no;
        a.vals64 = B.base.vals64 + no;
        a.vals32 = offset(B.base.vals32, no);
        a.base_vals = B.base.base_vals + no;
        a.base_b = B.base.base_b + ro;
        a.b = B.base.b + ro;
        a.x = B.base.x + ro;
        a.x_prev = B.base.x_prev + ro;
        a.r64 = B.base.r64 + ro;
        a.dx = B.base.dx + ro;
        a.partner = B.base.partner + ro;
        a.diag_slot = B.base.diag_slot + ro;
        a.off_slot = B.base.off_slot + ro;
        a.rowflag = offset(B.base.rowflag, ro);
        a.pc_part = (double *)B.base.pc_part + ro;
        a.rec0 = (double *)B.base.rec0 + 4 * ro;
        a.rec1 = (double *)B.base.rec1 + 4 * ro;
        a.rhat = (double *)B.base.rhat + ro;
        a.s = (double *)B.base.s + ro;
        a.t = (double *)B.base.t + ro;
        a.phat = (double *)B.base.phat + ro;
        a.shat = (double *)B.base.shat + ro;
        a.d = (double *)B.base.d + ro;
        a.nd = (int)(B.d_off[i + 1] - dq);
        a.nq = (int)(B.q_off[i + 1] - qq);
        a.nm = (int)(B.m_off[i + 1] - mq);
        a.diodes = B.base.diodes + dq;
        a.bjts = B.base.bjts + qq;
        a.mosfets = B.base.mosfets + mq;
        a.bjt_vaf = offset(B.base.bjt_vaf, qq);
        a.mstamp = B.base.mstamp + 4 * dq + 9 * qq + 6 * mq;
        a.rstamp = B.base.rstamp + 2 * dq + 3 * qq + 2 * mq;
        a.n_mslots = (int)(B.ms_off[i + 1] - B.ms_off[i]);
        a.mslot = B.base.mslot + B.ms_off[i];
        a.mslot_ptr = B.base.mslot_ptr + B.ms_off[i] + i;
        a.mslot_ids = B.base.mslot_ids + B.mid_off[i];
        a.n_rrows = (int)(B.rs_off[i + 1] - B.rs_off[i]);
        a.rrow = B.base.rrow + B.rs_off[i];
        a.rrow_ptr = B.base.rrow_ptr + B.rs_off[i] + i;
        a.rrow_ids = B.base.rrow_ids + B.rid_off[i];
        a.node_scale = (unsigned long long *)(B.node_scale_base + ro);
        a.trace = nullptr;
        a.n_nodes = B.n_nodes ? B.n_nodes[i] : 0;
        a.stampflag = B.stampflag + ro;
        a.x_good = B.x_good + ro;
        BlockTeam g;
        g.r0 = 0;
        g.r1 = a.n;
        g.gtid = threadIdx.x;
        g.gstride = blockDim.x;
        g.smem = smem;
        solve_body<LPR>(a, g, &B.infos[i]);
        __syncthreads();
    }
}

using BatchFn = void (*)(BatchArgs);

// Candidate launch shapes: threads per block and the blocks per SM the
// register budget is fitted to (256x2: 128 registers, 256x4 and 128x8: 64).
struct BatchShape { int block, min_blocks; };
constexpr BatchShape kBatchShapes[] = {{256, 2}, {256, 4}, {128, 8}};
constexpr int kNumBatchShapes = 3;

// Kernel for lanes per row 1, 2, 4 or 8 and a shape index.
BatchFn batch_kernel_lpr1(int shape);
BatchFn batch_kernel_lpr2(int shape);
BatchFn batch_kernel_lpr4(int shape);
BatchFn batch_kernel_lpr8(int shape);

inline BatchFn batch_kernel(int lpr, int shape) {
    switch (lpr) {
        case 1: return batch_kernel_lpr1(shape);
        case 2: return batch_kernel_lpr2(shape);
        case 4: return batch_kernel_lpr4(shape);
        default: return batch_kernel_lpr8(shape);
    }
}

}  // namespace ohm
