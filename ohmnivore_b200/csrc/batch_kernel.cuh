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
__host__ __device__ inline P *offset(P *p, int64_t k) { return p ? p + k : p; }

// Where instance i sits in the packed arrays (read from BatchArgs' device
// tables by the batch kernel, from host copies by the whole-GPU path).
struct InstanceOffsets {
    int64_t ro, ro1, no, no1, dq, dq1, qq, qq1, mq, mq1, ms, ms1, mid, rs, rs1, rid;
    int n_nodes;
};

// Kernel arguments of instance i: B.base with every per-row, per-nonzero and
// per-device pointer moved to the instance's slice.
__host__ __device__ inline void instance_args(const BatchArgs &B, int i, const InstanceOffsets &o, KernelArgs &a) {
    const int64_t ro = o.ro, no = o.no;
    const int64_t dq = o.dq, qq = o.qq, mq = o.mq;
    a = B.base;
    a.n = (int)(o.ro1 - ro);
    a.nnz = (int)(o.no1 - no);
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
    a.nd = (int)(o.dq1 - dq);
    a.nq = (int)(o.qq1 - qq);
    a.nm = (int)(o.mq1 - mq);
    a.diodes = B.base.diodes + dq;
    a.bjts = B.base.bjts + qq;
    a.mosfets = B.base.mosfets + mq;
    a.bjt_vaf = offset(B.base.bjt_vaf, qq);
    a.mstamp = B.base.mstamp + 4 * dq + 9 * qq + 6 * mq;
    a.rstamp = B.base.rstamp + 2 * dq + 3 * qq + 2 * mq;
    a.n_mslots = (int)(o.ms1 - o.ms);
    a.mslot = B.base.mslot + o.ms;
    a.mslot_ptr = B.base.mslot_ptr + o.ms + i;
    a.mslot_ids = B.base.mslot_ids + o.mid;
    a.n_rrows = (int)(o.rs1 - o.rs);
    a.rrow = B.base.rrow + o.rs;
    a.rrow_ptr = B.base.rrow_ptr + o.rs + i;
    a.rrow_ids = B.base.rrow_ids + o.rid;
    a.node_scale = (unsigned long long *)(B.node_scale_base + ro);
    a.trace = nullptr;
    a.n_nodes = o.n_nodes;
    a.stampflag = B.stampflag + ro;
    a.x_good = B.x_good + ro;
}

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
        InstanceOffsets o;
        o.ro = B.row_off[i]; o.ro1 = B.row_off[i + 1]; o.no = B.nnz_off[i]; o.no1 = B.nnz_off[i + 1];
        o.dq = B.d_off[i]; o.dq1 = B.d_off[i + 1]; o.qq = B.q_off[i]; o.qq1 = B.q_off[i + 1];
        o.mq = B.m_off[i]; o.mq1 = B.m_off[i + 1];
        o.ms = B.ms_off[i]; o.ms1 = B.ms_off[i + 1]; o.mid = B.mid_off[i];
        o.rs = B.rs_off[i]; o.rs1 = B.rs_off[i + 1]; o.rid = B.rid_off[i];
        o.n_nodes = B.n_nodes ? B.n_nodes[i] : 0;
        KernelArgs a;
        instance_args(B, i, o, a);
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
