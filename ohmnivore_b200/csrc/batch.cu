// Batched Newton: many independent circuits (Monte Carlo corners, parameter
// sweeps) solved by one launch.  Each block takes circuits from a work queue
// in decreasing order of nonzeros (longest-processing-time first) and runs the
// complete Newton loop of solve_body on it with block-level synchronisation
// only, so blocks never wait on each other.  The systems are stored packed:
// block-diagonal CSR with per-circuit local indices and offset tables.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "batch_kernel.cuh"
#include "host_util.h"

using namespace ohm;

struct ohm_batch {
    ohm_ctx *ctx = nullptr;
    int64_t n_inst = 0, rows = 0, nnz = 0, nd = 0, nq = 0, nm = 0;
    int lpr = 2, shape = 0;             // kernel choice (ohm_batch_autotune)
    std::vector<void *> allocs;
    int32_t *order = nullptr;           // instances by decreasing nnz
    int32_t *sample = nullptr;          // autotune sample (capacity n_inst)
    double *x_tune = nullptr;           // autotune scratch solution
    BatchArgs args{};
    std::vector<DeviceInfo> host_infos;
    DeviceInfo *infos = nullptr;
    unsigned int *queue = nullptr;
    // Host copies of the offset tables and of the largest-first order, for
    // instances solved one at a time by the whole GPU (ohm_batch_set_split).
    std::vector<InstanceOffsets> h_offsets;
    std::vector<int32_t> h_order;
    double *team_partials = nullptr;   // reduction partials of those solves
    int split = 1;

    template <typename T>
    cudaError_t put(T **dst, const T *src, size_t count) {
        cudaError_t e = dalloc(dst, count);
        if (e == cudaSuccess) allocs.push_back((void *)*dst);
        if (e == cudaSuccess && src && count)
            e = cudaMemcpyAsync(*dst, src, count * sizeof(T), cudaMemcpyHostToDevice, ctx->stream);
        return e;
    }
    template <typename T>
    cudaError_t zero(T **dst, size_t count) {
        cudaError_t e = put(dst, (const T *)nullptr, count);
        if (e == cudaSuccess) e = cudaMemsetAsync(*dst, 0, std::max<size_t>(count, 1) * sizeof(T), ctx->stream);
        return e;
    }
};

extern "C" ohm_status ohm_batch_create(ohm_ctx *c, int64_t n_inst, const int64_t *row_off, const int64_t *nnz_off,
                                       const uint32_t *row_ptrs, const uint32_t *col_indices,
                                       const double *base_g_values, const double *base_b,
                                       const int64_t *diode_off, const ohm_diode_desc *diodes,
                                       const int64_t *bjt_off, const ohm_bjt_desc *bjts, const double *bjt_vaf,
                                       const int64_t *mosfet_off, const ohm_mosfet_desc *mosfets,
                                       const int32_t *n_nodes, ohm_batch **out) {
    if (!c || !out || n_inst <= 0 || !row_off || !nnz_off || !row_ptrs || !base_g_values || !base_b ||
        !diode_off || !bjt_off || !mosfet_off)
        return ohm_fail(OHM_ERR_INVALID_ARG, "bad batch arguments");
    *out = nullptr;
    if (row_off[0] != 0 || nnz_off[0] != 0 || diode_off[0] != 0 || bjt_off[0] != 0 || mosfet_off[0] != 0)
        return ohm_fail(OHM_ERR_INVALID_ARG, "offset tables must start at 0");
    const int64_t rows = row_off[n_inst], nnz = nnz_off[n_inst];
    const int64_t nd = diode_off[n_inst], nq = bjt_off[n_inst], nm = mosfet_off[n_inst];
    if ((nnz && !col_indices) || (nd && !diodes) || (nq && !bjts) || (nm && !mosfets))
        return ohm_fail(OHM_ERR_INVALID_ARG, "null packed array");
    if (rows > 0x7fffffffLL || nnz > 0x7fffffffLL) return ohm_fail(OHM_ERR_INVALID_ARG, "batch too large");
    CUDA_TRY(cudaSetDevice(c->device));

    // per-instance validation, stamp maps and preconditioner structure (local indices)
    std::vector<int64_t> ms_off(n_inst + 1, 0), mid_off(n_inst + 1, 0), rs_off(n_inst + 1, 0), rid_off(n_inst + 1, 0);
    std::vector<uint32_t> mslot, mptr, mids, rrow, rptr, rids;
    std::vector<int32_t> partner(rows);
    std::vector<uint32_t> diag(rows), off(rows);
    std::vector<uint8_t> flag(rows), sflag(rows);
    bool any_pair = false;
    int64_t max_nnz_row = 0;
    for (int64_t i = 0; i < n_inst; ++i) {
        const int64_t n = row_off[i + 1] - row_off[i], z = nnz_off[i + 1] - nnz_off[i];
        if (n <= 0 || z < 0) return ohm_fail(OHM_ERR_INVALID_ARG, "instance %lld has no rows", (long long)i);
        const uint32_t *rp = row_ptrs + row_off[i] + i;
        const uint32_t *cl = col_indices + nnz_off[i];
        ohm_status st = check_csr(n, z, rp, cl);
        if (st != OHM_OK) return ohm_fail(st, "instance %lld: %s", (long long)i, ohm_last_error());
        const ohm_diode_desc *d = diodes + diode_off[i];
        const ohm_bjt_desc *q = bjts + bjt_off[i];
        const ohm_mosfet_desc *m = mosfets + mosfet_off[i];
        const int64_t dn = diode_off[i + 1] - diode_off[i], qn = bjt_off[i + 1] - bjt_off[i],
                      mn = mosfet_off[i + 1] - mosfet_off[i];
        st = check_devices(d, dn, q, qn, m, mn, n, z);
        if (st != OHM_OK) return ohm_fail(st, "instance %lld: %s", (long long)i, ohm_last_error());
        std::vector<std::pair<uint32_t, uint32_t>> mp, rp_;
        const uint32_t bq = 4u * (uint32_t)dn, bm = bq + 9u * (uint32_t)qn;
        const uint32_t rbq = 2u * (uint32_t)dn, rbm = rbq + 3u * (uint32_t)qn;
        for (int64_t k = 0; k < dn; ++k) {
            for (int j = 0; j < 4; ++j) if (d[k].g_row_col[j] != kSentinel) mp.push_back({d[k].g_row_col[j], (uint32_t)(4 * k + j)});
            for (int j = 0; j < 2; ++j) if (d[k].b_idx[j] != kSentinel) rp_.push_back({d[k].b_idx[j], (uint32_t)(2 * k + j)});
        }
        for (int64_t k = 0; k < qn; ++k) {
            for (int j = 0; j < 9; ++j) if (q[k].g_row_col[j] != kSentinel) mp.push_back({q[k].g_row_col[j], bq + (uint32_t)(9 * k + j)});
            for (int j = 0; j < 3; ++j) if (q[k].b_idx[j] != kSentinel) rp_.push_back({q[k].b_idx[j], rbq + (uint32_t)(3 * k + j)});
        }
        for (int64_t k = 0; k < mn; ++k) {
            for (int j = 0; j < 6; ++j) if (m[k].g_row_col[j] != kSentinel) mp.push_back({m[k].g_row_col[j], bm + (uint32_t)(6 * k + j)});
            for (int j = 0; j < 2; ++j) if (m[k].b_idx[j] != kSentinel) rp_.push_back({m[k].b_idx[j], rbm + (uint32_t)(2 * k + j)});
        }
        std::vector<uint32_t> s1, p1, i1, s2, p2, i2;
        build_stamp_map(mp, s1, p1, i1);
        build_stamp_map(rp_, s2, p2, i2);
        ms_off[i + 1] = ms_off[i] + (int64_t)s1.size();
        mid_off[i + 1] = mid_off[i] + (int64_t)i1.size();
        rs_off[i + 1] = rs_off[i] + (int64_t)s2.size();
        rid_off[i + 1] = rid_off[i] + (int64_t)i2.size();
        mslot.insert(mslot.end(), s1.begin(), s1.end());
        mptr.insert(mptr.end(), p1.begin(), p1.end());       // s1.size()+1 entries
        mids.insert(mids.end(), i1.begin(), i1.end());
        rrow.insert(rrow.end(), s2.begin(), s2.end());
        rptr.insert(rptr.end(), p2.begin(), p2.end());
        rids.insert(rids.end(), i2.begin(), i2.end());
        std::vector<char> touched(z, 0);
        for (uint32_t sl : s1) touched[sl] = 1;
        if (n_nodes && (n_nodes[i] < 0 || n_nodes[i] > n))
            return ohm_fail(OHM_ERR_INVALID_ARG, "instance %lld: n_nodes out of range", (long long)i);
        const std::vector<uint8_t> sf = stamp_flags(n, rp, cl, touched, s2);
        std::copy(sf.begin(), sf.end(), sflag.begin() + row_off[i]);
        PcHost pc;
        build_precond(n, rp, cl, base_g_values + nnz_off[i], touched, true, pc);
        std::copy(pc.partner.begin(), pc.partner.end(), partner.begin() + row_off[i]);
        std::copy(pc.diag_slot.begin(), pc.diag_slot.end(), diag.begin() + row_off[i]);
        std::copy(pc.off_slot.begin(), pc.off_slot.end(), off.begin() + row_off[i]);
        std::copy(pc.rowflag.begin(), pc.rowflag.end(), flag.begin() + row_off[i]);
        any_pair |= pc.any_pair;
        for (int64_t r = 0; r < n; ++r) max_nnz_row = std::max<int64_t>(max_nnz_row, rp[r + 1] - rp[r]);
    }
    // longest first
    std::vector<int32_t> order(n_inst);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int32_t x, int32_t y) {
        return (nnz_off[x + 1] - nnz_off[x]) > (nnz_off[y + 1] - nnz_off[y]);
    });

    ohm_batch *b = new ohm_batch();
    b->ctx = c;
    b->n_inst = n_inst; b->rows = rows; b->nnz = nnz; b->nd = nd; b->nq = nq; b->nm = nm;
    const double avg = (double)nnz / (double)rows;
    b->lpr = avg <= 5.5 ? 1 : (avg <= 12.0 ? 4 : 8);
    KernelArgs &a = b->args.base;
    a = KernelArgs{};
    uint32_t *u32 = nullptr;
    double *f64 = nullptr;
    cudaError_t e = cudaSuccess;
#define PUT(dst, src, cnt) do { if (e == cudaSuccess) e = b->put(&(dst), (src), (cnt)); } while (0)
#define ZERO(dst, cnt) do { if (e == cudaSuccess) e = b->zero(&(dst), (cnt)); } while (0)
    PUT(u32, row_ptrs, rows + n_inst); a.row_ptr = u32;
    PUT(u32, col_indices, nnz); a.col = u32;
    PUT(f64, base_g_values, nnz); a.base_vals = f64;
    PUT(f64, base_g_values, nnz); a.vals64 = f64;
    float *v32 = nullptr; ZERO(v32, nnz); a.vals32 = v32;
    PUT(f64, base_b, rows); a.base_b = f64;
    PUT(f64, base_b, rows); a.b = f64;
    ZERO(f64, rows); a.x_prev = f64;
    ZERO(f64, rows); a.r64 = f64;
    ZERO(f64, rows); a.dx = f64;
    ZERO(f64, rows); b->args.node_scale_base = f64;
    ZERO(f64, rows); b->args.x_good = f64;
    { uint8_t *sf = nullptr; PUT(sf, sflag.data(), rows); b->args.stampflag = sf; }
    if (n_nodes) { int32_t *nn = nullptr; PUT(nn, n_nodes, n_inst); b->args.n_nodes = nn; }
    int32_t *i32 = nullptr;
    PUT(i32, partner.data(), rows); a.partner = i32;
    PUT(u32, diag.data(), rows); a.diag_slot = u32;
    PUT(u32, off.data(), rows); a.off_slot = u32;
    uint8_t *u8 = nullptr;
    if (any_pair) { PUT(u8, flag.data(), rows); a.rowflag = u8; }
    ZERO(f64, 4 * rows); a.rec0 = f64;
    ZERO(f64, 4 * rows); a.rec1 = f64;
    void **vs[] = {&a.rhat, &a.s, &a.t, &a.phat, &a.shat, &a.d, &a.pc_part};
    for (void **slot : vs) { ZERO(f64, rows); *slot = f64; }
    DiodeDesc *dd = nullptr; PUT(dd, (const DiodeDesc *)diodes, nd); a.diodes = dd;
    BjtDesc *qd = nullptr; PUT(qd, (const BjtDesc *)bjts, nq); a.bjts = qd;
    MosfetDesc *md = nullptr; PUT(md, (const MosfetDesc *)mosfets, nm); a.mosfets = md;
    if (bjt_vaf && nq) { PUT(f64, bjt_vaf, nq); a.bjt_vaf = f64; }
    ZERO(f64, 4 * nd + 9 * nq + 6 * nm); a.mstamp = f64;
    ZERO(f64, 2 * nd + 3 * nq + 2 * nm); a.rstamp = f64;
    PUT(u32, mslot.data(), mslot.size()); a.mslot = u32;
    PUT(u32, mptr.data(), mptr.size()); a.mslot_ptr = u32;
    PUT(u32, mids.data(), mids.size()); a.mslot_ids = u32;
    PUT(u32, rrow.data(), rrow.size()); a.rrow = u32;
    PUT(u32, rptr.data(), rptr.size()); a.rrow_ptr = u32;
    PUT(u32, rids.data(), rids.size()); a.rrow_ids = u32;
    int64_t *i64 = nullptr;
    PUT(i64, row_off, n_inst + 1); b->args.row_off = i64;
    PUT(i64, nnz_off, n_inst + 1); b->args.nnz_off = i64;
    PUT(i64, diode_off, n_inst + 1); b->args.d_off = i64;
    PUT(i64, bjt_off, n_inst + 1); b->args.q_off = i64;
    PUT(i64, mosfet_off, n_inst + 1); b->args.m_off = i64;
    PUT(i64, ms_off.data(), n_inst + 1); b->args.ms_off = i64;
    PUT(i64, mid_off.data(), n_inst + 1); b->args.mid_off = i64;
    PUT(i64, rs_off.data(), n_inst + 1); b->args.rs_off = i64;
    PUT(i64, rid_off.data(), n_inst + 1); b->args.rid_off = i64;
    PUT(i32, order.data(), n_inst); b->args.order = i32; b->order = i32;
    ZERO(b->sample, n_inst);
    ZERO(b->team_partials, 8 * (size_t)c->num_sms * 8);
    ZERO(b->infos, n_inst);
    ZERO(b->queue, 4);
#undef PUT
#undef ZERO
    if (e == cudaSuccess && nnz) e = ohm_f64_to_f32(a.vals64, v32, nnz, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);   // host vectors go out of scope
    if (e != cudaSuccess) {
        for (void *p : b->allocs) ohm_pool_free(p);
        delete b;
        return ohm_fail(OHM_ERR_CUDA, "batch upload: %s", cudaGetErrorString(e));
    }
    b->args.n_inst = (int)n_inst;
    b->args.infos = b->infos;
    b->args.queue = b->queue;
    b->host_infos.resize(n_inst);
    b->h_order = order;
    b->h_offsets.resize(n_inst);
    for (int64_t i = 0; i < n_inst; ++i) {
        InstanceOffsets &o = b->h_offsets[i];
        o.ro = row_off[i]; o.ro1 = row_off[i + 1]; o.no = nnz_off[i]; o.no1 = nnz_off[i + 1];
        o.dq = diode_off[i]; o.dq1 = diode_off[i + 1]; o.qq = bjt_off[i]; o.qq1 = bjt_off[i + 1];
        o.mq = mosfet_off[i]; o.mq1 = mosfet_off[i + 1];
        o.ms = ms_off[i]; o.ms1 = ms_off[i + 1]; o.mid = mid_off[i];
        o.rs = rs_off[i]; o.rs1 = rs_off[i + 1]; o.rid = rid_off[i];
        o.n_nodes = n_nodes ? n_nodes[i] : 0;
    }
    ohm_ctx_retain(c);
    *out = b;
    return OHM_OK;
}

extern "C" ohm_status ohm_batch_destroy(ohm_batch *b) {
    if (!b) return OHM_OK;
    ohm_ctx *c = b->ctx;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    for (void *p : b->allocs) ohm_pool_free(p);
    delete b;
    ohm_ctx_release(c);
    return OHM_OK;
}

// Validated kernel arguments of one batched Newton call.
static ohm_status batch_args(ohm_batch *b, double *x_dev, const ohm_newton_params *np, BatchArgs &B) {
    if (!b || !x_dev || !np) return ohm_fail(OHM_ERR_INVALID_ARG, "null argument");
    if (np->max_iterations <= 0) return ohm_fail(OHM_ERR_NEWTON_NOT_CONVERGED, "Newton solver did not converge after 0 iterations");
    ohm_status st = ohm_check_krylov(&np->krylov);
    if (st != OHM_OK) return st;
    if (np->krylov.precond == OHM_PRECOND_ISAI1)
        return ohm_fail(OHM_ERR_INVALID_ARG, "batched solves use block Jacobi (ISAI(1) is for single systems)");
    if (np->continuation && !b->args.n_nodes)
        return ohm_fail(OHM_ERR_INVALID_ARG, "continuation needs the per-instance n_nodes given at creation");
    B = b->args;
    KernelArgs &a = B.base;
    a.x = x_dev;
    a.precond = np->krylov.precond == OHM_PRECOND_NONE ? kPcNone
              : (np->krylov.precond == OHM_PRECOND_JACOBI ? kPcJacobi : kPcAuto);
    if (a.precond != kPcAuto) a.rowflag = nullptr;
    a.newton = 1;
    const bool mixed = np->krylov.precision == OHM_PREC_MIXED;
    a.mixed = mixed ? 1 : 0;
    a.max_outer = np->max_iterations;
    a.abs_tol = np->abs_tol;
    a.rel_tol = np->rel_tol;
    a.max_krylov = np->krylov.max_iterations;
    a.krylov_tol = np->krylov.tolerance;
    a.inner_rtol = mixed ? (np->krylov.inner_rtol > 0.0 ? np->krylov.inner_rtol : 1e-4) : np->krylov.inner_rtol;
    a.forcing = np->forcing;
    a.eta_max = np->eta_max > 0.0 ? np->eta_max : 0.5;
    a.fp32_max_iterations = np->krylov.fp32_max_iterations > 0 ? np->krylov.fp32_max_iterations
                                                               : np->krylov.max_iterations;
    a.fp32_min_eta = np->krylov.fp32_min_eta_exp > 0 ? std::pow(10.0, -(double)np->krylov.fp32_min_eta_exp) : 0.0;
    a.max_restarts = std::max(0, np->krylov.max_restarts);
    a.continuation = np->continuation ? (1 | (np->continuation & OHM_CONT_TEST_PSEUDO)) : 0;
    return OHM_OK;
}

// One launch over `n` instances listed in `order` (device): a persistent grid
// of (blocks per SM) x SMs blocks, each taking instances from the queue.
static ohm_status launch_batch(ohm_batch *b, BatchArgs B, int lpr, int shape, int n, const int32_t *order) {
    ohm_ctx *c = b->ctx;
    B.order = order;
    B.n_inst = n;
    BatchFn fn = batch_kernel(lpr, shape);
    const int block = kBatchShapes[shape].block;
    int per_sm = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, block, 0));
    if (per_sm < 1) return ohm_fail(OHM_ERR_CUDA, "batch kernel does not fit on an SM");
    const int grid = (int)std::min<int64_t>((int64_t)per_sm * c->num_sms, n);
    CUDA_TRY(cudaMemsetAsync(b->queue, 0, sizeof(unsigned int), c->stream));
    fn<<<grid, block, 0, c->stream>>>(B);
    CUDA_TRY(cudaGetLastError());
    return OHM_OK;
}

// Split of one call: a circuit whose solve by one block would outlast the
// rest of the batch goes to the whole GPU instead.  A one-block solve is
// estimated as rows^1.5 (Krylov iterations grow about as the square root
// of a mesh's size); in largest-first order, circuits move while the next
// one's estimate exceeds the ideal length of the rest (the sum of their
// estimates over the resident blocks) and it has at least 2,048 rows (below
// that one block beats the grid, whose barriers cost microseconds each).
constexpr int64_t kSplitMinRows = 2048;

static void split_instances(const ohm_batch *b, int lpr, int shape, std::vector<int32_t> &team,
                            std::vector<int32_t> &rest) {
    team.clear();
    rest.clear();
    int per_sm = 0;
    const BatchFn fn = batch_kernel(lpr, shape);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kBatchShapes[shape].block, 0) != cudaSuccess)
        per_sm = 1;
    const double blocks = (double)std::max(per_sm, 1) * (double)b->ctx->num_sms;
    auto est = [&](int32_t i) {
        const double n = (double)(b->h_offsets[i].ro1 - b->h_offsets[i].ro);
        return n * std::sqrt(n);
    };
    double total = 0.0;
    for (int32_t i : b->h_order) total += est(i);
    size_t k = 0;
    if (b->split) {
        for (; k < b->h_order.size(); ++k) {
            const int32_t i = b->h_order[k];
            const double t = est(i);
            if (b->h_offsets[i].ro1 - b->h_offsets[i].ro < kSplitMinRows || t <= (total - t) / blocks) break;
            team.push_back(i);
            total -= t;
        }
    }
    rest.assign(b->h_order.begin() + (ptrdiff_t)k, b->h_order.end());
}

// Solves instance i alone with the single-system persistent solver over the
// batch's packed arrays; its status lands in the batch's per-instance info.
static ohm_status solve_instance_whole_gpu(ohm_batch *b, const BatchArgs &B, int32_t i, int *launches) {
    ohm_ctx *c = b->ctx;
    KernelArgs a;
    instance_args(B, i, b->h_offsets[i], a);
    a.partials = b->team_partials;
    const LaunchTarget t{c->num_sms, c->stream, c->sync_words, c->info_dev, c->info_host, 0, c->krylov_layout};
    ohm_status st = ohm_launch_persistent(t, a, a.nnz, launches);
    if (st != OHM_OK) return st;
    CUDA_TRY(cudaMemcpyAsync(b->infos + i, c->info_dev, sizeof(DeviceInfo), cudaMemcpyDeviceToDevice, c->stream));
    unsigned int words[4] = {0, 0, 0, 0};
    CUDA_TRY(cudaMemcpyAsync(words, c->sync_words, sizeof words, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (words[2] != 0)
        return ohm_fail(OHM_ERR_TIMEOUT, "instance %d: a device barrier wait gave up (error word %u)", (int)i,
                        words[2]);
    return OHM_OK;
}

extern "C" ohm_status ohm_batch_set_split(ohm_batch *b, int32_t on) {
    if (!b) return ohm_fail(OHM_ERR_INVALID_ARG, "batch is null");
    if (on != 0 && on != 1) return ohm_fail(OHM_ERR_INVALID_ARG, "split must be 0 or 1");
    b->split = on;
    return OHM_OK;
}

extern "C" ohm_status ohm_batch_newton_device(ohm_batch *b, double *x_dev, const ohm_newton_params *np,
                                              ohm_solve_info *summary) {
    BatchArgs B;
    ohm_status st = batch_args(b, x_dev, np, B);
    if (st != OHM_OK) return st;
    ohm_ctx *c = b->ctx;
    CUDA_TRY(cudaSetDevice(c->device));
    if (np->initial_guess)
        CUDA_TRY(cudaMemcpyAsync(x_dev, np->initial_guess, b->rows * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(cudaMemsetAsync(b->infos, 0, b->n_inst * sizeof(DeviceInfo), c->stream));
    std::vector<int32_t> team, rest;
    split_instances(b, b->lpr, b->shape, team, rest);
    int launches = 0;
    for (int32_t i : team) {
        st = solve_instance_whole_gpu(b, B, i, &launches);
        if (st != OHM_OK) return st;
    }
    if (!rest.empty()) {
        const int32_t *order = b->order;
        if (!team.empty()) {   // the rest of the largest-first order (the autotune sample array is free here)
            CUDA_TRY(cudaMemcpyAsync(b->sample, rest.data(), rest.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                                     c->stream));
            order = b->sample;
        }
        st = launch_batch(b, B, b->lpr, b->shape, (int)rest.size(), order);
        if (st != OHM_OK) return st;
        ++launches;
    }
    CUDA_TRY(cudaMemcpyAsync(b->host_infos.data(), b->infos, b->n_inst * sizeof(DeviceInfo), cudaMemcpyDeviceToHost,
                             c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    // summary: worst status, totals
    int64_t kit = 0, fb = 0, rs = 0, worst = -1, csteps = 0;
    int max_newton = 0, ckind = 0;
    for (int64_t i = 0; i < b->n_inst; ++i) {
        const DeviceInfo &d = b->host_infos[i];
        kit += d.krylov_iterations;
        fb += d.fp64_fallbacks;
        rs += d.krylov_restarts;
        csteps += d.continuation_steps;
        ckind = std::max(ckind, d.continuation_kind);
        max_newton = std::max(max_newton, d.iterations);
        if (d.status != 0 && worst < 0) worst = i;
    }
    if (summary) {
        std::memset(summary, 0, sizeof *summary);
        summary->iterations = max_newton;
        summary->krylov_iterations = kit;
        summary->fp64_fallbacks = (int32_t)fb;
        summary->krylov_restarts = (int32_t)rs;
        summary->kernel_launches = launches;
        summary->status = worst < 0 ? OHM_OK : b->host_infos[worst].status;
        summary->error_iteration = (int32_t)worst;
        summary->continuation_steps = (int32_t)std::min<int64_t>(csteps, 0x7fffffff);
        summary->continuation_kind = ckind;
    }
    if (worst >= 0) {
        const DeviceInfo &d = b->host_infos[worst];
        return ohm_fail(d.status == 1 ? OHM_ERR_SOLVE : (d.status == 3 ? OHM_ERR_NEWTON_NUMERICAL : OHM_ERR_NEWTON_NOT_CONVERGED),
                        "instance %lld failed: status %d (krylov code %d) after %d Newton iterations",
                        (long long)worst, d.status, d.krylov_code, d.iterations);
    }
    return OHM_OK;
}

extern "C" ohm_status ohm_batch_instance_info(ohm_batch *b, ohm_solve_info *infos, int64_t n) {
    if (!b || !infos || n != b->n_inst) return ohm_fail(OHM_ERR_INVALID_ARG, "bad arguments");
    for (int64_t i = 0; i < n; ++i) {
        const DeviceInfo &d = b->host_infos[i];
        ohm_solve_info &o = infos[i];
        std::memset(&o, 0, sizeof o);
        o.status = d.status == 0 ? OHM_OK : (d.status == 1 ? OHM_ERR_SOLVE : (d.status == 3 ? OHM_ERR_NEWTON_NUMERICAL : OHM_ERR_NEWTON_NOT_CONVERGED));
        o.krylov_code = d.krylov_code;
        o.iterations = d.iterations;
        o.error_iteration = d.error_iteration;
        o.krylov_iterations = d.krylov_iterations;
        o.fp64_fallbacks = d.fp64_fallbacks;
        o.krylov_restarts = d.krylov_restarts;
        o.max_residual = d.max_residual;
        o.b_norm = d.b_norm;
        o.kernel_launches = 1;
        o.continuation_steps = d.continuation_steps;
        o.continuation_kind = d.continuation_kind;
    }
    return OHM_OK;
}

extern "C" ohm_status ohm_batch_autotune(ohm_batch *b, const ohm_newton_params *np, int32_t sample_size,
                                         int32_t *lanes_per_row, int32_t *threads_per_block,
                                         int32_t *blocks_per_sm, double *sample_ms) {
    if (!b || !np) return ohm_fail(OHM_ERR_INVALID_ARG, "null argument");
    ohm_ctx *c = b->ctx;
    CUDA_TRY(cudaSetDevice(c->device));
    if (!b->x_tune) {
        cudaError_t e = b->zero(&b->x_tune, (size_t)b->rows);
        if (e != cudaSuccess) return ohm_fail(OHM_ERR_CUDA, "autotune scratch: %s", cudaGetErrorString(e));
    }
    BatchArgs B;
    ohm_status st = batch_args(b, b->x_tune, np, B);
    if (st != OHM_OK) return st;
    // a few Newton iterations show each variant's throughput; the
    // continuation (whose length depends on the path) stays off
    B.base.max_outer = std::min(B.base.max_outer, 3);
    B.base.continuation = 0;
    // sample: every k-th instance of the largest-first order, so the sample
    // spans the size distribution
    const int64_t n = b->n_inst;
    const int64_t m = sample_size <= 0 ? std::min<int64_t>(n, 512) : std::min<int64_t>(n, sample_size);
    std::vector<int32_t> order(n), pick(m);
    CUDA_TRY(cudaMemcpyAsync(order.data(), b->order, n * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    for (int64_t k = 0; k < m; ++k) pick[k] = order[(k * n) / m];
    CUDA_TRY(cudaMemcpyAsync(b->sample, pick.data(), m * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
    // candidates: lanes per row around the density heuristic, every shape
    const int base = b->lpr;
    std::vector<int> lprs = {base};
    if (base > 1) lprs.push_back(base / 2);
    if (base < 8) lprs.push_back(base * 2);
    cudaEvent_t e0, e1;
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    float best = -1.0f;
    int best_lpr = b->lpr, best_shape = b->shape;
    for (int lpr : lprs) {
        for (int sh = 0; sh < kNumBatchShapes; ++sh) {
            cudaMemsetAsync(b->x_tune, 0, b->rows * sizeof(double), c->stream);
            cudaEventRecord(e0, c->stream);
            st = launch_batch(b, B, lpr, sh, (int)m, b->sample);
            if (st != OHM_OK) break;
            cudaEventRecord(e1, c->stream);
            cudaError_t e = cudaEventSynchronize(e1);
            float ms = 0.0f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
            if (e != cudaSuccess) { st = ohm_fail(OHM_ERR_CUDA, "autotune: %s", cudaGetErrorString(e)); break; }
            if (best < 0.0f || ms < best) { best = ms; best_lpr = lpr; best_shape = sh; }
        }
        if (st != OHM_OK) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != OHM_OK) return st;
    b->lpr = best_lpr;
    b->shape = best_shape;
    if (lanes_per_row) *lanes_per_row = best_lpr;
    if (threads_per_block) *threads_per_block = kBatchShapes[best_shape].block;
    if (blocks_per_sm) *blocks_per_sm = kBatchShapes[best_shape].min_blocks;
    if (sample_ms) *sample_ms = best;
    return OHM_OK;
}

extern "C" ohm_status ohm_batch_set_kernel(ohm_batch *b, int32_t lanes_per_row, int32_t threads_per_block,
                                           int32_t blocks_per_sm) {
    if (!b) return ohm_fail(OHM_ERR_INVALID_ARG, "null batch");
    int shape = -1;
    for (int k = 0; k < kNumBatchShapes; ++k)
        if (kBatchShapes[k].block == threads_per_block && kBatchShapes[k].min_blocks == blocks_per_sm) shape = k;
    if (!(lanes_per_row == 1 || lanes_per_row == 2 || lanes_per_row == 4 || lanes_per_row == 8) || shape < 0)
        return ohm_fail(OHM_ERR_INVALID_ARG,
                        "lanes_per_row must be 1, 2, 4 or 8; (threads, blocks per SM) one of (256,2), (256,4), (128,8)");
    b->lpr = lanes_per_row;
    b->shape = shape;
    return OHM_OK;
}
