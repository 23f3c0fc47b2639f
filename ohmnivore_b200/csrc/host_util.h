// Host-side helpers shared by the C-ABI translation units: input
// validation, the block-Jacobi preconditioner structure and the stamp map.
#pragma once

#include <algorithm>
#include <cmath>
#include <utility>
#include <vector>

#include "internal.cuh"

namespace ohm {

// ------------------------------------------------------------- validation --
inline ohm_status check_csr(int64_t n, int64_t nnz, const uint32_t *rp, const uint32_t *col) {
    if (n < 0 || nnz < 0) return ohm_fail(OHM_ERR_INVALID_ARG, "negative size");
    if (n > 0x7fffffffLL || nnz > 0xfffffffeLL) return ohm_fail(OHM_ERR_INVALID_ARG, "size exceeds u32 indexing");
    if (!rp || (nnz > 0 && !col)) return ohm_fail(OHM_ERR_INVALID_ARG, "null CSR pointer");
    if (rp[0] != 0) return ohm_fail(OHM_ERR_COMPILE, "row_ptr[0] = %u, expected 0", rp[0]);
    for (int64_t i = 0; i < n; ++i)
        if (rp[i + 1] < rp[i]) return ohm_fail(OHM_ERR_COMPILE, "row_ptr decreases at row %lld", (long long)i);
    if ((int64_t)rp[n] != nnz) return ohm_fail(OHM_ERR_COMPILE, "row_ptr[n] = %u != nnz %lld", rp[n], (long long)nnz);
    for (int64_t k = 0; k < nnz; ++k)
        if ((int64_t)col[k] >= n) return ohm_fail(OHM_ERR_COMPILE, "column index %u out of range at %lld", col[k], (long long)k);
    return OHM_OK;
}

inline bool idx_ok(uint32_t v, int64_t lim) { return v == kSentinel || (int64_t)v < lim; }

inline ohm_status check_devices(const ohm_diode_desc *d, int64_t nd, const ohm_bjt_desc *q, int64_t nq,
                                const ohm_mosfet_desc *m, int64_t nm, int64_t size, int64_t nnz) {
    if (nd < 0 || nq < 0 || nm < 0) return ohm_fail(OHM_ERR_INVALID_ARG, "negative device count");
    if ((nd && !d) || (nq && !q) || (nm && !m)) return ohm_fail(OHM_ERR_INVALID_ARG, "null descriptor array");
    for (int64_t k = 0; k < nd; ++k) {
        const ohm_diode_desc &x = d[k];
        bool ok = idx_ok(x.anode_idx, size) && idx_ok(x.cathode_idx, size);
        for (int j = 0; j < 4; ++j) ok = ok && idx_ok(x.g_row_col[j], nnz);
        for (int j = 0; j < 2; ++j) ok = ok && idx_ok(x.b_idx[j], size);
        if (!ok) return ohm_fail(OHM_ERR_COMPILE, "diode %lld has an index out of range", (long long)k);
    }
    for (int64_t k = 0; k < nq; ++k) {
        const ohm_bjt_desc &x = q[k];
        bool ok = idx_ok(x.collector_idx, size) && idx_ok(x.base_idx, size) && idx_ok(x.emitter_idx, size);
        for (int j = 0; j < 9; ++j) ok = ok && idx_ok(x.g_row_col[j], nnz);
        for (int j = 0; j < 3; ++j) ok = ok && idx_ok(x.b_idx[j], size);
        if (!ok) return ohm_fail(OHM_ERR_COMPILE, "BJT %lld has an index out of range", (long long)k);
    }
    for (int64_t k = 0; k < nm; ++k) {
        const ohm_mosfet_desc &x = m[k];
        bool ok = idx_ok(x.drain_idx, size) && idx_ok(x.gate_idx, size) && idx_ok(x.source_idx, size);
        for (int j = 0; j < 6; ++j) ok = ok && idx_ok(x.g_row_col[j], nnz);
        for (int j = 0; j < 2; ++j) ok = ok && idx_ok(x.b_idx[j], size);
        if (!ok) return ohm_fail(OHM_ERR_COMPILE, "MOSFET %lld has an index out of range", (long long)k);
    }
    return OHM_OK;
}

// --------------------------------------------------- preconditioner setup --
// Block-Jacobi structure.  Rows whose diagonal is structurally zero (voltage
// source and inductor branch rows of an MNA matrix, src/compiler.rs:376-408)
// are paired with the off-diagonal column of largest magnitude whose row is
// unpaired and has a usable diagonal; the 2x2 block [[a_jj a_jk][a_kj 0]] has
// det = -a_jk a_kj != 0.  Unpaired zero-diagonal rows keep the reference's
// Jacobi rule (inverse 0).  `touched` marks diagonal slots the device stamps
// change; those rows never count as zero-diagonal.
struct PcHost {
    std::vector<int32_t> partner;
    std::vector<uint32_t> diag_slot, off_slot;
    std::vector<uint8_t> rowflag;   // row or one of its columns is paired
    bool any_pair = false;
};

inline void build_precond(int64_t n, const uint32_t *rp, const uint32_t *col, const double *val,
                          const std::vector<char> &touched_slot, bool pairs, PcHost &pc) {
    pc.partner.assign(n, -1);
    pc.diag_slot.assign(n, kSentinel);
    pc.off_slot.assign(n, kSentinel);
    pc.rowflag.clear();
    pc.any_pair = false;
    for (int64_t i = 0; i < n; ++i)
        for (uint32_t k = rp[i]; k < rp[i + 1]; ++k)
            if ((int64_t)col[k] == i) { pc.diag_slot[i] = k; break; }
    if (!pairs) {
        pc.rowflag.assign(n, 0);
        return;
    }
    auto zero_diag = [&](int64_t i) {
        const uint32_t s = pc.diag_slot[i];
        if (s == kSentinel) return true;
        if (!touched_slot.empty() && touched_slot[s]) return false;
        return std::fabs(val[s]) <= 1e-30;
    };
    auto slot_of = [&](int64_t r, int64_t c) -> uint32_t {
        for (uint32_t k = rp[r]; k < rp[r + 1]; ++k)
            if ((int64_t)col[k] == c) return k;
        return kSentinel;
    };
    for (int64_t k = 0; k < n; ++k) {
        if (!zero_diag(k) || pc.partner[k] >= 0) continue;
        int64_t best = -1;
        double best_mag = 0.0;
        uint32_t best_kj = kSentinel, best_jk = kSentinel;
        for (uint32_t e = rp[k]; e < rp[k + 1]; ++e) {
            const int64_t j = col[e];
            if (j == k || pc.partner[j] >= 0 || zero_diag(j)) continue;
            const double mag = std::fabs(val[e]);
            if (!(mag > 0.0)) continue;
            const uint32_t jk = slot_of(j, k);
            if (jk == kSentinel || !(std::fabs(val[jk]) > 0.0)) continue;
            if (mag > best_mag) { best_mag = mag; best = j; best_kj = e; best_jk = jk; }
        }
        if (best >= 0) {
            pc.partner[k] = (int32_t)best;
            pc.partner[best] = (int32_t)k;
            pc.off_slot[k] = best_kj;
            pc.off_slot[best] = best_jk;
            pc.any_pair = true;
        }
    }
    pc.rowflag.assign(n, 0);
    if (pc.any_pair)
        for (int64_t i = 0; i < n; ++i) {
            bool f = pc.partner[i] >= 0;
            for (uint32_t k = rp[i]; k < rp[i + 1] && !f; ++k) f = pc.partner[col[k]] >= 0;
            pc.rowflag[i] = f ? 1 : 0;
        }
}

// Stamp map: every (slot, contribution id) pair, grouped by slot.  Ids are
// assigned diodes first, then BJTs, then MOSFETs, device-major, so each slot
// sums its contributions in that fixed (canonical) order.
inline void build_stamp_map(const std::vector<std::pair<uint32_t, uint32_t>> &pairs_in,
                            std::vector<uint32_t> &slots, std::vector<uint32_t> &ptr, std::vector<uint32_t> &ids) {
    std::vector<std::pair<uint32_t, uint32_t>> pairs(pairs_in);
    std::stable_sort(pairs.begin(), pairs.end(),
                     [](const auto &x, const auto &y) { return x.first < y.first; });
    slots.clear(); ptr.clear(); ids.clear();
    for (size_t k = 0; k < pairs.size(); ++k) {
        if (k == 0 || pairs[k].first != pairs[k - 1].first) {
            slots.push_back(pairs[k].first);
            ptr.push_back((uint32_t)ids.size());
        }
        ids.push_back(pairs[k].second);
    }
    ptr.push_back((uint32_t)ids.size());
}


// Per-row flags for the DC continuation: bit 0 = the row's diagonal slot is
// written by the stamp map (touched_slot), bit 1 = its rhs entry is (rrows).
inline std::vector<uint8_t> stamp_flags(int64_t n, const uint32_t *rp, const uint32_t *col,
                                        const std::vector<char> &touched_slot, const std::vector<uint32_t> &rrows) {
    std::vector<uint8_t> f(n, 0);
    for (int64_t i = 0; i < n; ++i)
        for (uint32_t k = rp[i]; k < rp[i + 1]; ++k)
            if ((int64_t)col[k] == i && touched_slot[k]) f[i] |= 1;
    for (uint32_t r : rrows) f[r] |= 2;
    return f;
}

// Items whose range ptr[i]..ptr[i+1] is longer than min_len, each cut into
// consecutive chunks of at most `chunk` entries (long rows of a CSR matrix,
// stamp-map entries with many contributions).
struct LongSplit {
    std::vector<uint32_t> item, chunk_ptr, chunk_owner, chunk_beg, chunk_end;
    std::vector<uint8_t> flag;      // per item index: 1 if long
};

inline void split_long(int64_t count, const uint32_t *ptr, uint32_t min_len, uint32_t chunk, int64_t item_offset,
                       LongSplit &out) {
    if (out.chunk_ptr.empty()) out.chunk_ptr.push_back(0);
    for (int64_t i = 0; i < count; ++i) {
        const uint32_t b = ptr[i], e = ptr[i + 1];
        const bool long_item = e - b > min_len;
        out.flag.push_back(long_item ? 1 : 0);
        if (!long_item) continue;
        const uint32_t owner = (uint32_t)out.item.size();
        out.item.push_back((uint32_t)(i + item_offset));
        for (uint32_t c = b; c < e; c += chunk) {
            out.chunk_owner.push_back(owner);
            out.chunk_beg.push_back(c);
            out.chunk_end.push_back(std::min(e, c + chunk));
        }
        out.chunk_ptr.push_back((uint32_t)out.chunk_beg.size());
    }
}

// Thresholds: rows with more nonzeros than kLongRowMin, and stamp-map
// entries with more contributions than kLongSegMin, are handled by the whole
// team in chunks.
constexpr uint32_t kLongRowMin = 4096, kLongRowChunk = 128;
constexpr uint32_t kLongSegMin = 256, kLongSegChunk = 64;

}  // namespace ohm
