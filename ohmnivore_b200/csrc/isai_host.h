// Host-side symbolic set-up of the ISAI(1) preconditioner (all numeric work
// runs on the device, see isai.cuh).
//
// The reference builds ISAI from a full-fill LU with partial pivoting on the
// CPU every Newton iteration (src/solver/preconditioner.rs:54-277,
// newton.rs:368-406).  Here the factor is ILU(0) on A's pattern augmented with
// the diagonal (so a voltage-source branch row, whose diagonal is structurally
// zero, gets the nonzero pivot -1/U_jj of its node row), computed on the device
// by Chow-Patel fixed-point sweeps.  The ISAI(1) patterns follow the
// reference's level-1 rule (generate_patterns, preconditioner.rs:205-218):
// pattern(M_L) = pattern(L^2) with L's unit diagonal, pattern(M_U) =
// pattern(U^2); each column is the solution of the local system
// A[J, J] m = e_k (solve_column_isai, :316-367), triangular here because the
// factors are.
#pragma once

#include <algorithm>
#include <cstdint>
#include <vector>

namespace ohm {

// Columns with a larger local system keep the kIsaiMaxLocal rows nearest the
// diagonal (hub rows of a power rail would otherwise make dense columns).
constexpr int kIsaiMaxLocal = 32;

struct IsaiHost {
    int64_t n = 0, nnz_aug = 0;
    std::vector<uint32_t> arp, acol;     // augmented pattern A + diag (CSR, sorted)
    std::vector<int32_t> amap;           // aug slot -> A slot, -1 for an added diagonal
    std::vector<uint32_t> adiag;         // aug slot of (i, i)
    std::vector<uint32_t> cptr, cpair;   // Chow-Patel: per aug slot, pairs (slot(i,k), slot(k,j))
    std::vector<uint32_t> mlrp, mlcol;   // M_L CSR pattern (lower, incl. diagonal)
    std::vector<uint32_t> mlcp, mlrow, mlpos;  // M_L by column: rows (ascending), CSR position
    std::vector<uint32_t> murp, mucol;   // M_U CSR pattern (upper, incl. diagonal)
    std::vector<uint32_t> mucp, murow, mupos;

    int64_t find(uint32_t r, uint32_t c) const {
        const auto b = acol.begin() + arp[r], e = acol.begin() + arp[r + 1];
        const auto it = std::lower_bound(b, e, c);
        return (it != e && *it == c) ? (int64_t)(it - acol.begin()) : -1;
    }

    void build(int64_t n_, const uint32_t *rp, const uint32_t *col) {
        n = n_;
        // augmented pattern
        arp.assign(n + 1, 0);
        acol.clear();
        amap.clear();
        adiag.assign(n, 0);
        for (int64_t i = 0; i < n; ++i) {
            bool placed = false;                  // diagonal emitted for this row
            auto put_diag = [&]() {
                adiag[i] = (uint32_t)acol.size();
                acol.push_back((uint32_t)i);
                amap.push_back(-1);
                placed = true;
            };
            for (uint32_t k = rp[i]; k < rp[i + 1]; ++k) {
                const int64_t c = col[k];
                if (!placed && c > i) put_diag();   // structural zero diagonal
                if (c == i) { adiag[i] = (uint32_t)acol.size(); placed = true; }
                acol.push_back(col[k]);
                amap.push_back((int32_t)k);
            }
            if (!placed) put_diag();
            arp[i + 1] = (uint32_t)acol.size();
        }
        nnz_aug = (int64_t)acol.size();
        // Chow-Patel product lists
        cptr.assign(nnz_aug + 1, 0);
        cpair.clear();
        for (int64_t i = 0; i < n; ++i) {
            for (uint32_t s = arp[i]; s < arp[i + 1]; ++s) {
                const uint32_t j = acol[s];
                const uint32_t lim = std::min<uint32_t>((uint32_t)i, j);
                for (uint32_t t = arp[i]; t < arp[i + 1] && acol[t] < lim; ++t) {
                    const uint32_t k = acol[t];
                    const int64_t kj = find(k, j);
                    if (kj >= 0) { cpair.push_back(t); cpair.push_back((uint32_t)kj); }
                }
                cptr[s + 1] = (uint32_t)(cpair.size() / 2);
            }
        }
        // M_L = pattern((L + I)^2): row i = union over k in {i} + L-row(i) of {k} + L-row(k)
        std::vector<int64_t> mark(n, -1);
        std::vector<uint32_t> row;
        mlrp.assign(n + 1, 0);
        mlcol.clear();
        for (int64_t i = 0; i < n; ++i) {
            row.clear();
            auto add = [&](uint32_t c) { if (mark[c] != i) { mark[c] = i; row.push_back(c); } };
            add((uint32_t)i);
            for (uint32_t t = arp[i]; t < arp[i + 1] && (int64_t)acol[t] < i; ++t) {
                const uint32_t k = acol[t];
                add(k);
                for (uint32_t u = arp[k]; u < arp[k + 1] && acol[u] < k; ++u) add(acol[u]);
            }
            std::sort(row.begin(), row.end());
            mlcol.insert(mlcol.end(), row.begin(), row.end());
            mlrp[i + 1] = (uint32_t)mlcol.size();
        }
        // M_U = pattern(U^2): row i = union over k in U-row(i) (incl. i) of U-row(k)
        std::fill(mark.begin(), mark.end(), -1);
        murp.assign(n + 1, 0);
        mucol.clear();
        for (int64_t i = 0; i < n; ++i) {
            row.clear();
            auto add = [&](uint32_t c) { if (mark[c] != i) { mark[c] = i; row.push_back(c); } };
            for (uint32_t t = arp[i]; t < arp[i + 1]; ++t) {
                const uint32_t k = acol[t];
                if ((int64_t)k < i) continue;
                for (uint32_t u = arp[k]; u < arp[k + 1]; ++u)
                    if (acol[u] >= k) add(acol[u]);
            }
            std::sort(row.begin(), row.end());
            mucol.insert(mucol.end(), row.begin(), row.end());
            murp[i + 1] = (uint32_t)mucol.size();
        }
        columns(mlrp, mlcol, true, mlcp, mlrow, mlpos);
        columns(murp, mucol, false, mucp, murow, mupos);
    }

    // Column view of a CSR pattern, each column capped at kIsaiMaxLocal rows
    // nearest the diagonal (for M_L the rows just below it, for M_U above it).
    void columns(const std::vector<uint32_t> &rp, const std::vector<uint32_t> &cl, bool lower,
                 std::vector<uint32_t> &cp, std::vector<uint32_t> &rows, std::vector<uint32_t> &pos) const {
        std::vector<std::vector<std::pair<uint32_t, uint32_t>>> bycol(n);
        for (int64_t i = 0; i < n; ++i)
            for (uint32_t s = rp[i]; s < rp[i + 1]; ++s) bycol[cl[s]].push_back({(uint32_t)i, s});
        cp.assign(n + 1, 0);
        rows.clear();
        pos.clear();
        for (int64_t k = 0; k < n; ++k) {
            auto &v = bycol[k];                          // rows ascending
            size_t b = 0, e = v.size();
            if (e > (size_t)kIsaiMaxLocal) {
                if (lower) e = kIsaiMaxLocal;            // keep rows k, k+1, ...
                else b = e - kIsaiMaxLocal;              // keep ..., k-1, k
            }
            for (size_t t = b; t < e; ++t) { rows.push_back(v[t].first); pos.push_back(v[t].second); }
            cp[k + 1] = (uint32_t)rows.size();
        }
    }
};

}  // namespace ohm
