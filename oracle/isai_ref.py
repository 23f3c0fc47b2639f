"""ORACLE (test infrastructure only): restatement of the reference's ISAI
preconditioner (src/solver/preconditioner.rs), and of the ILU(0)-based
variant the device builds.

Only ``tests/`` and the other oracle entry points may use this module.

Reference algorithm (for small matrices, pure Python):
  ``ilu0``                 preconditioner.rs:64-153  (LU with partial pivoting and fill)
  ``generate_patterns``    :205-218   (level 0: L, U; level 1: L^2, U^2)
  ``solve_column_isai``    :316-367   (local system A[J, J] m = e_k)
  ``dense_solve``          :371-428   (GE with partial pivoting, zeros when singular)
  ``compute_isai``         :239-277   (M_L columns, permutation folded, M_U columns)

Device variant (numpy, exact sequential ILU(0)):
  ILU(0) on A's pattern plus the diagonal, no pivoting; ISAI(1) columns on the
  level-1 patterns as triangular solves.  The device computes the same factor
  approximately (Chow-Patel sweeps).

Device variant, step by step (``chow_patel_ref``, ``isai1_device_ref``):
  the factor after a fixed number of Jacobi-style Chow-Patel sweeps
  (E. Chow, A. Patel, "Fine-grained parallel incomplete LU factorization",
  SIAM J. Sci. Comput. 37(2), 2015), then ISAI(1) columns capped at 32 rows
  nearest the diagonal; the device result agrees to rounding.
"""
from __future__ import annotations

import numpy as np


def _rows(n, row_ptr, col, val):
    return [[(int(col[k]), float(val[k])) for k in range(row_ptr[i], row_ptr[i + 1])] for i in range(n)]


def _find(row, c):
    for cc, v in row:
        if cc == c:
            return v
    return 0.0


def ilu0_ref(n, row_ptr, col, val):
    """preconditioner.rs:64-153: returns dense L (unit), U and perm."""
    rows = _rows(n, row_ptr, col, val)
    perm = list(range(n))
    for j in range(n):
        best_row, best_val = j, abs(_find(rows[j], j))
        for i in range(j + 1, n):
            v = abs(_find(rows[i], j))
            if v > best_val:
                best_val, best_row = v, i
        if best_row != j:
            rows[j], rows[best_row] = rows[best_row], rows[j]
            perm[j], perm[best_row] = perm[best_row], perm[j]
        pivot = _find(rows[j], j)
        if abs(pivot) < 1e-30:
            continue
        upper = [(c, v) for c, v in rows[j] if c > j]
        for i in range(j + 1, n):
            a_ij = _find(rows[i], j)
            if abs(a_ij) < 1e-30:
                continue
            l_ij = a_ij / pivot
            d = dict(rows[i])
            d[j] = l_ij
            for k, u in upper:
                d[k] = d.get(k, 0.0) - l_ij * u
            rows[i] = sorted(d.items())
    L = np.eye(n)
    U = np.zeros((n, n))
    for i, row in enumerate(rows):
        for c, v in row:
            if c < i:
                L[i, c] = v
            else:
                U[i, c] = v
    return L, U, perm


def _pattern(M):
    return [sorted(np.nonzero(M[i])[0].tolist()) for i in range(M.shape[0])]


def _sym_mul(P, Q):
    out = []
    for row in P:
        s = set()
        for k in row:
            s.update(Q[k])
        out.append(sorted(s))
    return out


def dense_solve_ref(A, b):
    """preconditioner.rs:371-428 (zeros where singular)."""
    A = A.copy()
    b = b.copy()
    n = len(b)
    for c in range(n):
        # first maximum, as the reference's strict '>' scan
        best, bv = c, abs(A[c, c])
        for r in range(c + 1, n):
            if abs(A[r, c]) > bv:
                best, bv = r, abs(A[r, c])
        br = best
        if bv < 1e-30:
            continue
        if br != c:
            A[[c, br]] = A[[br, c]]
            b[[c, br]] = b[[br, c]]
        p = A[c, c]
        for r in range(c + 1, n):
            f = A[r, c] / p
            A[r, c] = 0.0
            A[r, c + 1:] -= f * A[c, c + 1:]
            b[r] -= f * b[c]
    x = np.zeros(n)
    for c in range(n - 1, -1, -1):
        if abs(A[c, c]) < 1e-30:
            continue
        x[c] = (b[c] - A[c, c + 1:] @ x[c + 1:]) / A[c, c]
    return x


def compute_isai_ref(n, row_ptr, col, val, level=1):
    """compute_isai (preconditioner.rs:239-277).  Returns dense (M_L, M_U, L, U, perm)."""
    L, U, perm = ilu0_ref(n, row_ptr, col, val)
    lp, up = _pattern(L), _pattern(U)
    if level == 1:
        lp, up = _sym_mul(lp, lp), _sym_mul(up, up)

    def columns(F, pat):
        M = np.zeros((n, n))
        colpat = [[] for _ in range(n)]
        for r, cs in enumerate(pat):
            for c in cs:
                colpat[c].append(r)
        for k in range(n):
            J = sorted(colpat[k])
            if not J:
                continue
            sub = F[np.ix_(J, J)]
            rhs = np.array([1.0 if j == k else 0.0 for j in J])
            m = dense_solve_ref(sub, rhs)
            M[J, k] = m
        return M

    ML = columns(L, lp)
    MLp = np.zeros_like(ML)                  # fold the permutation: column c -> perm[c]
    for c in range(n):
        MLp[:, perm[c]] += ML[:, c]
    MU = columns(U, up)
    return MLp, MU, L, U, perm


def ilu0_augmented(n, row_ptr, col, val):
    """Exact ILU(0) on A's pattern plus the diagonal, natural order, no
    pivoting (the device factor).  Returns dense L (unit) and U."""
    A = np.zeros((n, n))
    P = np.zeros((n, n), dtype=bool)
    for i in range(n):
        for k in range(row_ptr[i], row_ptr[i + 1]):
            A[i, col[k]] = val[k]
            P[i, col[k]] = True
        P[i, i] = True
    W = A.copy()
    for i in range(1, n):
        for k in range(i):
            if not P[i, k] or W[k, k] == 0.0:
                continue
            W[i, k] /= W[k, k]
            for j in range(k + 1, n):
                if P[i, j] and P[k, j]:
                    W[i, j] -= W[i, k] * W[k, j]
    L = np.tril(W, -1) * P + np.eye(n)
    U = np.triu(W) * P
    return L, U


def _augmented_pattern(n, row_ptr, col):
    P = np.zeros((n, n), dtype=bool)
    for i in range(n):
        for k in range(row_ptr[i], row_ptr[i + 1]):
            P[i, col[k]] = True
        P[i, i] = True
    return P


def chow_patel_ref(n, row_ptr, col, val, sweeps=6):
    """ILU(0) factor on the augmented pattern after ``sweeps`` Jacobi-style
    fixed-point sweeps.  Start: U = upper(A), L_ij = A_ij / A_jj (A_jj = 0
    leaves A_ij).  Sweep, every pattern entry from the previous iterate:
    l_ij = (a_ij - sum_{k<j} l_ik u_kj) / u_jj (j < i; u_jj = 0 leaves the
    numerator), u_ij = a_ij - sum_{k<i} l_ik u_kj (j >= i).  Returns dense L
    (unit diagonal) and U."""
    A = np.zeros((n, n))
    for i in range(n):
        for k in range(row_ptr[i], row_ptr[i + 1]):
            A[i, col[k]] = val[k]
    P = _augmented_pattern(n, row_ptr, col)
    Lo = np.zeros((n, n))
    Up = np.zeros((n, n))
    d = np.diag(A)
    for i in range(n):
        for j in np.nonzero(P[i])[0]:
            if j < i:
                Lo[i, j] = A[i, j] / d[j] if abs(d[j]) > 1e-300 else A[i, j]
            else:
                Up[i, j] = A[i, j]
    for _ in range(sweeps):
        Ln = np.zeros_like(Lo)
        Un = np.zeros_like(Up)
        for i in range(n):
            for j in np.nonzero(P[i])[0]:
                m = min(i, j)
                acc = A[i, j]
                for k in np.nonzero(P[i, :m])[0]:
                    if P[k, j]:
                        acc -= Lo[i, k] * Up[k, j]
                if j < i:
                    ujj = Up[j, j]
                    Ln[i, j] = acc / ujj if abs(ujj) > 1e-300 else acc
                else:
                    Un[i, j] = acc
        Lo, Up = Ln, Un
    return Lo + np.eye(n), Up, P


def isai1_device_ref(n, row_ptr, col, val, sweeps=6, cap=32):
    """ISAI(1) of the Chow-Patel factor: pattern(M_L) = pattern((L+I)^2),
    pattern(M_U) = pattern(U^2) over the augmented pattern; column k solves the
    local triangular system on its rows J (at most ``cap``: the smallest rows
    for M_L, the largest for M_U); a zero U pivot gives a zero entry.
    Returns dense M_L, M_U."""
    L, U, P = chow_patel_ref(n, row_ptr, col, val, sweeps)
    PL = np.tril(P)
    PU = np.triu(P)
    pat_l = (PL.astype(np.int64) @ PL.astype(np.int64)) > 0
    pat_u = (PU.astype(np.int64) @ PU.astype(np.int64)) > 0
    ML = np.zeros((n, n))
    MU = np.zeros((n, n))
    for k in range(n):
        J = np.nonzero(pat_l[:, k])[0][:cap]
        m = np.zeros(len(J))
        for x, rx in enumerate(J):
            acc = 1.0 if rx == k else 0.0
            for y in range(x):
                acc -= L[rx, J[y]] * m[y]
            m[x] = acc
        ML[J, k] = m
        J = np.nonzero(pat_u[:, k])[0]
        J = J[max(0, len(J) - cap):]
        m = np.zeros(len(J))
        for x in range(len(J) - 1, -1, -1):
            rx = J[x]
            acc = 1.0 if rx == k else 0.0
            for y in range(x + 1, len(J)):
                acc -= U[rx, J[y]] * m[y]
            m[x] = acc / U[rx, rx] if abs(U[rx, rx]) > 1e-300 else 0.0
        MU[J, k] = m
    return ML, MU
