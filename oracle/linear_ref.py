"""ORACLE (test infrastructure only): FP64 direct solvers and the reference
BiCGSTAB, restated on the CPU.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may use this module, and only as the checker / timed CPU baseline.

  dense_solve_real / _complex   C restatement of ``CpuSolver`` (src/solver/cpu.rs:28-171),
                                built from ``oracle/dense_ge.c`` by ``oracle/Makefile``.
  sparse_lu_solve               FP64 sparse direct solve standing in for the
                                reference's faer 0.24 ``sp_lu`` (src/solver/sparse_direct.rs:12-61;
                                faer is a Rust crate that is not available here).
                                SuperLU via scipy 1.18 ``splu``, natural column
                                order is not required: any exact FP64 LU pins the answer.
  bicgstab                      ``bicgstab_with_params`` (src/solver/bicgstab.rs:56-189)
                                statement by statement, FP64 numpy, right preconditioning.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


class SolveError(RuntimeError):
    """``OhmnivoreError::Solve`` (src/error.rs:12-13)."""


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"oracle library missing: {path} (run `make -C oracle`)")
        L = ctypes.CDLL(path)
        p64 = ctypes.POINTER(ctypes.c_int64)
        pd = ctypes.POINTER(ctypes.c_double)
        for fn in (L.oracle_dense_solve_real, L.oracle_dense_solve_complex):
            fn.restype = ctypes.c_int
            fn.argtypes = [ctypes.c_int64, ctypes.c_int64, p64, p64, pd, ctypes.c_int64, pd, pd,
                           ctypes.c_int]
        _LIB = L
    return _LIB


def _p(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


_ERR = {1: "singular matrix", 2: "dimension mismatch", 3: "out of memory"}


def dense_solve_real(nrows, ncols, row_ptr, col, val, b, skip_zero_factors=True):
    """CpuSolver::solve_real (cpu.rs:28-96)."""
    rp = np.ascontiguousarray(row_ptr, np.int64)
    ci = np.ascontiguousarray(col, np.int64)
    v = np.ascontiguousarray(val, np.float64)
    bb = np.ascontiguousarray(b, np.float64)
    x = np.zeros(nrows)
    rc = lib().oracle_dense_solve_real(nrows, ncols, _p(rp, ctypes.c_int64), _p(ci, ctypes.c_int64),
                                       _p(v, ctypes.c_double), bb.shape[0], _p(bb, ctypes.c_double),
                                       _p(x, ctypes.c_double), int(skip_zero_factors))
    if rc:
        raise SolveError(_ERR.get(rc, f"error {rc}"))
    return x


def dense_solve_complex(nrows, ncols, row_ptr, col, val, b, skip_zero_factors=True):
    """CpuSolver::solve_complex (cpu.rs:98-171)."""
    rp = np.ascontiguousarray(row_ptr, np.int64)
    ci = np.ascontiguousarray(col, np.int64)
    v = np.ascontiguousarray(np.asarray(val, np.complex128).view(np.float64))
    bb = np.ascontiguousarray(np.asarray(b, np.complex128).view(np.float64))
    x = np.zeros(2 * nrows)
    rc = lib().oracle_dense_solve_complex(nrows, ncols, _p(rp, ctypes.c_int64),
                                          _p(ci, ctypes.c_int64), _p(v, ctypes.c_double),
                                          bb.shape[0] // 2, _p(bb, ctypes.c_double),
                                          _p(x, ctypes.c_double), int(skip_zero_factors))
    if rc:
        raise SolveError(_ERR.get(rc, f"error {rc}"))
    return x.view(np.complex128)


def sparse_lu_solve(n, row_ptr, col, val, b):
    """FP64 sparse LU solve (stand-in for sparse_direct.rs:12-61)."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as sla
    A = sp.csr_matrix((np.asarray(val), np.asarray(col, np.int64), np.asarray(row_ptr, np.int64)),
                      shape=(n, n))
    try:
        lu = sla.splu(A.tocsc(), permc_spec="COLAMD", diag_pivot_thresh=1.0)
    except RuntimeError as e:   # exactly singular
        raise SolveError(f"sparse LU failed: {e}") from e
    x = lu.solve(np.asarray(b))
    if not np.all(np.isfinite(x)):
        raise SolveError("sparse LU produced non-finite solution")
    return x


def spmv(n, row_ptr, col, val, x):
    val = np.asarray(val)
    x = np.asarray(x)
    rows = np.repeat(np.arange(n), np.diff(np.asarray(row_ptr)))
    y = np.zeros(n, dtype=np.result_type(val.dtype, x.dtype))
    np.add.at(y, rows, val * x[np.asarray(col, dtype=np.int64)])
    return y


def bicgstab(n, row_ptr, col, val, b, precond, max_iterations=10_000, tolerance=1e-5):
    """Statement-by-statement restatement of ``bicgstab_with_params``
    (src/solver/bicgstab.rs:56-189).  ``precond(v) -> M^{-1} v``.
    Returns (x, iterations).  Raises SolveError on the same conditions."""
    if max_iterations == 0:
        raise SolveError("BiCGSTAB max_iterations must be > 0")
    if not (tolerance > 0.0 and np.isfinite(tolerance)):
        raise SolveError("BiCGSTAB tolerance must be finite and > 0")
    A = lambda v: spmv(n, row_ptr, col, val, v)  # noqa: E731
    x = np.zeros(n)
    r = np.array(b, dtype=np.float64)
    r_hat = r.copy()
    p = np.zeros(n); v = np.zeros(n)
    b_norm = np.sqrt(r @ r)
    if b_norm < 1e-30:
        return x, 0
    abs_tol = tolerance * b_norm
    rho = alpha = omega = 1.0
    for it in range(max_iterations):
        rho_new = r_hat @ r
        if abs(rho_new) < 1e-30:
            raise SolveError("BiCGSTAB breakdown: rho ~ 0")
        beta = (rho_new / rho) * (alpha / omega)
        rho = rho_new
        p = (p + (-omega) * v) * beta + r          # axpy(-w, v, p); scale(beta); axpy(1, r, p)
        p_hat = precond(p)
        v = A(p_hat)
        rv = r_hat @ v
        if abs(rv) < 1e-30:
            raise SolveError("BiCGSTAB breakdown: r_hat.v ~ 0")
        alpha = rho / rv
        s = r + (-alpha) * v
        if np.sqrt(s @ s) < abs_tol:
            x = x + alpha * p_hat
            return x, it + 1
        s_hat = precond(s)
        t = A(s_hat)
        ts = t @ s
        tt = t @ t
        if abs(tt) < 1e-30:
            raise SolveError("BiCGSTAB breakdown: ||t|| ~ 0")
        omega = ts / tt
        x = x + alpha * p_hat
        x = x + omega * s_hat
        r = s + (-omega) * t
        rn = np.sqrt(r @ r)
        if not np.isfinite(rn):
            raise SolveError("BiCGSTAB diverged: NaN/Inf in residual")
        if rn < abs_tol:
            return x, it + 1
        if abs(omega) < 1e-30:
            raise SolveError("BiCGSTAB breakdown: omega ~ 0")
    raise SolveError(f"BiCGSTAB did not converge within {max_iterations} iterations")


def jacobi_inverse_diagonal(n, row_ptr, col, val):
    """gpu.rs:177-190 / newton.rs:340-361: 1/a_ii when |a_ii| > 1e-30, else 0."""
    inv = np.zeros(n)
    rp = np.asarray(row_ptr)
    for i in range(n):
        for k in range(rp[i], rp[i + 1]):
            if col[k] == i:
                if abs(val[k]) > 1e-30:
                    inv[i] = 1.0 / val[k]
                break
    return inv
