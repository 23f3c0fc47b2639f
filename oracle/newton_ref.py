"""ORACLE (test infrastructure only): FP64 Newton-Raphson with a direct
sparse LU per iteration, and the BE transient step built on it.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may use this module, and only as the checker / timed CPU baseline.

Follows ``newton_solve`` (src/solver/newton.rs:153-488) with
``NewtonLinearMode::CpuSparseLu`` (newton.rs:282-317): per iteration
x_old = x; evaluate devices at x; assemble J and b_eq (base + stamps); solve
J x = b_eq directly; limit; converged when max|x - x_old| < abs_tol.
The oracle's own default tolerance is tight (abs_tol 1e-13 relative to
max(1, |x|_inf)) so that its answer is the FP64 fixed point.

Continuation fallbacks (GMIN stepping, src/analysis/dc.rs:160-292) are used
when the direct Newton does not converge.
"""
from __future__ import annotations

import numpy as np

from . import devices_ref as dev
from .linear_ref import SolveError, dense_solve_real, sparse_lu_solve


class NewtonNotConverged(RuntimeError):
    """``OhmnivoreError::NewtonNotConverged`` (src/error.rs:15-19)."""


def newton(sysm, base_vals=None, base_b=None, x0=None, max_iterations=100, abs_tol=None,
           rel_tol=1e-13, linear="splu", history=None):
    n = sysm.size
    vals0 = sysm.g.val if base_vals is None else base_vals
    b0 = sysm.b_dc if base_b is None else base_b
    x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64)
    rp, ci = sysm.g.row_ptr, sysm.g.col
    for it in range(max_iterations):
        x_old = x
        J, b = dev.assemble(sysm, vals0, b0, x)
        if not np.all(np.isfinite(J)):
            raise SolveError(f"numerical error at iteration {it}")
        if linear == "dense":
            x_new = dense_solve_real(n, n, rp, ci, J, b)
        else:
            x_new = sparse_lu_solve(n, rp, ci, J, b)
        x, _ = dev.limit(sysm, x_old, x_new)
        if not np.all(np.isfinite(x)):
            raise SolveError(f"numerical error at iteration {it}")
        d = float(np.max(np.abs(x - x_old))) if n else 0.0
        if history is not None:
            history.append(d)
        tol = abs_tol if abs_tol is not None else rel_tol * max(1.0, float(np.max(np.abs(x))))
        if d < tol:
            return x, it + 1
    raise NewtonNotConverged(f"no convergence after {max_iterations} iterations")


def dc_operating_point(sysm, **kw):
    """Direct Newton, then GMIN stepping (dc.rs:160-292) if it fails."""
    try:
        return newton(sysm, **kw)
    except (NewtonNotConverged, SolveError):
        pass
    diag = np.array([sysm.g.value_index(i, i) for i in range(sysm.n_nodes)], dtype=np.int64)
    x_prev = None
    gmin = 1e-1
    last_good = 1.0
    sub = 0
    while gmin > 1e-13:
        vals = sysm.g.val.copy()
        vals[diag] += gmin
        try:
            x_prev, _ = newton(sysm, base_vals=vals, x0=x_prev, max_iterations=50, abs_tol=1e-9)
            last_good = gmin
            sub = 0
            gmin *= 1e-3
        except (NewtonNotConverged, SolveError):
            sub += 1
            if sub > 13:
                raise
            gmin = last_good * 10.0 ** (-sub)
    return newton(sysm, x0=x_prev, **kw)


def residual(sysm, x, base_vals=None, base_b=None):
    """FP64 KCL residual b_eq(x) - J(x) x  (zero at the DC operating point)."""
    J, b = dev.assemble(sysm, sysm.g.val if base_vals is None else base_vals,
                        sysm.b_dc if base_b is None else base_b, x)
    rows = np.repeat(np.arange(sysm.size), np.diff(sysm.g.row_ptr))
    Ax = np.zeros(sysm.size)
    np.add.at(Ax, rows, J * x[sysm.g.col])
    return b - Ax
