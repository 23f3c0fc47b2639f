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

Continuation fallbacks: ``dc_operating_point`` adds GMIN stepping
(src/analysis/dc.rs:160-292) when the direct Newton does not converge;
``run_nonlinear`` restates the reference's whole DC strategy (source
stepping, GMIN stepping, pseudo-transient continuation, dc.rs:60-650).
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


def _node_diagonals(sysm):
    return np.array([sysm.g.value_index(i, i) for i in range(sysm.n_nodes)], dtype=np.int64)


def _step(sysm, diag, gmin=0.0, base_b=None, x0=None, max_iterations=50, abs_tol=1e-9):
    """``gmin_newton_step`` (dc.rs:293-330): one Newton solve with ``gmin``
    added to every node diagonal and the given rhs; every linear solve is the
    LU (the reference's CpuSparseLu retry of each step)."""
    vals = sysm.g.val.copy()
    if gmin != 0.0:
        vals[diag] += gmin
    x, _ = newton(sysm, base_vals=vals, base_b=base_b, x0=x0, max_iterations=max_iterations, abs_tol=abs_tol)
    return x


def run_nonlinear(sysm, step_tol=1e-9, stages=None):
    """The reference's nonlinear DC strategy, ``run_nonlinear``
    (src/analysis/dc.rs:60-290), with an LU per Newton iteration:

      1. direct Newton (50 iterations, NewtonParams::default, :72-121);
      2. for circuits with MOSFETs, source stepping (:495-645): alpha from
         0.1, on success grow by twice the last successful step, on failure
         halve towards the last good alpha, at most 20 subdivisions or a step
         below 1e-6; 30 Newton iterations per step;
      3. adaptive GMIN stepping (:160-253) from zeros: 1e-1, 1000x drops,
         10x subdivisions from the last good level, at most 13; 15 Newton
         iterations per step; then the true-GMIN solve (50 iterations);
      4. if that fails, pseudo-transient continuation (:331-490) from the
         last GMIN point: alpha from 1e-1, 100x drops, at most 7 10x
         subdivisions, gmin = alpha and b += alpha x_prev on node rows,
         20 Newton iterations per step; final solve with 25 iterations.

    Intermediate steps stop at max|dx| < ``step_tol``; the answer is then
    polished by the oracle's tight Newton.  ``stages`` (a list) receives the
    names of the stages that ran.  Returns x.
    """
    stages = [] if stages is None else stages
    n_nodes = sysm.n_nodes
    polish = lambda x: newton(sysm, x0=x, max_iterations=100)[0]   # noqa: E731
    stages.append("direct")
    try:
        return polish(newton(sysm, max_iterations=50, abs_tol=step_tol)[0])
    except (NewtonNotConverged, SolveError):
        pass
    diag = _node_diagonals(sysm)
    if len(sysm.mosfet_descriptors):
        stages.append("source")
        x_prev = None
        last, target, sub = 0.0, 0.1, 0
        try:
            while target <= 1.0:
                try:
                    x = _step(sysm, diag, 0.0, target * sysm.b_dc, x_prev, 30, step_tol)
                except (NewtonNotConverged, SolveError):
                    sub += 1
                    if sub > 20:
                        raise
                    target = last + (target - last) / 2.0
                    if target - last < 1e-6:
                        raise
                    continue
                x_prev = x
                prev_step = target - last
                last = target
                sub = 0
                if abs(target - 1.0) < 1e-12:
                    return polish(x)
                target = min(target + 2.0 * prev_step, 1.0)
        except (NewtonNotConverged, SolveError):
            pass
    stages.append("gmin")
    x_prev = None
    last, target, sub = 1.0, 1e-1, 0
    while target > 1e-13:
        try:
            x_prev = _step(sysm, diag, target, None, x_prev, 15, step_tol)
            last, sub = target, 0
            target *= 1e-3
        except (NewtonNotConverged, SolveError):
            sub += 1
            if sub > 13:
                raise
            target = last * 10.0 ** (-sub)
    try:
        return polish(_step(sysm, diag, 0.0, None, x_prev, 50, step_tol))
    except (NewtonNotConverged, SolveError):
        if x_prev is None:
            raise
    stages.append("pseudo")
    last, target, sub = 1.0, 1e-1, 0
    while target > 1e-8:
        b = sysm.b_dc.copy()
        b[:n_nodes] += target * x_prev[:n_nodes]
        try:
            x_prev = _step(sysm, diag, target, b, x_prev, 20, step_tol)
            last, sub = target, 0
            target *= 1e-2
        except (NewtonNotConverged, SolveError):
            sub += 1
            if sub > 7:
                raise
            target = last * 10.0 ** (-sub)
    return polish(_step(sysm, diag, 0.0, None, x_prev, 25, step_tol))


def residual(sysm, x, base_vals=None, base_b=None):
    """FP64 KCL residual b_eq(x) - J(x) x  (zero at the DC operating point)."""
    J, b = dev.assemble(sysm, sysm.g.val if base_vals is None else base_vals,
                        sysm.b_dc if base_b is None else base_b, x)
    rows = np.repeat(np.arange(sysm.size), np.diff(sysm.g.row_ptr))
    Ax = np.zeros(sysm.size)
    np.add.at(Ax, rows, J * x[sysm.g.col])
    return b - Ax
