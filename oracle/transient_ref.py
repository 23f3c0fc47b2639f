"""ORACLE (test infrastructure only): restatement of the reference's transient
source evaluation and backward-Euler companion system, with a Newton solve
(direct sparse LU) per step.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may use this module, and only as the checker / timed CPU baseline.

  ``eval_source``   PULSE / SIN / PWL / EXP, src/analysis/transient_source.rs:8-118
  ``b_at_time``     collect_source_info + evaluate_b_at_time, transient.rs:212-280
  ``companion``     A = G + C/h (BE), transient.rs:285-323
  ``be_transient``  b = b(t_n) + (C/h) x_{n-1} (transient.rs:326-333), then the
                    Newton loop of ``newton_ref.newton`` on (A, b) from x_{n-1}.
  ``adaptive_transient``  the adaptive BE / TRAP loop of transient::run
                    (transient.rs:77-178): TRAP rhs :336-352, LTE :355-362.
  ``uic_initial_conditions``  compute_uic_initial_conditions, transient.rs:364-482.

The reference's transient is linear only (one linear solve per step, devices
ignored); the Newton step per BE step is the nonlinear extension, so parity of
nonlinear transients is pinned by this restatement, not by reference output.
The source functions are pinned by the reference's known answers
(transient_source.rs tests).
"""
from __future__ import annotations

import math

import numpy as np

from . import newton_ref

PULSE, SIN, PWL, EXP = range(4)


def eval_source(kind, params, t):
    """transient_source.rs:8-118."""
    if kind == PULSE:
        v1, v2, td, tr, tf, pw, per = params
        if t < td:
            return v1
        t_rel = math.fmod(t - td, per) if (per > 0.0 and per < np.finfo(np.float64).max) else t - td
        if t_rel < tr:
            return v1 + (v2 - v1) * t_rel / tr if tr > 0.0 else v2
        if t_rel < tr + pw:
            return v2
        if t_rel < tr + pw + tf:
            return v2 + (v1 - v2) * (t_rel - tr - pw) / tf if tf > 0.0 else v1
        return v1
    if kind == SIN:
        vo, va, freq, td, theta = params[:5]
        if t < td:
            return vo
        dt = t - td
        env = math.exp(-dt * theta) if theta != 0.0 else 1.0
        return vo + va * math.sin(2.0 * math.pi * freq * dt) * env
    if kind == PWL:
        pairs = [tuple(p) for p in np.asarray(params, dtype=np.float64).reshape(-1, 2)]
        if not pairs:
            return 0.0
        if t <= pairs[0][0]:
            return pairs[0][1]
        if t >= pairs[-1][0]:
            return pairs[-1][1]
        for i in range(1, len(pairs)):
            if t <= pairs[i][0]:
                t0, v0 = pairs[i - 1]
                t1, v1 = pairs[i]
                return v0 + (v1 - v0) * ((t - t0) / (t1 - t0))
        return pairs[-1][1]
    if kind == EXP:
        v1, v2, td1, tau1, td2, tau2 = params[:6]
        if t < td1:
            return v1
        rise = (v2 - v1) * (1.0 - math.exp(-(t - td1) / tau1))
        if t < td2:
            return v1 + rise
        fall = (v1 - v2) * (1.0 - math.exp(-(t - td2) / tau2))
        return v1 + rise + fall
    raise ValueError(f"unknown source kind {kind}")


def b_at_time(sysm, t):
    """transient.rs:265-280: b starts at zero; every source adds sign * value."""
    b = np.zeros(sysm.size)
    for _, entries, dc, tran in sysm.sources:
        v = eval_source(tran[0], tran[1], t) if tran is not None else (0.0 if dc is None else dc)
        for row, sign in entries:
            b[row] += sign * v
    return b


def companion(sysm, h, alpha=1.0):
    """A = G + (alpha / h) C on G's pattern (every C entry must lie on it),
    form_companion_matrix, transient.rs:285-323."""
    factor = alpha / h
    a = sysm.g.val.astype(np.float64).copy()
    c = sysm.c
    for i in range(c.nrows):
        for k in range(int(c.row_ptr[i]), int(c.row_ptr[i + 1])):
            j = int(c.col[k])
            s = int(sysm.g.row_ptr[i]) + int(np.searchsorted(sysm.g.col[sysm.g.row_ptr[i]:sysm.g.row_ptr[i + 1]], j))
            assert sysm.g.col[s] == j, "capacitance entry off the conductance pattern"
            a[s] += factor * c.val[k]
    return a


def c_times(sysm, x):
    c = sysm.c
    rows = np.repeat(np.arange(c.nrows), np.diff(c.row_ptr))
    y = np.zeros(c.nrows)
    np.add.at(y, rows, c.val * x[c.col])
    return y


def be_transient(sysm, x0, t0, h, n_steps, probes, **newton_kw):
    """Returns (x at the end, waveform n_steps x len(probes), Newton iterations per step)."""
    A = companion(sysm, h)
    x = np.array(x0, dtype=np.float64)
    wave = np.zeros((n_steps, len(probes)))
    its = []
    for s in range(n_steps):
        tn = t0 + (s + 1) * h
        b = b_at_time(sysm, tn) + (1.0 / h) * c_times(sysm, x)
        x, it = newton_ref.newton(sysm, base_vals=A, base_b=b, x0=x, **newton_kw)
        wave[s] = x[list(probes)]
        its.append(it)
    return x, wave, its


class TimestepError(RuntimeError):
    """``OhmnivoreError::Timestep`` (src/error.rs)."""


def f_of_x(sysm, x):
    """f(x) = G x + i(x): J(x) x - b of the system stamped at x on the base
    (G, 0).  For a linear circuit this is the reference's G x."""
    return -newton_ref.residual(sysm, x, base_vals=sysm.g.val, base_b=np.zeros(sysm.size))


def adaptive_transient(sysm, x0, tstep, tstop, tstart, probes, **newton_kw):
    """transient::run's stepping loop (transient.rs:77-178) from t = 0, each
    companion solve a Newton solve (LU) from x_{n-1}.  Returns
    (times, waveforms n_points x n_probes, stats)."""
    h_min = tstep / 10_000.0
    h_max = tstep
    lte_tol = 1e-3
    max_consecutive_failures = 10
    probes = list(probes)
    x = np.array(x0, dtype=np.float64)
    times, wave = [], []
    stats = {"accepted": 0, "rejected": 0, "linear_solves": 0}
    if tstart <= 0.0:
        times.append(0.0)
        wave.append(x[probes].copy())
    t = 0.0
    h = min(tstep, h_max)
    b_prev = b_at_time(sysm, 0.0)
    use_be = True
    fails = 0

    def solve(alpha, rhs):
        xs, _ = newton_ref.newton(sysm, base_vals=companion(sysm, h, alpha), base_b=rhs, x0=x, **newton_kw)
        stats["linear_solves"] += 1
        return xs

    while t < tstop:
        if t + h > tstop:
            h = tstop - t
        if h < h_min * 0.5:
            break
        t_next = t + h
        b_next = b_at_time(sysm, t_next)
        cx = c_times(sysm, x)
        if use_be:
            x_be = solve(1.0, b_next + (1.0 / h) * cx)
            x_trap = x_be
        else:
            rhs = ((b_next + (2.0 / h) * cx) - f_of_x(sysm, x)) + b_prev
            x_trap = solve(2.0, rhs)
            x_be = solve(1.0, b_next + (1.0 / h) * cx)
        if not use_be:
            lte = (2.0 / 3.0) * float(np.max(np.abs(x_trap - x_be)))
            ratio = lte_tol / lte if lte > 0.0 else math.inf
            factor = min(max(0.9 * math.sqrt(ratio), 0.5), 2.0)
            if lte > lte_tol:
                h = max(h * factor, h_min)
                fails += 1
                if fails >= max_consecutive_failures and h <= h_min * 1.01:
                    raise TimestepError(f"{fails} consecutive failures at minimum timestep near t={t:.2e}")
                stats["rejected"] += 1
                use_be = True
                continue
            h = min(max(h * factor, h_min), h_max)
        else:
            use_be = False
        fails = 0
        stats["accepted"] += 1
        x = x_trap
        b_prev = b_next
        t = t_next
        if t >= tstart:
            times.append(t)
            wave.append(x[probes].copy())
    return np.array(times), np.array(wave).reshape(len(times), len(probes)), stats


def uic_initial_conditions(sysm, ckt):
    """compute_uic_initial_conditions (transient.rs:364-482): inductor branch
    rows become I_L = 0; per capacitor, in component order, the first
    unconstrained terminal row becomes V(i) - V(j) = 0 (V(i) = 0 to ground);
    then one direct solve."""
    from ohmnivore_b200 import circuits as ck

    g = sysm.g
    vals = g.val.astype(np.float64).copy()
    b = sysm.b_dc.astype(np.float64).copy()
    n_nodes = sysm.n_nodes

    def zero_row(r):
        vals[int(g.row_ptr[r]):int(g.row_ptr[r + 1])] = 0.0

    def put(r, c, v):
        k = g.value_index(r, c)
        if k is not None:
            vals[k] = v

    branch_row = {int(ci): n_nodes + k for k, ci in enumerate(sysm.branch_components)}
    for ci in range(ckt.n_components):
        if ckt.kind[ci] == ck.L:
            bk = branch_row[ci]
            zero_row(bk)
            put(bk, bk, 1.0)
            b[bk] = 0.0
    constrained = [False] * n_nodes

    def idx(label):
        return None if label == 0 else sysm.node_index(int(label))

    for ci in range(ckt.n_components):
        if ckt.kind[ci] != ck.C:
            continue
        i, j = idx(ckt.nodes[ci, 0]), idx(ckt.nodes[ci, 1])
        if i is not None and j is None:
            if not constrained[i]:
                zero_row(i); put(i, i, 1.0); b[i] = 0.0; constrained[i] = True
        elif i is None and j is not None:
            if not constrained[j]:
                zero_row(j); put(j, j, 1.0); b[j] = 0.0; constrained[j] = True
        elif i is not None and j is not None:
            if not constrained[i]:
                zero_row(i); put(i, i, 1.0); put(i, j, -1.0); b[i] = 0.0; constrained[i] = True
            elif not constrained[j]:
                zero_row(j); put(j, j, 1.0); put(j, i, -1.0); b[j] = 0.0; constrained[j] = True
    from .linear_ref import sparse_lu_solve
    return sparse_lu_solve(sysm.size, g.row_ptr, g.col, vals, b)
