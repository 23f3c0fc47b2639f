"""ORACLE (test infrastructure only): restatement of the reference's transient
source evaluation and backward-Euler companion system, with a Newton solve
(direct sparse LU) per step.

Only ``tests/`` and ``bench.py``'s CPU-baseline leg may use this module, and
only as the checker / timed CPU baseline.

  ``eval_source``   PULSE / SIN / PWL / EXP, src/analysis/transient_source.rs:8-118
  ``b_at_time``     collect_source_info + evaluate_b_at_time, transient.rs:212-280
  ``companion``     A = G + C/h (BE), transient.rs:285-323
  ``be_transient``  b = b(t_n) + (C/h) x_{n-1} (transient.rs:326-333), then the
                    Newton loop of ``newton_ref.newton`` on (A, b) from x_{n-1}.

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


def companion(sysm, h):
    """A = G + C/h on G's pattern (every C entry must lie on it)."""
    a = sysm.g.val.astype(np.float64).copy()
    c = sysm.c
    for i in range(c.nrows):
        for k in range(int(c.row_ptr[i]), int(c.row_ptr[i + 1])):
            j = int(c.col[k])
            s = int(sysm.g.row_ptr[i]) + int(np.searchsorted(sysm.g.col[sysm.g.row_ptr[i]:sysm.g.row_ptr[i + 1]], j))
            assert sysm.g.col[s] == j, "capacitance entry off the conductance pattern"
            a[s] += c.val[k] / h
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
        b = b_at_time(sysm, tn) + c_times(sysm, x) / h
        x, it = newton_ref.newton(sysm, base_vals=A, base_b=b, x0=x, **newton_kw)
        wave[s] = x[list(probes)]
        its.append(it)
    return x, wave, its
