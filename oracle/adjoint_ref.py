"""ORACLE (test infrastructure only): sensitivities of one output of a DC
solve or of a backward-Euler transient, by the adjoint method with a direct
sparse LU, by FP64 forward sensitivities, and by central finite differences.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may use this module, and only as the checker / timed CPU baseline.  The reference has no sensitivity
analysis; the equations are the BE companion of src/analysis/transient.rs
(:285-333) with a Newton solve per step, written as residuals

    F_0(x_0) = G x_0 + i(x_0) - b(t_0)                          (DC start)
    F_n(x_n) = (G + C/h) x_n - (C/h) x_{n-1} + i(x_n) - b(t_n)

for an output o = w . x_N.  Parameters: every resistance R (conductance 1/R
between its terminals), capacitance C, diode saturation current Is
(i_d = Is (exp(v / nVt) - 1), the stored f32 value), and every MOSFET's
threshold magnitude |VTO| and transconductance KP (the descriptor values;
the drain current of ds_nonlinear_shaders.rs:746-849 depends on them through
v_ov = V_GS - |VTO| and linearly on KP).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spl

from . import devices_ref as dev
from . import transient_ref as tref


def _at(v, idx):
    idx = np.asarray(idx)
    out = np.zeros(idx.shape)
    ok = idx >= 0
    out[ok] = v[idx[ok]]
    return out


def _jacobian(sysm, base_vals, x):
    J, _ = dev.assemble(sysm, base_vals, sysm.b_dc, x)
    n = sysm.size
    return sp.csr_matrix((J, sysm.g.col, sysm.g.row_ptr), shape=(n, n))


def _diode_terms(sysm, x):
    d = sysm.diode_descriptors
    an = d["anode"].astype(np.int64)
    ca = d["cathode"].astype(np.int64)
    an = np.where(an == 0xFFFFFFFF, -1, an)
    ca = np.where(ca == 0xFFFFFFFF, -1, ca)
    v = _at(x, an) - _at(x, ca)
    e = np.exp(np.clip(v / d["n_vt"].astype(np.float64), -80.0, 80.0))
    return an, ca, e - 1.0


def _mosfet_terms(sysm, x):
    """Drain/source rows (-1 = ground), dI/d|VTO| and dI/dKP of the drain
    current I (polarity applied) at x."""
    m = sysm.mosfet_descriptors
    dr = m["drain"].astype(np.int64)
    so = m["source"].astype(np.int64)
    dr = np.where(dr == 0xFFFFFFFF, -1, dr)
    so = np.where(so == 0xFFFFFFFF, -1, so)
    i_d, g_m, _ = dev.mosfet_eval(m, x)
    pol = m["polarity"].astype(np.float64)
    return dr, so, -pol * g_m, i_d / m["kp"].astype(np.float64)


def backstamp(sysm, comps, x, xprev, lam, h):
    """-lambda^T dF/dp per component (xprev None: the DC equation); MOSFET
    gradients are returned by ``backstamp_mosfets``."""
    dv = _at(x, comps.r_a) - _at(x, comps.r_b)
    gr = dv * (_at(lam, comps.r_a) - _at(lam, comps.r_b)) / comps.r_ohms ** 2
    gc = np.zeros(len(comps.c_farads))
    if xprev is not None:
        ddv = (_at(x, comps.c_a) - _at(x, comps.c_b)) - (_at(xprev, comps.c_a) - _at(xprev, comps.c_b))
        gc = -ddv / h * (_at(lam, comps.c_a) - _at(lam, comps.c_b))
    an, ca, em1 = _diode_terms(sysm, x)
    gd = -(_at(lam, an) - _at(lam, ca)) * em1
    return gr, gc, gd


def backstamp_mosfets(sysm, x, lam):
    """-lambda^T dF/d|VTO| and -lambda^T dF/dKP per MOSFET: the drain current
    enters F at the drain row and leaves at the source row."""
    if not len(sysm.mosfet_descriptors):
        return np.zeros(0), np.zeros(0)
    dr, so, di_dvto, di_dkp = _mosfet_terms(sysm, x)
    dl = _at(lam, dr) - _at(lam, so)
    return -dl * di_dvto, -dl * di_dkp


def dc_adjoint(sysm, comps, x, w):
    J = _jacobian(sysm, sysm.g.val, x)
    lam = spl.splu(J.T.tocsc()).solve(np.asarray(w, dtype=np.float64))
    gr, _, gd = backstamp(sysm, comps, x, None, lam, 1.0)
    gv, gk = backstamp_mosfets(sysm, x, lam)
    return {"R": gr, "Is": gd, "VTO": gv, "KP": gk}, lam


def transient_states(sysm, x0, t0, h, n_steps):
    states = [np.array(x0, dtype=np.float64)]
    A = tref.companion(sysm, h)
    x = states[0]
    for s in range(n_steps):
        b = tref.b_at_time(sysm, t0 + (s + 1) * h) + tref.c_times(sysm, x) / h
        from . import newton_ref
        x, _ = newton_ref.newton(sysm, base_vals=A, base_b=b, x0=x)
        states.append(x)
    return states


def transient_adjoint(sysm, comps, states, h, w):
    """Gradients of o = w . x_N; states = [x_0 .. x_N] (x_0 the DC point)."""
    A = tref.companion(sysm, h)
    n = sysm.size
    cm = sp.csr_matrix((sysm.c.val, sysm.c.col, sysm.c.row_ptr), shape=(n, n))
    rhs = np.asarray(w, dtype=np.float64)
    gr = np.zeros(len(comps.r_ohms))
    gc = np.zeros(len(comps.c_farads))
    gd = np.zeros(len(sysm.diode_descriptors))
    gv = np.zeros(len(sysm.mosfet_descriptors))
    gk = np.zeros(len(sysm.mosfet_descriptors))
    N = len(states) - 1
    for k in range(N, 0, -1):
        J = _jacobian(sysm, A, states[k])
        lam = spl.splu(J.T.tocsc()).solve(rhs)
        a, b, c = backstamp(sysm, comps, states[k], states[k - 1], lam, h)
        mv, mk = backstamp_mosfets(sysm, states[k], lam)
        gr += a
        gc += b
        gd += c
        gv += mv
        gk += mk
        rhs = cm.T @ lam / h
    J0 = _jacobian(sysm, sysm.g.val, states[0])
    lam0 = spl.splu(J0.T.tocsc()).solve(rhs)
    a, _, c = backstamp(sysm, comps, states[0], None, lam0, h)
    mv, mk = backstamp_mosfets(sysm, states[0], lam0)
    return {"R": gr + a, "C": gc, "Is": gd + c, "VTO": gv + mv, "KP": gk + mk}


def _dF_dp(sysm, comps, kind, j, x, xprev, h):
    """dF/dp of one parameter as a dense vector."""
    n = sysm.size
    f = np.zeros(n)

    def put(i, v):
        if i >= 0:
            f[i] += v
    if kind == "R":
        a, b, r = int(comps.r_a[j]), int(comps.r_b[j]), comps.r_ohms[j]
        dv = (x[a] if a >= 0 else 0.0) - (x[b] if b >= 0 else 0.0)
        put(a, -dv / r ** 2)
        put(b, dv / r ** 2)
    elif kind == "C":
        if xprev is None:
            return f
        a, b = int(comps.c_a[j]), int(comps.c_b[j])
        v = lambda z, i: z[i] if i >= 0 else 0.0  # noqa: E731
        ddv = (v(x, a) - v(x, b)) - (v(xprev, a) - v(xprev, b))
        put(a, ddv / h)
        put(b, -ddv / h)
    elif kind in ("VTO", "KP"):
        dr, so, di_dvto, di_dkp = _mosfet_terms(sysm, x)
        d = di_dvto[j] if kind == "VTO" else di_dkp[j]
        put(int(dr[j]), d)
        put(int(so[j]), -d)
    else:
        an, ca, em1 = _diode_terms(sysm, x)
        put(int(an[j]), em1[j])
        put(int(ca[j]), -em1[j])
    return f


def forward_sensitivity(sysm, comps, states, h, w, kind, j):
    """d(w . x_N)/dp by the FP64 forward recursion J_0 s_0 = -dF_0/dp,
    J_n s_n = -dF_n/dp + (C/h) s_{n-1}."""
    A = tref.companion(sysm, h)
    n = sysm.size
    cm = sp.csr_matrix((sysm.c.val, sysm.c.col, sysm.c.row_ptr), shape=(n, n))
    J0 = _jacobian(sysm, sysm.g.val, states[0])
    s = spl.splu(J0.tocsc()).solve(-_dF_dp(sysm, comps, kind, j, states[0], None, h))
    for k in range(1, len(states)):
        J = _jacobian(sysm, A, states[k])
        s = spl.splu(J.tocsc()).solve(-_dF_dp(sysm, comps, kind, j, states[k], states[k - 1], h) + cm @ s / h)
    return float(np.dot(w, s))
