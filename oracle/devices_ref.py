"""ORACLE (test infrastructure only): FP64 restatement of the reference's
nonlinear device evaluation, Norton-companion stamping and voltage limiting.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may use this module, and only as the checker.

The reference evaluates these in double-single (hi/lo f32) arithmetic; this
restatement runs the same equations in plain FP64 with the f32-rounded
descriptor parameters promoted to f64 (the values the reference stores).

  diode     src/solver/ds_nonlinear_shaders.rs:40-76   (eval)
            :128-164, :211-248                          (matrix / rhs stamps)
  BJT       :280-367 (eval), :393-453 (matrix), :478-573 (rhs)
  MOSFET    :746-849 (eval), :873-911 (matrix), :932-996 (rhs)
  limiting  :1173-1234 (diode pnjlim), :600-714 (BJT), :1051-1130 (MOSFET)
  converge  :1256-1297

Deliberate, documented differences from the reference shaders:
  * the floating diode's matrix stamp uses +g at (a,a) and (c,c) and -g at
    (a,c) and (c,a), in the slot order the compiler writes
    ([aa, cc, ac, ca], src/compiler.rs:625-631); the shader indexes the four
    slots as [aa, ac, ca, cc] (ds_nonlinear_shaders.rs:144-163), which flips
    the sign of the (c,c) and (c,a) stamps when both terminals are non-ground;
  * MOSFET soft-overdrive middle region in FP64 (the shader uses f32 there),
    with log1p(exp(arg)) for the softplus;
  * limiting control flow in FP64 (the shader uses the f32 hi parts) and
    sqrt(2) in FP64;
  * the voltage limiters of all device kinds propose a damping factor per
    terminal node and each node takes the smallest proposal; the reference
    applies BJT, MOSFET and diode limiting in sequence with unsynchronised
    read-modify-writes where devices share a node.  For devices that share no
    node (e.g. every diode to ground on its own node) the result is the same.
  * optional BJT Early voltage VAF (extension; VAF = inf reproduces the
    reference's equations exactly).
"""
from __future__ import annotations

import math

import numpy as np

SENT = 0xFFFFFFFF
VT_MOS = float(np.float32(0.02585))   # shader constant `let VT: f32 = 0.02585;` (:774)
MOS_STEP_LIMIT = 0.5                  # :1028


def _v(x, idx):
    idx = np.asarray(idx, np.int64)
    out = np.zeros(idx.shape)
    ok = idx != SENT
    out[ok] = x[idx[ok]]
    return out


def diode_eval(desc, x):
    """Returns (i_d, g_d) per diode (ds_nonlinear_shaders.rs:40-76)."""
    is_ = desc["is_val"].astype(np.float64)
    nvt = desc["n_vt"].astype(np.float64)
    v = _v(x, desc["anode"]) - _v(x, desc["cathode"])
    e = np.exp(np.clip(v / nvt, -80.0, 80.0))
    return is_ * (e - 1.0), is_ * e / nvt, v


def bjt_eval(desc, x, vaf=None):
    """Ebers-Moll transport model (ds_nonlinear_shaders.rs:280-367).

    Returns currents (I_C, I_B) with polarity applied and the four partials
    dI_C/dVbe, dI_C/dVbc, dI_B/dVbe, dI_B/dVbc (polarity-free, as the shader).
    With a finite VAF the collector transport current is multiplied by
    (1 + Vce/VAF), Vce = Vbe - Vbc, and the partials follow.
    """
    pol = desc["polarity"].astype(np.float64)
    is_ = desc["is_val"].astype(np.float64)
    bf = desc["bf"].astype(np.float64)
    br = desc["br"].astype(np.float64)
    nf = desc["nf_vt"].astype(np.float64)
    nr = desc["nr_vt"].astype(np.float64)
    vb = _v(x, desc["base"]); ve = _v(x, desc["emitter"]); vc = _v(x, desc["collector"])
    vbe = pol * (vb - ve)
    vbc = pol * (vb - vc)
    ef = np.exp(np.clip(vbe / nf, -80.0, 80.0))
    er = np.exp(np.clip(vbc / nr, -80.0, 80.0))
    i_f = is_ * (ef - 1.0)
    i_r = is_ * (er - 1.0)
    bf_frac = bf / (bf + 1.0)
    br1 = br + 1.0
    i_c = bf_frac * i_f - i_r / br1
    i_b = i_f / (bf + 1.0) + i_r / br1
    gf = is_ * ef / nf
    gr = is_ * er / nr
    dic_dvbe = bf_frac * gf
    dic_dvbc = -(gr / br1)
    dib_dvbe = gf / (bf + 1.0)
    dib_dvbc = gr / br1
    if vaf is not None:
        vaf = np.asarray(vaf, np.float64)
        fin = np.isfinite(vaf)
        if fin.any():
            inv = np.where(fin, 1.0 / np.where(fin, vaf, 1.0), 0.0)
            vce = vbe - vbc
            k = 1.0 + vce * inv
            ict = bf_frac * i_f           # transport part carrying the Early factor
            i_c = np.where(fin, ict * k - i_r / br1, i_c)
            dic_dvbe = np.where(fin, dic_dvbe * k + ict * inv, dic_dvbe)
            dic_dvbc = np.where(fin, dic_dvbc - ict * inv, dic_dvbc)
    return pol * i_c, pol * i_b, dic_dvbe, dic_dvbc, dib_dvbe, dib_dvbc


def mosfet_eval(desc, x):
    """Shichman-Hodges with soft overdrive (ds_nonlinear_shaders.rs:746-849).
    Returns (polarity * I_D, g_m, g_ds)."""
    pol = desc["polarity"].astype(np.float64)
    vto = desc["vto"].astype(np.float64)
    kp = desc["kp"].astype(np.float64)
    lam = desc["lam"].astype(np.float64)
    vg = _v(x, desc["gate"]); vs = _v(x, desc["source"]); vd = _v(x, desc["drain"])
    vgs = pol * (vg - vs)
    vds = pol * (vd - vs)
    v_ov = vgs - vto
    arg = v_ov / VT_MOS
    hi = arg > 20.0
    lo = arg < -20.0
    mid = ~(hi | lo)
    e_lo = np.exp(np.clip(arg, -80.0, 80.0))
    veff = np.where(hi, v_ov, np.where(lo, VT_MOS * e_lo, 0.0))
    sig = np.where(hi, 1.0, np.where(lo, e_lo, 0.0))
    am = np.where(mid, arg, 0.0)
    veff = np.where(mid, VT_MOS * np.log1p(np.exp(am)), veff)
    sig = np.where(mid, 1.0 / (1.0 + np.exp(-am)), sig)
    lamf = 1.0 + lam * vds
    lin = vds < veff
    inner = veff * vds - 0.5 * (vds * vds)
    kp_inner = kp * inner
    i_lin = kp_inner * lamf
    gm_lin = (kp * vds) * lamf * sig
    gds_lin = (kp * (veff - vds)) * lamf + kp_inner * lam
    kh_vov2 = (kp / 2.0) * (veff * veff)
    i_sat = kh_vov2 * lamf
    gm_sat = (kp * veff) * lamf * sig
    gds_sat = kh_vov2 * lam
    i_d = np.where(lin, i_lin, i_sat)
    g_m = np.where(lin, gm_lin, gm_sat)
    g_ds = np.where(lin, gds_lin, gds_sat)
    return pol * i_d, g_m, g_ds


def stamp_contributions(sysm, x):
    """All device contributions in canonical order: diodes, then BJTs, then
    MOSFETs; device-major; stamp-position minor.  Returns
    (mat_slots, mat_vals, rhs_rows, rhs_vals) with SENTINEL entries removed."""
    ms, mv, rs, rv = [], [], [], []

    dd = sysm.diode_descriptors
    if len(dd):
        i_d, g_d, v = diode_eval(dd, x)
        ieq = i_d - g_d * v
        slots = dd["g_row_col"].astype(np.int64)                      # [aa, cc, ac, ca]
        vals = np.stack([g_d, g_d, -g_d, -g_d], axis=1)
        ms.append(slots); mv.append(vals)
        rs.append(dd["b_idx"].astype(np.int64)); rv.append(np.stack([-ieq, ieq], axis=1))

    qd = sysm.bjt_descriptors
    if len(qd):
        ic, ib, a, b_, c_, d_ = bjt_eval(qd, x, sysm.bjt_vaf)
        g_cc = -b_; g_cb = a + b_; g_ce = -a
        g_bc = -d_; g_bb = c_ + d_; g_be = -c_
        g_ec = b_ + d_; g_eb = -(((a + b_) + c_) + d_); g_ee = a + c_
        G = np.stack([g_cc, g_cb, g_ce, g_bc, g_bb, g_be, g_ec, g_eb, g_ee], axis=1)
        ms.append(qd["g_row_col"].astype(np.int64)); mv.append(G)
        vc = _v(x, qd["collector"]); vb = _v(x, qd["base"]); ve = _v(x, qd["emitter"])
        ie = -(ic + ib)
        ilc = (g_cc * vc + g_cb * vb) + g_ce * ve
        ilb = (g_bc * vc + g_bb * vb) + g_be * ve
        ile = (g_ec * vc + g_eb * vb) + g_ee * ve
        rs.append(qd["b_idx"].astype(np.int64))
        rv.append(np.stack([-(ic - ilc), -(ib - ilb), -(ie - ile)], axis=1))

    md = sysm.mosfet_descriptors
    if len(md):
        i_d, gm, gds = mosfet_eval(md, x)
        s = gm + gds
        G = np.stack([gds, gm, -s, -gds, -gm, s], axis=1)             # [DD,DG,DS,SD,SG,SS]
        ms.append(md["g_row_col"].astype(np.int64)); mv.append(G)
        vd = _v(x, md["drain"]); vg = _v(x, md["gate"]); vs = _v(x, md["source"])
        ild = (gds * vd + gm * vg) + (-s) * vs
        ieq_d = i_d - ild
        ils = ((-gds) * vd + (-gm) * vg) + s * vs
        ieq_s = (-i_d) - ils
        rs.append(md["b_idx"].astype(np.int64)); rv.append(np.stack([-ieq_d, -ieq_s], axis=1))

    def flat(a, b):
        if not a:
            return np.zeros(0, np.int64), np.zeros(0)
        s = np.concatenate([z.reshape(-1) for z in a])
        v = np.concatenate([z.reshape(-1) for z in b])
        ok = s != SENT
        return s[ok], v[ok]

    a, b = flat(ms, mv)
    c, d = flat(rs, rv)
    return a, b, c, d


def assemble(sysm, base_vals, base_b, x):
    """J = base + device conductance stamps; b = base + Norton currents.
    Contributions are added to each slot left to right in canonical order."""
    ms, mv, rs, rv = stamp_contributions(sysm, x)
    vals = base_vals.astype(np.float64).copy()
    b = base_b.astype(np.float64).copy()
    np.add.at(vals, ms, mv)
    np.add.at(b, rs, rv)
    return vals, b


def pnjlim(vnew, vold, vt, vcrit):
    """Modified SPICE3f5 pnjlim (ds_nonlinear_shaders.rs:1173-1187), FP64."""
    vnew = np.asarray(vnew, np.float64); vold = np.asarray(vold, np.float64)
    out = vnew.copy()
    cond = (vnew > vcrit) & (np.abs(vnew - vold) > vt + vt)
    pos = cond & (vold > 0.0)
    arg = 1.0 + (vnew - vold) / vt
    with np.errstate(invalid="ignore", divide="ignore"):
        a1 = vold + vt * (2.0 + np.log(np.where(arg > 2.0, arg - 2.0, 1.0)))
        a2 = vt * np.log(np.where(vnew > 0, vnew / vt, 1.0))
    out = np.where(pos & (arg > 0.0), a1, out)
    out = np.where(pos & ~(arg > 0.0), vcrit, out)
    out = np.where(cond & ~(vold > 0.0), a2, out)
    return out


def limit(sysm, x_old, x_new):
    """Per-node damping: every device proposes scale = (v_lim - v_old)/(v_new - v_old)
    for its terminal nodes (skipping V-source-fixed nodes for BJT and MOSFET),
    each node keeps the smallest proposal, and nodes with a proposal below 1
    become x_old + (x_new - x_old)*scale; all other entries keep x_new."""
    n = x_new.shape[0]
    scale = np.ones(n)

    def propose(idx, s, ok):
        idx = np.asarray(idx, np.int64)
        m = ok & (idx != SENT)
        np.minimum.at(scale, idx[m], s[m])

    dd = sysm.diode_descriptors
    if len(dd):
        is_ = dd["is_val"].astype(np.float64); nvt = dd["n_vt"].astype(np.float64)
        vcrit = nvt * np.log(nvt / (math.sqrt(2.0) * is_))
        vo = _v(x_old, dd["anode"]) - _v(x_old, dd["cathode"])
        vn = _v(x_new, dd["anode"]) - _v(x_new, dd["cathode"])
        vl = pnjlim(vn, vo, nvt, vcrit)
        dlt = vn - vo
        act = (vl != vn) & (np.abs(dlt) > 1e-30)
        s = np.where(act, (vl - vo) / np.where(act, dlt, 1.0), 1.0)
        propose(dd["anode"], s, act)
        propose(dd["cathode"], s, act)

    qd = sysm.bjt_descriptors
    if len(qd):
        pol = qd["polarity"].astype(np.float64); is_ = qd["is_val"].astype(np.float64)
        fx = qd["node_fixed"] != 0
        for (j, vtk, other, ofix) in ((0, "nf_vt", "emitter", 2), (1, "nr_vt", "collector", 0)):
            vt = qd[vtk].astype(np.float64)
            vcrit = vt * np.log(vt / (math.sqrt(2.0) * is_))
            vo = pol * (_v(x_old, qd["base"]) - _v(x_old, qd[other]))
            vn = pol * (_v(x_new, qd["base"]) - _v(x_new, qd[other]))
            vl = pnjlim(vn, vo, vt, vcrit)
            dlt = vn - vo
            act = (vl != vn) & (np.abs(dlt) > 1e-30)
            s = np.where(act, (vl - vo) / np.where(act, dlt, 1.0), 1.0)
            propose(qd["base"], s, act & ~fx[:, 1])
            propose(qd[other], s, act & ~fx[:, ofix])

    md = sysm.mosfet_descriptors
    if len(md):
        fp = md["node_fixed_packed"].astype(np.int64)
        dfx, gfx, sfx = (fp & 1) != 0, (fp & 2) != 0, (fp & 4) != 0
        for (a_, afx) in (("gate", gfx), ("drain", dfx)):
            vo = _v(x_old, md[a_]) - _v(x_old, md["source"])
            vn = _v(x_new, md[a_]) - _v(x_new, md["source"])
            d = np.abs(vn - vo)
            act = d > MOS_STEP_LIMIT
            s = np.where(act, MOS_STEP_LIMIT / np.where(act, d, 1.0), 1.0)
            propose(md[a_], s, act & ~afx)
            propose(md["source"], s, act & ~sfx)

    damped = scale < 1.0
    out = x_new.copy()
    out[damped] = x_old[damped] + (x_new[damped] - x_old[damped]) * scale[damped]
    return out, scale
