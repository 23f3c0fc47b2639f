// Nonlinear device models in FP64: evaluation, Norton-companion stamps and
// voltage-limiting proposals.
//
// Equations follow the reference shaders (src/solver/ds_nonlinear_shaders.rs):
//   diode   eval :40-76,   stamps :128-164 and :211-248
//   BJT     eval :280-367, stamps :393-453 and :478-573, limiting :600-714
//   MOSFET  eval :746-849, stamps :873-911 and :932-996, limiting :1051-1130
//   diode   limiting (modified pnjlim) :1173-1234
// evaluated in FP64 instead of double-single, with these fixed choices:
//   * floating-diode matrix stamps +g at (a,a),(c,c) and -g at (a,c),(c,a) in
//     the compiler's slot order [aa, cc, ac, ca] (src/compiler.rs:625-631);
//   * the MOSFET soft-overdrive middle region in FP64 with log1p(exp(arg));
//   * limiting decisions in FP64; each device proposes a damping factor per
//     terminal node and every node keeps the smallest proposal (deterministic
//     where the reference's unsynchronised read-modify-writes race);
//   * optional BJT Early voltage (VAF = +inf reproduces the reference).
#pragma once

#include <cstdint>

#include "common.cuh"

namespace ohm {

struct DiodeDesc {      // GpuDiodeDescriptor, 48 B (src/compiler.rs:52-73)
    uint32_t anode, cathode;
    float is_val, n_vt;
    uint32_t g_row_col[4];
    uint32_t b_idx[2];
    uint32_t pad[2];
};
struct BjtDesc {        // GpuBjtDescriptor, 96 B (src/compiler.rs:79-113)
    uint32_t collector, base, emitter;
    float polarity, is_val, bf, br, nf_vt, nr_vt;
    uint32_t node_fixed[3];
    uint32_t g_row_col[9];
    uint32_t b_idx[3];
};
struct MosfetDesc {     // GpuMosfetDescriptor, 64 B (src/compiler.rs:119-149)
    uint32_t drain, gate, source;
    float polarity, vto, kp, lambda;
    uint32_t node_fixed_packed;
    uint32_t g_row_col[6];
    uint32_t b_idx[2];
};
static_assert(sizeof(DiodeDesc) == 48, "diode descriptor layout");
static_assert(sizeof(BjtDesc) == 96, "bjt descriptor layout");
static_assert(sizeof(MosfetDesc) == 64, "mosfet descriptor layout");

// f32 shader constant `let VT: f32 = 0.02585;` promoted to f64.
constexpr double kVtMos = (double)0.02585f;
constexpr double kMosStepLimit = 0.5;

__device__ __forceinline__ double node_v(const double *x, uint32_t idx) {
    return idx == kSentinel ? 0.0 : x[idx];
}

__device__ __forceinline__ double clamp_exp(double a) {
    return exp(fmin(fmax(a, -80.0), 80.0));
}

// Stamp-value layout per device (matrix slots, then rhs rows):
//   diode  : 4 matrix [aa, cc, ac, ca],          2 rhs [a, c]
//   BJT    : 9 matrix [CC..EE],                  3 rhs [C, B, E]
//   MOSFET : 6 matrix [DD, DG, DS, SD, SG, SS],  2 rhs [D, S]
__device__ __forceinline__ void diode_stamps(const DiodeDesc &d, const double *x, double *ms,
                                             double *rs) {
    const double is_ = (double)d.is_val, nvt = (double)d.n_vt;
    const double v = node_v(x, d.anode) - node_v(x, d.cathode);
    const double e = clamp_exp(v / nvt);
    const double i_d = is_ * (e - 1.0);
    const double g = is_ * e / nvt;
    const double ieq = i_d - g * v;
    ms[0] = g; ms[1] = g; ms[2] = -g; ms[3] = -g;
    rs[0] = -ieq; rs[1] = ieq;
}

__device__ __forceinline__ void bjt_stamps(const BjtDesc &q, double vaf, const double *x,
                                           double *ms, double *rs) {
    const double pol = (double)q.polarity, is_ = (double)q.is_val;
    const double bf = (double)q.bf, br = (double)q.br;
    const double nf = (double)q.nf_vt, nr = (double)q.nr_vt;
    const double vc = node_v(x, q.collector), vb = node_v(x, q.base), ve = node_v(x, q.emitter);
    const double vbe = pol * (vb - ve), vbc = pol * (vb - vc);
    const double ef = clamp_exp(vbe / nf), er = clamp_exp(vbc / nr);
    const double i_f = is_ * (ef - 1.0), i_r = is_ * (er - 1.0);
    const double bf_frac = bf / (bf + 1.0), br1 = br + 1.0;
    double ic = bf_frac * i_f - i_r / br1;
    const double ib = i_f / (bf + 1.0) + i_r / br1;
    const double gf = is_ * ef / nf, gr = is_ * er / nr;
    double a = bf_frac * gf;            // dIc/dVbe
    double b = -(gr / br1);             // dIc/dVbc
    const double c = gf / (bf + 1.0);   // dIb/dVbe
    const double dd = gr / br1;         // dIb/dVbc
    if (isfinite(vaf)) {                // Early effect extension
        const double inv = 1.0 / vaf;
        const double k = 1.0 + (vbe - vbc) * inv;
        const double ict = bf_frac * i_f;
        ic = ict * k - i_r / br1;
        a = a * k + ict * inv;
        b = b - ict * inv;
    }
    ic *= pol;
    const double ibp = pol * ib;
    const double g_cc = -b, g_cb = a + b, g_ce = -a;
    const double g_bc = -dd, g_bb = c + dd, g_be = -c;
    const double g_ec = b + dd, g_eb = -(((a + b) + c) + dd), g_ee = a + c;
    ms[0] = g_cc; ms[1] = g_cb; ms[2] = g_ce;
    ms[3] = g_bc; ms[4] = g_bb; ms[5] = g_be;
    ms[6] = g_ec; ms[7] = g_eb; ms[8] = g_ee;
    const double ie = -(ic + ibp);
    const double ilc = (g_cc * vc + g_cb * vb) + g_ce * ve;
    const double ilb = (g_bc * vc + g_bb * vb) + g_be * ve;
    const double ile = (g_ec * vc + g_eb * vb) + g_ee * ve;
    rs[0] = -(ic - ilc); rs[1] = -(ibp - ilb); rs[2] = -(ie - ile);
}

// MOSFET drain current at x (ds_nonlinear_shaders.rs:746-849): i_d with the
// polarity applied, g_m = dI/dV_GS and g_ds = dI/dV_DS (polarity-free), and
// i_per_kp = i_d / KP (the current is linear in KP), plus the terminal
// voltages.  d i_d / d|VTO| = -polarity * g_m.
struct MosEval {
    double i_d, gm, gds, i_per_kp, vd, vg, vs;
};

__device__ __forceinline__ MosEval mosfet_eval(const MosfetDesc &m, const double *x) {
    const double pol = (double)m.polarity, vto = (double)m.vto;
    const double kp = (double)m.kp, lam = (double)m.lambda;
    const double vd = node_v(x, m.drain), vg = node_v(x, m.gate), vs = node_v(x, m.source);
    const double vgs = pol * (vg - vs), vds = pol * (vd - vs);
    const double v_ov = vgs - vto;
    const double arg = v_ov / kVtMos;
    double veff, sig;
    if (arg > 20.0) {
        veff = v_ov; sig = 1.0;
    } else if (arg < -20.0) {
        const double e = clamp_exp(arg);
        veff = kVtMos * e; sig = e;
    } else {
        veff = kVtMos * log1p(exp(arg));
        sig = 1.0 / (1.0 + exp(-arg));
    }
    const double lamf = 1.0 + lam * vds;
    double i_d, gm, gds, ipk;
    if (vds < veff) {                      // linear region
        const double inner = veff * vds - 0.5 * (vds * vds);
        const double kp_inner = kp * inner;
        i_d = kp_inner * lamf;
        gm = (kp * vds) * lamf * sig;
        gds = (kp * (veff - vds)) * lamf + kp_inner * lam;
        ipk = inner * lamf;
    } else {                               // saturation
        const double kh_vov2 = (kp / 2.0) * (veff * veff);
        i_d = kh_vov2 * lamf;
        gm = (kp * veff) * lamf * sig;
        gds = kh_vov2 * lam;
        ipk = 0.5 * (veff * veff) * lamf;
    }
    return MosEval{i_d * pol, gm, gds, ipk * pol, vd, vg, vs};
}

__device__ __forceinline__ void mosfet_stamps(const MosfetDesc &m, const double *x, double *ms,
                                              double *rs) {
    const MosEval ev = mosfet_eval(m, x);
    const double i_d = ev.i_d, gm = ev.gm, gds = ev.gds, vd = ev.vd, vg = ev.vg, vs = ev.vs;
    const double s = gm + gds;
    ms[0] = gds; ms[1] = gm; ms[2] = -s; ms[3] = -gds; ms[4] = -gm; ms[5] = s;
    const double ild = (gds * vd + gm * vg) + (-s) * vs;
    const double ils = ((-gds) * vd + (-gm) * vg) + s * vs;
    rs[0] = -(i_d - ild);
    rs[1] = -((-i_d) - ils);
}

// Modified SPICE3f5 pnjlim (ds_nonlinear_shaders.rs:1173-1187) in FP64.
__device__ __forceinline__ double pnjlim(double vnew, double vold, double vt, double vcrit) {
    if (vnew > vcrit && fabs(vnew - vold) > vt + vt) {
        if (vold > 0.0) {
            const double arg = 1.0 + (vnew - vold) / vt;
            if (arg > 0.0) return vold + vt * (2.0 + log(arg - 2.0));
            return vcrit;
        }
        return vt * log(vnew / vt);
    }
    return vnew;
}

// Node damping factors are kept as the bit patterns of non-negative doubles,
// whose unsigned order equals their numeric order, so atomicMin gives the
// smallest proposal independent of arrival order.
__device__ __forceinline__ void propose_scale(unsigned long long *scale, uint32_t node, double s) {
    if (node == kSentinel) return;
    if (!(s < 1.0)) return;              // proposals >= 1 (or NaN) never damp
    s = fmax(s, 0.0);
    atomicMin(&scale[node], (unsigned long long)__double_as_longlong(s));
}

__device__ __forceinline__ double junction_scale(double vnew, double vold, double vt,
                                                 double vcrit, bool *active) {
    const double vl = pnjlim(vnew, vold, vt, vcrit);
    const double dlt = vnew - vold;
    *active = (vl != vnew) && (fabs(dlt) > 1e-30);
    return *active ? (vl - vold) / dlt : 1.0;
}

__device__ __forceinline__ void diode_limit(const DiodeDesc &d, const double *xo, const double *xn,
                                            unsigned long long *scale) {
    const double is_ = (double)d.is_val, nvt = (double)d.n_vt;
    const double vcrit = nvt * log(nvt / (1.4142135623730951 * is_));
    const double vo = node_v(xo, d.anode) - node_v(xo, d.cathode);
    const double vn = node_v(xn, d.anode) - node_v(xn, d.cathode);
    bool act;
    const double s = junction_scale(vn, vo, nvt, vcrit, &act);
    if (act) {
        propose_scale(scale, d.anode, s);
        propose_scale(scale, d.cathode, s);
    }
}

__device__ __forceinline__ void bjt_limit(const BjtDesc &q, const double *xo, const double *xn,
                                          unsigned long long *scale) {
    const double pol = (double)q.polarity, is_ = (double)q.is_val;
    const double nf = (double)q.nf_vt, nr = (double)q.nr_vt;
    {
        const double vcrit = nf * log(nf / (1.4142135623730951 * is_));
        const double vo = pol * (node_v(xo, q.base) - node_v(xo, q.emitter));
        const double vn = pol * (node_v(xn, q.base) - node_v(xn, q.emitter));
        bool act;
        const double s = junction_scale(vn, vo, nf, vcrit, &act);
        if (act) {
            if (!q.node_fixed[1]) propose_scale(scale, q.base, s);
            if (!q.node_fixed[2]) propose_scale(scale, q.emitter, s);
        }
    }
    {
        const double vcrit = nr * log(nr / (1.4142135623730951 * is_));
        const double vo = pol * (node_v(xo, q.base) - node_v(xo, q.collector));
        const double vn = pol * (node_v(xn, q.base) - node_v(xn, q.collector));
        bool act;
        const double s = junction_scale(vn, vo, nr, vcrit, &act);
        if (act) {
            if (!q.node_fixed[1]) propose_scale(scale, q.base, s);
            if (!q.node_fixed[0]) propose_scale(scale, q.collector, s);
        }
    }
}

__device__ __forceinline__ void mosfet_limit(const MosfetDesc &m, const double *xo,
                                             const double *xn, unsigned long long *scale) {
    const uint32_t f = m.node_fixed_packed;
    const bool dfx = f & 1u, gfx = f & 2u, sfx = f & 4u;
    {
        const double vo = node_v(xo, m.gate) - node_v(xo, m.source);
        const double vn = node_v(xn, m.gate) - node_v(xn, m.source);
        const double d = fabs(vn - vo);
        if (d > kMosStepLimit) {
            const double s = kMosStepLimit / d;
            if (!gfx) propose_scale(scale, m.gate, s);
            if (!sfx) propose_scale(scale, m.source, s);
        }
    }
    {
        const double vo = node_v(xo, m.drain) - node_v(xo, m.source);
        const double vn = node_v(xn, m.drain) - node_v(xn, m.source);
        const double d = fabs(vn - vo);
        if (d > kMosStepLimit) {
            const double s = kMosStepLimit / d;
            if (!dfx) propose_scale(scale, m.drain, s);
            if (!sfx) propose_scale(scale, m.source, s);
        }
    }
}

}  // namespace ohm
