"""The reference's nonlinear end-to-end test circuits and their assertions,
transcribed for the oracle (CPU) and the GPU path.

Test infrastructure only.  Each case cites the reference test it comes from.
The reference runs these through ``analysis::dc::run`` on its GPU backend and
checks physical windows (``tests/transistor_integration_test.rs``,
``tests/diode_integration_test.rs``); its regression suite
(``tests/regression/manifest.toml``) compares four of them with ngspice, which
is not installed here, so for those the expected value is computed in closed
form from the model equations with the reference's constants (VT = 0.02585 V,
GMIN = 1e-12 S, parameters rounded to f32 as the descriptors store them).

Netlist node names map to integer labels by first appearance ("0" is ground),
which reproduces the reference's node numbering.
"""
from __future__ import annotations

import math

import numpy as np


def npn(is_, bf, br=1.0, nf=1.0, nr=1.0):
    return {"is_": is_, "bf": bf, "br": br, "nf": nf, "nr": nr, "npn": True}


def pnp(is_, bf, br=1.0, nf=1.0, nr=1.0):
    return {"is_": is_, "bf": bf, "br": br, "nf": nf, "nr": nr, "npn": False}


def nmos(vto, kp, lam=0.0):
    return {"vto": vto, "kp": kp, "lam": lam, "nmos": True}


def pmos(vto, kp, lam=0.0):
    return {"vto": vto, "kp": kp, "lam": lam, "nmos": False}


def dmod(is_, n=1.0):
    return {"is_": is_, "n": n}


_NMOD = nmos(0.7, 1.1e-4, 0.04)
_PMOD = pmos(-0.7, 5.5e-5, 0.04)


def _chain(n_stages, names):
    comps = [("V", "VDD", ("vdd", "0"), 5.0), ("V", "VIN", ("in", "0"), 5.0)]
    for i in range(n_stages):
        inp = "in" if i == 0 else names(i - 1)
        out = names(i)
        comps.append(("M", f"MP{i}", (out, inp, "vdd"), _PMOD))
        comps.append(("M", f"MN{i}", (out, inp, "0"), _NMOD))
    return comps


def _alternating(names, n):
    def check(v):
        for i in range(n):
            if i % 2 == 0:
                assert v[names(i)] < 1.0, (names(i), v[names(i)])
            else:
                assert v[names(i)] > 4.0, (names(i), v[names(i)])
    return check


# name -> {src, comps, check(v: dict node -> volts), must_converge}
CASES = {
    "npn_common_emitter": {
        "src": "tests/transistor_integration_test.rs:241-272",
        "comps": [("V", "V1", ("vcc", "0"), 5.0), ("V", "V2", ("vb", "0"), 1.0),
                  ("R", "R1", ("vcc", "vc"), 1e3), ("R", "R2", ("vb", "base"), 100e3),
                  ("Q", "Q1", ("vc", "base", "0"), npn(1e-14, 200.0, 2.0, 1.0, 1.0))],
        "check": lambda v: (0.3 < v["base"] < 1.0 or _fail("base", v)) and (v["vc"] < 4.5 or _fail("vc", v)),
    },
    "pnp_basic": {
        "src": "tests/transistor_integration_test.rs:274-298",
        "comps": [("V", "V1", ("vcc", "0"), 5.0), ("V", "V2", ("base", "0"), 4.3),
                  ("R", "R1", ("0", "vc"), 1e3), ("Q", "Q1", ("vc", "base", "vcc"), pnp(1e-14, 100.0))],
        "check": lambda v: 0.0 < v["vc"] < 5.0 or _fail("vc", v),
    },
    "bjt_cutoff": {
        "src": "tests/transistor_integration_test.rs:300-326",
        "comps": [("V", "V1", ("vcc", "0"), 5.0), ("V", "V2", ("base", "0"), 0.0),
                  ("R", "R1", ("vcc", "vc"), 1e3), ("Q", "Q1", ("vc", "base", "0"), npn(1e-14, 200.0))],
        "check": lambda v: (abs(v["base"]) < 0.1 or _fail("base", v)) and (abs(v["vc"] - 5.0) < 0.5 or _fail("vc", v)),
    },
    "nmos_common_source": {
        "src": "tests/transistor_integration_test.rs:328-354",
        "comps": [("V", "V1", ("vdd", "0"), 5.0), ("V", "V2", ("gate", "0"), 2.0),
                  ("R", "R1", ("vdd", "drain"), 1e3), ("M", "M1", ("drain", "gate", "0"), _NMOD)],
        "check": lambda v: 4.0 < v["drain"] < 5.1 or _fail("drain", v),
    },
    "pmos_basic": {
        "src": "tests/transistor_integration_test.rs:356-380",
        "comps": [("V", "V1", ("vdd", "0"), 5.0), ("V", "V2", ("gate", "0"), 3.0),
                  ("R", "R1", ("0", "drain"), 1e3), ("M", "M1", ("drain", "gate", "vdd"), pmos(0.7, 4.5e-5, 0.05))],
        "check": lambda v: 0.0 < v["drain"] < 5.0 or _fail("drain", v),
    },
    "mosfet_cutoff": {
        "src": "tests/transistor_integration_test.rs:382-405",
        "comps": [("V", "V1", ("vdd", "0"), 5.0), ("V", "V2", ("gate", "0"), 0.3),
                  ("R", "R1", ("vdd", "drain"), 1e3), ("M", "M1", ("drain", "gate", "0"), nmos(0.7, 1.1e-4))],
        "check": lambda v: abs(v["drain"] - 5.0) < 0.5 or _fail("drain", v),
    },
    "mixed_diode_bjt_mosfet": {
        "src": "tests/transistor_integration_test.rs:407-448",
        "comps": [("V", "V1", ("vcc", "0"), 5.0), ("R", "R1", ("vcc", "n1"), 1e3),
                  ("D", "D1", ("n1", "n2"), dmod(1e-14, 1.0)), ("R", "R2", ("n2", "n3"), 10e3),
                  ("Q", "Q1", ("vcc", "n2", "n3"), npn(1e-14, 100.0)), ("R", "R3", ("n3", "n4"), 1e3),
                  ("M", "M1", ("n4", "n2", "0"), nmos(0.7, 1e-4))],
        "check": lambda v: all(-0.5 <= x <= 5.5 for x in v.values()) or _fail(None, v),
    },
    "bjt_high_bf_convergence": {
        "src": "tests/transistor_integration_test.rs:450-470",
        "comps": [("V", "V1", ("vcc", "0"), 5.0), ("V", "V2", ("base", "0"), 0.7),
                  ("R", "R1", ("vcc", "vc"), 1e3), ("Q", "Q1", ("vc", "base", "0"), npn(1e-14, 1000.0))],
        "check": lambda v: 0.0 <= v["vc"] <= 5.0 or _fail("vc", v),
    },
    "mosfet_4terminal_syntax": {
        "src": "tests/transistor_integration_test.rs:472-497 (bulk terminal ignored)",
        "comps": [("V", "V1", ("vdd", "0"), 5.0), ("V", "V2", ("gate", "0"), 2.0),
                  ("R", "R1", ("vdd", "drain"), 1e3), ("M", "M1", ("drain", "gate", "0"), nmos(0.7, 1.1e-4))],
        "check": lambda v: 4.0 < v["drain"] < 5.1 or _fail("drain", v),
    },
    "cmos_inverter_dc": {
        "src": "tests/transistor_integration_test.rs:499-517 (must converge)",
        "comps": [("V", "VDD", ("vdd", "0"), 5.0), ("V", "VIN", ("in", "0"), 5.0),
                  ("M", "MP1", ("out", "in", "vdd"), _PMOD), ("M", "MN1", ("out", "in", "0"), _NMOD)],
        "check": lambda v: v["out"] < 0.5 or _fail("out", v),
    },
    "linear_divider": {
        "src": "tests/transistor_integration_test.rs:519-541, tests/diode_integration_test.rs:208-236",
        "comps": [("V", "V1", ("1", "0"), 10.0), ("R", "R1", ("1", "2"), 1e3), ("R", "R2", ("2", "0"), 1e3)],
        "check": lambda v: abs(v["2"] - 5.0) < 1e-6 or _fail("2", v),
    },
    "cmos_inverter_chain_10_dc": {
        "src": "tests/transistor_integration_test.rs:545-599",
        "comps": _chain(10, lambda i: f"n{i}"),
        "check": _alternating(lambda i: f"n{i}", 10),
    },
    "mosfet_at_threshold_bias": {
        "src": "tests/transistor_integration_test.rs:601-626",
        "comps": [("V", "V1", ("vdd", "0"), 5.0), ("V", "V2", ("gate", "0"), 0.7),
                  ("R", "R1", ("vdd", "drain"), 10e3), ("M", "M1", ("drain", "gate", "0"), _NMOD)],
        "check": lambda v: 3.0 < v["drain"] <= 5.01 or _fail("drain", v),
    },
    "mosfet_subthreshold_current": {
        "src": "tests/transistor_integration_test.rs:628-658",
        "comps": [("V", "V1", ("vdd", "0"), 5.0), ("V", "V2", ("gate", "0"), 0.5),
                  ("R", "R1", ("vdd", "drain"), 10e3), ("M", "M1", ("drain", "gate", "0"), _NMOD)],
        "check": lambda v: abs(v["drain"] - 5.0) < 0.5 or _fail("drain", v),
    },
    "diode_resistor_vsource": {
        "src": "tests/diode_integration_test.rs:160-206; tests/regression/circuits/diode_forward.spice",
        "comps": [("V", "V1", ("1", "0"), 5.0), ("R", "R1", ("1", "2"), 1e3),
                  ("D", "D1", ("2", "0"), dmod(1e-14, 1.0))],
        "check": lambda v: ((abs(v["1"] - 5.0) < 0.1 or _fail("1", v))
                            and (0.3 < v["2"] < 1.0 or _fail("2", v))
                            and (0.003 < (v["1"] - v["2"]) / 1000.0 < 0.006 or _fail("i(R1)", v))),
    },
    "cmos_inverter_chain_dc_regression": {
        "src": "tests/regression/circuits/cmos_inverter_chain_dc.spice (stages out_1..out_10)",
        "comps": _chain(10, lambda i: f"out_{i + 1}"),
        "check": _alternating(lambda i: f"out_{i + 1}", 10),
    },
}


def _fail(node, v):
    raise AssertionError(f"window violated at {node}: {v}")


def labels(comps):
    """Netlist node name -> integer label, by first appearance; "0" -> 0."""
    out = {"0": 0}
    for c in comps:
        for nd in c[2]:
            if nd not in out:
                out[nd] = len(out)
    return out


def build(case):
    """Circuit of a case (components in netlist order) and its name -> label map."""
    from tests.golden.known_answers import build_circuit
    lab = labels(case["comps"])
    comps = [(k, name, tuple(lab[nd] for nd in nodes)) + tuple(rest) for (k, name, nodes, *rest) in case["comps"]]
    return build_circuit(comps), lab


def node_voltages(sysm, lab, x):
    """{node name: volts} for every non-ground node of the case."""
    return {name: float(x[sysm.node_index(label)]) for name, label in lab.items() if label != 0}


# ---------------------------------------------------------------------------
# Closed-form values for the regression circuits (tests/regression/manifest.toml)
# ---------------------------------------------------------------------------
VT = 0.02585
GMIN = 1e-12
f32 = lambda x: float(np.float32(x))   # noqa: E731  (descriptor parameters are f32)


def diode_forward_v2():
    """diode_forward.spice: (5 - V)/1k = Is (exp(V / (N VT)) - 1) + GMIN V, by
    bisection on the monotone residual."""
    is_, nvt = f32(1e-14), f32(1.0 * VT)
    f = lambda v: (5.0 - v) / 1e3 - is_ * math.expm1(v / nvt) - GMIN * v   # noqa: E731
    lo, hi = 0.0, 1.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if f(mid) > 0.0:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def nmos_common_source_vd():
    """nmos_common_source.spice: V_GS = 2 V, so the soft overdrive argument
    (V_GS - VTO)/VT = 50 is above 20 and v_eff = V_GS - VTO exactly; the drain
    is in saturation, I_D = KP/2 v_eff^2 (1 + lambda V_D), and
    (5 - V_D)/1k = I_D + GMIN V_D is linear in V_D."""
    kp, vto, lam = f32(1.1e-4), f32(0.7), f32(0.04)
    veff = 2.0 - vto
    a = 0.5 * kp * veff * veff
    # 5e-3 - V/1e3 = a + a lam V + GMIN V  ->  V (1e-3 + a lam + GMIN) = 5e-3 - a
    return (5.0 / 1e3 - a) / (1.0 / 1e3 + a * lam + GMIN)
