"""The reference's nonlinear end-to-end tests on the oracle (CPU): the
compile round trips of tests/transistor_integration_test.rs and
tests/diode_integration_test.rs (descriptor fields and sentinels), the DC
windows of their GPU end-to-end tests (the oracle's FP64 Newton with a
sparse LU per iteration must land inside every window), and the closed-form
values of the regression circuits (tests/regression/manifest.toml).

These pin the oracle's diode, BJT and MOSFET equations and its Newton loop to
answers the reference itself asserts; the GPU path is checked against the
oracle on the same circuits in test_gpu_reference_circuits.py.
"""
import numpy as np
import pytest

from oracle import newton_ref
from ohmnivore_b200 import mna
from tests.golden import reference_circuits as RC
from tests.golden.known_answers import build_circuit

SENT = mna.SENTINEL
f32 = RC.f32


def _compile(comps):
    lab = RC.labels(comps)
    cc = [(k, name, tuple(lab[nd] for nd in nodes)) + tuple(rest) for (k, name, nodes, *rest) in comps]
    return mna.compile_circuit(build_circuit(cc)), lab


def oracle_dc(sysm, stages=None):
    """The oracle's DC operating point by the reference's strategy (direct
    Newton, source stepping for MOSFET circuits, GMIN stepping, pseudo-transient)."""
    return newton_ref.run_nonlinear(sysm, stages=stages)


@pytest.mark.parametrize("name", sorted(RC.CASES))
def test_oracle_within_reference_windows(name):
    case = RC.CASES[name]
    ckt, lab = RC.build(case)
    sysm = mna.compile_circuit(ckt)
    x = oracle_dc(sysm)
    v = RC.node_voltages(sysm, lab, x)
    case["check"](v)
    # the operating point satisfies KCL in FP64
    r = newton_ref.residual(sysm, x)
    assert np.max(np.abs(r)) < 1e-12 * max(1.0, np.max(np.abs(sysm.b_dc)))


def test_regression_diode_forward_closed_form():
    """tests/regression/circuits/diode_forward.spice, V(2)."""
    sysm, lab = _compile(RC.CASES["diode_resistor_vsource"]["comps"])
    x = oracle_dc(sysm)
    v2 = x[sysm.node_index(lab["2"])]
    ref = RC.diode_forward_v2()
    assert abs(v2 - ref) < 1e-9 * abs(ref)
    # the manifest's tolerance against ngspice (5 % / 10 mV) holds for the
    # closed form at the reference's VT; ngspice itself is not installed
    assert 0.6 < ref < 0.75


def test_regression_nmos_common_source_closed_form():
    """tests/regression/circuits/nmos_common_source.spice, V(drain)."""
    sysm, lab = _compile(RC.CASES["nmos_common_source"]["comps"])
    x = oracle_dc(sysm)
    vd = x[sysm.node_index(lab["drain"])]
    ref = RC.nmos_common_source_vd()
    assert abs(vd - ref) < 1e-9 * abs(ref)
    assert 4.85 < ref < 4.95            # ~93 uA through 1k (transistor_integration_test.rs:346-352)


# ---- compile round trips (parse -> compile -> descriptors) ----

def test_bjt_compile_descriptor():
    """transistor_integration_test.rs:131-170."""
    sysm, _ = _compile([("V", "V1", ("vcc", "0"), 5.0), ("R", "R1", ("vcc", "vc"), 1e3),
                        ("Q", "Q1", ("vc", "base", "0"), RC.npn(1e-14, 200.0, 2.0, 1.0, 1.0))])
    assert len(sysm.bjt_descriptors) == 1
    d = sysm.bjt_descriptors[0]
    assert abs(d["polarity"] - 1.0) < 1e-6
    assert abs(float(d["is_val"]) - f32(1e-14)) < 1e-20
    assert abs(d["bf"] - 200.0) < 1e-3 and abs(d["br"] - 2.0) < 1e-3
    assert abs(float(d["nf_vt"]) - f32(1.0 * 0.02585)) < 1e-5
    assert abs(float(d["nr_vt"]) - f32(1.0 * 0.02585)) < 1e-5
    assert d["emitter"] == SENT and d["collector"] != SENT and d["base"] != SENT
    assert len(sysm.diode_descriptors) == 0 and len(sysm.mosfet_descriptors) == 0


def test_mosfet_compile_descriptor():
    """transistor_integration_test.rs:172-205."""
    sysm, _ = _compile([("V", "V1", ("vdd", "0"), 5.0), ("R", "R1", ("vdd", "drain"), 1e3),
                        ("M", "M1", ("drain", "gate", "0"), RC.nmos(0.7, 1.1e-4, 0.04))])
    assert len(sysm.mosfet_descriptors) == 1
    d = sysm.mosfet_descriptors[0]
    assert abs(d["polarity"] - 1.0) < 1e-6
    assert abs(d["vto"] - 0.7) < 1e-5 and abs(float(d["kp"]) - 1.1e-4) < 1e-10 and abs(d["lam"] - 0.04) < 1e-5
    assert d["source"] == SENT and d["drain"] != SENT and d["gate"] != SENT
    assert len(sysm.diode_descriptors) == 0 and len(sysm.bjt_descriptors) == 0


def test_mixed_devices_compile():
    """transistor_integration_test.rs:207-237 and :407-424."""
    for comps in ([("V", "V1", ("vcc", "0"), 5.0), ("R", "R1", ("vcc", "n1"), 1e3),
                   ("D", "D1", ("n1", "0"), RC.dmod(1e-14)), ("R", "R2", ("vcc", "n2"), 1e3),
                   ("Q", "Q1", ("n2", "n1", "0"), RC.npn(1e-14, 100.0)), ("R", "R3", ("vcc", "n3"), 1e3),
                   ("M", "M1", ("n3", "n1", "0"), RC.nmos(0.7, 1e-4))],
                  RC.CASES["mixed_diode_bjt_mosfet"]["comps"]):
        sysm, _ = _compile(comps)
        assert (len(sysm.diode_descriptors), len(sysm.bjt_descriptors), len(sysm.mosfet_descriptors)) == (1, 1, 1)


def test_diode_compile_descriptor():
    """diode_integration_test.rs:10-34: anode is node "2" (index 1), cathode ground."""
    sysm, _ = _compile([("V", "V1", ("1", "0"), 5.0), ("R", "R1", ("1", "2"), 1e3),
                        ("D", "D1", ("2", "0"), RC.dmod(2.52e-9, 1.752))])
    assert len(sysm.diode_descriptors) == 1
    d = sysm.diode_descriptors[0]
    assert d["anode"] == 1 and d["cathode"] == SENT
    assert abs(float(d["is_val"]) - f32(2.52e-9)) < 1e-15
    assert abs(float(d["n_vt"]) - f32(1.752 * 0.02585)) < 1e-5


def test_diodes_to_ground_and_floating_compile():
    """diode_integration_test.rs:36-53 (two diodes to ground) and :55-84 (a
    diode between two non-ground nodes has all four matrix slots)."""
    sysm, _ = _compile([("V", "V1", ("1", "0"), 5.0), ("R", "R1", ("1", "2"), 1e3), ("R", "R2", ("2", "3"), 1e3),
                        ("D", "D1", ("2", "0"), RC.dmod(1e-14)), ("D", "D2", ("3", "0"), RC.dmod(1e-14))])
    assert len(sysm.diode_descriptors) == 2
    assert all(d["cathode"] == SENT for d in sysm.diode_descriptors)
    sysm, _ = _compile([("V", "V1", ("1", "0"), 5.0), ("R", "R1", ("1", "2"), 1e3), ("R", "R2", ("3", "0"), 1e3),
                        ("D", "D1", ("2", "3"), RC.dmod(1e-14))])
    d = sysm.diode_descriptors[0]
    assert d["anode"] != SENT and d["cathode"] != SENT
    assert all(int(s) != SENT for s in d["g_row_col"])
