"""CPU: the oracle's adaptive BE / TRAP transient (transient.rs:77-178) and
UIC initial conditions (:364-482) pinned by the reference's own known
answers (tests/transient_integration_test.rs), and the host UIC system of
the library checked against the oracle's."""
import math

import numpy as np
import pytest

from oracle import newton_ref
from oracle import transient_ref as tref
from oracle.linear_ref import sparse_lu_solve
from ohmnivore_b200 import circuits as ck
from ohmnivore_b200 import mna


def rc_charging():
    """transient_integration_test.rs:52-87: V1 5 V, R 1k, C 1u, .TRAN 10u 5m UIC."""
    b = ck.CircuitBuilder()
    b.vsource(1, 0, dc=5.0, name="V1")
    b.resistors([1], [2], [1e3])
    b.capacitors([2], [0], [1e-6])
    return b.build(), 10e-6, 5e-3, True


def rl_step():
    """:89-132: V1 5 V, R 100, L 10m, .TRAN 1u 500u UIC."""
    b = ck.CircuitBuilder()
    b.vsource(1, 0, dc=5.0, name="V1")
    b.resistors([1], [2], [100.0])
    b.inductors([2], [0], [10e-3], names=["L1"])
    return b.build(), 1e-6, 500e-6, True


def lc_oscillation():
    """:134-161: V1 5 V, L 1m, C 1u, .TRAN 1u 200u (DC start)."""
    b = ck.CircuitBuilder()
    b.vsource(1, 0, dc=5.0, name="V1")
    b.inductors([1], [2], [1e-3])
    b.capacitors([2], [0], [1e-6])
    return b.build(), 1e-6, 200e-6, False


def pulse_rc():
    """:163-194: PULSE(0 5 0 0 0 50u 100u), R 1k, C 100n, .TRAN 1u 200u."""
    b = ck.CircuitBuilder()
    b.vsource(1, 0, dc=0.0, name="V1", tran=(ck.TRAN_PULSE, (0.0, 5.0, 0.0, 0.0, 0.0, 50e-6, 100e-6)))
    b.resistors([1], [2], [1e3])
    b.capacitors([2], [0], [100e-9])
    return b.build(), 1e-6, 200e-6, False


def sin_source():
    """:196-219: SIN(0 1 10k) across R 1k, .TRAN 1u 200u."""
    b = ck.CircuitBuilder()
    b.vsource(1, 0, dc=0.0, name="V1", tran=(ck.TRAN_SIN, (0.0, 1.0, 10e3, 0.0, 0.0)))
    b.resistors([1], [0], [1e3])
    return b.build(), 1e-6, 200e-6, False


CASES = {"rc_charging": rc_charging, "rl_step": rl_step, "lc_oscillation": lc_oscillation,
         "pulse_rc": pulse_rc, "sin_source": sin_source}


def start(ckt, s, uic):
    return tref.uic_initial_conditions(s, ckt) if uic else newton_ref.dc_operating_point(s)[0]


def run(name):
    ckt, tstep, tstop, uic = CASES[name]()
    s = mna.compile_circuit(ckt)
    x0 = start(ckt, s, uic)
    probes = list(range(s.size))
    times, wave, stats = tref.adaptive_transient(s, x0, tstep, tstop, 0.0, probes)
    return ckt, s, times, wave, stats


def test_rc_charging_known_answer():
    _, s, times, wave, stats = run("rc_charging")
    v = wave[:, s.node_index(2)]
    for t, vt in zip(times, v):
        if t > 0.0:
            assert abs(vt - 5.0 * (1.0 - math.exp(-t / 1e-3))) < 0.02 * 5.0 + 1e-6
    assert times[-1] == pytest.approx(5e-3, rel=1e-12)
    assert stats["accepted"] >= 500               # h never exceeds tstep


def test_rl_step_known_answer():
    ckt, s, times, wave, _ = run("rl_step")
    k = s.n_nodes + list(s.branch_components).index(ckt.names.index("L1"))
    for t, i in zip(times, wave[:, k]):
        if t > 1e-6:
            assert abs(i - 5.0 / 100.0 * (1.0 - math.exp(-t / 1e-4))) < 0.02 * (5.0 / 100.0) + 1e-6


def test_lc_oscillation_known_answer():
    _, s, times, wave, _ = run("lc_oscillation")
    assert np.max(wave[:, s.node_index(2)]) > 4.9
    assert len(times) > 10


def test_pulse_rc_known_answer():
    _, s, times, wave, _ = run("pulse_rc")
    assert len(times) > 10
    k = int(np.flatnonzero(times >= 25e-6)[0])
    assert 0.5 < wave[k, s.node_index(2)] < 5.0


def test_sin_source_known_answer():
    _, s, times, wave, _ = run("sin_source")
    for t, v in zip(times, wave[:, s.node_index(1)]):
        assert abs(v - math.sin(2.0 * math.pi * 10e3 * t)) < 0.05


def test_step_control_rejects_and_recovers():
    """A sharp PULSE edge inside a step: LTE > 1e-3 rejects the TRAP step,
    the retry is BE with the reduced h (transient.rs:126-146)."""
    b = ck.CircuitBuilder()
    b.vsource(1, 0, dc=0.0, name="V1", tran=(ck.TRAN_PULSE, (0.0, 5.0, 30e-6, 1e-9, 1e-9, 50e-6, 200e-6)))
    b.resistors([1], [2], [1e3])
    b.capacitors([2], [0], [10e-9])
    s = mna.compile_circuit(b.build())
    x0 = newton_ref.dc_operating_point(s)[0]
    times, _, stats = tref.adaptive_transient(s, x0, 10e-6, 100e-6, 0.0, [0, 1])
    assert stats["rejected"] >= 1
    # two solves per TRAP attempt, one per BE-only step (the first, and one
    # after each rejection)
    n_be = 1 + stats["rejected"]
    assert stats["linear_solves"] == 2 * (stats["accepted"] - n_be + stats["rejected"]) + n_be
    assert np.all(np.diff(times) > 0)


def test_tstart_skips_early_points():
    ckt, tstep, tstop, uic = CASES["rc_charging"]()
    s = mna.compile_circuit(ckt)
    x0 = start(ckt, s, uic)
    times, wave, _ = tref.adaptive_transient(s, x0, 100e-6, 1e-3, 0.5e-3, [1])
    assert times[0] >= 0.5e-3 and len(times) == len(wave)


@pytest.mark.parametrize("name", ["rc_charging", "rl_step"])
def test_host_uic_system_matches_oracle(name):
    """The library's UIC system (host logic) solved by LU equals the
    oracle's UIC start: V(C) = 0, I_L = 0, sources satisfied."""
    ckt, _, _, _ = CASES[name]()
    s = mna.compile_circuit(ckt)
    vals, b = mna.uic_system(ckt, s)
    x = sparse_lu_solve(s.size, s.g.row_ptr, s.g.col, vals, b)
    ref = tref.uic_initial_conditions(s, ckt)
    np.testing.assert_allclose(x, ref, rtol=0, atol=1e-15)
    assert x[s.node_index(1)] == pytest.approx(5.0)


def test_uic_two_terminal_capacitor_chain():
    """Capacitors between two non-ground nodes: the first unconstrained
    terminal row takes V(i) - V(j) = 0; a node is constrained once."""
    b = ck.CircuitBuilder()
    b.vsource(1, 0, dc=2.0, name="V1")
    b.resistors([1, 2, 3], [2, 3, 0], [1e3, 2e3, 3e3])
    b.capacitors([2, 3, 2], [3, 0, 3], [1e-9, 1e-9, 2e-9])   # the third finds both rows taken
    ckt = b.build()
    s = mna.compile_circuit(ckt)
    vals, rhs = mna.uic_system(ckt, s)
    x = sparse_lu_solve(s.size, s.g.row_ptr, s.g.col, vals, rhs)
    ref = tref.uic_initial_conditions(s, ckt)
    np.testing.assert_allclose(x, ref, rtol=0, atol=1e-15)
    assert x[s.node_index(3)] == 0.0 and x[s.node_index(2)] == pytest.approx(x[s.node_index(3)], abs=1e-15)
