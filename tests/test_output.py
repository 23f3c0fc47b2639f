"""CPU: CSV output in the reference's format (src/output.rs:16-93), with the
reference's CSV tests (tests/integration_test.rs:220-313) ported onto oracle
solutions, and Rust's f64 Display rules for the numbers."""
import io
import math

import numpy as np
import pytest

from oracle import ac_ref, newton_ref
from oracle import transient_ref as tref
from ohmnivore_b200 import circuits as ck
from ohmnivore_b200 import mna
from ohmnivore_b200.output import fmt, write_ac_csv, write_dc_csv, write_tran_csv
from ohmnivore_b200.solver import ac_frequencies


@pytest.mark.parametrize("x, s", [
    (5.0, "5"), (3.3, "3.3"), (0.001, "0.001"), (-0.005, "-0.005"), (1e-9, "0.000000001"),
    (2.5e-12, "0.0000000000025"), (1e21, "1000000000000000000000"), (-0.0, "-0"), (0.0, "0"),
    (0.1 + 0.2, "0.30000000000000004"), (123456789.125, "123456789.125"), (float("nan"), "NaN"),
    (float("inf"), "inf"), (float("-inf"), "-inf")])
def test_rust_float_display(x, s):
    assert fmt(x) == s


def test_display_round_trips():
    rng = np.random.default_rng(0)
    xs = np.concatenate([rng.standard_normal(500) * 10.0 ** rng.integers(-30, 30, 500),
                         rng.uniform(-1, 1, 100)])
    for x in xs:
        s = fmt(x)
        assert "e" not in s and float(s) == x


def _divider():
    b = ck.CircuitBuilder()
    b.vsource(1, 0, dc=10.0, name="V1")
    b.resistors([1, 2], [2, 0], [1e3, 1e3], names=["R1", "R2"])
    return b.build()


def test_dc_csv_output():
    """integration_test.rs:220-243."""
    ckt = _divider()
    s = mna.compile_circuit(ckt)
    x, _ = newton_ref.dc_operating_point(s)
    buf = io.StringIO()
    write_dc_csv(ckt, s, x, buf)
    csv = buf.getvalue()
    assert csv.startswith("Variable,Value\n")
    assert "V(1)," in csv and "V(2)," in csv and "I(V1)," in csv
    rows = dict(line.split(",") for line in csv.strip().splitlines()[1:])
    assert rows["V(1)"] == "10" and abs(float(rows["V(2)"]) - 5.0) < 1e-6
    assert float(rows["I(V1)"]) == x[s.n_nodes]


def test_ac_csv_output():
    """integration_test.rs:245-283: header + 3 rows, magnitude and phase
    columns, the same number of columns in every row."""
    b = ck.CircuitBuilder()
    b.vsource(1, 0, dc=None, ac=(1.0, 0.0), name="V1")
    b.resistors([1], [2], [1e3])
    b.capacitors([2], [0], [1e-6])
    ckt = b.build()
    s = mna.compile_circuit(ckt)
    freqs = ac_frequencies("lin", 3, 100.0, 1000.0)
    xs = ac_ref.ac_sweep(s, freqs)
    buf = io.StringIO()
    write_ac_csv(ckt, s, freqs, xs, buf)
    lines = buf.getvalue().splitlines()
    assert len(lines) == 4
    assert lines[0].startswith("Frequency") and "_mag" in lines[0] and "_phase_deg" in lines[0]
    assert all(line.count(",") == lines[0].count(",") for line in lines[1:])
    # V(2) of an RC low-pass: |H| = 1 / sqrt(1 + (w R C)^2), phase -atan(w R C)
    cols = lines[0].split(",")
    row = lines[2].split(",")
    w = 2 * math.pi * float(row[0])
    assert abs(float(row[cols.index("V(2)_mag")]) - 1 / math.hypot(1.0, w * 1e-3)) < 1e-9
    assert abs(float(row[cols.index("V(2)_phase_deg")]) + math.degrees(math.atan(w * 1e-3))) < 1e-7


def test_tran_csv_output():
    b = ck.CircuitBuilder()
    b.vsource(1, 0, dc=5.0, name="V1")
    b.resistors([1], [2], [1e3])
    b.capacitors([2], [0], [1e-6])
    ckt = b.build()
    s = mna.compile_circuit(ckt)
    x0 = tref.uic_initial_conditions(s, ckt)
    times, wave, _ = tref.adaptive_transient(s, x0, 100e-6, 1e-3, 0.0, list(range(s.size)))
    buf = io.StringIO()
    write_tran_csv(ckt, s, times, wave, buf)
    lines = buf.getvalue().splitlines()
    assert lines[0] == "time,V(1),V(2),I(V1)"
    assert len(lines) == len(times) + 1
    assert lines[1].split(",")[0] == "0" and float(lines[-1].split(",")[0]) == times[-1]
    np.testing.assert_array_equal(np.array([[float(v) for v in ln.split(",")[1:]] for ln in lines[1:]]), wave)
