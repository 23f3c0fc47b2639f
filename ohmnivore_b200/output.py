"""CSV output of DC, AC and transient results in the reference's format
(``src/output.rs:16-93``), so that files written from this library's results
compare byte for byte with the reference CLI's.

Columns: nodes in matrix order as ``V(name)``, then branch currents as
``I(component)`` (V sources and inductors in component order).  Numbers are
written as Rust's ``{}`` formats an ``f64``: the shortest decimal that reads
back to the same double, in positional notation (never an exponent), ``5``
for 5.0, ``-0`` for -0.0, ``NaN``, ``inf``, ``-inf``.  AC entries are the
magnitude (``hypot``) and the phase in degrees (``atan2`` times 180 / pi, the
constant of Rust's ``to_degrees``).
"""
from __future__ import annotations

import io
import math

import numpy as np

from . import circuits as ck


def fmt(x: float) -> str:
    """Rust's ``Display`` of an ``f64``."""
    x = float(x)
    if math.isnan(x):
        return "NaN"
    if math.isinf(x):
        return "inf" if x > 0 else "-inf"
    return np.format_float_positional(x, unique=True, trim="-")


def names(ckt: ck.Circuit, sysm) -> tuple[list[str], list[str]]:
    """Node names in matrix order and branch (component) names in branch order."""
    nodes = [str(int(lbl)) for lbl in sysm.node_labels]
    if ckt.names is not None:
        branches = [str(ckt.names[int(c)]) for c in sysm.branch_components]
    else:
        branches = [f"{ck.KIND_NAMES[int(ckt.kind[c])]}{int(c)}" for c in sysm.branch_components]
    return nodes, branches


def write_dc_csv(ckt: ck.Circuit, sysm, x, out: io.TextIOBase) -> None:
    """write_dc_csv (output.rs:16-25): ``Variable,Value`` then one row per
    node voltage and branch current."""
    nodes, branches = names(ckt, sysm)
    x = np.asarray(x, dtype=np.float64)
    out.write("Variable,Value\n")
    for k, n in enumerate(nodes):
        out.write(f"V({n}),{fmt(x[k])}\n")
    for k, b in enumerate(branches):
        out.write(f"I({b}),{fmt(x[sysm.n_nodes + k])}\n")


def write_ac_csv(ckt: ck.Circuit, sysm, freqs, xs, out: io.TextIOBase) -> None:
    """write_ac_csv (output.rs:36-62): ``Frequency`` then magnitude and phase
    (degrees) of every node voltage and branch current, one row per point.
    ``xs``: n_freq x size complex (the AC sweep's solutions)."""
    nodes, branches = names(ckt, sysm)
    xs = np.asarray(xs, dtype=np.complex128)
    out.write("Frequency")
    for n in nodes:
        out.write(f",V({n})_mag,V({n})_phase_deg")
    for b in branches:
        out.write(f",I({b})_mag,I({b})_phase_deg")
    out.write("\n")
    to_deg = 180.0 / math.pi
    for fi, f in enumerate(freqs):
        row = xs[fi]
        out.write(fmt(f))
        for k in range(sysm.size):
            z = row[k]
            out.write(f",{fmt(np.hypot(z.real, z.imag))},{fmt(math.atan2(z.imag, z.real) * to_deg)}")
        out.write("\n")


def write_tran_csv(ckt: ck.Circuit, sysm, times, states, out: io.TextIOBase) -> None:
    """write_tran_csv (output.rs:72-93): ``time`` then every node voltage and
    branch current, one row per output point.  ``states``: n_points x size
    (e.g. the waveforms of a transient run probing every row)."""
    nodes, branches = names(ckt, sysm)
    states = np.asarray(states, dtype=np.float64)
    out.write("time")
    for n in nodes:
        out.write(f",V({n})")
    for b in branches:
        out.write(f",I({b})")
    out.write("\n")
    for ti, t in enumerate(times):
        out.write(fmt(t))
        for k in range(sysm.size):
            out.write("," + fmt(states[ti, k]))
        out.write("\n")
