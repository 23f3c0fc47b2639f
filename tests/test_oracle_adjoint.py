"""The oracle's MOSFET sensitivities (|VTO| and KP of every MOSFET) pinned on
the CPU: the LU adjoint, the FP64 forward sensitivity and central finite
differences of the oracle's own Newton solve agree, at DC and through a
backward-Euler transient, on a small inverter chain biased into its
switching region.  The GPU adjoint is checked against this oracle in
test_gpu_adjoint.py."""
import copy

import numpy as np
import pytest

from oracle import adjoint_ref, newton_ref
from ohmnivore_b200 import circuits as ck
from ohmnivore_b200 import mna

H = 5e-12


def analog_chain(stages=4, vin=0.82):
    """Inverter chain (the transient workload's recipe, seed 2) with the input
    held at ``vin`` volts at DC.  At 0.82 V the first stage sits on its
    transfer curve (output ~1.66 V), so that output depends on the stage's
    |VTO| and KP; the later stages are driven to the rails."""
    ckt = ck.inverter_chain(stages=stages, seed=2)
    vi = int(np.flatnonzero(ckt.kind == ck.V)[1])
    ckt.value[vi] = vin
    return ckt


class _Comps:
    """No resistors or capacitors differentiated (MOSFET terms only)."""
    r_a = r_b = c_a = c_b = np.zeros(0, np.int64)
    r_ohms = c_farads = np.zeros(0)


def _fd(sysm, kind, j, output, rel=1e-6):
    """Central difference of output(sysm') over the f32-rounded perturbed
    descriptor values (the parameter is stored as f32)."""
    field = {"VTO": "vto", "KP": "kp"}[kind]
    v0 = float(sysm.mosfet_descriptors[field][j])
    outs, vals = [], []
    for sign in (1, -1):
        s2 = copy.deepcopy(sysm)
        s2.mosfet_descriptors[field][j] = np.float32(v0 * (1 + sign * rel))
        vals.append(float(s2.mosfet_descriptors[field][j]))
        outs.append(output(s2))
    assert vals[0] != vals[1]
    return (outs[0] - outs[1]) / (vals[0] - vals[1])


@pytest.mark.parametrize("kind", ["VTO", "KP"])
def test_dc_mosfet_gradients_agree(kind):
    s = mna.compile_circuit(analog_chain())
    probe = s.node_index(2 + 1)                    # first stage output
    w = np.zeros(s.size)
    w[probe] = 1.0
    x, _ = newton_ref.newton(s)
    g, _ = adjoint_ref.dc_adjoint(s, _Comps, x, w)
    scale = np.max(np.abs(g[kind]))
    assert scale > 0.0
    for j in range(len(s.mosfet_descriptors)):
        fs = adjoint_ref.forward_sensitivity(s, _Comps, [x], 1.0, w, kind, j)
        assert abs(g[kind][j] - fs) <= 1e-10 * max(abs(fs), scale), (kind, j)
    for j in (0, 1):                               # the first stage's PMOS and NMOS
        fd = _fd(s, kind, j, lambda s2: newton_ref.newton(s2, x0=x)[0][probe])
        assert abs(g[kind][j] - fd) <= 1e-6 * max(abs(fd), 1e-3 * scale), (kind, j, g[kind][j], fd)


def test_transient_mosfet_gradients_agree():
    """Backward Euler from the DC point through the input's rising PULSE edge
    (0 -> 1.8 V in 50 ps), output = the first stage's output at step 12
    (60 ps), while that stage switches."""
    ckt = analog_chain(stages=3, vin=0.0)
    s = mna.compile_circuit(ckt)
    probe = s.node_index(2 + 1)
    w = np.zeros(s.size)
    w[probe] = 1.0
    n_steps = 12

    def run(s2):
        x0, _ = newton_ref.dc_operating_point(s2)
        return adjoint_ref.transient_states(s2, x0, 0.0, H, n_steps)

    states = run(s)
    g = adjoint_ref.transient_adjoint(s, _Comps, states, H, w)
    for kind in ("VTO", "KP"):
        scale = np.max(np.abs(g[kind]))
        assert scale > 0.0
        for j in (0, 1, 4):
            fs = adjoint_ref.forward_sensitivity(s, _Comps, states, H, w, kind, j)
            assert abs(g[kind][j] - fs) <= 1e-9 * max(abs(fs), scale), (kind, j)
            # a relative step of 1e-6 in KP moves this output by ~1e-11 V,
            # a few ulps of its FP64 value: KP takes a step of 1e-4
            # (central differences: truncation ~1e-8 relative)
            fd = _fd(s, kind, j, lambda s2: run(s2)[-1][probe], rel=1e-6 if kind == "VTO" else 1e-4)
            assert abs(g[kind][j] - fd) <= 1e-6 * max(abs(fd), 1e-3 * scale), (kind, j, g[kind][j], fd)
