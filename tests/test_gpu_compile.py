"""GPU: the device-side MNA compile (ohm_compile) against the host compiler
(the restatement of src/compiler.rs:194-754 that the oracle pins), bit for
bit: CSR patterns and values, right-hand sides, node and branch order,
descriptor bytes; every component kind, arbitrary node labels, duplicate
stamps, compile errors, and the headline's 250k-row mesh."""
import numpy as np
import pytest

from ohmnivore_b200 import circuits as ck
from ohmnivore_b200 import mna
from ohmnivore_b200 import solver as S

pytestmark = pytest.mark.gpu


def _bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint8) if a.size else a


def assert_same_system(dev, host):
    assert (dev.size, dev.n_nodes) == (host.size, host.n_nodes)
    for name in ("g", "c"):
        d, h = getattr(dev, name), getattr(host, name)
        np.testing.assert_array_equal(d.row_ptr, h.row_ptr, err_msg=name)
        np.testing.assert_array_equal(d.col, h.col, err_msg=name)
        np.testing.assert_array_equal(_bits(d.val.astype(np.float64)), _bits(h.val.astype(np.float64)),
                                      err_msg=name)
    np.testing.assert_array_equal(_bits(dev.b_dc), _bits(host.b_dc))
    np.testing.assert_array_equal(dev.b_ac, host.b_ac)
    np.testing.assert_array_equal(dev.node_labels, host.node_labels)
    np.testing.assert_array_equal(dev.branch_components, host.branch_components)
    for name in ("diode_descriptors", "bjt_descriptors", "mosfet_descriptors"):
        np.testing.assert_array_equal(_bits(getattr(dev, name)), _bits(getattr(host, name)), err_msg=name)
    np.testing.assert_array_equal(dev.bjt_vaf, host.bjt_vaf)
    for name in ("diode_components", "bjt_components", "mosfet_components"):
        np.testing.assert_array_equal(getattr(dev, name), getattr(host, name))
    assert dev.sources == host.sources


def _mixed_circuit():
    """Every component kind: inductors, V and I sources with DC and AC values
    (two current sources into one node), a floating diode, BJTs of both
    polarities with and without an emitter at ground, MOSFETs with terminals
    on a V-source node (node_fixed), a self-loop resistor, capacitors
    between two nodes."""
    b = ck.CircuitBuilder()
    b.vsource(1, 0, dc=5.0, ac=(1.0, 30.0), name="V1")
    b.vsource(7, 3, dc=None, name="V2", tran=(ck.TRAN_SIN, (0.0, 1.0, 1e6, 0.0, 0.0)))
    b.resistors([1, 2, 3, 4, 5, 6, 4], [2, 3, 4, 5, 6, 0, 4], [100.0, 220.0, 330.0, 1e3, 2.2e3, 4.7e3, 50.0])
    b.inductors([2, 6], [0, 5], [1e-6, 3e-9])
    b.capacitors([3, 5, 2], [0, 4, 6], [1e-12, 2e-12, 5e-13])
    b.isource(0, 4, dc=1e-3, ac=(0.5, -45.0), name="I1")
    b.isource(5, 4, dc=2.5e-4, name="I2")
    b.isource(0, 0, dc=1.0, name="I3")
    b.diodes([3, 5], [4, 0], is_=1e-14, n=1.5)
    b.bjts([4, 6], [3, 5], [0, 2], is_=1e-16, bf=80.0, npn=True)
    b.bjts([2], [6], [1], is_=2e-16, bf=50.0, npn=False, vaf=75.0)
    b.mosfets([5, 7], [1, 3], [0, 1], vto=0.7, kp=1.1e-4, lam=0.02, nmos=True)
    b.mosfets([2], [4], [1], vto=-0.7, kp=5e-5, lam=0.01, nmos=False)
    return b.build()


CIRCUITS = {
    "diode_mesh": lambda: ck.diode_mesh(30, 30, seed=2),
    "rc_diode_mesh": lambda: ck.rc_diode_mesh(20, 20, seed=4),
    "inverter_chain": lambda: ck.inverter_chain(stages=60, seed=2),
    "monte_carlo_bjt": lambda: ck.monte_carlo_batch(1, seed=5, n_lo=300, n_hi=400, vaf=100.0)[0],
    "resistor_ladder": lambda: ck.resistor_ladder(500, seed=0),
    "mixed": _mixed_circuit,
}


@pytest.mark.parametrize("name", list(CIRCUITS))
def test_device_compile_equals_host(ctx, name):
    ckt = CIRCUITS[name]()
    assert_same_system(S.compile_circuit_device(ckt, ctx), mna.compile_circuit(ckt))


def test_arbitrary_labels(ctx):
    """Node labels are only names: scattered 62-bit labels (and negative
    third terminals) number the same way as small ones."""
    ckt = _mixed_circuit()
    rng = np.random.default_rng(7)
    labels = np.unique(ckt.nodes[ckt.nodes > 0])
    new = rng.choice(np.arange(1, 2 ** 62, 2 ** 40, dtype=np.int64), size=labels.size, replace=False)
    remap = dict(zip(labels.tolist(), new.tolist()))
    nodes = ckt.nodes.copy()
    for idx in np.ndindex(nodes.shape):
        if nodes[idx] > 0:
            nodes[idx] = remap[int(nodes[idx])]
    two = ~np.isin(ckt.kind, [ck.Q, ck.M])
    nodes[two, 2] = -5
    ckt.nodes = nodes
    assert_same_system(S.compile_circuit_device(ckt, ctx), mna.compile_circuit(ckt))


def test_empty_and_ground_only(ctx):
    b = ck.CircuitBuilder()
    b.resistors([0], [0], [10.0])
    ckt = b.build()
    dev = S.compile_circuit_device(ckt, ctx)
    assert dev.size == 0 and dev.g.nnz == 0
    assert_same_system(dev, mna.compile_circuit(ckt))


@pytest.mark.parametrize("bad", ["zero_r", "negative_c", "no_model"])
def test_compile_errors(ctx, bad):
    ckt = _mixed_circuit()
    if bad == "zero_r":
        ckt.value[np.flatnonzero(ckt.kind == ck.R)[3]] = 0.0
    elif bad == "negative_c":
        ckt.value[np.flatnonzero(ckt.kind == ck.C)[1]] = -1e-12
    else:
        ckt.params[np.flatnonzero(ckt.kind == ck.M)[0], 0] = np.nan
    with pytest.raises(mna.CompileError):
        mna.compile_circuit(ckt)
    with pytest.raises(mna.CompileError):
        S.compile_circuit_device(ckt, ctx)


def test_headline_mesh_and_solve(ctx):
    """The 250k-row diode mesh: identical system, and the Newton solve on the
    device-compiled system is bit-identical to the one on the host's."""
    import torch
    ckt = ck.diode_mesh(500, 500, seed=1)
    dev = S.compile_circuit_device(ckt, ctx)
    host = mna.compile_circuit(ckt)
    assert_same_system(dev, host)
    params = S.NewtonParams(max_iterations=200, abs_tol=1e-9, bicgstab_max_iterations=20000,
                            bicgstab_tolerance=1e-14, inner_rtol=1e-4, forcing=1, eta_max=0.7)
    xs = []
    for s in (dev, host):
        plan = S.NewtonPlan(s, ctx)
        try:
            x = torch.zeros(s.size, dtype=torch.float64, device="cuda")
            plan.newton_device(x.data_ptr(), params)
            xs.append(x.cpu().numpy())
        finally:
            plan.close()
    np.testing.assert_array_equal(xs[0], xs[1])
