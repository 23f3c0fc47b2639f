"""CPU: the host half of the device compile.  `system_from_device_compile`
fills in the AC rhs, the transient source list, the BJT Early voltages and
the per-kind index maps from the arrays the device returns; fed with the
host compiler's arrays it must rebuild the host compiler's system."""
import numpy as np
import pytest

from ohmnivore_b200 import circuits as ck
from ohmnivore_b200 import mna
from tests.test_gpu_compile import CIRCUITS, _mixed_circuit


@pytest.mark.parametrize("name", ["mixed", "inverter_chain", "monte_carlo_bjt", "rc_diode_mesh"])
def test_assembly_from_compiled_arrays(name):
    ckt = CIRCUITS[name]()
    h = mna.compile_circuit(ckt)
    d = mna.system_from_device_compile(ckt, h.g, h.c, h.b_dc, h.node_labels, h.branch_components,
                                       h.diode_descriptors, h.bjt_descriptors, h.mosfet_descriptors)
    assert (d.size, d.n_nodes) == (h.size, h.n_nodes)
    np.testing.assert_array_equal(d.b_ac, h.b_ac)
    assert d.sources == h.sources
    np.testing.assert_array_equal(d.bjt_vaf, h.bjt_vaf)
    for k in ("diode_components", "bjt_components", "mosfet_components"):
        np.testing.assert_array_equal(getattr(d, k), getattr(h, k))


def test_assembly_with_scattered_labels():
    ckt = _mixed_circuit()
    ckt.nodes = np.where(ckt.nodes > 0, ckt.nodes * 1_000_003 + 17, ckt.nodes)
    h = mna.compile_circuit(ckt)
    d = mna.system_from_device_compile(ckt, h.g, h.c, h.b_dc, h.node_labels, h.branch_components,
                                       h.diode_descriptors, h.bjt_descriptors, h.mosfet_descriptors)
    np.testing.assert_array_equal(d.b_ac, h.b_ac)
    assert d.sources == h.sources
