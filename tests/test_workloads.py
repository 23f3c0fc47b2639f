"""CPU: the seeded synthetic workloads follow their recipes (the configs the
measurements are quoted on): sizes, component counts, value ranges, seeds
and draw order, sources, and the compiled system sizes the bench reports."""
import math

import numpy as np

from ohmnivore_b200 import circuits as ck
from ohmnivore_b200 import mna


def _vals(ckt, kind):
    return ckt.value[ckt.kind == kind]


def test_resistor_ladder_10k():
    """Config 1: 10,000-node chain, V1 = 10 V at node 1, series R
    log-uniform [100, 100k] drawn first, shunt R log-uniform [1k, 1M]."""
    n = 10_000
    ckt = ck.resistor_ladder(n, seed=0)
    assert ckt.count(ck.V) == 1 and _vals(ckt, ck.V)[0] == 10.0
    r = _vals(ckt, ck.R)
    assert r.size == 2 * n - 1
    rng = np.random.default_rng(0)
    series = np.exp(rng.uniform(math.log(100.0), math.log(1e5), n - 1))
    shunt = np.exp(rng.uniform(math.log(1e3), math.log(1e6), n))
    np.testing.assert_array_equal(r[: n - 1], series)
    np.testing.assert_array_equal(r[n - 1:], shunt)
    assert mna.compile_circuit(ckt).size == n + 1


def test_diode_mesh_500():
    """Config 2: 500x500 mesh, edge R log-uniform [10, 10k], 25,000 diodes
    (10 %, without replacement) to ground, Is 1e-14, N 1, 5 V through 100
    ohm into corner (0, 0); 250,002 unknowns, 1,248,005 nonzeros."""
    ckt = ck.diode_mesh(500, 500, seed=1)
    assert _vals(ckt, ck.V).tolist() == [5.0]
    r = _vals(ckt, ck.R)
    assert r[0] == 100.0 and r.size == 1 + 2 * 500 * 499
    assert r[1:].min() >= 10.0 and r[1:].max() <= 1e4
    d = ckt.kind == ck.D
    assert d.sum() == 25_000
    assert np.all(ckt.nodes[d, 1] == 0) and np.unique(ckt.nodes[d, 0]).size == 25_000
    assert np.all(ckt.params[d, 0] == 1e-14) and np.all(ckt.params[d, 1] == 1.0)
    s = mna.compile_circuit(ckt)
    assert (s.size, s.g.nnz, len(s.diode_descriptors)) == (250_002, 1_248_005, 25_000)


def test_inverter_chain():
    """Config 3: NMOS VTO 0.7 / KP 110u, PMOS -0.7 / 50u, W/L uniform [1, 4]
    per device (PMOS drawn first), 10 fF per output, VDD 1.8 V, input PULSE
    0 -> 1.8 V with 50 ps edges, 0.95 ns width, 2 ns period."""
    stages = 2000
    ckt = ck.inverter_chain(stages=stages, seed=2)
    assert ckt.count(ck.M) == 2 * stages and ckt.count(ck.C) == stages
    v = np.flatnonzero(ckt.kind == ck.V)
    assert ckt.value[v[0]] == 1.8
    kind, params = ckt.tran[int(v[1])]
    assert kind == ck.TRAN_PULSE and tuple(params) == (0.0, 1.8, 0.0, 50e-12, 50e-12, 0.95e-9, 2e-9)
    m = ckt.kind == ck.M
    nmos = m & (ckt.params[:, 3] != 0)
    pmos = m & (ckt.params[:, 3] == 0)
    assert nmos.sum() == pmos.sum() == stages
    assert np.all(ckt.params[nmos, 0] == 0.7) and np.all(ckt.params[pmos, 0] == -0.7)
    rng = np.random.default_rng(2)
    wl_p = rng.uniform(1.0, 4.0, stages)
    wl_n = rng.uniform(1.0, 4.0, stages)
    np.testing.assert_allclose(ckt.params[pmos, 1], 50e-6 * wl_p, rtol=1e-15)
    np.testing.assert_allclose(ckt.params[nmos, 1], 110e-6 * wl_n, rtol=1e-15)
    assert np.all(_vals(ckt, ck.C) == 10e-15)
    assert mna.compile_circuit(ck.inverter_chain(stages=100_000, seed=2)).size == 100_004


def test_monte_carlo_batch():
    """Config 4: sizes log-uniform [50, 20,000] from default_rng(3), BJT
    differential pairs (Is 1e-16, BF 100, +-5 % Gaussian spread, VAF 100 V
    or infinite) and diode loads on resistor meshes."""
    n = 128
    ckts = ck.monte_carlo_batch(n, seed=3, vaf=100.0)
    rng = np.random.default_rng(3)
    sizes = np.round(np.exp(rng.uniform(math.log(50), math.log(20_000), n))).astype(np.int64)
    for c, target in zip(ckts, sizes):
        w = max(3, math.ceil(math.sqrt(max(int(target), 9))))
        assert np.count_nonzero(np.unique(c.nodes[c.nodes > 0])) >= w * w     # mesh nodes at least
        q = c.kind == ck.Q
        assert q.sum() >= 2 and np.all(c.params[q, 6] == 100.0)
        assert np.all(np.abs(c.params[q, 0] / 1e-16 - 1.0) < 0.5)
        assert np.all(np.abs(c.params[q, 1] / 100.0 - 1.0) < 0.5)
    assert all(np.all(np.isnan(c.params[c.kind == ck.Q, 6]) | np.isinf(c.params[c.kind == ck.Q, 6]))
               for c in ck.monte_carlo_batch(4, seed=3))


def test_rc_diode_mesh_1000():
    """Config 5: 1000x1000 RC mesh, R log-uniform [10, 10k], C log-uniform
    [1 fF, 1 pF] at every node, diodes at 5 % of the nodes, a 1 V step through
    50 ohm; 1,000,002 unknowns."""
    ckt = ck.rc_diode_mesh(1000, 1000, seed=4)
    v = int(np.flatnonzero(ckt.kind == ck.V)[0])
    kind, params = ckt.tran[v]
    assert kind == ck.TRAN_PULSE and params[0] == 0.0 and params[1] == 1.0
    r = _vals(ckt, ck.R)
    assert r[0] == 50.0 and r[1:].min() >= 10.0 and r[1:].max() <= 1e4
    c = _vals(ckt, ck.C)
    assert c.size == 1_000_000 and c.min() >= 1e-15 and c.max() <= 1e-12
    assert ckt.count(ck.D) == 50_000
    assert mna.compile_circuit(ckt).size == 1_000_002
