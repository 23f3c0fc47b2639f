"""Columnar circuit description and seeded generators for the benchmark circuits.

The reference describes a circuit as an ordered list of ``Component`` values
(``src/ir.rs:11-178``).  Ordering matters: node indices are assigned by first
appearance over the component list and branch indices by the order of voltage
sources and inductors (``src/compiler.rs:196-252``).  This module keeps the
same ordered list, but stored column-wise (one numpy array per field) so that
circuits with millions of elements can be built and compiled quickly.

Node labels are integers; label ``0`` is ground (the reference treats ``"0"``
and ``"GND"`` as ground, ``src/compiler.rs:177-179``).  Unused terminals are
``-1``.

Device parameters are stored per element (one ``.MODEL`` per instance), which
is how per-instance W/L and Monte Carlo perturbations are expressed.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# Component kinds, in the order of the reference's ``Component`` enum.
R, C, L, V, I, D, Q, M = range(8)
KIND_NAMES = "RCLVIDQM"

# Parameter columns (``params[:, k]``).
#   D: is, n
#   Q: is, bf, br, nf, nr, npn(1/0), vaf (inf = no Early effect; extension)
#   M: vto, kp, lambda, nmos(1/0)
N_PARAMS = 7

# Transient source functions (``src/ir.rs`` ``TransientFunc``).
TRAN_PULSE, TRAN_SIN, TRAN_PWL, TRAN_EXP = range(4)


@dataclass
class Circuit:
    """Ordered component list in column form.

    Attributes are numpy arrays of equal length ``m`` (number of components):
    ``kind`` (int8), ``nodes`` (m x 3 int64 labels), ``value`` (R ohms, C farads,
    L henries, V/I DC value; NaN = no DC value), ``ac`` (m x 2: magnitude,
    phase in degrees; NaN = none), ``params`` (m x N_PARAMS).
    ``tran`` maps a component index to ``(func_kind, tuple_of_params)``.
    """

    kind: np.ndarray
    nodes: np.ndarray
    value: np.ndarray
    ac: np.ndarray
    params: np.ndarray
    tran: dict = field(default_factory=dict)
    names: list | None = None

    @property
    def n_components(self) -> int:
        return int(self.kind.shape[0])

    def count(self, kind: int) -> int:
        return int(np.count_nonzero(self.kind == kind))


class CircuitBuilder:
    """Appends blocks of same-kind components; ``build()`` concatenates in order."""

    def __init__(self):
        self._blocks = []
        self._tran = {}
        self._count = 0
        self._names = []

    def _add(self, kind, n0, n1, n2=None, value=None, ac=None, params=None, names=None):
        n0 = np.atleast_1d(np.asarray(n0, dtype=np.int64))
        m = n0.shape[0]
        n1 = np.broadcast_to(np.asarray(n1, dtype=np.int64), (m,))
        n2 = (np.full(m, -1, np.int64) if n2 is None
              else np.broadcast_to(np.asarray(n2, dtype=np.int64), (m,)))
        nodes = np.stack([n0, n1, n2], axis=1)
        val = (np.full(m, np.nan) if value is None
               else np.broadcast_to(np.asarray(value, dtype=np.float64), (m,)).copy())
        acv = np.full((m, 2), np.nan)
        if ac is not None:
            acv[:] = np.asarray(ac, dtype=np.float64)
        par = np.full((m, N_PARAMS), np.nan)
        if params is not None:
            p = np.asarray(params, dtype=np.float64)
            if p.ndim == 1:
                p = np.broadcast_to(p, (m, p.shape[0]))
            par[:, : p.shape[1]] = p
        self._blocks.append((np.full(m, kind, np.int8), nodes, val, acv, par))
        if names is None:
            names = [f"{KIND_NAMES[kind]}{self._count + k + 1}" for k in range(m)]
        self._names.extend(names)
        first = self._count
        self._count += m
        return first

    def resistors(self, a, b, ohms, names=None):
        return self._add(R, a, b, value=ohms, names=names)

    def capacitors(self, a, b, farads, names=None):
        return self._add(C, a, b, value=farads, names=names)

    def inductors(self, a, b, henries, names=None):
        return self._add(L, a, b, value=henries, names=names)

    def vsource(self, a, b, dc=None, ac=None, tran=None, name=None):
        idx = self._add(V, a, b, value=np.nan if dc is None else dc, ac=ac,
                        names=None if name is None else [name])
        if tran is not None:
            self._tran[idx] = tran
        return idx

    def isource(self, a, b, dc=None, ac=None, tran=None, name=None):
        idx = self._add(I, a, b, value=np.nan if dc is None else dc, ac=ac,
                        names=None if name is None else [name])
        if tran is not None:
            self._tran[idx] = tran
        return idx

    def diodes(self, anode, cathode, is_=1e-14, n=1.0, names=None):
        a = np.atleast_1d(np.asarray(anode, np.int64))
        par = np.stack(np.broadcast_arrays(np.asarray(is_, float) * np.ones(a.shape[0]),
                                           np.asarray(n, float)), axis=1)
        return self._add(D, a, cathode, params=par, names=names)

    def bjts(self, c, b, e, is_=1e-16, bf=100.0, br=1.0, nf=1.0, nr=1.0, npn=True,
             vaf=math.inf, names=None):
        c = np.atleast_1d(np.asarray(c, np.int64))
        m = c.shape[0]
        cols = [np.broadcast_to(np.asarray(v, float), (m,))
                for v in (is_, bf, br, nf, nr, np.where(np.asarray(npn), 1.0, 0.0), vaf)]
        return self._add(Q, c, b, e, params=np.stack(cols, axis=1), names=names)

    def mosfets(self, d, g, s, vto=1.0, kp=2e-5, lam=0.0, nmos=True, names=None):
        d = np.atleast_1d(np.asarray(d, np.int64))
        m = d.shape[0]
        cols = [np.broadcast_to(np.asarray(v, float), (m,))
                for v in (vto, kp, lam, np.where(np.asarray(nmos), 1.0, 0.0))]
        return self._add(M, d, g, s, params=np.stack(cols, axis=1), names=names)

    def build(self) -> Circuit:
        if not self._blocks:
            z = np.zeros(0)
            return Circuit(np.zeros(0, np.int8), np.zeros((0, 3), np.int64), z,
                           np.zeros((0, 2)), np.zeros((0, N_PARAMS)), {}, [])
        cat = [np.concatenate([b[k] for b in self._blocks]) for k in range(5)]
        return Circuit(*cat, tran=dict(self._tran), names=list(self._names))


def _log_uniform(rng, lo, hi, size):
    return np.exp(rng.uniform(math.log(lo), math.log(hi), size))


# ---------------------------------------------------------------------------
# Benchmark circuits (seeded).  Component order is part of each recipe because
# it fixes the node/branch numbering.
# ---------------------------------------------------------------------------

def resistor_ladder(n_nodes: int = 10_000, seed: int = 0, v_dc: float = 10.0) -> Circuit:
    """Linear resistor chain: ``n_nodes`` nodes in series, a DC source at node 1,
    series R log-uniform in [100, 100k] ohm and a shunt R from every node to
    ground log-uniform in [1k, 1M] ohm.  ``default_rng(seed)`` draws the series
    values first, then the shunts.  Order: V1, series R, shunt R.
    The reference's chain generator (``bench/generate_chain.py:8-48``) emits
    inverter chains; this ladder follows its style (seeded, fixed line order).
    """
    rng = np.random.default_rng(seed)
    series = _log_uniform(rng, 100.0, 1e5, n_nodes - 1)
    shunt = _log_uniform(rng, 1e3, 1e6, n_nodes)
    b = CircuitBuilder()
    b.vsource(1, 0, dc=v_dc, name="V1")
    k = np.arange(1, n_nodes, dtype=np.int64)
    b.resistors(k, k + 1, series)
    b.resistors(np.arange(1, n_nodes + 1, dtype=np.int64), 0, shunt)
    return b.build()


def diode_mesh(rows: int = 500, cols: int = 500, seed: int = 1, diode_frac: float = 0.10,
               r_lo: float = 10.0, r_hi: float = 1e4, v_src: float = 5.0,
               r_src: float = 100.0, is_: float = 1e-14, n: float = 1.0) -> Circuit:
    """2-D resistor mesh with diodes to ground and a source driving a corner.

    Labels: mesh node (i, j) is ``2 + i*cols + j``; the source node is ``1``.
    ``default_rng(seed)`` draws the horizontal edge resistors (row-major), then
    the vertical edge resistors (row-major), then the diode sites (uniform,
    without replacement, ``round(diode_frac * rows * cols)`` of them, in
    ascending node order).
    Order: V1 (node 1 to ground), Rsrc (node 1 to corner (0,0)), horizontal
    edges, vertical edges, diodes (anode at the site, cathode at ground).
    """
    rng = np.random.default_rng(seed)
    nh = rows * (cols - 1)
    nv = (rows - 1) * cols
    rh = _log_uniform(rng, r_lo, r_hi, nh)
    rv = _log_uniform(rng, r_lo, r_hi, nv)
    n_mesh = rows * cols
    n_d = int(round(diode_frac * n_mesh))
    sites = np.sort(rng.choice(n_mesh, size=n_d, replace=False))
    lab = lambda i, j: 2 + i * cols + j  # noqa: E731
    b = CircuitBuilder()
    b.vsource(1, 0, dc=v_src, name="V1")
    b.resistors([1], [lab(0, 0)], [r_src], names=["RSRC"])
    ii, jj = np.meshgrid(np.arange(rows), np.arange(cols - 1), indexing="ij")
    b.resistors(lab(ii, jj).ravel(), lab(ii, jj + 1).ravel(), rh)
    ii, jj = np.meshgrid(np.arange(rows - 1), np.arange(cols), indexing="ij")
    b.resistors(lab(ii, jj).ravel(), lab(ii + 1, jj).ravel(), rv)
    b.diodes(2 + sites, 0, is_=is_, n=n)
    return b.build()


def rc_diode_mesh(rows: int = 1000, cols: int = 1000, seed: int = 4, diode_frac: float = 0.05,
                  v_step: float = 1.0, r_src: float = 50.0) -> Circuit:
    """RC mesh with diodes: edge R log-uniform [10, 10k] ohm, a capacitor from
    every mesh node to ground log-uniform [1 fF, 1 pF], diodes at
    ``diode_frac`` of the nodes, a step source through ``r_src`` into corner
    (0, 0).  Same labelling and draw order as :func:`diode_mesh`, with the
    capacitor values drawn last.  The source carries a PULSE 0 -> v_step with
    a 1 ps rise so that DC sees 0 V and the transient sees the step.
    """
    rng = np.random.default_rng(seed)
    nh = rows * (cols - 1)
    nv = (rows - 1) * cols
    rh = _log_uniform(rng, 10.0, 1e4, nh)
    rv = _log_uniform(rng, 10.0, 1e4, nv)
    n_mesh = rows * cols
    n_d = int(round(diode_frac * n_mesh))
    sites = np.sort(rng.choice(n_mesh, size=n_d, replace=False))
    caps = _log_uniform(rng, 1e-15, 1e-12, n_mesh)
    lab = lambda i, j: 2 + i * cols + j  # noqa: E731
    b = CircuitBuilder()
    b.vsource(1, 0, dc=0.0, name="V1",
              tran=(TRAN_PULSE, (0.0, v_step, 0.0, 1e-12, 1e-12, 1.0, 2.0)))
    b.resistors([1], [lab(0, 0)], [r_src], names=["RSRC"])
    ii, jj = np.meshgrid(np.arange(rows), np.arange(cols - 1), indexing="ij")
    b.resistors(lab(ii, jj).ravel(), lab(ii, jj + 1).ravel(), rh)
    ii, jj = np.meshgrid(np.arange(rows - 1), np.arange(cols), indexing="ij")
    b.resistors(lab(ii, jj).ravel(), lab(ii + 1, jj).ravel(), rv)
    b.diodes(2 + sites, 0, is_=1e-14, n=1.0)
    b.capacitors(2 + np.arange(n_mesh), 0, caps)
    return b.build()


def inverter_chain(stages: int = 100_000, seed: int = 2, vdd: float = 1.8,
                   c_load: float = 10e-15, lam: float = 0.04,
                   pulse=(0.0, 1.8, 0.0, 50e-12, 50e-12, 0.95e-9, 2e-9)) -> Circuit:
    """CMOS inverter chain.  NMOS VTO=0.7, KP=110u; PMOS VTO=-0.7, KP=50u;
    W/L uniform in [1, 4] per device from ``default_rng(seed)`` (PMOS values
    first, then NMOS), realised as KP_eff = KP * W/L.  A load capacitor per
    stage output.  Labels: vdd=1, in=2, out_k = 2 + k (k = 1..stages).
    Order: VDD, VIN (PULSE), then per stage MP, MN, CL (as the reference's
    chain generator orders MP before MN, ``bench/generate_chain.py:33-38``).
    """
    rng = np.random.default_rng(seed)
    wl_p = rng.uniform(1.0, 4.0, stages)
    wl_n = rng.uniform(1.0, 4.0, stages)
    b = CircuitBuilder()
    b.vsource(1, 0, dc=vdd, name="VDD")
    b.vsource(2, 0, dc=pulse[0], name="VIN", tran=(TRAN_PULSE, tuple(pulse)))
    k = np.arange(1, stages + 1, dtype=np.int64)
    gate = np.where(k == 1, 2, 1 + k)
    out = 2 + k
    # Build the MP, MN and CL columns separately, then interleave them
    # stage-major (MP1, MN1, CL1, MP2, ...).
    pm = CircuitBuilder()
    pm.mosfets(out, gate, 1, vto=-0.7, kp=50e-6 * wl_p, lam=lam, nmos=False)
    pn = CircuitBuilder()
    pn.mosfets(out, gate, 0, vto=0.7, kp=110e-6 * wl_n, lam=lam, nmos=True)
    pc = CircuitBuilder()
    pc.capacitors(out, 0, c_load)
    head = b.build()
    cp, cn, cc = pm.build(), pn.build(), pc.build()
    m = stages

    def merge(field):
        a = np.stack([getattr(cp, field), getattr(cn, field), getattr(cc, field)], axis=1)
        return a.reshape((3 * m,) + a.shape[2:])

    body = Circuit(merge("kind"), merge("nodes"), merge("value"), merge("ac"), merge("params"))
    names = head.names + [f"{p}{s}" for s in range(1, m + 1) for p in ("MP", "MN", "CL")]
    return Circuit(np.concatenate([head.kind, body.kind]),
                   np.concatenate([head.nodes, body.nodes]),
                   np.concatenate([head.value, body.value]),
                   np.concatenate([head.ac, body.ac]),
                   np.concatenate([head.params, body.params]),
                   tran=dict(head.tran), names=names)


def bjt_diffpair_mesh(n_target: int, rng: np.random.Generator, sigma: float = 0.05,
                      vaf: float = math.inf) -> Circuit:
    """One Monte Carlo instance: a resistor mesh with BJT differential pairs
    and diode loads, about ``n_target`` nodes.

    Recipe (documented choice): a ``w x w`` resistor mesh (w = ceil(sqrt(n))),
    edge R log-uniform [100, 10k] ohm; VCC = 5 V at node 1 feeding mesh corner
    (0,0) through 100 ohm; one NPN differential pair per 100 mesh nodes: the
    two collectors sit on mesh nodes, the bases on mesh nodes two columns
    away, the shared emitter node goes to ground through a 4.3k tail resistor;
    one diode load (anode on a mesh node, cathode to ground) per pair.
    Every R, Is and BF is multiplied by ``1 + sigma * N(0, 1)``.
    """
    w = max(3, int(math.ceil(math.sqrt(max(n_target, 9)))))
    n_mesh = w * w
    lab = lambda i, j: 2 + i * w + j  # noqa: E731
    pert = lambda x: x * (1.0 + sigma * rng.standard_normal(np.shape(x)))  # noqa: E731
    rh = pert(_log_uniform(rng, 100.0, 1e4, w * (w - 1)))
    rv = pert(_log_uniform(rng, 100.0, 1e4, (w - 1) * w))
    n_pairs = max(1, n_mesh // 100)
    sites = np.sort(rng.choice(n_mesh - 2 * w, size=n_pairs, replace=False))
    b = CircuitBuilder()
    b.vsource(1, 0, dc=5.0, name="VCC")
    b.resistors([1], [lab(0, 0)], [pert(100.0)], names=["RSRC"])
    ii, jj = np.meshgrid(np.arange(w), np.arange(w - 1), indexing="ij")
    b.resistors(lab(ii, jj).ravel(), lab(ii, jj + 1).ravel(), rh)
    ii, jj = np.meshgrid(np.arange(w - 1), np.arange(w), indexing="ij")
    b.resistors(lab(ii, jj).ravel(), lab(ii + 1, jj).ravel(), rv)
    c1 = 2 + sites
    c2 = 2 + sites + 1
    b1 = 2 + sites + w
    b2 = 2 + sites + w + 1
    tail = 2 + n_mesh + np.arange(n_pairs)
    b.resistors(tail, 0, pert(np.full(n_pairs, 4300.0)))
    is_ = pert(np.full(n_pairs, 1e-16))
    bf = pert(np.full(n_pairs, 100.0))
    b.bjts(c1, b1, tail, is_=is_, bf=bf, vaf=vaf)
    is2 = pert(np.full(n_pairs, 1e-16))
    bf2 = pert(np.full(n_pairs, 100.0))
    b.bjts(c2, b2, tail, is_=is2, bf=bf2, vaf=vaf)
    b.diodes(2 + sites + 2 * w, 0, is_=pert(np.full(n_pairs, 1e-14)))
    return b.build()


def monte_carlo_batch(n_instances: int = 4096, seed: int = 3, n_lo: int = 50,
                      n_hi: int = 20_000, vaf: float = math.inf):
    """Sizes log-uniform in [n_lo, n_hi] from ``default_rng(seed)``, then one
    :func:`bjt_diffpair_mesh` per instance drawn from the same generator."""
    rng = np.random.default_rng(seed)
    sizes = np.round(_log_uniform(rng, n_lo, n_hi, n_instances)).astype(np.int64)
    return [bjt_diffpair_mesh(int(s), rng, vaf=vaf) for s in sizes]
