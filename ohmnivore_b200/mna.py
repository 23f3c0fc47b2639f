"""MNA compiler: circuit -> CSR conductance/capacitance matrices + device descriptors.

This is the host-side counterpart of ``compile`` (``src/compiler.rs:194-754``)
for callers that do not run the reference's Rust front end.  Its output is the
input contract of the hot path: the CSR pattern, the values and the CSR
value-array indices stored in the device descriptors match the reference
bit for bit (node order, branch order, triplet summation order, GMIN, the
C-pattern zero fill and the ``u32::MAX`` sentinels).

It is vectorised with numpy so that million-node circuits compile in seconds.
Duplicate triplets are summed strictly left to right in the reference's
triplet order, as ``CsrMatrix::from_triplets`` does after its stable sort
(``src/sparse.rs:51-104``), so that the floating-point sums are identical.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import circuits as ck

VT_300K = 0.02585          # src/compiler.rs:40
GMIN = 1e-12               # src/compiler.rs:44
SENTINEL = 0xFFFFFFFF      # u32::MAX, src/compiler.rs:600

# Byte-identical to the reference's #[repr(C)] descriptor structs.
DIODE_DTYPE = np.dtype([            # GpuDiodeDescriptor, src/compiler.rs:52-73 (48 B)
    ("anode", "<u4"), ("cathode", "<u4"), ("is_val", "<f4"), ("n_vt", "<f4"),
    ("g_row_col", "<u4", (4,)), ("b_idx", "<u4", (2,)), ("pad", "<u4", (2,)),
])
BJT_DTYPE = np.dtype([              # GpuBjtDescriptor, src/compiler.rs:79-113 (96 B)
    ("collector", "<u4"), ("base", "<u4"), ("emitter", "<u4"), ("polarity", "<f4"),
    ("is_val", "<f4"), ("bf", "<f4"), ("br", "<f4"), ("nf_vt", "<f4"), ("nr_vt", "<f4"),
    ("node_fixed", "<u4", (3,)), ("g_row_col", "<u4", (9,)), ("b_idx", "<u4", (3,)),
])
MOSFET_DTYPE = np.dtype([           # GpuMosfetDescriptor, src/compiler.rs:119-149 (64 B)
    ("drain", "<u4"), ("gate", "<u4"), ("source", "<u4"), ("polarity", "<f4"),
    ("vto", "<f4"), ("kp", "<f4"), ("lam", "<f4"), ("node_fixed_packed", "<u4"),
    ("g_row_col", "<u4", (6,)), ("b_idx", "<u4", (2,)),
])
assert DIODE_DTYPE.itemsize == 48 and BJT_DTYPE.itemsize == 96 and MOSFET_DTYPE.itemsize == 64


class CompileError(ValueError):
    """``OhmnivoreError::Compile`` (``src/error.rs:9-10``)."""


@dataclass
class Csr:
    """CSR matrix; ``row_ptr`` int64 (n+1), ``col`` int64, ``val`` float64/complex."""
    nrows: int
    ncols: int
    row_ptr: np.ndarray
    col: np.ndarray
    val: np.ndarray

    @property
    def nnz(self) -> int:
        return int(self.col.shape[0])

    def value_index(self, row: int, col: int):
        """``CsrMatrix::value_index`` (``src/sparse.rs:27-31``)."""
        s, e = int(self.row_ptr[row]), int(self.row_ptr[row + 1])
        hit = np.nonzero(self.col[s:e] == col)[0]
        return int(s + hit[0]) if hit.size else None

    def to_dense(self):
        d = np.zeros((self.nrows, self.ncols), dtype=self.val.dtype)
        rows = np.repeat(np.arange(self.nrows), np.diff(self.row_ptr))
        d[rows, self.col] = self.val
        return d

    def spmv(self, x):
        rows = np.repeat(np.arange(self.nrows), np.diff(self.row_ptr))
        y = np.zeros(self.nrows, dtype=np.result_type(self.val, x))
        np.add.at(y, rows, self.val * x[self.col])
        return y

    def keys(self):
        rows = np.repeat(np.arange(self.nrows, dtype=np.int64), np.diff(self.row_ptr))
        return rows * np.int64(max(self.ncols, 1)) + self.col

    def positions(self, rows, cols):
        """Vectorised value_index; returns SENTINEL where absent."""
        rows = np.asarray(rows, np.int64)
        cols = np.asarray(cols, np.int64)
        out = np.full(rows.shape, SENTINEL, dtype=np.int64)
        ok = (rows >= 0) & (cols >= 0)
        if self.nnz == 0 or not ok.any():
            return out
        keys = self.keys()
        q = rows[ok] * np.int64(max(self.ncols, 1)) + cols[ok]
        pos = np.searchsorted(keys, q)
        pos_c = np.minimum(pos, keys.shape[0] - 1)
        hit = keys[pos_c] == q
        res = np.where(hit, pos_c, SENTINEL)
        out[ok] = res
        return out


@dataclass
class MnaSystem:
    """``MnaSystem`` (``src/compiler.rs:153-175``) plus index maps used by the
    analyses (V-source branch rows and constrained nodes)."""
    g: Csr
    c: Csr
    b_dc: np.ndarray
    b_ac: np.ndarray
    size: int
    n_nodes: int
    node_labels: np.ndarray          # matrix index -> node label
    branch_components: np.ndarray    # branch k -> component index
    diode_descriptors: np.ndarray
    bjt_descriptors: np.ndarray
    mosfet_descriptors: np.ndarray
    bjt_vaf: np.ndarray = field(default=None)        # extension: Early voltage per BJT
    diode_components: np.ndarray = field(default=None)
    bjt_components: np.ndarray = field(default=None)
    mosfet_components: np.ndarray = field(default=None)
    sources: list = field(default_factory=list)     # [(comp_idx, [(row, sign)], dc, tran)]

    @property
    def n_branches(self) -> int:
        return self.size - self.n_nodes

    @property
    def nonlinear(self) -> bool:
        return (len(self.diode_descriptors) + len(self.bjt_descriptors)
                + len(self.mosfet_descriptors)) > 0

    def node_index(self, label: int):
        hit = np.nonzero(self.node_labels == label)[0]
        return int(hit[0]) if hit.size else None


def _seq_group_sum(keys, seq, vals):
    """Sum ``vals`` grouped by ``keys``, left to right in ``seq`` order.

    Returns (unique_keys, sums).  Within a group the additions run strictly
    sequentially (a loop over the rank inside the group, vectorised across
    groups), which reproduces the order of ``CsrMatrix::from_triplets``.
    """
    if keys.size == 0:
        return keys, vals
    order = np.lexsort((seq, keys))
    k = keys[order]
    v = vals[order]
    starts = np.flatnonzero(np.r_[True, k[1:] != k[:-1]])
    lens = np.diff(np.r_[starts, k.size])
    acc = v[starts].copy()
    for r in range(1, int(lens.max())):
        m = lens > r
        acc[m] = acc[m] + v[starts[m] + r]
    return k[starts], acc


def _build_csr(n, rows, cols, vals, seq):
    """``CsrMatrix::from_triplets``: pattern = unique (row, col); value = ordered sum.

    Zero-valued triplets only add pattern entries: adding +0.0 never changes a
    sum (up to the sign of zero), so they are left out of the summation.
    """
    key = rows * np.int64(max(n, 1)) + cols
    pattern = np.unique(key)
    nzm = vals != 0
    uk, us = _seq_group_sum(key[nzm], seq[nzm], vals[nzm])
    val = np.zeros(pattern.shape[0], dtype=vals.dtype)
    if uk.size:
        val[np.searchsorted(pattern, uk)] = us
    prow = pattern // max(n, 1)
    pcol = pattern % max(n, 1)
    row_ptr = np.zeros(n + 1, dtype=np.int64)
    np.add.at(row_ptr, prow + 1, 1)
    row_ptr = np.cumsum(row_ptr)
    return Csr(n, n, row_ptr, pcol.astype(np.int64), val)


def compile_circuit(ckt: ck.Circuit) -> MnaSystem:
    """Compile a circuit into an :class:`MnaSystem` (``src/compiler.rs:194-754``)."""
    kind = ckt.kind
    m = kind.shape[0]
    nodes = ckt.nodes

    # Step 1 (compiler.rs:196-235): node index = first appearance, ground excluded.
    three = (kind == ck.Q) | (kind == ck.M)
    term = nodes.copy()
    term[~three, 2] = -1
    flat = term.ravel()
    valid = flat > 0
    labels_seq = flat[valid]
    if labels_seq.size:
        uniq, first = np.unique(labels_seq, return_index=True)
        node_labels = uniq[np.argsort(first, kind="stable")]
    else:
        uniq = np.zeros(0, np.int64)
        node_labels = np.zeros(0, np.int64)
    n_nodes = int(node_labels.shape[0])
    # label -> matrix index
    lab_sorted = uniq
    idx_of_sorted = np.empty(lab_sorted.shape[0], dtype=np.int64)
    idx_of_sorted[np.searchsorted(lab_sorted, node_labels)] = np.arange(n_nodes)

    def nidx(lbl):
        lbl = np.asarray(lbl, np.int64)
        out = np.full(lbl.shape, -1, np.int64)
        ok = lbl > 0
        if ok.any():
            out[ok] = idx_of_sorted[np.searchsorted(lab_sorted, lbl[ok])]
        return out

    # Step 2 (compiler.rs:237-252): branches = V and L in component order.
    is_branch = (kind == ck.V) | (kind == ck.L)
    branch_components = np.flatnonzero(is_branch)
    n_br = int(branch_components.shape[0])
    size = n_nodes + n_br
    bk_of = np.full(m, -1, np.int64)
    bk_of[branch_components] = n_nodes + np.arange(n_br)

    # Validation (compiler.rs:310-316, 336-340).
    rmask = kind == ck.R
    if np.any(ckt.value[rmask] == 0.0):
        bad = int(np.flatnonzero(rmask & (ckt.value == 0.0))[0])
        raise CompileError(f"Resistor {_name(ckt, bad)} has zero resistance")
    cmask = kind == ck.C
    if np.any(ckt.value[cmask] < 0.0):
        bad = int(np.flatnonzero(cmask & (ckt.value < 0.0))[0])
        raise CompileError(f"Capacitor {_name(ckt, bad)} has negative capacitance")
    for kk, what in ((ck.D, "Diode"), (ck.Q, "BJT"), (ck.M, "MOSFET")):
        km = kind == kk
        if np.any(np.isnan(ckt.params[km, 0])):
            bad = int(np.flatnonzero(km & np.isnan(ckt.params[:, 0]))[0])
            raise CompileError(f"{what} {_name(ckt, bad)} references undefined model")

    ni = nidx(nodes[:, 0])
    nj = nidx(nodes[:, 1])
    nk = nidx(nodes[:, 2])
    comp = np.arange(m, dtype=np.int64)

    g_rows, g_cols, g_vals, g_seq = [], [], [], []
    c_rows, c_cols, c_vals, c_seq = [], [], [], []

    def push(lst, sel, r, c, v, sub):
        rows, cols, vals, seq = lst
        ok = sel & (r >= 0) & (c >= 0)
        rows.append(r[ok])
        cols.append(c[ok])
        vals.append(np.broadcast_to(v, sel.shape)[ok].astype(np.float64))
        seq.append(comp[ok] * 16 + sub)

    G = (g_rows, g_cols, g_vals, g_seq)
    Cm = (c_rows, c_cols, c_vals, c_seq)

    # Resistors (compiler.rs:310-330): (i,i,g) (j,j,g) (i,j,-g) (j,i,-g)
    with np.errstate(divide="ignore"):
        gcond = np.where(rmask, 1.0 / np.where(rmask, ckt.value, 1.0), 0.0)
    both = (ni >= 0) & (nj >= 0)
    push(G, rmask, ni, ni, gcond, 0)
    push(G, rmask, nj, nj, gcond, 1)
    push(G, rmask & both, ni, nj, -gcond, 2)
    push(G, rmask & both, nj, ni, -gcond, 3)
    # Capacitors (compiler.rs:332-355) into C.
    cap = np.where(cmask, ckt.value, 0.0)
    push(Cm, cmask, ni, ni, cap, 0)
    push(Cm, cmask, nj, nj, cap, 1)
    push(Cm, cmask & both, ni, nj, -cap, 2)
    push(Cm, cmask & both, nj, ni, -cap, 3)
    # Inductors and V sources (compiler.rs:357-408): KCL/KVL couplings.
    bk = bk_of
    push(G, is_branch, ni, bk, 1.0, 0)
    push(G, is_branch, bk, ni, 1.0, 1)
    push(G, is_branch, nj, bk, -1.0, 2)
    push(G, is_branch, bk, nj, -1.0, 3)
    lmask = kind == ck.L
    push(Cm, lmask, bk, bk, -np.where(lmask, ckt.value, 0.0), 4)
    # Diode placeholders (compiler.rs:427-437).
    dmask = kind == ck.D
    push(G, dmask, ni, ni, 0.0, 0)
    push(G, dmask, nj, nj, 0.0, 1)
    push(G, dmask & both, ni, nj, 0.0, 2)
    push(G, dmask & both, nj, ni, 0.0, 3)
    # BJT 3x3 placeholders (compiler.rs:489-497), rows/cols over (C, B, E).
    qmask = kind == ck.Q
    trip = (ni, nj, nk)
    for a in range(3):
        for b in range(3):
            push(G, qmask, trip[a], trip[b], 0.0, 4 + 3 * a + b)
    # MOSFET 6 placeholders (compiler.rs:533-542): rows (D, S) x cols (D, G, S).
    mmask = kind == ck.M
    for a, rr in enumerate((ni, nk)):
        for b, cc in enumerate((ni, nj, nk)):
            push(G, mmask, rr, cc, 0.0, 4 + 3 * a + b)

    # GMIN (compiler.rs:571-574) then the C-pattern zero fill (compiler.rs:576-579).
    diag = np.arange(n_nodes, dtype=np.int64)
    g_rows.append(diag)
    g_cols.append(diag)
    g_vals.append(np.full(n_nodes, GMIN))
    g_seq.append(np.int64(m) * 16 + diag * 0)
    cr = np.concatenate(c_rows) if c_rows else np.zeros(0, np.int64)
    cc_ = np.concatenate(c_cols) if c_cols else np.zeros(0, np.int64)
    g_rows.append(cr)
    g_cols.append(cc_)
    g_vals.append(np.zeros(cr.shape[0]))
    g_seq.append(np.full(cr.shape[0], (m + 1) * 16, np.int64))

    cat = lambda l: np.concatenate(l) if l else np.zeros(0, np.int64)  # noqa: E731
    g = _build_csr(size, cat(g_rows), cat(g_cols), np.concatenate(g_vals) if g_vals else np.zeros(0),
                   cat(g_seq))
    c = _build_csr(size, cat(c_rows), cat(c_cols), np.concatenate(c_vals) if c_vals else np.zeros(0),
                   cat(c_seq))

    # RHS (compiler.rs:391-398 V sources, 440-468 I sources).
    b_dc = np.zeros(size)
    vmask = kind == ck.V
    vdc = vmask & ~np.isnan(ckt.value)
    b_dc[bk[vdc]] = ckt.value[vdc]
    imask = kind == ck.I
    idc = np.flatnonzero(imask & ~np.isnan(ckt.value))
    if idc.size:
        ii = ni[idc]
        jj = nj[idc]
        val = ckt.value[idc]
        # interleave (b[i] -= I, b[j] += I) per source, in component order
        tgt = np.stack([ii, jj], axis=1).ravel()
        amt = np.stack([-val, val], axis=1).ravel()
        ok = tgt >= 0
        np.add.at(b_dc, tgt[ok], amt[ok])
    b_ac, sources = _ac_rhs_and_sources(ckt, ni, nj, bk, size)

    # V-source constrained nodes (compiler.rs:582-595).
    fixed = np.zeros(max(n_nodes, 1), dtype=bool)
    vs_i = ni[vmask]
    vs_j = nj[vmask]
    fixed[vs_i[vs_i >= 0]] = True
    fixed[vs_j[vs_j >= 0]] = True

    u32 = lambda a: np.where(a >= 0, a, SENTINEL).astype(np.uint32)  # noqa: E731
    fx = lambda a: np.where(a >= 0, fixed[np.maximum(a, 0)], False).astype(np.uint32)  # noqa: E731

    # Diode descriptors (compiler.rs:597-640).
    di = np.flatnonzero(dmask)
    dd = np.zeros(di.size, dtype=DIODE_DTYPE)
    a_, c_ = ni[di], nj[di]
    dd["anode"] = u32(a_)
    dd["cathode"] = u32(c_)
    dd["is_val"] = ckt.params[di, 0].astype(np.float32)
    dd["n_vt"] = (ckt.params[di, 1] * VT_300K).astype(np.float32)
    dd["g_row_col"] = np.stack([g.positions(a_, a_), g.positions(c_, c_),
                                g.positions(a_, c_), g.positions(c_, a_)], axis=1).astype(np.uint32)
    dd["b_idx"] = np.stack([u32(a_), u32(c_)], axis=1)

    # BJT descriptors (compiler.rs:642-690).
    qi = np.flatnonzero(qmask)
    qd = np.zeros(qi.size, dtype=BJT_DTYPE)
    tc, tb, te = ni[qi], nj[qi], nk[qi]
    qd["collector"], qd["base"], qd["emitter"] = u32(tc), u32(tb), u32(te)
    qd["polarity"] = np.where(ckt.params[qi, 5] != 0, 1.0, -1.0).astype(np.float32)
    qd["is_val"] = ckt.params[qi, 0].astype(np.float32)
    qd["bf"] = ckt.params[qi, 1].astype(np.float32)
    qd["br"] = ckt.params[qi, 2].astype(np.float32)
    qd["nf_vt"] = (ckt.params[qi, 3] * VT_300K).astype(np.float32)
    qd["nr_vt"] = (ckt.params[qi, 4] * VT_300K).astype(np.float32)
    qd["node_fixed"] = np.stack([fx(tc), fx(tb), fx(te)], axis=1)
    tri = (tc, tb, te)
    qd["g_row_col"] = np.stack([g.positions(tri[a], tri[b]) for a in range(3) for b in range(3)],
                               axis=1).astype(np.uint32)
    qd["b_idx"] = np.stack([u32(tc), u32(tb), u32(te)], axis=1)
    vaf = ckt.params[qi, 6].copy()
    vaf[np.isnan(vaf)] = np.inf

    # MOSFET descriptors (compiler.rs:692-740).
    mi = np.flatnonzero(mmask)
    md = np.zeros(mi.size, dtype=MOSFET_DTYPE)
    td, tg, ts = ni[mi], nj[mi], nk[mi]
    md["drain"], md["gate"], md["source"] = u32(td), u32(tg), u32(ts)
    md["polarity"] = np.where(ckt.params[mi, 3] != 0, 1.0, -1.0).astype(np.float32)
    md["vto"] = np.abs(ckt.params[mi, 0]).astype(np.float32)
    md["kp"] = ckt.params[mi, 1].astype(np.float32)
    md["lam"] = ckt.params[mi, 2].astype(np.float32)
    md["node_fixed_packed"] = fx(td) | (fx(tg) << 1) | (fx(ts) << 2)
    md["g_row_col"] = np.stack([g.positions(r, cc) for r in (td, ts) for cc in (td, tg, ts)],
                               axis=1).astype(np.uint32)
    md["b_idx"] = np.stack([u32(td), u32(ts)], axis=1)

    return MnaSystem(g=g, c=c, b_dc=b_dc, b_ac=b_ac, size=size, n_nodes=n_nodes,
                     node_labels=node_labels, branch_components=branch_components,
                     diode_descriptors=dd, bjt_descriptors=qd, mosfet_descriptors=md,
                     bjt_vaf=vaf, diode_components=di, bjt_components=qi,
                     mosfet_components=mi, sources=sources)


def _ac_rhs_and_sources(ckt: ck.Circuit, ni, nj, bk, size):
    """AC right-hand side (compiler.rs:391-398, 440-468: V sources at their
    branch rows, current sources -I / +I at their nodes in component order)
    and the time-dependent sources of the transient driver
    (transient.rs:232-262) as [(component, [(row, sign)], dc, tran)]."""
    kind = ckt.kind
    b_ac = np.zeros(size, dtype=np.complex128)
    vmask = kind == ck.V
    imask = kind == ck.I
    vac = vmask & ~np.isnan(ckt.ac[:, 0])
    if vac.any():
        b_ac[bk[vac]] = _ac_to_complex(ckt.ac[vac, 0], ckt.ac[vac, 1])
    iac = np.flatnonzero(imask & ~np.isnan(ckt.ac[:, 0]))
    if iac.size:
        z = _ac_to_complex(ckt.ac[iac, 0], ckt.ac[iac, 1])
        tgt = np.stack([ni[iac], nj[iac]], axis=1).ravel()
        amt = np.stack([-z, z], axis=1).ravel()
        ok = tgt >= 0
        np.add.at(b_ac, tgt[ok], amt[ok])
    sources = []
    for ci in np.flatnonzero(vmask | imask):
        ci = int(ci)
        if kind[ci] == ck.V:
            entries = [(int(bk[ci]), 1.0)]
        else:
            entries = [(int(x), sg) for x, sg in ((ni[ci], -1.0), (nj[ci], 1.0)) if x >= 0]
        dcv = None if np.isnan(ckt.value[ci]) else float(ckt.value[ci])
        sources.append((ci, entries, dcv, ckt.tran.get(ci)))
    return b_ac, sources


def system_from_device_compile(ckt: ck.Circuit, g: Csr, c: Csr, b_dc, node_labels, branch_components,
                               dd, qd, md) -> MnaSystem:
    """An :class:`MnaSystem` from the arrays of the device compile: the AC
    rhs, the source list and the per-kind index maps are filled in on the
    host (small, per-source work)."""
    n_nodes = int(node_labels.shape[0])
    size = n_nodes + int(branch_components.shape[0])
    order = np.argsort(node_labels, kind="stable")
    sorted_labels = node_labels[order]

    def nidx(lbl):
        lbl = np.asarray(lbl, np.int64)
        out = np.full(lbl.shape, -1, np.int64)
        ok = lbl > 0
        if ok.any() and n_nodes:
            out[ok] = order[np.searchsorted(sorted_labels, lbl[ok])]
        return out

    ni, nj = nidx(ckt.nodes[:, 0]), nidx(ckt.nodes[:, 1])
    bk = np.full(ckt.n_components, -1, np.int64)
    bk[branch_components] = n_nodes + np.arange(branch_components.shape[0])
    b_ac, sources = _ac_rhs_and_sources(ckt, ni, nj, bk, size)
    qi = np.flatnonzero(ckt.kind == ck.Q)
    vaf = ckt.params[qi, 6].copy()
    vaf[np.isnan(vaf)] = np.inf
    return MnaSystem(g=g, c=c, b_dc=b_dc, b_ac=b_ac, size=size, n_nodes=n_nodes,
                     node_labels=node_labels, branch_components=branch_components,
                     diode_descriptors=dd, bjt_descriptors=qd, mosfet_descriptors=md,
                     bjt_vaf=vaf, diode_components=np.flatnonzero(ckt.kind == ck.D), bjt_components=qi,
                     mosfet_components=np.flatnonzero(ckt.kind == ck.M), sources=sources)


def uic_system(ckt: ck.Circuit, sysm: MnaSystem):
    """The system of ``compute_uic_initial_conditions``
    (``src/analysis/transient.rs:364-482``): G and b_dc with every inductor
    branch row replaced by I_L = 0 and, per capacitor in component order,
    the first unconstrained terminal row replaced by V(i) - V(j) = 0
    (V(i) = 0 for a capacitor to ground); a node row is replaced once.
    Returns (values on G's pattern, rhs); its solution is the UIC start."""
    g = sysm.g
    vals = g.val.astype(np.float64).copy()
    b = sysm.b_dc.astype(np.float64).copy()
    rp = g.row_ptr

    def replace_row(r, entries):
        vals[int(rp[r]):int(rp[r + 1])] = 0.0
        for c, v in entries:
            k = g.value_index(r, c)
            if k is not None:
                vals[k] = v
        b[r] = 0.0

    branch_row = np.full(ckt.n_components, -1, np.int64)
    branch_row[sysm.branch_components] = sysm.n_nodes + np.arange(len(sysm.branch_components))
    for ci in np.flatnonzero(ckt.kind == ck.L):
        bk = int(branch_row[ci])
        replace_row(bk, [(bk, 1.0)])
    order = np.argsort(sysm.node_labels)
    sorted_labels = sysm.node_labels[order]

    def idx(label):
        if label == 0:
            return None
        k = int(np.searchsorted(sorted_labels, label))
        return int(order[k])

    constrained = np.zeros(sysm.n_nodes, dtype=bool)
    for ci in np.flatnonzero(ckt.kind == ck.C):
        i, j = idx(int(ckt.nodes[ci, 0])), idx(int(ckt.nodes[ci, 1]))
        if i is not None and j is None:
            if not constrained[i]:
                replace_row(i, [(i, 1.0)])
                constrained[i] = True
        elif i is None and j is not None:
            if not constrained[j]:
                replace_row(j, [(j, 1.0)])
                constrained[j] = True
        elif i is not None and j is not None:
            if not constrained[i]:
                replace_row(i, [(i, 1.0), (j, -1.0)])
                constrained[i] = True
            elif not constrained[j]:
                replace_row(j, [(j, 1.0), (i, -1.0)])
                constrained[j] = True
    return vals, b


def _ac_to_complex(mag, phase_deg):
    """``ac_to_complex`` (``src/compiler.rs:182-185``)."""
    ph = np.radians(phase_deg)
    return mag * np.cos(ph) + 1j * (mag * np.sin(ph))


def _name(ckt, idx):
    return ckt.names[idx] if ckt.names else f"#{idx}"
