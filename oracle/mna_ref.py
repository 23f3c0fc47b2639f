"""ORACLE (test infrastructure only): plain-Python restatement of the
reference's MNA compiler and CSR builder.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may use this module, and only as the checker.  It is never part of the
product path.

Follows, statement by statement:
  * ``src/compiler.rs:194-754``  ``compile``: node/branch numbering, stamps,
    GMIN, C-pattern zero fill, descriptor resolution;
  * ``src/sparse.rs:51-104``     ``CsrMatrix::from_triplets`` (stable sort by
    (row, col), duplicates summed left to right);
  * ``src/sparse.rs:27-31``      ``value_index`` (linear scan in the row).

Pure Python loops: use for circuits up to a few hundred thousand triplets.
"""
from __future__ import annotations

import math

import numpy as np

VT_300K = 0.02585
GMIN = 1e-12
SENTINEL = 0xFFFFFFFF
R, C, L, V, I, D, Q, M = range(8)


def f32(x: float) -> float:
    """``x as f32`` then back to f64 (round to nearest even)."""
    return float(np.float32(x))


class RefCsr:
    def __init__(self, nrows, ncols, values, col_indices, row_pointers):
        self.nrows, self.ncols = nrows, ncols
        self.values, self.col_indices, self.row_pointers = values, col_indices, row_pointers

    @staticmethod
    def from_triplets(nrows, ncols, triplets):
        """``CsrMatrix::from_triplets`` (src/sparse.rs:51-104)."""
        if not triplets:
            return RefCsr(nrows, ncols, [], [], [0] * (nrows + 1))
        idx = sorted(range(len(triplets)), key=lambda i: (triplets[i][0], triplets[i][1]))
        values, cols = [], []
        rp = [0] * (nrows + 1)
        r0, c0, v0 = triplets[idx[0]]
        for i in idx[1:]:
            r, c, v = triplets[i]
            if r == r0 and c == c0:
                v0 = v0 + v
            else:
                values.append(v0)
                cols.append(c0)
                rp[r0 + 1] += 1
                r0, c0, v0 = r, c, v
        values.append(v0)
        cols.append(c0)
        rp[r0 + 1] += 1
        for i in range(1, nrows + 1):
            rp[i] += rp[i - 1]
        return RefCsr(nrows, ncols, values, cols, rp)

    def value_index(self, row, col):
        """src/sparse.rs:27-31."""
        for i in range(self.row_pointers[row], self.row_pointers[row + 1]):
            if self.col_indices[i] == col:
                return i
        return None

    def to_dense(self):
        d = np.zeros((self.nrows, self.ncols), dtype=np.result_type(*(self.values or [0.0])))
        for r in range(self.nrows):
            for i in range(self.row_pointers[r], self.row_pointers[r + 1]):
                d[r, self.col_indices[i]] = self.values[i]
        return d


def compile_ref(ckt):
    """Restatement of ``compile`` (src/compiler.rs:194-754) over a column-form
    circuit (see ``ohmnivore_b200.circuits.Circuit``).  Returns a dict."""
    kind = [int(k) for k in ckt.kind]
    nodes = [[int(v) for v in row] for row in ckt.nodes]
    m = len(kind)

    node_map, node_names = {}, []

    def reg(lbl):
        if lbl <= 0:          # ground ("0"/"GND") or unused terminal
            return
        if lbl not in node_map:
            node_map[lbl] = len(node_names)
            node_names.append(lbl)

    for k in range(m):                               # compiler.rs:213-233
        if kind[k] in (Q, M):
            reg(nodes[k][0]); reg(nodes[k][1]); reg(nodes[k][2])
        else:
            reg(nodes[k][0]); reg(nodes[k][1])
    n_nodes = len(node_names)
    branch_map, branch_comp = {}, []
    for k in range(m):                               # compiler.rs:241-250
        if kind[k] in (V, L):
            branch_map[k] = len(branch_comp)
            branch_comp.append(k)
    size = n_nodes + len(branch_comp)

    def ni(lbl):
        return None if lbl <= 0 else node_map.get(lbl)

    g_t, c_t = [], []
    b_dc = [0.0] * size
    b_ac = [0j] * size
    pend_d, pend_q, pend_m = [], [], []
    for k in range(m):
        t = kind[k]
        a, b = ni(nodes[k][0]), ni(nodes[k][1])
        val = float(ckt.value[k])
        if t == R:                                   # compiler.rs:310-330
            if val == 0.0:
                raise ValueError("zero resistance")
            g = 1.0 / val
            if a is not None: g_t.append((a, a, g))
            if b is not None: g_t.append((b, b, g))
            if a is not None and b is not None:
                g_t.append((a, b, -g)); g_t.append((b, a, -g))
        elif t == C:                                 # compiler.rs:332-355
            if val < 0.0:
                raise ValueError("negative capacitance")
            if a is not None: c_t.append((a, a, val))
            if b is not None: c_t.append((b, b, val))
            if a is not None and b is not None:
                c_t.append((a, b, -val)); c_t.append((b, a, -val))
        elif t in (L, V):                            # compiler.rs:357-408
            bk = n_nodes + branch_map[k]
            if a is not None: g_t.append((a, bk, 1.0)); g_t.append((bk, a, 1.0))
            if b is not None: g_t.append((b, bk, -1.0)); g_t.append((bk, b, -1.0))
            if t == L:
                c_t.append((bk, bk, -val))
            else:
                if not math.isnan(val):
                    b_dc[bk] = val
                mag, ph = float(ckt.ac[k, 0]), float(ckt.ac[k, 1])
                if not math.isnan(mag):
                    r = ph * (math.pi / 180.0)
                    b_ac[bk] = complex(mag * math.cos(r), mag * math.sin(r))
        elif t == D:                                 # compiler.rs:412-447
            if a is not None: g_t.append((a, a, 0.0))
            if b is not None: g_t.append((b, b, 0.0))
            if a is not None and b is not None:
                g_t.append((a, b, 0.0)); g_t.append((b, a, 0.0))
            p = ckt.params[k]
            pend_d.append((a, b, f32(p[0]), f32(p[1] * VT_300K)))
        elif t == I:                                 # compiler.rs:449-477
            if not math.isnan(val):
                if a is not None: b_dc[a] -= val
                if b is not None: b_dc[b] += val
            mag, ph = float(ckt.ac[k, 0]), float(ckt.ac[k, 1])
            if not math.isnan(mag):
                r = ph * (math.pi / 180.0)
                z = complex(mag * math.cos(r), mag * math.sin(r))
                if a is not None: b_ac[a] -= z
                if b is not None: b_ac[b] += z
        elif t == Q:                                 # compiler.rs:479-515
            e = ni(nodes[k][2])
            tri = [a, b, e]
            for r_ in tri:
                for c_ in tri:
                    if r_ is not None and c_ is not None:
                        g_t.append((r_, c_, 0.0))
            p = ckt.params[k]
            pend_q.append((a, b, e, 1.0 if p[5] != 0 else -1.0, f32(p[0]), f32(p[1]), f32(p[2]),
                           f32(p[3] * VT_300K), f32(p[4] * VT_300K)))
        elif t == M:                                 # compiler.rs:519-566
            s = ni(nodes[k][2])
            for r_ in (a, s):
                for c_ in (a, b, s):
                    if r_ is not None and c_ is not None:
                        g_t.append((r_, c_, 0.0))
            p = ckt.params[k]
            pend_m.append((a, b, s, 1.0 if p[3] != 0 else -1.0, f32(abs(p[0])), f32(p[1]),
                           f32(p[2])))
    for i in range(n_nodes):                         # compiler.rs:571-574
        g_t.append((i, i, GMIN))
    for (r_, c_, _) in c_t:                          # compiler.rs:576-579
        g_t.append((r_, c_, 0.0))
    g = RefCsr.from_triplets(size, size, g_t)
    c = RefCsr.from_triplets(size, size, c_t)

    fixed = set()                                    # compiler.rs:582-595
    for k in range(m):
        if kind[k] == V:
            for lbl in nodes[k][:2]:
                x = ni(lbl)
                if x is not None:
                    fixed.add(x)

    S = SENTINEL
    u = lambda x: S if x is None else x  # noqa: E731
    vi = lambda r_, c_: S if (r_ is None or c_ is None) else u(g.value_index(r_, c_))  # noqa: E731
    diodes = [dict(anode=u(a), cathode=u(b), is_val=is_, n_vt=nvt,
                   g_row_col=[vi(a, a), vi(b, b), vi(a, b), vi(b, a)], b_idx=[u(a), u(b)])
              for (a, b, is_, nvt) in pend_d]
    bjts = []
    for (cc, bb, ee, pol, is_, bf, br, nfv, nrv) in pend_q:
        tri = [cc, bb, ee]
        bjts.append(dict(collector=u(cc), base=u(bb), emitter=u(ee), polarity=pol, is_val=is_,
                         bf=bf, br=br, nf_vt=nfv, nr_vt=nrv,
                         node_fixed=[int(x is not None and x in fixed) for x in tri],
                         g_row_col=[vi(r_, c_) for r_ in tri for c_ in tri],
                         b_idx=[u(cc), u(bb), u(ee)]))
    mos = []
    for (dd, gg, ss, pol, vto, kp, lam) in pend_m:
        fxb = lambda x: int(x is not None and x in fixed)  # noqa: E731
        mos.append(dict(drain=u(dd), gate=u(gg), source=u(ss), polarity=pol, vto=vto, kp=kp,
                        lam=lam, node_fixed_packed=fxb(dd) | (fxb(gg) << 1) | (fxb(ss) << 2),
                        g_row_col=[vi(r_, c_) for r_ in (dd, ss) for c_ in (dd, gg, ss)],
                        b_idx=[u(dd), u(ss)]))
    return dict(g=g, c=c, b_dc=b_dc, b_ac=b_ac, size=size, n_nodes=n_nodes,
                node_labels=node_names, branch_components=branch_comp,
                diodes=diodes, bjts=bjts, mosfets=mos)
