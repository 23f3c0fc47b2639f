"""ORACLE (test infrastructure only): the reference's AC sweep restated with a
direct complex sparse LU per frequency point.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may use this module, and only as the checker / timed CPU baseline.

  ``form_complex_matrix``  A = G + j w C from triplets (src/sparse.rs:149-178)
  ``generate_frequencies`` DEC / OCT / LIN points (src/analysis/ac.rs:80-109)
  ``ac_sweep``             per point: w = 2 pi f, solve A x = b_ac
                           (ac.rs:56-70, with the CPU direct solve of
                           src/solver/cpu.rs instead of the GPU BiCGSTAB)
"""
from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spl


def form_complex_matrix(sysm, omega):
    n = sysm.size
    g, c = sysm.g, sysm.c
    gr = np.repeat(np.arange(n), np.diff(g.row_ptr))
    cr = np.repeat(np.arange(n), np.diff(c.row_ptr))
    rows = np.concatenate([gr, cr])
    cols = np.concatenate([g.col, c.col])
    vals = np.concatenate([g.val.astype(np.complex128), 1j * omega * c.val])
    return sp.csr_matrix((vals, (rows, cols)), shape=(n, n))    # duplicates are summed


def generate_frequencies(kind, n_points, f_start, f_stop):
    if kind == "dec":
        total = math.ceil(n_points * math.log10(f_stop / f_start))
        return [f_start * 10.0 ** (i / n_points) for i in range(total)]
    if kind == "oct":
        total = math.ceil(n_points * math.log2(f_stop / f_start))
        return [f_start * 2.0 ** (i / n_points) for i in range(total)]
    if n_points <= 1:
        return [f_start]
    step = (f_stop - f_start) / (n_points - 1)
    return [f_start + step * i for i in range(n_points)]


def ac_sweep(sysm, freqs):
    out = np.zeros((len(freqs), sysm.size), dtype=np.complex128)
    for k, f in enumerate(freqs):
        a = form_complex_matrix(sysm, 2.0 * math.pi * f).tocsc()
        out[k] = spl.splu(a).solve(np.asarray(sysm.b_ac, dtype=np.complex128))
    return out
