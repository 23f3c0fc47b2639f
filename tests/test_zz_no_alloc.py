"""ohm_solve_real_noalloc: the linear solve for callers that cannot allocate
device memory (a host program that owns every device byte through its own
pool, or a latency-critical path where cudaMalloc/cudaFree would synchronise
or fail).  The caller owns the inputs and the output; the entry point works in
a fixed device array inside the library.

Checked through the C ABI against the allocating entry point ohm_solve_real,
on two calls in a row (the second must not see the first call's leftovers).
This file is collected last so a failure here leaves every other test run.
"""
import ctypes as C

import numpy as np
import pytest

from ohmnivore_b200 import _lib
from ohmnivore_b200 import circuits as ck
from ohmnivore_b200 import mna
from ohmnivore_b200 import solver as S

pytestmark = pytest.mark.gpu


def _noalloc_solve(sysm, b, params):
    import torch
    dev = torch.device("cuda", 0)
    rp = torch.from_numpy(sysm.g.row_ptr.astype(np.int32)).to(dev)      # u32 bit patterns
    ci = torch.from_numpy(sysm.g.col.astype(np.int32)).to(dev)
    vals = torch.from_numpy(np.ascontiguousarray(sysm.g.val, np.float64)).to(dev)
    bb = torch.from_numpy(np.ascontiguousarray(b, np.float64)).to(dev)
    x = torch.full((sysm.size,), 123.0, dtype=torch.float64, device=dev)  # garbage in the output
    torch.cuda.synchronize()
    info = _lib.SolveInfo()
    p = params.to_c()
    st = _lib.load().ohm_solve_real_noalloc(None, sysm.size, sysm.g.nnz, C.c_void_p(rp.data_ptr()),
                                            C.c_void_p(ci.data_ptr()), C.c_void_p(vals.data_ptr()),
                                            C.c_void_p(bb.data_ptr()), C.c_void_p(x.data_ptr()),
                                            C.byref(p), C.byref(info))
    assert st == _lib.OK, _lib.last_error()
    return x.cpu().numpy(), info


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def test_noalloc_matches_allocating_entry_point_twice():
    ctx = S.Context(0)
    try:
        params = S.BiCgStabParams(tolerance=1e-13)
        cases = [mna.compile_circuit(ck.resistor_ladder(3000, seed=0)),
                 mna.compile_circuit(ck.diode_mesh(40, 40, seed=2, diode_frac=0.0))]
        for sysm in cases:                                   # two calls in a row
            b = sysm.b_dc
            ref = S.GpuSolver(ctx, params).solve_real(sysm.g, b)
            got, info = _noalloc_solve(sysm, b, params)
            nn = slice(0, sysm.n_nodes)
            assert _rel(got[nn], ref[nn]) < 1e-9
            assert info.kernel_launches >= 1
    finally:
        ctx.close()


def test_noalloc_mixed_precision_twice():
    ctx = S.Context(0)
    try:
        params = S.BiCgStabParams(tolerance=1e-14, precision=1, max_refinements=20)
        sysm = mna.compile_circuit(ck.resistor_ladder(2000, seed=4))
        ref = S.GpuSolver(ctx, params).solve_real(sysm.g, sysm.b_dc)
        for scale in (1.0, -2.5):                             # two calls in a row
            got, _ = _noalloc_solve(sysm, scale * sysm.b_dc, params)
            nn = slice(0, sysm.n_nodes)
            assert _rel(got[nn], scale * ref[nn]) < 1e-9
    finally:
        ctx.close()


def test_noalloc_rejects_oversize():
    x = np.zeros(1)
    p = S.BiCgStabParams().to_c()
    st = _lib.load().ohm_solve_real_noalloc(None, 40000, 100000, None, None, None, None,
                                            C.c_void_p(x.ctypes.data), C.byref(p), None)
    assert st == _lib.ERR_INVALID_ARG
    assert "exceeds the fixed scratch limit" in _lib.last_error()
