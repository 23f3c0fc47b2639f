"""ohm_solve_real_noalloc: the linear solve for callers that cannot allocate
device memory (a host program that owns every device byte through its own
pool, or a latency-critical path where cudaMalloc/cudaFree would synchronise
or fail).  The caller owns the inputs and the output; the entry point works in
a fixed device array inside the library.

Checked through the C ABI against the allocating entry point ohm_solve_real,
on two calls in a row (the second must not see the first call's leftovers),
with every preconditioner it accepts run on a smaller system right after a
larger one, and on an empty matrix.  This file is collected last so a failure
here leaves every other test run.
"""
import ctypes as C

import numpy as np
import pytest

from ohmnivore_b200 import _lib
from ohmnivore_b200 import circuits as ck
from ohmnivore_b200 import mna
from ohmnivore_b200 import solver as S

pytestmark = pytest.mark.gpu


def _noalloc_call(n, row_ptr, col, vals, b, params):
    """One call through the C ABI on device copies of the arrays; col / vals
    may be empty, in which case NULL is passed for them."""
    import torch
    dev = torch.device("cuda", 0)
    rp = torch.from_numpy(np.asarray(row_ptr, np.uint32).view(np.int32).copy()).to(dev)   # u32 bit patterns
    ci = vv = None
    if len(col):
        ci = torch.from_numpy(np.asarray(col, np.uint32).view(np.int32).copy()).to(dev)
        vv = torch.from_numpy(np.ascontiguousarray(vals, np.float64)).to(dev)
    bb = torch.from_numpy(np.ascontiguousarray(b, np.float64)).to(dev)
    x = torch.full((n,), 123.0, dtype=torch.float64, device=dev)   # garbage in the output
    torch.cuda.synchronize()
    info = _lib.SolveInfo()
    p = params.to_c()
    ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None   # noqa: E731
    st = _lib.load().ohm_solve_real_noalloc(None, n, len(col), ptr(rp), ptr(ci), ptr(vv), ptr(bb), ptr(x),
                                            C.byref(p), C.byref(info))
    assert st == _lib.OK, _lib.last_error()
    return x.cpu().numpy(), info


def _noalloc_solve(sysm, b, params):
    return _noalloc_call(sysm.size, sysm.g.row_ptr, sysm.g.col, sysm.g.val, b, params)


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def _current_fed_ladder(n=300, seed=5):
    """A ladder fed by a 10 A current source: no zero diagonal, so plain and
    Jacobi BiCGSTAB converge without the 2x2 pairing."""
    rng = np.random.default_rng(seed)
    b = ck.CircuitBuilder()
    b.isource(0, 1, dc=10.0)
    k = np.arange(1, n, dtype=np.int64)
    b.resistors(k, k + 1, np.exp(rng.uniform(np.log(100.0), np.log(1e4), n - 1)))
    b.resistors(np.arange(1, n + 1, dtype=np.int64), 0, np.exp(rng.uniform(np.log(1e3), np.log(1e5), n)))
    return mna.compile_circuit(b.build())


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


def test_noalloc_every_precond_after_a_larger_system():
    """NONE and JACOBI right after a larger AUTO solve: the diagonal-slot
    table must be this call's, not the larger system's."""
    ctx = S.Context(0)
    try:
        big = mna.compile_circuit(ck.resistor_ladder(3000, seed=0))
        small = _current_fed_ladder()
        assert small.g.nnz < big.g.nnz and small.size < big.size
        for precond in (_lib.PRECOND_NONE, _lib.PRECOND_JACOBI, _lib.PRECOND_NONE):
            auto = S.BiCgStabParams(tolerance=1e-13)
            ref_big = S.GpuSolver(ctx, auto).solve_real(big.g, big.b_dc)
            got_big, _ = _noalloc_solve(big, big.b_dc, auto)          # the larger system first
            assert _rel(got_big[:big.n_nodes], ref_big[:big.n_nodes]) < 1e-9
            params = S.BiCgStabParams(tolerance=1e-12, precond=precond)
            ref = S.GpuSolver(ctx, params).solve_real(small.g, small.b_dc)
            got, info = _noalloc_solve(small, small.b_dc, params)
            assert _rel(got, ref) < 1e-9
            assert info.krylov_iterations > 0
    finally:
        ctx.close()


def test_noalloc_empty_matrix():
    """nnz = 0 with NULL column and value pointers: b = 0 gives x = 0, as
    ohm_solve_real does, even after a larger system left its tables behind."""
    ctx = S.Context(0)
    try:
        big = mna.compile_circuit(ck.resistor_ladder(3000, seed=0))
        _noalloc_solve(big, big.b_dc, S.BiCgStabParams(tolerance=1e-12))
        n = 5
        rp = np.zeros(n + 1, np.uint32)
        for precond in (_lib.PRECOND_NONE, _lib.PRECOND_JACOBI, _lib.PRECOND_AUTO):
            params = S.BiCgStabParams(precond=precond)
            got, _ = _noalloc_call(n, rp, np.zeros(0, np.uint32), np.zeros(0), np.zeros(n), params)
            assert np.all(got == 0.0)
            x = np.full(n, 7.0)
            info = _lib.SolveInfo()
            p = params.to_c()
            st = ctx.lib.ohm_solve_real(ctx.handle, n, 0, S.u32ptr(rp), None, None, S.dptr(np.zeros(n)),
                                        S.dptr(x), C.byref(p), C.byref(info))
            assert st == _lib.OK, _lib.last_error()
            assert np.all(x == got)
    finally:
        ctx.close()


def test_noalloc_mixed_precision_twice():
    ctx = S.Context(0)
    try:
        params = S.BiCgStabParams(tolerance=1e-14, precision=1, max_refinements=20, fp32_max_iterations=10_000)
        sysm = mna.compile_circuit(ck.resistor_ladder(2000, seed=4))
        solver = S.GpuSolver(ctx, params)
        ref = solver.solve_real(sysm.g, sysm.b_dc)
        assert solver.last_info["fp64_fallbacks"] == 0
        for scale in (1.0, -2.5):                             # two calls in a row
            got, info = _noalloc_solve(sysm, scale * sysm.b_dc, params)
            nn = slice(0, sysm.n_nodes)
            assert _rel(got[nn], scale * ref[nn]) < 1e-9
            assert info.fp64_fallbacks == 0                   # the FP32 bulk did the work
    finally:
        ctx.close()


def test_noalloc_rejects_oversize():
    x = np.zeros(1)
    p = S.BiCgStabParams().to_c()
    st = _lib.load().ohm_solve_real_noalloc(None, 40000, 100000, None, None, None, None,
                                            C.c_void_p(x.ctypes.data), C.byref(p), None)
    assert st == _lib.ERR_INVALID_ARG
    assert "exceeds the fixed scratch limit" in _lib.last_error()
