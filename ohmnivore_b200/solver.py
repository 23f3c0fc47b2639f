"""Host-side mirror of the reference's solver interfaces over the C ABI.

  ``LinearSolver`` / ``GpuSolver.solve_real``   src/solver/mod.rs:27-34, gpu.rs:107-208
  ``SolverBackend`` (buffers, spmv, dot, ...)   src/solver/backend.rs:51-96
  ``BiCgStabParams``                            src/solver/bicgstab.rs:14-27
  ``NewtonParams``, ``newton_solve``            src/solver/newton.rs:34-78
  error taxonomy                                src/error.rs:4-33

Every call goes through ``libohm_b200.so``; nothing here computes on the CPU.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib, mna
from ._lib import dptr, u32ptr, vptr

DEFAULT_MAX_ITERATIONS = 10_000   # bicgstab.rs:10
DEFAULT_TOLERANCE = 1e-5          # bicgstab.rs:11


class OhmnivoreError(RuntimeError):
    """Base of the error taxonomy (src/error.rs:4-33)."""


class CompileError(OhmnivoreError):
    pass


class SolveError(OhmnivoreError):
    def __init__(self, msg, krylov_code=None):
        super().__init__(msg)
        self.krylov_code = krylov_code


class NewtonNotConverged(OhmnivoreError):
    def __init__(self, msg, iterations, max_residual, x=None):
        super().__init__(msg)
        self.iterations = iterations
        self.max_residual = max_residual
        self.x = x


class NewtonNumericalError(OhmnivoreError):
    def __init__(self, msg, iteration):
        super().__init__(msg)
        self.iteration = iteration


class DeviceTimeout(OhmnivoreError):
    pass


class InvalidArgument(OhmnivoreError, ValueError):
    pass


class TimestepError(OhmnivoreError):
    """``OhmnivoreError::Timestep``: the adaptive step control gave up."""


def _raise(st, info=None, x=None):
    msg = _lib.last_error()
    if st == _lib.ERR_SOLVE:
        raise SolveError(msg, None if info is None else info.krylov_code)
    if st == _lib.ERR_NEWTON_NOT_CONVERGED:
        raise NewtonNotConverged(msg, 0 if info is None else info.iterations,
                                 0.0 if info is None else info.max_residual, x)
    if st == _lib.ERR_NEWTON_NUMERICAL:
        raise NewtonNumericalError(msg, 0 if info is None else info.error_iteration)
    if st == _lib.ERR_COMPILE:
        raise CompileError(msg)
    if st == _lib.ERR_TIMEOUT:
        raise DeviceTimeout(msg)
    if st == _lib.ERR_INVALID_ARG:
        raise InvalidArgument(msg)
    if st == _lib.ERR_TIMESTEP:
        raise TimestepError(msg)
    raise OhmnivoreError(f"status {st}: {msg}")


@dataclass
class BiCgStabParams:
    """``BiCgStabParams`` (bicgstab.rs:14-27) plus the B200 extensions."""
    max_iterations: int = DEFAULT_MAX_ITERATIONS
    tolerance: float = DEFAULT_TOLERANCE
    precision: int = _lib.PREC_FP64
    precond: int = _lib.PRECOND_AUTO
    inner_rtol: float = 0.0
    max_refinements: int = 1
    max_restarts: int = 50
    fp32_max_iterations: int = 600
    fp32_min_eta_exp: int = 0

    def to_c(self) -> _lib.KrylovParams:
        p = _lib.KrylovParams()
        _lib.load().ohm_krylov_params_default(C.byref(p))
        p.max_iterations = int(self.max_iterations)
        p.tolerance = float(self.tolerance)
        p.precision = int(self.precision)
        p.precond = int(self.precond)
        p.inner_rtol = float(self.inner_rtol)
        p.max_refinements = int(self.max_refinements)
        p.max_restarts = int(self.max_restarts)
        p.fp32_max_iterations = int(self.fp32_max_iterations)
        p.fp32_min_eta_exp = int(self.fp32_min_eta_exp)
        return p


@dataclass
class NewtonParams:
    """``NewtonParams`` (newton.rs:34-55) plus extensions (rel_tol, precision)."""
    max_iterations: int = 50
    abs_tol: float = 1e-4
    bicgstab_max_iterations: int = DEFAULT_MAX_ITERATIONS
    initial_guess: np.ndarray | None = None
    rel_tol: float = 0.0
    bicgstab_tolerance: float = DEFAULT_TOLERANCE
    precision: int = _lib.PREC_FP64
    precond: int = _lib.PRECOND_AUTO
    inner_rtol: float = 0.0
    forcing: int = 0              # 0 constant inner_rtol, 1 Eisenstat-Walker
    eta_max: float = 0.5
    fp32_max_iterations: int = 600
    fp32_min_eta_exp: int = 0     # mixed: inner tolerances below 10^-k go straight to FP64 (0 = off)
    continuation: int = 0         # 1: reference DC strategy on failure (src/analysis/dc.rs:60-290);
                                  # | CONT_TEST_PSEUDO (testing): force the pseudo-transient stage
    n_nodes: int = 0              # node rows; filled from the system by NewtonPlan / NewtonBatch

    def to_c(self):
        p = _lib.NewtonParamsC()
        _lib.load().ohm_newton_params_default(C.byref(p))
        p.max_iterations = int(self.max_iterations)
        p.abs_tol = float(self.abs_tol)
        p.rel_tol = float(self.rel_tol)
        p.krylov = BiCgStabParams(self.bicgstab_max_iterations, self.bicgstab_tolerance,
                                  self.precision, self.precond, self.inner_rtol,
                                  fp32_max_iterations=self.fp32_max_iterations,
                                  fp32_min_eta_exp=self.fp32_min_eta_exp).to_c()
        p.forcing = int(self.forcing)
        p.eta_max = float(self.eta_max)
        p.continuation = int(self.continuation)
        p.n_nodes = int(self.n_nodes)
        keep = None
        if self.initial_guess is not None:
            keep = np.ascontiguousarray(self.initial_guess, dtype=np.float64)
            p.initial_guess = dptr(keep)
        return p, keep


class Context:
    """One CUDA device + stream (``WgpuDsBackend::new``)."""

    def __init__(self, device: int = 0):
        lib = _lib.load()
        h = C.c_void_p()
        st = lib.ohm_ctx_create(int(device), C.byref(h))
        if st != _lib.OK:
            _raise(st)
        self._h = h
        self.lib = lib

    @property
    def handle(self):
        return self._h

    def synchronize(self):
        st = self.lib.ohm_ctx_synchronize(self._h)
        if st:
            _raise(st)

    def set_krylov_layout(self, layout: int):
        """Where single-system Krylov solves keep their working set:
        ``_lib.KRYLOV_LAYOUT_AUTO`` (each block's slice in shared memory where
        it fits, else global memory) or ``KRYLOV_LAYOUT_GLOBAL`` (global
        memory for every block, the path of large systems, at any size)."""
        st = self.lib.ohm_ctx_set_krylov_layout(self._h, int(layout))
        if st:
            _raise(st)

    def close(self):
        if getattr(self, "_h", None):
            self.lib.ohm_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_DEFAULT_CTX = None


def default_context() -> Context:
    global _DEFAULT_CTX
    if _DEFAULT_CTX is None:
        _DEFAULT_CTX = Context(0)
    return _DEFAULT_CTX


def _csr_u32(a):
    rp = np.ascontiguousarray(a.row_ptr, dtype=np.uint32)
    ci = np.ascontiguousarray(a.col, dtype=np.uint32)
    return rp, ci


class GpuSolver:
    """``LinearSolver`` implementation (src/solver/gpu.rs:107-208)."""

    def __init__(self, ctx: Context | None = None, params: BiCgStabParams | None = None):
        self.ctx = ctx or default_context()
        self.params = params or BiCgStabParams()
        self.last_info = None

    def solve_real(self, a, b, params: BiCgStabParams | None = None) -> np.ndarray:
        n = int(a.nrows)
        if a.ncols != n or len(b) != n:
            raise SolveError(f"dimension mismatch: matrix is {a.nrows}x{a.ncols}, rhs length is {len(b)}")
        if n == 0:
            return np.zeros(0)
        rp, ci = _csr_u32(a)
        val = np.ascontiguousarray(a.val, dtype=np.float64)
        bb = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(n)
        info = _lib.SolveInfo()
        p = (params or self.params).to_c()
        st = self.ctx.lib.ohm_solve_real(self.ctx.handle, n, len(ci), u32ptr(rp), u32ptr(ci), dptr(val),
                                         dptr(bb), dptr(x), C.byref(p), C.byref(info))
        self.last_info = info.as_dict()
        if st != _lib.OK:
            _raise(st, info)
        return x

    def solve_complex(self, a, b, params: BiCgStabParams | None = None) -> np.ndarray:
        """``LinearSolver::solve_complex`` (src/solver/gpu.rs:210-735) through
        ``ohm_solve_complex``: complex FP64 BiCGSTAB, ||r|| < tol ||b||."""
        n = int(a.nrows)
        if a.ncols != n or len(b) != n:
            raise SolveError(f"dimension mismatch: matrix is {a.nrows}x{a.ncols}, rhs length is {len(b)}")
        if n == 0:
            return np.zeros(0, dtype=np.complex128)
        rp, ci = _csr_u32(a)
        val = np.asarray(a.val, dtype=np.complex128)
        v = np.ascontiguousarray(np.stack([val.real, val.imag], axis=1).reshape(-1))
        bc = np.asarray(b, dtype=np.complex128)
        bb = np.ascontiguousarray(np.stack([bc.real, bc.imag], axis=1).reshape(-1))
        x = np.zeros(2 * n)
        info = _lib.AcPointInfo()
        p = (params or self.params).to_c()
        st = self.ctx.lib.ohm_solve_complex(self.ctx.handle, n, len(ci), u32ptr(rp), u32ptr(ci), dptr(v), dptr(bb),
                                            dptr(x), C.byref(p), C.byref(info))
        self.last_info = info.as_dict()
        if st != _lib.OK:
            _raise(st, info)
        return x[0::2] + 1j * x[1::2]


def newton_solve(ctx, base_g_values, col_indices, row_ptrs, base_b, diode_descriptors,
                 bjt_descriptors, mosfet_descriptors, system_size, matrix_nnz,
                 params: NewtonParams | None = None, stats: dict | None = None) -> np.ndarray:
    """``newton_solve`` (src/solver/newton.rs:65-78), same argument order.

    Descriptor arrays are numpy structured arrays with the reference byte
    layout (``ohmnivore_b200.mna.DIODE_DTYPE`` etc.).  Returns x (FP64).
    """
    ctx = ctx or default_context()
    params = params or NewtonParams()
    vals = np.ascontiguousarray(base_g_values, dtype=np.float64)
    ci = np.ascontiguousarray(col_indices, dtype=np.uint32)
    rp = np.ascontiguousarray(row_ptrs, dtype=np.uint32)
    bb = np.ascontiguousarray(base_b, dtype=np.float64)
    dd = np.ascontiguousarray(diode_descriptors)
    qd = np.ascontiguousarray(bjt_descriptors)
    md = np.ascontiguousarray(mosfet_descriptors)
    x = np.zeros(int(system_size))
    info = _lib.SolveInfo()
    p, keep = params.to_c()
    st = ctx.lib.ohm_newton_solve(ctx.handle, dptr(vals), u32ptr(ci), u32ptr(rp), dptr(bb),
                                  vptr(dd), len(dd), vptr(qd), len(qd), vptr(md), len(md),
                                  int(system_size), int(matrix_nnz), C.byref(p), dptr(x),
                                  C.byref(info))
    del keep
    if stats is not None:
        stats.update(info.as_dict())
    if st != _lib.OK:
        _raise(st, info, x)
    return x


class NewtonPlan:
    """Device-resident nonlinear system: uploads once, solves many times."""

    def __init__(self, sysm, ctx: Context | None = None, base_vals=None, base_b=None):
        self.ctx = ctx or default_context()
        self.sysm = sysm
        self.n = int(sysm.size)
        self.nnz = int(sysm.g.nnz)
        vals = np.ascontiguousarray(sysm.g.val if base_vals is None else base_vals, dtype=np.float64)
        rp, ci = _csr_u32(sysm.g)
        bb = np.ascontiguousarray(sysm.b_dc if base_b is None else base_b, dtype=np.float64)
        dd = np.ascontiguousarray(sysm.diode_descriptors)
        qd = np.ascontiguousarray(sysm.bjt_descriptors)
        md = np.ascontiguousarray(sysm.mosfet_descriptors)
        vaf = None
        if len(qd) and sysm.bjt_vaf is not None and np.any(np.isfinite(sysm.bjt_vaf)):
            vaf = np.ascontiguousarray(sysm.bjt_vaf, dtype=np.float64)
        h = C.c_void_p()
        st = self.ctx.lib.ohm_plan_create(self.ctx.handle, dptr(vals), u32ptr(ci), u32ptr(rp), dptr(bb),
                                          vptr(dd), len(dd), vptr(qd), len(qd), vptr(md), len(md),
                                          None if vaf is None else dptr(vaf), self.n, self.nnz,
                                          C.byref(h))
        if st != _lib.OK:
            _raise(st)
        self._h = h
        self.last_info = None

    def close(self):
        if getattr(self, "_h", None):
            self.ctx.lib.ohm_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_base(self, base_vals=None, base_b=None):
        v = None if base_vals is None else np.ascontiguousarray(base_vals, dtype=np.float64)
        b = None if base_b is None else np.ascontiguousarray(base_b, dtype=np.float64)
        st = self.ctx.lib.ohm_plan_set_base(self._h, None if v is None else dptr(v),
                                            None if b is None else dptr(b))
        if st:
            _raise(st)

    def newton_device(self, x_dev_ptr: int, params: NewtonParams | None = None) -> dict:
        """Run Newton on a device vector (raw CUDA pointer, e.g. torch ``data_ptr()``)."""
        p, keep = (params or NewtonParams()).to_c()
        if p.continuation and p.n_nodes <= 0:
            p.n_nodes = int(self.sysm.n_nodes)
        info = _lib.SolveInfo()
        st = self.ctx.lib.ohm_plan_newton_device(self._h, C.c_void_p(int(x_dev_ptr)), C.byref(p),
                                                 C.byref(info))
        del keep
        self.last_info = info.as_dict()
        if st != _lib.OK:
            _raise(st, info)
        return self.last_info

    def trace(self):
        """Per-Newton-iteration record of the last newton_device call (rows x 6)."""
        out = np.zeros((256, 6))
        rows = C.c_int32()
        st = self.ctx.lib.ohm_plan_trace(self._h, dptr(out), 256, C.byref(rows))
        if st:
            _raise(st)
        t = out[: rows.value]
        keep = ~np.all(np.isnan(t), axis=1)
        return t[keep]

    def assemble(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        vals = np.zeros(self.nnz)
        rhs = np.zeros(self.n)
        st = self.ctx.lib.ohm_plan_assemble(self._h, dptr(x), dptr(vals), dptr(rhs))
        if st:
            _raise(st)
        return vals, rhs

    def limit(self, x_old, x_new):
        xo = np.ascontiguousarray(x_old, dtype=np.float64)
        xn = np.array(x_new, dtype=np.float64, copy=True)
        st = self.ctx.lib.ohm_plan_limit(self._h, dptr(xo), dptr(xn))
        if st:
            _raise(st)
        return xn


class NewtonBatch:
    """Many independent nonlinear systems (``MnaSystem`` each) packed into one
    block-diagonal CSR and solved by one launch, one thread block per system.

    The reference solves one circuit per ``newton_solve`` call
    (src/solver/newton.rs:62-430); every instance here runs that loop.
    ``row_off`` gives each instance's rows in the packed solution vector.
    """

    def __init__(self, systems, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        systems = list(systems)
        if not systems:
            raise InvalidArgument("empty batch")
        self.n_instances = len(systems)
        sizes = np.array([int(s.size) for s in systems], dtype=np.int64)
        nnzs = np.array([int(s.g.nnz) for s in systems], dtype=np.int64)
        self.row_off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        self.nnz_off = np.concatenate([[0], np.cumsum(nnzs)]).astype(np.int64)
        self.rows = int(self.row_off[-1])
        rp = np.concatenate([np.asarray(s.g.row_ptr, dtype=np.uint32) for s in systems])
        ci = np.concatenate([np.asarray(s.g.col, dtype=np.uint32) for s in systems])
        vals = np.concatenate([np.asarray(s.g.val, dtype=np.float64) for s in systems])
        bb = np.concatenate([np.asarray(s.b_dc, dtype=np.float64) for s in systems])

        def pack(attr):
            parts = [np.ascontiguousarray(getattr(s, attr)) for s in systems]
            off = np.concatenate([[0], np.cumsum([len(p) for p in parts])]).astype(np.int64)
            return np.ascontiguousarray(np.concatenate(parts)), off

        dd, doff = pack("diode_descriptors")
        qd, qoff = pack("bjt_descriptors")
        md, moff = pack("mosfet_descriptors")
        vaf = None
        if len(qd):
            v = [np.full(len(s.bjt_descriptors), np.inf) if s.bjt_vaf is None else np.asarray(s.bjt_vaf, dtype=np.float64)
                 for s in systems]
            v = np.ascontiguousarray(np.concatenate(v))
            if np.any(np.isfinite(v)):
                vaf = v
        rp = np.ascontiguousarray(rp)
        ci = np.ascontiguousarray(ci)
        self.n_nodes = np.array([int(s.n_nodes) for s in systems], dtype=np.int32)
        h = C.c_void_p()
        st = self.ctx.lib.ohm_batch_create(
            self.ctx.handle, self.n_instances, vptr(self.row_off), vptr(self.nnz_off), u32ptr(rp), u32ptr(ci),
            dptr(vals), dptr(bb), vptr(doff), vptr(dd), vptr(qoff), vptr(qd),
            None if vaf is None else dptr(vaf), vptr(moff), vptr(md), vptr(self.n_nodes), C.byref(h))
        if st != _lib.OK:
            _raise(st)
        self._h = h
        self.last_info = None

    def close(self):
        if getattr(self, "_h", None):
            self.ctx.lib.ohm_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def split(self, x):
        """Per-instance views of a packed solution vector."""
        return [x[self.row_off[i]:self.row_off[i + 1]] for i in range(self.n_instances)]

    def newton_device(self, x_dev_ptr: int, params: NewtonParams | None = None, check: bool = True) -> dict:
        """Newton on every instance over the packed device vector ``x_dev_ptr``
        (``rows`` doubles, initial guess in, solution out)."""
        p, keep = (params or NewtonParams()).to_c()
        info = _lib.SolveInfo()
        st = self.ctx.lib.ohm_batch_newton_device(self._h, C.c_void_p(int(x_dev_ptr)), C.byref(p),
                                                  C.byref(info))
        del keep
        self.last_info = info.as_dict()
        if st != _lib.OK and check:
            _raise(st, info)
        return self.last_info

    def autotune(self, params: NewtonParams | None = None, sample_size: int = 0) -> dict:
        """Pick the fastest kernel variant on a sample of the batch (kept for
        later ``newton_device`` calls)."""
        p, keep = (params or NewtonParams()).to_c()
        lpr, tpb, bps = C.c_int32(), C.c_int32(), C.c_int32()
        ms = C.c_double()
        st = self.ctx.lib.ohm_batch_autotune(self._h, C.byref(p), int(sample_size), C.byref(lpr), C.byref(tpb),
                                             C.byref(bps), C.byref(ms))
        del keep
        if st:
            _raise(st)
        return {"lanes_per_row": lpr.value, "threads_per_block": tpb.value, "blocks_per_sm": bps.value,
                "sample_ms": ms.value}

    def set_kernel(self, lanes_per_row: int, threads_per_block: int, blocks_per_sm: int):
        st = self.ctx.lib.ohm_batch_set_kernel(self._h, int(lanes_per_row), int(threads_per_block),
                                               int(blocks_per_sm))
        if st:
            _raise(st)

    def set_split(self, on: bool):
        """Solve the circuits that would set a call's time alone on the whole
        GPU before the batch kernel takes the rest (default on)."""
        st = self.ctx.lib.ohm_batch_set_split(self._h, 1 if on else 0)
        if st:
            _raise(st)

    def instance_info(self):
        arr = (_lib.SolveInfo * self.n_instances)()
        st = self.ctx.lib.ohm_batch_instance_info(self._h, arr, self.n_instances)
        if st:
            _raise(st)
        return [a.as_dict() for a in arr]


def ac_frequencies(sweep: str, n_points: int, f_start: float, f_stop: float) -> np.ndarray:
    """Frequency points of an AC sweep (``generate_frequencies``,
    src/analysis/ac.rs:80-109): DEC / OCT points per decade / octave from
    f_start, ceil(n_points * decades) of them; LIN n_points from f_start to
    f_stop."""
    kind = sweep.lower()
    if kind == "dec":
        total = int(np.ceil(n_points * np.log10(f_stop / f_start)))
        return np.array([f_start * 10.0 ** (i / n_points) for i in range(total)])
    if kind == "oct":
        total = int(np.ceil(n_points * np.log2(f_stop / f_start)))
        return np.array([f_start * 2.0 ** (i / n_points) for i in range(total)])
    if kind == "lin":
        if n_points <= 1:
            return np.array([f_start])
        step = (f_stop - f_start) / (n_points - 1)
        return np.array([f_start + step * i for i in range(n_points)])
    raise InvalidArgument(f"unknown sweep type {sweep!r}")


def ac_sweep(sysm, freqs, params: BiCgStabParams | None = None, ctx: Context | None = None, g_values=None):
    """``analysis::ac::run`` over the given frequency points, all points in one
    launch.  Returns (x: n_freq x size complex, per-point info)."""
    ctx = ctx or default_context()
    params = params or BiCgStabParams()
    n = int(sysm.size)
    rp, ci = _csr_u32(sysm.g)
    g = np.ascontiguousarray(sysm.g.val if g_values is None else g_values, dtype=np.float64)
    cv = c_on_g_pattern(sysm)
    b = np.ascontiguousarray(np.stack([sysm.b_ac.real, sysm.b_ac.imag], axis=1).reshape(-1))
    f = np.ascontiguousarray(freqs, dtype=np.float64)
    x = np.zeros(2 * n * len(f))
    pts = (_lib.AcPointInfo * max(1, len(f)))()
    p = params.to_c()
    st = ctx.lib.ohm_ac_sweep(ctx.handle, n, len(ci), u32ptr(rp), u32ptr(ci), dptr(g), dptr(cv), dptr(b), len(f),
                              dptr(f), C.byref(p), dptr(x), pts)
    infos = [pts[k].as_dict() for k in range(len(f))]
    if st != _lib.OK:
        _raise(st)
    xr = x.reshape(len(f), n, 2)
    return xr[..., 0] + 1j * xr[..., 1], infos


def c_on_g_pattern(sysm) -> np.ndarray:
    """C values placed on G's pattern (the compiler zero-fills G with C's
    pattern, src/compiler.rs:576-579)."""
    g, c = sysm.g, sysm.c
    n = np.int64(max(int(sysm.size), 1))
    gk = np.repeat(np.arange(g.nrows, dtype=np.int64), np.diff(g.row_ptr)) * n + g.col
    ck = np.repeat(np.arange(c.nrows, dtype=np.int64), np.diff(c.row_ptr)) * n + c.col
    pos = np.searchsorted(gk, ck)
    ok = (pos < len(gk)) & (gk[np.minimum(pos, len(gk) - 1)] == ck) if len(gk) else np.zeros(len(ck), bool)
    if not np.all(ok):
        k = int(np.flatnonzero(~ok)[0])
        raise CompileError(f"capacitance entry ({ck[k] // n}, {ck[k] % n}) is not on the conductance pattern")
    out = np.zeros(g.nnz)
    out[pos] = c.val
    return out


class ComponentTable:
    """Resistors and capacitors of a circuit as system rows (-1 = ground) and
    values, in circuit order (the parameters the adjoint differentiates)."""

    def __init__(self, ckt, sysm):
        from . import circuits as ck
        labels = np.asarray(sysm.node_labels, dtype=np.int64)
        order = np.argsort(labels, kind="stable")
        sl = labels[order]

        def rows(lab):
            lab = np.asarray(lab, dtype=np.int64)
            if not len(sl):
                return np.full(lab.shape, -1, np.int32)
            pos = np.minimum(np.searchsorted(sl, lab), len(sl) - 1)
            ok = (lab != 0) & (sl[pos] == lab)
            return np.where(ok, order[pos], -1).astype(np.int32)

        r = np.flatnonzero(ckt.kind == ck.R)
        c = np.flatnonzero(ckt.kind == ck.C)
        self.r_index, self.c_index = r, c
        self.r_a, self.r_b = rows(ckt.nodes[r, 0]), rows(ckt.nodes[r, 1])
        self.r_ohms = np.ascontiguousarray(ckt.value[r], dtype=np.float64)
        self.c_a, self.c_b = rows(ckt.nodes[c, 0]), rows(ckt.nodes[c, 1])
        self.c_farads = np.ascontiguousarray(ckt.value[c], dtype=np.float64)

    def to_c(self):
        return _lib.Components(len(self.r_ohms), vptr(self.r_a), vptr(self.r_b), vptr(self.r_ohms),
                               len(self.c_farads), vptr(self.c_a), vptr(self.c_b), vptr(self.c_farads))


def adjoint_dc(plan: "NewtonPlan", x_dev_ptr: int, w, comps: ComponentTable, params: BiCgStabParams | None = None):
    """do/dp of o = w . x at the DC operating point x (device pointer) for
    every resistor, diode Is and MOSFET |VTO| and KP (the descriptor values:
    the threshold magnitude, and KP with W/L folded in).
    Returns (dict of gradients, lambda, info)."""
    kp = (params or BiCgStabParams(max_iterations=20000, tolerance=1e-14)).to_c()
    w = np.ascontiguousarray(w, dtype=np.float64)
    gr = np.zeros(len(comps.r_ohms))
    gd = np.zeros(len(plan.sysm.diode_descriptors))
    nm = len(plan.sysm.mosfet_descriptors)
    gvto, gkp = np.zeros(nm), np.zeros(nm)
    lam = np.zeros(plan.n)
    info = _lib.AdjointInfo()
    cc = comps.to_c()
    opt = lambda a: dptr(a) if len(a) else None   # noqa: E731
    st = plan.ctx.lib.ohm_plan_adjoint_dc(plan._h, C.c_void_p(int(x_dev_ptr)), dptr(w), C.byref(cc), C.byref(kp),
                                          opt(gr), opt(gd), opt(gvto), opt(gkp), dptr(lam), C.byref(info))
    if st != _lib.OK:
        _raise(st)
    return {"R": gr, "Is": gd, "VTO": gvto, "KP": gkp}, lam, info.as_dict()


def compile_circuit_device(ckt, ctx: Context | None = None) -> "mna.MnaSystem":
    """``compile`` (src/compiler.rs:194-754) on the GPU (``ohm_compile``):
    the same :class:`mna.MnaSystem` as ``mna.compile_circuit``, bit for bit.
    Raises ``mna.CompileError`` for the reference's compile errors."""
    ctx = ctx or default_context()
    m = ckt.n_components
    kind = np.ascontiguousarray(ckt.kind, dtype=np.int32)
    nodes = np.ascontiguousarray(ckt.nodes, dtype=np.int64).reshape(m, 3)
    value = np.ascontiguousarray(ckt.value, dtype=np.float64)
    params = np.ascontiguousarray(ckt.params, dtype=np.float64).reshape(m, 7)
    h = C.c_void_p()
    st = ctx.lib.ohm_compile(ctx.handle, m, kind.ctypes.data_as(C.POINTER(C.c_int32)),
                             nodes.ctypes.data_as(C.POINTER(C.c_int64)), dptr(value), dptr(params), C.byref(h))
    if st == _lib.ERR_COMPILE:
        raise mna.CompileError(_lib.last_error())
    if st != _lib.OK:
        _raise(st)
    try:
        z = _lib.NetlistSizes()
        st = ctx.lib.ohm_netlist_get_sizes(h, C.byref(z))
        if st != _lib.OK:
            _raise(st)
        n = int(z.size)
        g_rp = np.zeros(n + 1, np.uint32)
        g_col = np.zeros(z.g_nnz, np.uint32)
        g_val = np.zeros(z.g_nnz)
        c_rp = np.zeros(n + 1, np.uint32)
        c_col = np.zeros(z.c_nnz, np.uint32)
        c_val = np.zeros(z.c_nnz)
        b_dc = np.zeros(n)
        labels = np.zeros(z.n_nodes, np.int64)
        branches = np.zeros(z.n_branches, np.int64)
        dd = np.zeros(z.n_diodes, dtype=mna.DIODE_DTYPE)
        qd = np.zeros(z.n_bjts, dtype=mna.BJT_DTYPE)
        md = np.zeros(z.n_mosfets, dtype=mna.MOSFET_DTYPE)
        i64 = lambda a: a.ctypes.data_as(C.POINTER(C.c_int64))  # noqa: E731
        st = ctx.lib.ohm_netlist_download(h, u32ptr(g_rp), u32ptr(g_col), dptr(g_val), u32ptr(c_rp), u32ptr(c_col),
                                          dptr(c_val), dptr(b_dc), i64(labels), i64(branches),
                                          C.c_void_p(dd.ctypes.data), C.c_void_p(qd.ctypes.data),
                                          C.c_void_p(md.ctypes.data))
        if st != _lib.OK:
            _raise(st)
    finally:
        ctx.lib.ohm_netlist_destroy(h)
    g = mna.Csr(n, n, g_rp.astype(np.int64), g_col.astype(np.int64), g_val)
    c = mna.Csr(n, n, c_rp.astype(np.int64), c_col.astype(np.int64), c_val)
    return mna.system_from_device_compile(ckt, g, c, b_dc, labels, branches, dd, qd, md)


def uic_initial_conditions(ckt, sysm, params: BiCgStabParams | None = None, ctx: Context | None = None):
    """x(0) of a transient with UIC: the solution of ``mna.uic_system`` by
    the GPU BiCGSTAB (compute_uic_initial_conditions,
    src/analysis/transient.rs:364-482)."""
    vals, b = mna.uic_system(ckt, sysm)
    a = mna.Csr(sysm.size, sysm.size, sysm.g.row_ptr, sysm.g.col, vals)
    return GpuSolver(ctx or default_context(), params or BiCgStabParams(tolerance=1e-14)).solve_real(a, b)


def pack_sources(sysm):
    """``ohm_source`` records and PWL points for the sources of an MnaSystem
    (``collect_source_info``, src/analysis/transient.rs:212-262): a source
    with a transient function (kind, params) uses it, otherwise its DC value."""
    srcs = np.zeros(len(sysm.sources), dtype=_lib.SOURCE_DTYPE)
    pwl = []
    for k, (_, entries, dc, tran) in enumerate(sysm.sources):
        rec = srcs[k]
        rec["n_rows"] = len(entries)
        for j, (row, sign) in enumerate(entries):
            rec["rows"][j] = row
            rec["sign"][j] = sign
        rec["dc"] = 0.0 if dc is None else dc
        if tran is None:
            rec["kind"] = -1
        else:
            kind, params = tran
            rec["kind"] = int(kind)
            if int(kind) == 2:                       # PWL: (t, v) pairs
                pts = np.asarray(params, dtype=np.float64).reshape(-1, 2)
                rec["pwl_offset"] = len(pwl)
                rec["pwl_count"] = len(pts)
                pwl.extend(map(tuple, pts))
            else:
                p = np.zeros(7)
                p[: len(params)] = params
                rec["p"] = p
    pts = np.ascontiguousarray(np.asarray(pwl, dtype=np.float64).reshape(-1))
    return srcs, pts


class Transient:
    """Fixed-step backward-Euler transient with a Newton solve per step on a
    :class:`NewtonPlan` (companion system of src/analysis/transient.rs:285-333
    plus device evaluation); every step runs on the device."""

    def __init__(self, plan: NewtonPlan, probes=()):
        self.plan = plan
        self.ctx = plan.ctx
        sysm = plan.sysm
        c = sysm.c
        rp = np.ascontiguousarray(c.row_ptr, dtype=np.uint32)
        ci = np.ascontiguousarray(c.col, dtype=np.uint32)
        cv = np.ascontiguousarray(c.val, dtype=np.float64)
        self.sources, self.pwl = pack_sources(sysm)
        self.probes = np.ascontiguousarray(probes, dtype=np.uint32)
        h = C.c_void_p()
        st = self.ctx.lib.ohm_transient_create(
            plan._h, len(cv), u32ptr(rp), u32ptr(ci), dptr(cv) if len(cv) else None, vptr(self.sources),
            len(self.sources), dptr(self.pwl) if len(self.pwl) else None, len(self.pwl) // 2,
            u32ptr(self.probes) if len(self.probes) else None, len(self.probes), C.byref(h))
        if st != _lib.OK:
            _raise(st)
        self._h = h
        self.last_info = None

    def close(self):
        if getattr(self, "_h", None):
            self.ctx.lib.ohm_transient_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def adjoint(self, x0_dev_ptr: int, t0: float, h: float, n_steps: int, w, comps: ComponentTable,
                params: NewtonParams | None = None, checkpoint_every: int = 50,
                krylov: BiCgStabParams | None = None):
        """do/dp of o = w . x(t0 + n_steps h) for every resistor, capacitor,
        diode Is and MOSFET |VTO| and KP (the DC start x0 included).  x0 is
        left unchanged.  Returns (dict of gradients, info)."""
        p, keep = (params or NewtonParams()).to_c()
        kp = (krylov or BiCgStabParams(max_iterations=20000, tolerance=1e-14)).to_c()
        w = np.ascontiguousarray(w, dtype=np.float64)
        gr = np.zeros(len(comps.r_ohms))
        gc = np.zeros(len(comps.c_farads))
        gd = np.zeros(len(self.plan.sysm.diode_descriptors))
        nm = len(self.plan.sysm.mosfet_descriptors)
        gvto, gkp = np.zeros(nm), np.zeros(nm)
        info = _lib.AdjointInfo()
        cc = comps.to_c()
        opt = lambda a: dptr(a) if len(a) else None   # noqa: E731
        st = self.ctx.lib.ohm_transient_adjoint(self._h, C.c_void_p(int(x0_dev_ptr)), float(t0), float(h),
                                                int(n_steps), int(checkpoint_every), C.byref(p), dptr(w),
                                                C.byref(cc), C.byref(kp), opt(gr), opt(gc), opt(gd), opt(gvto),
                                                opt(gkp), C.byref(info))
        del keep
        if st != _lib.OK:
            _raise(st)
        return {"R": gr, "C": gc, "Is": gd, "VTO": gvto, "KP": gkp}, info.as_dict()

    def set_predictor(self, order: int):
        """Newton start of each fixed step after the first: 0 = x_{n-1}, 1 = the
        linear extrapolation 2 x_{n-1} - x_{n-2}, 2 = the quadratic
        3 x_{n-1} - 3 x_{n-2} + x_{n-3} (same BE solution, usually fewer
        Newton iterations)."""
        st = self.ctx.lib.ohm_transient_set_predictor(self._h, int(order))
        if st != _lib.OK:
            _raise(st)

    def run(self, x_dev_ptr: int, t0: float, h: float, n_steps: int, params: NewtonParams | None = None,
            steps_per_launch: int = 100, graph: bool = True, check: bool = True):
        """Advance x (device pointer, x(t0) in, x(t0 + n_steps h) out).
        Returns the probe waveforms (n_steps x n_probes)."""
        p, keep = (params or NewtonParams()).to_c()
        wave = np.zeros((int(n_steps), len(self.probes)))
        info = _lib.TransientInfo()
        st = self.ctx.lib.ohm_transient_run(self._h, C.c_void_p(int(x_dev_ptr)), float(t0), float(h), int(n_steps),
                                            int(steps_per_launch), C.byref(p), 1 if graph else 0,
                                            dptr(wave) if wave.size else None, C.byref(info))
        del keep
        self.last_info = info.as_dict()
        if st != _lib.OK and check:
            _raise(st)
        return wave

    def run_adaptive(self, x_dev_ptr: int, tstep: float, tstop: float, tstart: float = 0.0,
                     params: NewtonParams | None = None, max_points: int | None = None, check: bool = True):
        """The reference's adaptive BE / TRAP transient (transient::run,
        src/analysis/transient.rs:77-178) from t = 0 to tstop on the device:
        x (device pointer) holds x(0) and receives the last accepted state.
        Returns (times, waveforms n_points x n_probes).  ``max_points``
        defaults to 8 tstop / tstep + 2; a run that produced more points
        returns the first max_points and reports the total in
        ``last_info["points"]``."""
        if max_points is None:
            ok = tstep > 0 and np.isfinite(tstop) and tstop >= 0
            max_points = int(8 * np.ceil(tstop / tstep)) + 2 if ok else 2   # bad values: the C call rejects them
        p, keep = (params or NewtonParams()).to_c()
        times = np.zeros(int(max_points))
        wave = np.zeros((int(max_points), len(self.probes)))
        info = _lib.AdaptiveInfo()
        st = self.ctx.lib.ohm_transient_run_adaptive(self._h, C.c_void_p(int(x_dev_ptr)), float(tstep), float(tstop),
                                                     float(tstart), C.byref(p), int(max_points),
                                                     dptr(times) if times.size else None,
                                                     dptr(wave) if wave.size else None, C.byref(info))
        del keep
        self.last_info = info.as_dict()
        if st != _lib.OK and check:
            _raise(st)
        kept = min(info.points, int(max_points))
        return times[:kept], wave[:kept]


class DeviceBuffer:
    """``SolverBackend::Buffer``: FP64 device vector."""

    def __init__(self, ctx: Context, n: int):
        self.ctx, self.n = ctx, int(n)
        h = C.c_void_p()
        st = ctx.lib.ohm_buf_create(ctx.handle, self.n, C.byref(h))
        if st:
            _raise(st)
        self._h = h

    def upload(self, host):
        a = np.ascontiguousarray(host, dtype=np.float64)
        st = self.ctx.lib.ohm_buf_upload(self.ctx.handle, self._h, dptr(a), len(a))
        if st:
            _raise(st)

    def download(self) -> np.ndarray:
        out = np.zeros(self.n)
        st = self.ctx.lib.ohm_buf_download(self.ctx.handle, self._h, dptr(out), self.n)
        if st:
            _raise(st)
        return out

    def close(self):
        if getattr(self, "_h", None):
            self.ctx.lib.ohm_buf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DeviceCsr:
    """``GpuCsrMatrix``."""

    def __init__(self, ctx: Context, a):
        self.ctx, self.n, self.nnz = ctx, int(a.nrows), int(a.nnz)
        rp, ci = _csr_u32(a)
        val = np.ascontiguousarray(a.val, dtype=np.float64)
        h = C.c_void_p()
        st = ctx.lib.ohm_csr_upload(ctx.handle, self.n, self.nnz, u32ptr(rp), u32ptr(ci), dptr(val),
                                    C.byref(h))
        if st:
            _raise(st)
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self.ctx.lib.ohm_csr_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SolverBackend:
    """``SolverBackend`` trait operations (backend.rs:51-96) on device buffers."""

    def __init__(self, ctx: Context | None = None):
        self.ctx = ctx or default_context()

    def new_buffer(self, n):
        return DeviceBuffer(self.ctx, n)

    def upload_matrix(self, a):
        return DeviceCsr(self.ctx, a)

    def _chk(self, st):
        if st:
            _raise(st)

    def spmv(self, a: DeviceCsr, x: DeviceBuffer, y: DeviceBuffer):
        self._chk(self.ctx.lib.ohm_spmv(self.ctx.handle, a._h, x._h, y._h))

    def dot(self, a: DeviceBuffer, b: DeviceBuffer) -> float:
        out = C.c_double()
        self._chk(self.ctx.lib.ohm_dot(self.ctx.handle, a._h, b._h, C.byref(out)))
        return out.value

    def dot_n(self, a: DeviceBuffer, b: DeviceBuffer, n: int) -> float:
        """``dot_n`` (backend.rs:60-68): the dot product over the first n entries."""
        out = C.c_double()
        self._chk(self.ctx.lib.ohm_dot_n(self.ctx.handle, a._h, b._h, int(n), C.byref(out)))
        return out.value

    def axpy(self, alpha, x, y):
        self._chk(self.ctx.lib.ohm_axpy(self.ctx.handle, float(alpha), x._h, y._h))

    def copy(self, src, dst):
        self._chk(self.ctx.lib.ohm_copy(self.ctx.handle, src._h, dst._h))

    def scale(self, alpha, x):
        self._chk(self.ctx.lib.ohm_scale(self.ctx.handle, float(alpha), x._h))

    def solve_real_device(self, a: DeviceCsr, b: DeviceBuffer, x: DeviceBuffer,
                          params: BiCgStabParams | None = None) -> dict:
        p = (params or BiCgStabParams()).to_c()
        info = _lib.SolveInfo()
        st = self.ctx.lib.ohm_solve_real_device(self.ctx.handle, a._h, b._h, x._h, C.byref(p),
                                                C.byref(info))
        if st:
            _raise(st, info)
        return info.as_dict()
