"""ctypes binding of ``libohm_b200.so`` (declared in ``include/ohm.h``).

The shared library is built in-tree by ``ohmnivore_b200/csrc/Makefile``.
There is no fallback: importing the solver without the library raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libohm_b200.so")

# ohm_status
OK, ERR_SOLVE, ERR_NEWTON_NOT_CONVERGED, ERR_NEWTON_NUMERICAL, ERR_COMPILE, ERR_TIMEOUT, \
    ERR_INVALID_ARG, ERR_CUDA, ERR_TIMESTEP = range(9)
PREC_FP64, PREC_MIXED = 0, 1
PRECOND_AUTO, PRECOND_JACOBI, PRECOND_ISAI1, PRECOND_NONE = 0, 1, 2, 3
CONT_ON, CONT_TEST_PSEUDO = 1, 2   # ohm_newton_params.continuation bits
KRYLOV_LAYOUT_AUTO, KRYLOV_LAYOUT_GLOBAL = 0, 1   # ohm_ctx_set_krylov_layout


class KrylovParams(C.Structure):
    _fields_ = [("max_iterations", C.c_int32), ("tolerance", C.c_double), ("precision", C.c_int32),
                ("precond", C.c_int32), ("inner_rtol", C.c_double), ("max_refinements", C.c_int32),
                ("max_restarts", C.c_int32), ("fp32_max_iterations", C.c_int32),
                ("fp32_min_eta_exp", C.c_int32)]


class Components(C.Structure):
    _fields_ = [("n_resistors", C.c_int64), ("r_a", C.c_void_p), ("r_b", C.c_void_p), ("r_ohms", C.c_void_p),
                ("n_capacitors", C.c_int64), ("c_a", C.c_void_p), ("c_b", C.c_void_p), ("c_farads", C.c_void_p)]


class AdjointInfo(C.Structure):
    _fields_ = [("status", C.c_int32), ("steps", C.c_int32), ("linear_solves", C.c_int32),
                ("recompute_launches", C.c_int32), ("krylov_iterations", C.c_int64), ("output", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class AcPointInfo(C.Structure):
    _fields_ = [("krylov_code", C.c_int32), ("iterations", C.c_int32), ("restarts", C.c_int32),
                ("reserved", C.c_int32), ("residual_norm", C.c_double), ("b_norm", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class TransientInfo(C.Structure):
    _fields_ = [("status", C.c_int32), ("steps_done", C.c_int32), ("failed_step", C.c_int32),
                ("krylov_code", C.c_int32), ("newton_iterations", C.c_int64), ("krylov_iterations", C.c_int64),
                ("fp64_fallbacks", C.c_int32), ("launches", C.c_int32), ("graph", C.c_int32),
                ("reserved", C.c_int32), ("max_residual", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class AdaptiveInfo(C.Structure):
    _fields_ = [("status", C.c_int32), ("accepted", C.c_int32), ("rejected", C.c_int32), ("points", C.c_int32),
                ("newton_iterations", C.c_int64), ("krylov_iterations", C.c_int64),
                ("linear_solves", C.c_int32), ("fp64_fallbacks", C.c_int32), ("krylov_code", C.c_int32),
                ("failed_solve", C.c_int32), ("t_end", C.c_double), ("h_last", C.c_double),
                ("t_failed", C.c_double), ("max_residual", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class NetlistSizes(C.Structure):
    _fields_ = [(k, C.c_int64) for k in ("n_nodes", "size", "n_branches", "g_nnz", "c_nnz", "n_diodes",
                                          "n_bjts", "n_mosfets")]


# ohm_source (include/ohm.h), 104 bytes
SOURCE_DTYPE = np.dtype([("kind", "<i4"), ("n_rows", "<i4"), ("rows", "<u4", (2,)), ("sign", "<f8", (2,)),
                         ("dc", "<f8"), ("p", "<f8", (7,)), ("pwl_offset", "<i4"), ("pwl_count", "<i4")],
                        align=True)


class NewtonParamsC(C.Structure):
    _fields_ = [("max_iterations", C.c_int32), ("abs_tol", C.c_double), ("rel_tol", C.c_double),
                ("krylov", KrylovParams), ("initial_guess", C.POINTER(C.c_double)),
                ("forcing", C.c_int32), ("eta_max", C.c_double), ("continuation", C.c_int32),
                ("n_nodes", C.c_int32)]


class SolveInfo(C.Structure):
    _fields_ = [("status", C.c_int32), ("krylov_code", C.c_int32), ("iterations", C.c_int32),
                ("error_iteration", C.c_int32), ("krylov_iterations", C.c_int64),
                ("fp64_fallbacks", C.c_int32), ("krylov_restarts", C.c_int32),
                ("max_residual", C.c_double), ("final_residual_norm", C.c_double),
                ("b_norm", C.c_double), ("kernel_launches", C.c_int64),
                ("continuation_steps", C.c_int32), ("continuation_kind", C.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_vp = C.c_void_p
_i64 = C.c_int64
_dp = C.POINTER(C.c_double)
_u32p = C.POINTER(C.c_uint32)

# name -> (restype, argtypes)
SIGNATURES = {
    "ohm_last_error": (C.c_char_p, []),
    "ohm_version": (C.c_char_p, []),
    "ohm_krylov_params_default": (None, [C.POINTER(KrylovParams)]),
    "ohm_newton_params_default": (None, [C.POINTER(NewtonParamsC)]),
    "ohm_ctx_create": (C.c_int, [C.c_int, C.POINTER(_vp)]),
    "ohm_ctx_destroy": (C.c_int, [_vp]),
    "ohm_ctx_synchronize": (C.c_int, [_vp]),
    "ohm_ctx_stream": (_vp, [_vp]),
    "ohm_ctx_set_krylov_layout": (C.c_int, [_vp, C.c_int32]),
    "ohm_batch_set_split": (C.c_int, [_vp, C.c_int32]),
    "ohm_buf_create": (C.c_int, [_vp, _i64, C.POINTER(_vp)]),
    "ohm_buf_destroy": (C.c_int, [_vp]),
    "ohm_buf_upload": (C.c_int, [_vp, _vp, _dp, _i64]),
    "ohm_buf_download": (C.c_int, [_vp, _vp, _dp, _i64]),
    "ohm_buf_device_ptr": (_vp, [_vp]),
    "ohm_csr_upload": (C.c_int, [_vp, _i64, _i64, _u32p, _u32p, _dp, C.POINTER(_vp)]),
    "ohm_csr_update_values": (C.c_int, [_vp, _vp, _dp, _i64]),
    "ohm_csr_destroy": (C.c_int, [_vp]),
    "ohm_spmv": (C.c_int, [_vp, _vp, _vp, _vp]),
    "ohm_dot": (C.c_int, [_vp, _vp, _vp, _dp]),
    "ohm_dot_n": (C.c_int, [_vp, _vp, _vp, _i64, _dp]),
    "ohm_axpy": (C.c_int, [_vp, C.c_double, _vp, _vp]),
    "ohm_copy": (C.c_int, [_vp, _vp, _vp]),
    "ohm_scale": (C.c_int, [_vp, C.c_double, _vp]),
    "ohm_solve_real": (C.c_int, [_vp, _i64, _i64, _u32p, _u32p, _dp, _dp, _dp,
                                 C.POINTER(KrylovParams), C.POINTER(SolveInfo)]),
    "ohm_solve_real_device": (C.c_int, [_vp, _vp, _vp, _vp, C.POINTER(KrylovParams),
                                        C.POINTER(SolveInfo)]),
    "ohm_solve_real_noalloc": (C.c_int, [_vp, _i64, _i64, _vp, _vp, _vp, _vp, _vp,
                                         C.POINTER(KrylovParams), C.POINTER(SolveInfo)]),
    "ohm_newton_solve": (C.c_int, [_vp, _dp, _u32p, _u32p, _dp, _vp, _i64, _vp, _i64, _vp, _i64,
                                   _i64, _i64, C.POINTER(NewtonParamsC), _dp, C.POINTER(SolveInfo)]),
    "ohm_plan_create": (C.c_int, [_vp, _dp, _u32p, _u32p, _dp, _vp, _i64, _vp, _i64, _vp, _i64, _dp,
                                  _i64, _i64, C.POINTER(_vp)]),
    "ohm_plan_destroy": (C.c_int, [_vp]),
    "ohm_plan_set_base": (C.c_int, [_vp, _dp, _dp]),
    "ohm_plan_newton_device": (C.c_int, [_vp, _vp, C.POINTER(NewtonParamsC), C.POINTER(SolveInfo)]),
    "ohm_plan_download_system": (C.c_int, [_vp, _dp, _dp]),
    "ohm_plan_assemble": (C.c_int, [_vp, _dp, _dp, _dp]),
    "ohm_plan_limit": (C.c_int, [_vp, _dp, _dp]),
    "ohm_plan_trace": (C.c_int, [_vp, _dp, C.c_int32, C.POINTER(C.c_int32)]),
    "ohm_batch_create": (C.c_int, [_vp, _i64, _vp, _vp, _u32p, _u32p, _dp, _dp, _vp, _vp, _vp, _vp, _dp,
                                   _vp, _vp, _vp, C.POINTER(_vp)]),
    "ohm_batch_destroy": (C.c_int, [_vp]),
    "ohm_transient_create": (C.c_int, [_vp, _i64, _u32p, _u32p, _dp, _vp, C.c_int32, _dp, C.c_int32, _u32p,
                                       C.c_int32, C.POINTER(_vp)]),
    "ohm_transient_destroy": (C.c_int, [_vp]),
    "ohm_plan_adjoint_dc": (C.c_int, [_vp, _vp, _dp, C.POINTER(Components), C.POINTER(KrylovParams), _dp, _dp, _dp,
                                      _dp, _dp, C.POINTER(AdjointInfo)]),
    "ohm_transient_adjoint": (C.c_int, [_vp, _vp, C.c_double, C.c_double, C.c_int32, C.c_int32,
                                        C.POINTER(NewtonParamsC), _dp, C.POINTER(Components),
                                        C.POINTER(KrylovParams), _dp, _dp, _dp, _dp, _dp, C.POINTER(AdjointInfo)]),
    "ohm_ac_sweep": (C.c_int, [_vp, _i64, _i64, _u32p, _u32p, _dp, _dp, _dp, _i64, _dp, C.POINTER(KrylovParams),
                               _dp, C.POINTER(AcPointInfo)]),
    "ohm_transient_run": (C.c_int, [_vp, _vp, C.c_double, C.c_double, C.c_int32, C.c_int32,
                                    C.POINTER(NewtonParamsC), C.c_int32, _dp, C.POINTER(TransientInfo)]),
    "ohm_transient_set_predictor": (C.c_int, [_vp, C.c_int32]),
    "ohm_solve_complex": (C.c_int, [_vp, _i64, _i64, _u32p, _u32p, _dp, _dp, _dp, C.POINTER(KrylovParams),
                                    C.POINTER(AcPointInfo)]),
    "ohm_compile": (C.c_int, [_vp, _i64, C.POINTER(C.c_int32), C.POINTER(C.c_int64), _dp, _dp,
                              C.POINTER(C.c_void_p)]),
    "ohm_netlist_get_sizes": (C.c_int, [_vp, C.POINTER(NetlistSizes)]),
    "ohm_netlist_download": (C.c_int, [_vp, _u32p, _u32p, _dp, _u32p, _u32p, _dp, _dp, C.POINTER(C.c_int64),
                                       C.POINTER(C.c_int64), _vp, _vp, _vp]),
    "ohm_netlist_destroy": (C.c_int, [_vp]),
    "ohm_transient_run_adaptive": (C.c_int, [_vp, _vp, C.c_double, C.c_double, C.c_double,
                                             C.POINTER(NewtonParamsC), C.c_int32, _dp, _dp,
                                             C.POINTER(AdaptiveInfo)]),
    "ohm_batch_autotune": (C.c_int, [_vp, C.POINTER(NewtonParamsC), C.c_int32, C.POINTER(C.c_int32),
                                     C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_double)]),
    "ohm_batch_set_kernel": (C.c_int, [_vp, C.c_int32, C.c_int32, C.c_int32]),
    "ohm_isai_apply": (C.c_int, [_vp, _i64, _i64, _u32p, _u32p, _dp, _dp, _dp, _i64]),
    "ohm_batch_newton_device": (C.c_int, [_vp, _vp, C.POINTER(NewtonParamsC), C.POINTER(SolveInfo)]),
    "ohm_batch_instance_info": (C.c_int, [_vp, C.POINTER(SolveInfo), _i64]),
}

_LIB = None


def load():
    """Load the library (once).  Raises if it is missing or lacks a symbol."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing; build it with `make -C ohmnivore_b200/csrc` "
                          "or __graft_entry__.build()")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def last_error() -> str:
    return load().ohm_last_error().decode(errors="replace")


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def u32ptr(a: np.ndarray):
    assert a.dtype == np.uint32 and a.flags.c_contiguous
    return a.ctypes.data_as(_u32p)


def vptr(a):
    return None if a is None or len(a) == 0 else C.c_void_p(a.ctypes.data)
