"""The C-ABI library loads and exports every symbol include/ohm.h declares;
struct layouts agree between the header, ctypes and numpy.  No GPU needed."""
import ctypes
import os
import re
import subprocess

import numpy as np

from ohmnivore_b200 import _lib, mna

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    text = open(os.path.join(ROOT, "include", "ohm.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ohm_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = _declared_symbols()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # ctypes signatures cover every declared entry point
    assert set(names) <= set(_lib.SIGNATURES), set(names) - set(_lib.SIGNATURES)


def test_struct_layouts(tmp_path):
    """ctypes mirrors agree with the C compiler's view of include/ohm.h."""
    src = tmp_path / "sz.c"
    src.write_text('#include <stdio.h>\n#include "ohm.h"\nint main(void){printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu",'
                   ' sizeof(ohm_krylov_params), sizeof(ohm_newton_params), sizeof(ohm_solve_info),'
                   ' sizeof(ohm_diode_desc), sizeof(ohm_bjt_desc), sizeof(ohm_mosfet_desc),'
                   ' sizeof(ohm_source), sizeof(ohm_transient_info), sizeof(ohm_adaptive_info)); return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    sizes = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    assert sizes == [ctypes.sizeof(_lib.KrylovParams), ctypes.sizeof(_lib.NewtonParamsC),
                     ctypes.sizeof(_lib.SolveInfo), 48, 96, 64, _lib.SOURCE_DTYPE.itemsize,
                     ctypes.sizeof(_lib.TransientInfo), ctypes.sizeof(_lib.AdaptiveInfo)]
    assert ctypes.sizeof(_lib.AdaptiveInfo) == 80
    assert mna.DIODE_DTYPE.itemsize == 48
    assert mna.BJT_DTYPE.itemsize == 96
    assert mna.MOSFET_DTYPE.itemsize == 64


def test_defaults_match_reference():
    lib = _lib.load()
    k = _lib.KrylovParams()
    lib.ohm_krylov_params_default(ctypes.byref(k))
    assert k.max_iterations == 10_000 and k.tolerance == 1e-5      # bicgstab.rs:10-11
    n = _lib.NewtonParamsC()
    lib.ohm_newton_params_default(ctypes.byref(n))
    assert n.max_iterations == 50 and n.abs_tol == 1e-4            # newton.rs:48-49


def test_host_validation_without_gpu():
    """Calls that fail argument validation return an error code (no device work)."""
    lib = _lib.load()
    h = ctypes.c_void_p()
    st = lib.ohm_ctx_create(-1, ctypes.byref(h))
    assert st != _lib.OK
    assert _lib.last_error()
    assert lib.ohm_ctx_destroy(None) == _lib.OK
    x = np.zeros(2)
    st = lib.ohm_solve_real(None, 2, 0, None, None, None, _lib.dptr(x), _lib.dptr(x), None, None)
    assert st == _lib.ERR_INVALID_ARG
    st = lib.ohm_solve_complex(None, 2, 0, None, None, None, _lib.dptr(x), _lib.dptr(x), None, None)
    assert st == _lib.ERR_INVALID_ARG
    st = lib.ohm_compile(None, 0, None, None, None, None, None)
    assert st == _lib.ERR_INVALID_ARG
