"""GPU parity: device evaluation, stamping, limiting and the persistent
Newton solve through the C ABI vs the FP64 oracle."""
import numpy as np
import pytest

from oracle import devices_ref, newton_ref
from ohmnivore_b200 import circuits as ck
from ohmnivore_b200 import mna
from ohmnivore_b200 import solver as S

pytestmark = pytest.mark.gpu


def _bjt_circuit():
    b = ck.CircuitBuilder()
    b.vsource(1, 0, dc=5.0, name="VCC")
    b.vsource(6, 0, dc=0.8, name="VB")
    b.resistors([1, 6, 1, 4, 3, 5], [2, 3, 5, 0, 0, 4], [1000.0, 5e3, 2000.0, 470.0, 1e5, 300.0])
    b.bjts([2, 5], [3, 3], [4, 0], is_=1e-16, bf=[100.0, 80.0], br=[1.0, 2.0], npn=[True, True])
    b.bjts([0], [4], [5], is_=1e-15, bf=50.0, npn=False)            # PNP
    b.diodes([2, 5], [0, 4], is_=1e-14, n=[1.0, 1.5])               # one floating diode
    return b.build()


def _mos_circuit():
    return ck.inverter_chain(stages=12, seed=2)


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("make", [lambda: ck.diode_mesh(15, 15, seed=1), _bjt_circuit, _mos_circuit],
                         ids=["diode_mesh", "bjt_diode", "cmos_chain"])
def test_assemble_matches_oracle(ctx, make):
    s = mna.compile_circuit(make())
    plan = S.NewtonPlan(s, ctx)
    try:
        rng = np.random.default_rng(7)
        for trial in range(3):
            x = rng.uniform(-0.5, 1.2, s.size)
            vals, rhs = plan.assemble(x)
            rv, rb = devices_ref.assemble(s, s.g.val, s.b_dc, x)
            np.testing.assert_allclose(vals, rv, rtol=1e-13, atol=1e-300)
            np.testing.assert_allclose(rhs, rb, rtol=1e-12, atol=1e-15 * max(1.0, np.abs(rb).max()))
            # untouched slots are bit-identical to the base values
            ms, _, _, _ = devices_ref.stamp_contributions(s, x)
            untouched = np.ones(s.g.nnz, bool)
            untouched[ms] = False
            np.testing.assert_array_equal(vals[untouched], s.g.val[untouched])
    finally:
        plan.close()


@pytest.mark.parametrize("make", [lambda: ck.diode_mesh(15, 15, seed=1), _bjt_circuit, _mos_circuit],
                         ids=["diode_mesh", "bjt_diode", "cmos_chain"])
def test_limit_matches_oracle(ctx, make):
    s = mna.compile_circuit(make())
    plan = S.NewtonPlan(s, ctx)
    try:
        rng = np.random.default_rng(9)
        for trial in range(4):
            xo = rng.uniform(-0.2, 0.9, s.size)
            xn = xo + rng.normal(0, 2.0, s.size)
            got = plan.limit(xo, xn)
            ref, _ = devices_ref.limit(s, xo, xn)
            np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-14)
    finally:
        plan.close()


def _newton_params(prec, abs_tol=1e-10, tol=1e-14):
    """Tight settings for the 1e-9 bar: Newton stops at max|dx| < 1e-10; each
    linear solve is inexact (relative 1e-4 on the correction) down to an
    absolute floor of 1e-14 ||b||; the same settings for FP64 and mixed."""
    return S.NewtonParams(max_iterations=100, abs_tol=abs_tol, bicgstab_max_iterations=20000,
                          bicgstab_tolerance=tol, precision=prec, inner_rtol=1e-4)


@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "mixed"])
@pytest.mark.parametrize("make", [lambda: ck.diode_mesh(20, 20, seed=1), _bjt_circuit],
                         ids=["diode_mesh", "bjt_diode"])
def test_newton_matches_oracle(ctx, make, prec):
    s = mna.compile_circuit(make())
    ref, _ = newton_ref.newton(s)
    stats = {}
    x = S.newton_solve(ctx, s.g.val, s.g.col, s.g.row_ptr, s.b_dc, s.diode_descriptors,
                       s.bjt_descriptors, s.mosfet_descriptors, s.size, s.g.nnz,
                       _newton_params(prec), stats)
    nn = slice(0, s.n_nodes)
    br = slice(s.n_nodes, s.size)
    assert _rel(x[nn], ref[nn]) < 1e-9
    assert _rel(x[br], ref[br]) < 1e-9
    assert stats["kernel_launches"] == 1


@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "mixed"])
def test_newton_isai_matches_oracle(ctx, prec):
    """Newton with the ISAI(1) preconditioner refactored on the device every iteration."""
    s = mna.compile_circuit(ck.diode_mesh(24, 24, seed=3))
    ref, _ = newton_ref.newton(s)
    p = _newton_params(prec)
    p.precond = 2
    stats = {}
    x = S.newton_solve(ctx, s.g.val, s.g.col, s.g.row_ptr, s.b_dc, s.diode_descriptors,
                       s.bjt_descriptors, s.mosfet_descriptors, s.size, s.g.nnz, p, stats)
    assert _rel(x[: s.n_nodes], ref[: s.n_nodes]) < 1e-9
    assert _rel(x[s.n_nodes:], ref[s.n_nodes:]) < 1e-9


def test_newton_reference_defaults(ctx):
    """Reference NewtonParams defaults (abs_tol 1e-4, BiCGSTAB tol 1e-5 of
    ||b||) reach the operating point within the reference's own GPU-vs-CPU
    check, 0.1 V (src/solver/gpu.rs:946-981)."""
    s = mna.compile_circuit(ck.diode_mesh(10, 10, seed=2))
    ref, _ = newton_ref.newton(s)
    x = S.newton_solve(ctx, s.g.val, s.g.col, s.g.row_ptr, s.b_dc, s.diode_descriptors,
                       s.bjt_descriptors, s.mosfet_descriptors, s.size, s.g.nnz, S.NewtonParams())
    assert np.max(np.abs(x[: s.n_nodes] - ref[: s.n_nodes])) < 0.1


def test_newton_not_converged_reports(ctx):
    s = mna.compile_circuit(ck.diode_mesh(10, 10, seed=2))
    with pytest.raises(S.NewtonNotConverged) as ei:
        S.newton_solve(ctx, s.g.val, s.g.col, s.g.row_ptr, s.b_dc, s.diode_descriptors,
                       s.bjt_descriptors, s.mosfet_descriptors, s.size, s.g.nnz,
                       S.NewtonParams(max_iterations=2, abs_tol=1e-12, bicgstab_tolerance=1e-12))
    assert ei.value.iterations == 2
    assert ei.value.max_residual > 0


def test_newton_rejects_bad_descriptor(ctx):
    s = mna.compile_circuit(ck.diode_mesh(5, 5, seed=2))
    bad = s.diode_descriptors.copy()
    bad["g_row_col"][0, 0] = s.g.nnz + 5
    with pytest.raises(S.CompileError):
        S.newton_solve(ctx, s.g.val, s.g.col, s.g.row_ptr, s.b_dc, bad, s.bjt_descriptors,
                       s.mosfet_descriptors, s.size, s.g.nnz, S.NewtonParams())


def test_newton_nan_in_base_is_numerical_error(ctx):
    s = mna.compile_circuit(ck.diode_mesh(5, 5, seed=2))
    b = s.b_dc.copy()
    b[0] = np.nan
    with pytest.raises((S.NewtonNumericalError, S.SolveError)):
        S.newton_solve(ctx, s.g.val, s.g.col, s.g.row_ptr, b, s.diode_descriptors,
                       s.bjt_descriptors, s.mosfet_descriptors, s.size, s.g.nnz, S.NewtonParams())


@pytest.mark.slow
@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "mixed"])
def test_diode_mesh_500_matches_oracle(ctx, prec):
    """The 500x500 diode mesh (250k nodes, 25k diodes): GPU Newton vs the
    FP64 Newton + sparse LU oracle, 1e-9 norm-wise for voltages and currents."""
    s = mna.compile_circuit(ck.diode_mesh())
    ref = _mesh500_reference(s)
    plan = S.NewtonPlan(s, ctx)
    try:
        import torch
        x = torch.zeros(s.size, dtype=torch.float64, device="cuda")
        info = plan.newton_device(x.data_ptr(), _newton_params(prec))
        xh = x.cpu().numpy()
    finally:
        plan.close()
    assert _rel(xh[: s.n_nodes], ref[: s.n_nodes]) < 1e-9
    assert _rel(xh[s.n_nodes:], ref[s.n_nodes:]) < 1e-9
    assert info["kernel_launches"] == 1


_MESH500 = {}


def _mesh500_reference(s):
    if "x" not in _MESH500:
        _MESH500["x"], _ = newton_ref.newton(s)
    return _MESH500["x"]
