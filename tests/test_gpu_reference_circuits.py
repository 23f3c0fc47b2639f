"""GPU: the reference's nonlinear end-to-end tests (tests/transistor_integration_test.rs,
tests/diode_integration_test.rs, the DC circuits of tests/regression/manifest.toml)
through the persistent Newton solver with the device-side DC continuation,
checked against the reference's own windows, the closed-form regression
values and the FP64 oracle (1e-9 norm-wise); and the ill-conditioned MNA
system of tests/gpu_integration_test.rs:195-235 through the linear solve."""
import numpy as np
import pytest

from oracle import linear_ref, newton_ref
from ohmnivore_b200 import mna
from ohmnivore_b200 import solver as S
from tests.golden import reference_circuits as RC

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)) if len(b) else 0.0


def _gpu_dc(ctx, sysm, precision=0):
    import torch
    params = S.NewtonParams(max_iterations=50, abs_tol=1e-12, bicgstab_max_iterations=20000,
                            bicgstab_tolerance=1e-15, inner_rtol=1e-6, precision=precision, continuation=1)
    plan = S.NewtonPlan(sysm, ctx)
    try:
        x = torch.zeros(sysm.size, dtype=torch.float64, device="cuda")
        info = plan.newton_device(x.data_ptr(), params)
        return x.cpu().numpy(), info
    finally:
        plan.close()


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "mixed"])
@pytest.mark.parametrize("name", sorted(RC.CASES))
def test_gpu_within_reference_windows_and_oracle(ctx, name, precision):
    case = RC.CASES[name]
    ckt, lab = RC.build(case)
    sysm = mna.compile_circuit(ckt)
    x, info = _gpu_dc(ctx, sysm, precision)
    case["check"](RC.node_voltages(sysm, lab, x))
    ref = newton_ref.run_nonlinear(sysm)
    nn, br = slice(0, sysm.n_nodes), slice(sysm.n_nodes, sysm.size)
    assert _rel(x[nn], ref[nn]) < 1e-9, info
    # branch currents: norm-wise, floored at 1 pA for circuits in cutoff
    assert np.max(np.abs(x[br] - ref[br])) <= 1e-9 * max(np.max(np.abs(ref[br])), 1e-3), info


def test_gpu_regression_closed_forms(ctx):
    """diode_forward.spice V(2) and nmos_common_source.spice V(drain)."""
    for name, node, ref in (("diode_resistor_vsource", "2", RC.diode_forward_v2()),
                            ("nmos_common_source", "drain", RC.nmos_common_source_vd())):
        ckt, lab = RC.build(RC.CASES[name])
        sysm = mna.compile_circuit(ckt)
        x, _ = _gpu_dc(ctx, sysm)
        assert abs(x[sysm.node_index(lab[node])] - ref) < 1e-9 * abs(ref), name


def test_gpu_mixed_device_circuit_takes_source_stepping(ctx):
    """transistor_integration_test.rs:407-448 needs source stepping in the
    reference ("mixed circuits ... need source stepping continuation"): the
    direct Newton diverges, and the device-side continuation recovers it."""
    ckt, lab = RC.build(RC.CASES["mixed_diode_bjt_mosfet"])
    sysm = mna.compile_circuit(ckt)
    stages = []
    ref = newton_ref.run_nonlinear(sysm, stages=stages)
    assert "source" in stages
    x, info = _gpu_dc(ctx, sysm)
    assert info["continuation_kind"] != 0 and info["continuation_steps"] > 0
    assert _rel(x[: sysm.n_nodes], ref[: sysm.n_nodes]) < 1e-9


def test_gpu_ill_conditioned_mna_3x3(ctx):
    """tests/gpu_integration_test.rs:195-235: GMIN = 1e-12 diagonals with a
    voltage-source stamp (condition ~1e12); the reference requires agreement
    with the CPU solver within 1e-4, here 1e-9 relative to the dense GE."""
    from ohmnivore_b200.mna import Csr
    gmin = 1e-12
    cols, vals = [0, 2, 1, 0], [gmin, 1.0, gmin, 1.0]            # rows 0, 0, 1, 2
    rp = np.array([0, 2, 3, 4], np.int64)
    a = Csr(3, 3, rp, np.array(cols, np.int64), np.array(vals))
    b = np.array([0.0, 0.0, 5.0])
    ref = linear_ref.dense_solve_real(3, 3, rp, a.col, a.val, b)
    for precond in (S._lib.PRECOND_AUTO, S._lib.PRECOND_ISAI1):   # gpu.rs:139 takes ISAI on a zero diagonal
        x = S.GpuSolver(ctx, S.BiCgStabParams(tolerance=1e-12, precond=precond)).solve_real(a, b)
        assert np.max(np.abs(x - ref)) < 1e-4
        assert _rel(x, ref) < 1e-9
