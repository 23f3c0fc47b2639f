"""GPU: the reference's DC continuation (source stepping, GMIN stepping,
pseudo-transient; src/analysis/dc.rs:60-290) run on the device after a failed
direct Newton solve, single-circuit and batched, against the FP64 oracle."""
import numpy as np
import pytest

from oracle import newton_ref
from ohmnivore_b200 import circuits as ck
from ohmnivore_b200 import mna
from ohmnivore_b200 import solver as S

pytestmark = pytest.mark.gpu

CONT_SOURCE, CONT_GMIN, CONT_PSEUDO = 1, 2, 3


def _params(max_iterations, continuation=True, **kw):
    p = S.NewtonParams(max_iterations=max_iterations, abs_tol=1e-10, bicgstab_max_iterations=20000,
                       bicgstab_tolerance=1e-14, inner_rtol=1e-4, continuation=continuation)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _plan_solve(ctx, s, params):
    import torch
    plan = S.NewtonPlan(s, ctx)
    try:
        x = torch.zeros(s.size, dtype=torch.float64, device="cuda")
        info = plan.newton_device(x.data_ptr(), params)
        return x.cpu().numpy(), info
    finally:
        plan.close()


def test_gmin_stepping_recovers_capped_direct_solve(ctx):
    """A direct solve capped at 3 Newton iterations fails on a diode mesh;
    GMIN stepping (15 iterations per level) then a true-GMIN solve from the
    last level reach the oracle's operating point."""
    s = mna.compile_circuit(ck.diode_mesh(10, 10, seed=2))
    ref, _ = newton_ref.newton(s)
    with pytest.raises(S.NewtonNotConverged):
        _plan_solve(ctx, s, _params(3, continuation=False))
    x, info = _plan_solve(ctx, s, _params(3))
    assert info["continuation_kind"] == CONT_GMIN
    assert info["continuation_steps"] >= 5          # 0.1, 1e-4, 1e-7, 1e-10, 1e-13, final
    assert _rel(x[: s.n_nodes], ref[: s.n_nodes]) < 1e-9
    assert _rel(x[s.n_nodes:], ref[s.n_nodes:]) < 1e-9


def test_pseudo_transient_stage_runs_and_converges(ctx):
    """Pseudo-transient continuation (dc.rs:331-490) after GMIN stepping: the
    testing flag makes the true-GMIN solve count as failed, so the stage runs
    from the last GMIN point (alpha from 0.1, 100x drops, b += alpha x_good on
    node rows) and its final 25-iteration true-DC solve reaches the oracle's
    operating point."""
    s = mna.compile_circuit(ck.diode_mesh(10, 10, seed=2))
    ref, _ = newton_ref.newton(s)
    x, info = _plan_solve(ctx, s, _params(3, continuation=S._lib.CONT_ON | S._lib.CONT_TEST_PSEUDO))
    assert info["continuation_kind"] == CONT_PSEUDO
    # GMIN levels 0.1 .. 1e-13 (5), the true-GMIN solve, alpha 0.1 .. 1e-7 (4), the final solve
    assert info["continuation_steps"] >= 11
    assert _rel(x[: s.n_nodes], ref[: s.n_nodes]) < 1e-9
    assert _rel(x[s.n_nodes:], ref[s.n_nodes:]) < 1e-9
    # without the flag the same call ends after GMIN stepping
    x2, info2 = _plan_solve(ctx, s, _params(3))
    assert info2["continuation_kind"] == CONT_GMIN
    assert info2["continuation_steps"] < info["continuation_steps"]


def test_source_stepping_for_mosfet_circuit(ctx):
    """Circuits with MOSFETs try source stepping first (dc.rs:133-152); its
    last step (all sources at full value) is the true DC solve."""
    s = mna.compile_circuit(ck.inverter_chain(stages=12, seed=2))
    ref, _ = newton_ref.newton(s)
    x, info = _plan_solve(ctx, s, _params(2))
    assert info["continuation_kind"] in (CONT_SOURCE, CONT_GMIN, CONT_PSEUDO)
    assert info["continuation_steps"] >= 1
    assert _rel(x[: s.n_nodes], ref[: s.n_nodes]) < 1e-9


def test_direct_success_runs_no_continuation(ctx):
    s = mna.compile_circuit(ck.diode_mesh(8, 8, seed=2))
    _, info = _plan_solve(ctx, s, _params(100))
    assert info["continuation_steps"] == 0 and info["continuation_kind"] == 0


def test_continuation_needs_node_count(ctx):
    s = mna.compile_circuit(ck.diode_mesh(5, 5, seed=2))
    with pytest.raises(S.InvalidArgument):
        S.newton_solve(ctx, s.g.val, s.g.col, s.g.row_ptr, s.b_dc, s.diode_descriptors, s.bjt_descriptors,
                       s.mosfet_descriptors, s.size, s.g.nnz, _params(3))
    x = S.newton_solve(ctx, s.g.val, s.g.col, s.g.row_ptr, s.b_dc, s.diode_descriptors, s.bjt_descriptors,
                       s.mosfet_descriptors, s.size, s.g.nnz, _params(100, n_nodes=s.n_nodes))
    ref, _ = newton_ref.newton(s)
    assert _rel(x[: s.n_nodes], ref[: s.n_nodes]) < 1e-9


def test_batched_continuation(ctx):
    """Every instance of a batch runs its own continuation schedule in its
    block; all reach the oracle's operating points."""
    import torch
    systems = [mna.compile_circuit(c) for c in ck.monte_carlo_batch(8, seed=3, n_lo=50, n_hi=300)]
    systems.append(mna.compile_circuit(ck.inverter_chain(stages=6, seed=2)))
    batch = S.NewtonBatch(systems, ctx)
    try:
        x = torch.zeros(batch.rows, dtype=torch.float64, device="cuda")
        batch.newton_device(x.data_ptr(), _params(3))
        per = batch.instance_info()
        xs = batch.split(x.cpu().numpy())
    finally:
        batch.close()
    assert all(p["status"] == 0 for p in per)
    assert all(p["continuation_steps"] > 0 for p in per)
    for s, xi in zip(systems, xs):
        ref, _ = newton_ref.newton(s)
        assert _rel(xi[: s.n_nodes], ref[: s.n_nodes]) < 1e-9
