"""GPU parity of the batched Newton path (many circuits, one launch, one
thread block per circuit) against the FP64 Newton + sparse LU oracle run on
each instance, and against the single-circuit GPU path."""
import numpy as np
import pytest

from oracle import newton_ref
from ohmnivore_b200 import circuits as ck
from ohmnivore_b200 import mna
from ohmnivore_b200 import solver as S

pytestmark = pytest.mark.gpu


def _params(prec, **kw):
    p = S.NewtonParams(max_iterations=100, abs_tol=1e-10, bicgstab_max_iterations=20000,
                       bicgstab_tolerance=1e-14, precision=prec, inner_rtol=1e-4)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _solve(batch, x0=None, params=None, check=True):
    import torch
    x = torch.zeros(batch.rows, dtype=torch.float64, device="cuda")
    if x0 is not None:
        x.copy_(torch.from_numpy(x0))
    info = batch.newton_device(x.data_ptr(), params, check=check)
    return x.cpu().numpy(), info


def _check_all(systems, xs, tol=1e-9, current_floor=0.0):
    """Norm-wise relative error, node voltages and branch currents separately.
    ``current_floor`` (amperes) bounds the current norm from below for
    circuits whose branch currents are leakage-level."""
    for i, (s, x) in enumerate(zip(systems, xs)):
        ref, _ = newton_ref.newton(s)
        assert _rel(x[: s.n_nodes], ref[: s.n_nodes]) < tol, i
        ib, rb = x[s.n_nodes:], ref[s.n_nodes:]
        if len(rb):
            scale = max(float(np.max(np.abs(rb))), current_floor, 1e-300)
            assert float(np.max(np.abs(ib - rb))) / scale < tol, i


@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "mixed"])
@pytest.mark.parametrize("vaf", [np.inf, 100.0], ids=["vaf_inf", "vaf_100"])
def test_monte_carlo_batch_matches_oracle(ctx, prec, vaf):
    """24 Monte Carlo instances (BJT differential pairs + diode loads on
    resistor meshes, 50-600 nodes, uneven sizes) in one launch."""
    systems = [mna.compile_circuit(c) for c in ck.monte_carlo_batch(24, seed=3, n_lo=50, n_hi=600, vaf=vaf)]
    batch = S.NewtonBatch(systems, ctx)
    try:
        x, info = _solve(batch, params=_params(prec))
        per = batch.instance_info()
    finally:
        batch.close()
    assert info["kernel_launches"] == 1
    assert info["status"] == 0 and info["error_iteration"] == -1
    assert all(p["status"] == 0 and p["iterations"] >= 1 for p in per)
    assert info["iterations"] == max(p["iterations"] for p in per)
    _check_all(systems, batch.split(x))


def test_heterogeneous_batch(ctx):
    """Diode meshes, a CMOS chain, BJT circuits and a linear ladder in one
    batch.  The static CMOS chain draws only ~10 pA of leakage from VDD; Newton
    resolves node voltages to ~1e-10 V, which through an on-transistor
    (~1e-4 S) bounds that current to ~1e-14 A absolute, so branch currents are
    compared against a 1e-4 A current scale (1e-13 A at the 1e-9 gate)."""
    cs = [ck.diode_mesh(12, 12, seed=1), ck.inverter_chain(stages=10, seed=2),
          ck.resistor_ladder(200, seed=0), ck.diode_mesh(7, 30, seed=5)]
    cs += ck.monte_carlo_batch(3, seed=11, n_lo=60, n_hi=300, vaf=np.inf)
    systems = [mna.compile_circuit(c) for c in cs]
    batch = S.NewtonBatch(systems, ctx)
    try:
        x, _ = _solve(batch, params=_params(0))
    finally:
        batch.close()
    _check_all(systems, batch.split(x), current_floor=1e-4)


def test_batch_agrees_with_single_circuit_path(ctx):
    """The same instance solved alone (grid-wide kernel) and inside a batch
    (one block) converges to the same point."""
    systems = [mna.compile_circuit(c) for c in ck.monte_carlo_batch(6, seed=5, n_lo=100, n_hi=400)]
    batch = S.NewtonBatch(systems, ctx)
    try:
        x, _ = _solve(batch, params=_params(0))
    finally:
        batch.close()
    for s, xb in zip(systems, batch.split(x)):
        xs = S.newton_solve(ctx, s.g.val, s.g.col, s.g.row_ptr, s.b_dc, s.diode_descriptors,
                            s.bjt_descriptors, s.mosfet_descriptors, s.size, s.g.nnz, _params(0))
        assert _rel(xb, xs) < 1e-10


def test_batch_repeat_and_initial_guess(ctx):
    """A second call on the same batch object reuses its device state: from the
    converged point it stops after one or two iterations with the same answer."""
    systems = [mna.compile_circuit(c) for c in ck.monte_carlo_batch(5, seed=8, n_lo=50, n_hi=200)]
    batch = S.NewtonBatch(systems, ctx)
    try:
        x1, i1 = _solve(batch, params=_params(0))
        x2, i2 = _solve(batch, x0=x1, params=_params(0))
    finally:
        batch.close()
    assert i2["iterations"] <= 2 < i1["iterations"]
    assert _rel(x2, x1) < 1e-10


def test_batch_failure_is_per_instance(ctx):
    """A Newton cap too small for the instances is reported per instance, and
    the call's status is the first failure's."""
    systems = [mna.compile_circuit(c) for c in ck.monte_carlo_batch(4, seed=3, n_lo=50, n_hi=120)]
    batch = S.NewtonBatch(systems, ctx)
    try:
        with pytest.raises(S.NewtonNotConverged):
            _solve(batch, params=_params(0, max_iterations=2))
        _, info = _solve(batch, params=_params(0, max_iterations=2), check=False)
        per = batch.instance_info()
    finally:
        batch.close()
    assert info["status"] == 2
    assert 0 <= info["error_iteration"] < 4
    assert all(p["status"] == 2 and p["iterations"] == 2 for p in per)


def test_batch_rejects_isai(ctx):
    systems = [mna.compile_circuit(ck.diode_mesh(5, 5, seed=2))]
    batch = S.NewtonBatch(systems, ctx)
    try:
        p = _params(0)
        p.precond = 2
        with pytest.raises(S.InvalidArgument):
            _solve(batch, params=p)
    finally:
        batch.close()


def test_batch_rejects_bad_instance(ctx):
    s = mna.compile_circuit(ck.diode_mesh(5, 5, seed=2))
    bad = mna.compile_circuit(ck.diode_mesh(5, 5, seed=2))
    bad.diode_descriptors = bad.diode_descriptors.copy()
    bad.diode_descriptors["g_row_col"][0, 0] = bad.g.nnz + 3
    with pytest.raises(S.CompileError):
        S.NewtonBatch([s, bad], ctx)


def test_batch_kernel_variants_agree(ctx):
    """Every kernel variant the autotuner can choose (lanes per row x launch
    shape) converges to the same operating points.  The variants reduce in
    different orders, so an instance's Krylov path can differ (and break
    down in one variant but not another); continuation is on, as in use."""
    systems = [mna.compile_circuit(c) for c in ck.monte_carlo_batch(12, seed=4, n_lo=50, n_hi=400)]
    batch = S.NewtonBatch(systems, ctx)
    try:
        ref, _ = _solve(batch, params=_params(0, continuation=True))
        for lpr in (1, 2, 4, 8):
            for tpb, bps in ((256, 2), (256, 4), (128, 8)):
                batch.set_kernel(lpr, tpb, bps)
                x, _ = _solve(batch, params=_params(0, continuation=True))
                assert _rel(x, ref) < 1e-9, (lpr, tpb, bps)
        with pytest.raises(S.InvalidArgument):
            batch.set_kernel(3, 256, 2)
    finally:
        batch.close()


def test_batch_autotune(ctx):
    systems = [mna.compile_circuit(c) for c in ck.monte_carlo_batch(40, seed=6, n_lo=50, n_hi=800)]
    batch = S.NewtonBatch(systems, ctx)
    try:
        choice = batch.autotune(_params(0, continuation=True), sample_size=16)
        assert choice["lanes_per_row"] in (1, 2, 4, 8)
        assert (choice["threads_per_block"], choice["blocks_per_sm"]) in ((256, 2), (256, 4), (128, 8))
        assert choice["sample_ms"] > 0
        x, info = _solve(batch, params=_params(0, continuation=True))
    finally:
        batch.close()
    assert info["status"] == 0
    _check_all(systems, batch.split(x))


def test_batch_split_solves_large_circuit_on_whole_gpu(ctx):
    """One 3,600-row diode mesh among small Monte Carlo circuits: its
    one-block solve would outlast the rest of the batch, so the split solves
    it alone on the whole GPU first (two launches); the results match the
    oracle and the unsplit batch."""
    cs = [ck.diode_mesh(60, 60, seed=2)] + ck.monte_carlo_batch(24, seed=3, n_lo=50, n_hi=600, vaf=np.inf)[:7]
    systems = [mna.compile_circuit(c) for c in cs]
    assert systems[0].size >= 2048
    batch = S.NewtonBatch(systems, ctx)
    try:
        x_split, info_split = _solve(batch, params=_params(0))
        per = batch.instance_info()
        batch.set_split(False)
        x_one, info_one = _solve(batch, params=_params(0))
    finally:
        batch.close()
    assert info_split["kernel_launches"] == 2
    assert info_one["kernel_launches"] == 1
    assert all(p["status"] == 0 and p["iterations"] >= 1 for p in per)
    assert info_split["iterations"] == max(p["iterations"] for p in per)
    _check_all(systems, batch.split(x_split))
    assert _rel(x_split, x_one) < 1e-10
