"""GPU: fixed-step backward-Euler transient with a Newton solve per step, all
steps on the device (chunked persistent launches, optionally one CUDA graph),
against the oracle restatement (BE companion of src/analysis/transient.rs
plus LU Newton per step); and long rows / long stamp segments (a supply rail
shared by thousands of transistors) in DC and transient solves."""
import numpy as np
import pytest

from oracle import newton_ref
from oracle import transient_ref as tref
from ohmnivore_b200 import circuits as ck
from ohmnivore_b200 import mna
from ohmnivore_b200 import solver as S

pytestmark = pytest.mark.gpu


def _params(**kw):
    p = S.NewtonParams(max_iterations=100, abs_tol=1e-11, bicgstab_max_iterations=20000,
                       bicgstab_tolerance=1e-14, inner_rtol=1e-6)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _wave_err(w, ref):
    return float(np.max(np.abs(w - ref)) / max(np.max(np.abs(ref)), 1e-300))


def _run(s, x0, t0, h, n, probes, predictor=0, **kw):
    import torch
    ctx = S.default_context()
    plan = S.NewtonPlan(s, ctx)
    tr = S.Transient(plan, probes)
    tr.set_predictor(predictor)
    try:
        x = torch.from_numpy(np.ascontiguousarray(x0, dtype=np.float64)).cuda()
        params = kw.pop("params", _params())
        wave = tr.run(x.data_ptr(), t0, h, n, params, **kw)
        return wave, x.cpu().numpy(), tr.last_info
    finally:
        tr.close()
        plan.close()


def _rc_sources_circuit():
    """Four RC sections driven by PULSE, SIN, PWL and EXP voltage sources, a
    DC current source and a diode clamp."""
    b = ck.CircuitBuilder()
    b.vsource(1, 0, dc=0.0, name="VP", tran=(ck.TRAN_PULSE, (0.0, 1.0, 2e-9, 1e-9, 1e-9, 5e-9, 20e-9)))
    b.vsource(2, 0, dc=0.0, name="VS", tran=(ck.TRAN_SIN, (0.5, 0.4, 1e8, 1e-9, 1e7)))
    b.vsource(3, 0, dc=0.0, name="VW", tran=(ck.TRAN_PWL, ((0.0, 0.0), (5e-9, 2.0), (10e-9, -1.0), (30e-9, 0.5))))
    b.vsource(4, 0, dc=0.0, name="VE", tran=(ck.TRAN_EXP, (0.0, 1.5, 1e-9, 3e-9, 12e-9, 4e-9)))
    b.resistors([1, 2, 3, 4, 5, 6, 7], [5, 6, 7, 8, 6, 7, 8], [1e3, 2e3, 500.0, 1.5e3, 5e3, 4e3, 3e3])
    b.capacitors([5, 6, 7, 8], [0, 0, 0, 0], [1e-12, 2e-12, 0.5e-12, 3e-12])
    b.isource(0, 8, dc=1e-4, name="I1")
    b.diodes([6], [0], is_=1e-14)
    return b.build()


@pytest.mark.parametrize("graph", [True, False], ids=["graph", "launches"])
def test_sources_rc_transient_matches_oracle(graph):
    s = mna.compile_circuit(_rc_sources_circuit())
    x0, _ = newton_ref.newton(s)
    probes = list(range(s.size))
    h, n = 2e-10, 150
    wave, x_end, info = _run(s, x0, 0.0, h, n, probes, steps_per_launch=40, graph=graph)
    _, ref, _ = tref.be_transient(s, x0, 0.0, h, n, probes)
    nn = slice(0, s.n_nodes)
    assert _wave_err(wave[:, nn], ref[:, nn]) < 1e-9
    assert info["steps_done"] == n and info["failed_step"] == -1
    assert info["launches"] == 4 and info["graph"] == (1 if graph else 0)
    np.testing.assert_array_equal(x_end, wave[-1])


def test_inverter_chain_transient_matches_oracle():
    """A CMOS chain switching: PULSE input, 10 fF loads, 5 ps BE steps."""
    s = mna.compile_circuit(ck.inverter_chain(stages=8, seed=2))
    x0, _ = newton_ref.dc_operating_point(s)
    probes = list(range(s.n_nodes))
    h, n = 5e-12, 120
    wave, _, info = _run(s, x0, 0.0, h, n, probes, steps_per_launch=50)
    _, ref, _ = tref.be_transient(s, x0, 0.0, h, n, probes)
    assert _wave_err(wave, ref) < 1e-9
    assert info["newton_iterations"] >= n
    # the chain switches: the first stage output falls from VDD within the run
    assert wave[0, s.node_index(3)] > 1.7 and wave[-1, s.node_index(3)] < 0.1


def test_graph_and_chunking_do_not_change_results():
    s = mna.compile_circuit(ck.inverter_chain(stages=6, seed=3))
    x0, _ = newton_ref.dc_operating_point(s)
    probes = list(range(s.n_nodes))
    w1, _, _ = _run(s, x0, 0.0, 5e-12, 60, probes, steps_per_launch=7, graph=True)
    w2, _, _ = _run(s, x0, 0.0, 5e-12, 60, probes, steps_per_launch=60, graph=False)
    np.testing.assert_array_equal(w1, w2)


def _star(branches=5000, seed=7):
    """A hub node fed from 2 V through 10 ohm, with `branches` diodes from the
    hub to their own nodes, each loaded by a resistor to ground: the hub row
    has a nonzero per branch and its diagonal / rhs a stamp per diode."""
    rng = np.random.default_rng(seed)
    b = ck.CircuitBuilder()
    b.vsource(1, 0, dc=2.0, name="V1")
    b.resistors([1], [2], [10.0])
    k = 3 + np.arange(branches)
    b.diodes(np.full(branches, 2), k, is_=1e-14 * (1.0 + 0.05 * rng.standard_normal(branches)))
    b.resistors(k, 0, rng.uniform(1e3, 1e5, branches))
    return b.build()


def test_long_rows_and_segments_match_oracle():
    import torch
    s = mna.compile_circuit(_star())
    hub = s.node_index(2)
    assert s.g.row_ptr[hub + 1] - s.g.row_ptr[hub] > 4096
    ref, _ = newton_ref.newton(s)
    for prec in (0, 1):
        plan = S.NewtonPlan(s)
        try:
            x = torch.zeros(s.size, dtype=torch.float64, device="cuda")
            plan.newton_device(x.data_ptr(), _params(precision=prec, abs_tol=1e-10))
            xd = x.cpu().numpy()
            vals, rhs = plan.assemble(ref)
        finally:
            plan.close()
        assert _wave_err(xd[: s.n_nodes], ref[: s.n_nodes]) < 1e-9, prec
        assert _wave_err(xd[s.n_nodes:], ref[s.n_nodes:]) < 1e-9, prec


def test_supply_rail_chain_dc_and_transient():
    """4,500 stages: the VDD row holds ~4,500 nonzeros (one per stage) and its
    diagonal ~4,500 stamp contributions, so both take the team-cooperative
    long-row and long-segment paths.  Newton starts from logic levels; the
    oracle's LU Newton started from the GPU point must leave it in place, and
    30 BE steps match the oracle."""
    import torch
    s = mna.compile_circuit(ck.inverter_chain(stages=4500, seed=2))
    vdd = s.node_index(1)
    assert s.g.row_ptr[vdd + 1] - s.g.row_ptr[vdd] > 4096
    x0 = np.zeros(s.size)
    x0[s.node_index(1)] = 1.8
    for k in range(1, 4501):
        x0[s.node_index(2 + k)] = 1.8 if k % 2 else 0.0
    plan = S.NewtonPlan(s)
    try:
        x = torch.from_numpy(x0).cuda()
        plan.newton_device(x.data_ptr(), _params(abs_tol=1e-10))
        xd = x.cpu().numpy()
    finally:
        plan.close()
    ref_dc, _ = newton_ref.newton(s, x0=xd)
    assert _wave_err(xd[: s.n_nodes], ref_dc[: s.n_nodes]) < 1e-9
    probes = [s.node_index(k) for k in (2, 3, 4, 5, 1000, 4502)]
    wave, _, _ = _run(s, ref_dc, 0.0, 5e-12, 30, probes, steps_per_launch=30)
    _, ref, _ = tref.be_transient(s, ref_dc, 0.0, 5e-12, 30, probes)
    assert _wave_err(wave, ref) < 1e-9
    # the linear predictor starts each step's Newton elsewhere and reaches
    # the same backward-Euler solutions, in fewer iterations
    wave_p, _, info_p = _run(s, ref_dc, 0.0, 5e-12, 30, probes, predictor=1, steps_per_launch=7)
    _, _, info_0 = _run(s, ref_dc, 0.0, 5e-12, 30, probes, steps_per_launch=7)
    assert _wave_err(wave_p, ref) < 1e-9
    assert info_p["newton_iterations"] <= info_0["newton_iterations"]
    # the quadratic predictor (from the third step on, across launch boundaries)
    wave_q, _, info_q = _run(s, ref_dc, 0.0, 5e-12, 30, probes, predictor=2, steps_per_launch=7)
    assert _wave_err(wave_q, ref) < 1e-9
    assert info_q["newton_iterations"] <= info_0["newton_iterations"]


def test_failed_step_is_reported():
    s = mna.compile_circuit(ck.inverter_chain(stages=6, seed=3))
    x0, _ = newton_ref.dc_operating_point(s)
    import torch
    plan = S.NewtonPlan(s)
    tr = S.Transient(plan, [0])
    try:
        x = torch.from_numpy(x0).cuda()
        with pytest.raises(S.NewtonNotConverged):
            tr.run(x.data_ptr(), 0.0, 5e-12, 40, _params(max_iterations=1, abs_tol=1e-14))
        info = tr.last_info
    finally:
        tr.close()
        plan.close()
    assert info["failed_step"] >= 0 and info["steps_done"] == info["failed_step"]


def test_capacitance_off_pattern_rejected():
    """The compiler zero-fills G with C's pattern (as src/compiler.rs:576-579
    does), so only a hand-made C can miss it; the C ABI rejects that."""
    import ctypes as C
    from ohmnivore_b200 import _lib
    s = mna.compile_circuit(ck.diode_mesh(4, 4, seed=2))
    n = s.size
    far = n - 1
    assert s.g.value_index(2, far) is None
    rp = np.zeros(n + 1, dtype=np.uint32)
    rp[3:] = 1                                   # one entry, in row 2
    col = np.array([far], dtype=np.uint32)
    val = np.array([1e-12])
    plan = S.NewtonPlan(s)
    try:
        h = C.c_void_p()
        st = plan.ctx.lib.ohm_transient_create(plan._h, 1, _lib.u32ptr(rp), _lib.u32ptr(col), _lib.dptr(val),
                                               None, 0, None, 0, None, 0, C.byref(h))
        assert st == _lib.ERR_COMPILE and not h.value
    finally:
        plan.close()


def test_dc_solve_after_transient_on_the_same_plan():
    """A transient run assembles the backward-Euler rhs into the plan; the
    plan's rhs is restored afterwards, so a DC solve on the same plan (which
    re-stamps only the rows that devices touch) gives the same operating
    point, bit for bit, as before the run; likewise after the adaptive run
    and the transient adjoint."""
    import torch
    s = mna.compile_circuit(_rc_sources_circuit())
    plan = S.NewtonPlan(s)
    tr = S.Transient(plan, [0])
    try:
        def dc():
            x = torch.zeros(s.size, dtype=torch.float64, device="cuda")
            plan.newton_device(x.data_ptr(), _params())
            return x.cpu().numpy()
        x_dc = dc()
        x = torch.from_numpy(x_dc).cuda()
        tr.run(x.data_ptr(), 0.0, 1e-10, 40, _params())
        np.testing.assert_array_equal(dc(), x_dc)
        x = torch.from_numpy(x_dc).cuda()
        tr.run_adaptive(x.data_ptr(), 1e-10, 4e-9, 0.0, _params())
        np.testing.assert_array_equal(dc(), x_dc)
        comps = S.ComponentTable(_rc_sources_circuit(), s)
        x = torch.from_numpy(x_dc).cuda()
        w = np.zeros(s.size)
        w[0] = 1.0
        tr.adjoint(x.data_ptr(), 0.0, 1e-10, 20, w, comps, _params(), 5)
        np.testing.assert_array_equal(dc(), x_dc)
    finally:
        tr.close()
        plan.close()
