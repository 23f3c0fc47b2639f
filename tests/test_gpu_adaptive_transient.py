"""GPU: the adaptive BE / TRAP transient (transient.rs:77-178) in one
persistent launch against the oracle's restatement: the reference's own
transient circuits (tests/transient_integration_test.rs), nonlinear circuits
(TRAP with device currents), rejections, output truncation and tstart; and
the UIC start through the GPU solver."""
import numpy as np
import pytest

from oracle import newton_ref
from oracle import transient_ref as tref
from ohmnivore_b200 import circuits as ck
from ohmnivore_b200 import mna
from ohmnivore_b200 import solver as S
from tests.test_oracle_adaptive_transient import CASES

pytestmark = pytest.mark.gpu


def _params():
    return S.NewtonParams(max_iterations=100, abs_tol=1e-12, bicgstab_max_iterations=20000,
                          bicgstab_tolerance=1e-15, inner_rtol=1e-8)


def _gpu_adaptive(s, x0, tstep, tstop, tstart=0.0, probes=None, max_points=None):
    import torch
    probes = list(range(s.size)) if probes is None else probes
    plan = S.NewtonPlan(s)
    tr = S.Transient(plan, probes)
    try:
        x = torch.from_numpy(np.ascontiguousarray(x0, dtype=np.float64)).cuda()
        times, wave = tr.run_adaptive(x.data_ptr(), tstep, tstop, tstart, _params(), max_points)
        return times, wave, tr.last_info, x.cpu().numpy()
    finally:
        tr.close()
        plan.close()


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _start(ckt, s, uic):
    return tref.uic_initial_conditions(s, ckt) if uic else newton_ref.dc_operating_point(s)[0]


@pytest.mark.parametrize("name", list(CASES))
def test_reference_circuits_match_oracle(name):
    ckt, tstep, tstop, uic = CASES[name]()
    s = mna.compile_circuit(ckt)
    x0 = _start(ckt, s, uic)
    rt, rw, rst = tref.adaptive_transient(s, x0, tstep, tstop, 0.0, list(range(s.size)))
    times, wave, info, x_end = _gpu_adaptive(s, x0, tstep, tstop)
    assert info["status"] == 0
    assert (info["accepted"], info["rejected"], info["linear_solves"]) == \
        (rst["accepted"], rst["rejected"], rst["linear_solves"])
    assert info["points"] == len(rt) == len(times)
    np.testing.assert_allclose(times, rt, rtol=1e-12, atol=0)
    assert _rel(wave, rw) < 1e-9
    np.testing.assert_array_equal(x_end, wave[-1])          # x receives the last accepted state
    assert info["t_end"] == pytest.approx(tstop, rel=1e-12)


@pytest.mark.parametrize("name", ["rc_charging", "rl_step"])
def test_uic_start_on_gpu(name):
    ckt, _, _, _ = CASES[name]()
    s = mna.compile_circuit(ckt)
    x = S.uic_initial_conditions(ckt, s)
    np.testing.assert_allclose(x, tref.uic_initial_conditions(s, ckt), rtol=0, atol=1e-12)


def _rc_diode_sources():
    """RC sections driven by PULSE, SIN, PWL and EXP sources, a current
    source and a diode clamp: TRAP steps carry the diode current in f(x)."""
    b = ck.CircuitBuilder()
    b.vsource(1, 0, dc=0.0, name="VP", tran=(ck.TRAN_PULSE, (0.0, 1.0, 2e-9, 1e-9, 1e-9, 5e-9, 20e-9)))
    b.vsource(2, 0, dc=0.0, name="VS", tran=(ck.TRAN_SIN, (0.5, 0.4, 1e8, 1e-9, 1e7)))
    b.vsource(3, 0, dc=0.0, name="VW", tran=(ck.TRAN_PWL, ((0.0, 0.0), (5e-9, 2.0), (10e-9, -1.0), (30e-9, 0.5))))
    b.vsource(4, 0, dc=0.0, name="VE", tran=(ck.TRAN_EXP, (0.0, 1.5, 1e-9, 3e-9, 12e-9, 4e-9)))
    b.resistors([1, 2, 3, 4, 5, 6, 7], [5, 6, 7, 8, 6, 7, 8], [1e3, 2e3, 500.0, 1.5e3, 5e3, 4e3, 3e3])
    b.capacitors([5, 6, 7, 8], [0, 0, 0, 0], [1e-12, 2e-12, 0.5e-12, 3e-12])
    b.isource(0, 8, dc=1e-4, name="I1")
    b.diodes([6, 7], [0, 8], is_=1e-14)
    return b.build()


def test_nonlinear_sources_and_diodes_match_oracle():
    s = mna.compile_circuit(_rc_diode_sources())
    x0, _ = newton_ref.newton(s)
    rt, rw, rst = tref.adaptive_transient(s, x0, 0.5e-9, 30e-9, 0.0, list(range(s.size)))
    times, wave, info, _ = _gpu_adaptive(s, x0, 0.5e-9, 30e-9)
    assert rst["rejected"] >= 1                    # the edges force rejections
    assert (info["accepted"], info["rejected"]) == (rst["accepted"], rst["rejected"])
    np.testing.assert_allclose(times, rt, rtol=1e-12, atol=0)
    assert _rel(wave, rw) < 1e-9


def test_mosfet_chain_matches_oracle():
    s = mna.compile_circuit(ck.inverter_chain(stages=6, seed=2))
    x0, _ = newton_ref.newton(s)
    rt, rw, rst = tref.adaptive_transient(s, x0, 5e-12, 300e-12, 0.0, list(range(s.size)))
    times, wave, info, _ = _gpu_adaptive(s, x0, 5e-12, 300e-12)
    assert (info["accepted"], info["rejected"]) == (rst["accepted"], rst["rejected"])
    np.testing.assert_allclose(times, rt, rtol=1e-12, atol=0)
    assert _rel(wave, rw) < 1e-9


def test_truncated_output_and_tstart():
    ckt, tstep, tstop, uic = CASES["pulse_rc"]()
    s = mna.compile_circuit(ckt)
    x0 = _start(ckt, s, uic)
    full_t, full_w, full_i, _ = _gpu_adaptive(s, x0, tstep, tstop)
    t5, w5, i5, _ = _gpu_adaptive(s, x0, tstep, tstop, max_points=5)
    assert i5["points"] == full_i["points"] > 5 and len(t5) == 5
    np.testing.assert_array_equal(t5, full_t[:5])
    np.testing.assert_array_equal(w5, full_w[:5])
    tl, wl, il, _ = _gpu_adaptive(s, x0, tstep, tstop, tstart=100e-6)
    keep = full_t >= 100e-6
    np.testing.assert_array_equal(tl, full_t[keep])
    np.testing.assert_array_equal(wl, full_w[keep])


def test_bad_arguments():
    ckt, _, _, _ = CASES["rc_charging"]()
    s = mna.compile_circuit(ckt)
    with pytest.raises(S.InvalidArgument):
        _gpu_adaptive(s, np.zeros(s.size), 0.0, 1e-3)
    with pytest.raises(S.InvalidArgument):
        _gpu_adaptive(s, np.zeros(s.size), 1e-6, float("inf"))
