"""GPU: adjoint sensitivities (J^T lambda = w by the library's BiCGSTAB on the
transposed CSR, device back-stamping; checkpointed transient adjoint) against
the oracle's LU adjoint, its FP64 forward sensitivities and central finite
differences, plus a thin torch.autograd.Function wrapper."""
import copy

import numpy as np
import pytest

from oracle import adjoint_ref, newton_ref
from ohmnivore_b200 import circuits as ck
from ohmnivore_b200 import mna
from ohmnivore_b200 import solver as S

pytestmark = pytest.mark.gpu

H = 2e-12


def _newton():
    return S.NewtonParams(max_iterations=100, abs_tol=1e-12, bicgstab_max_iterations=20000,
                          bicgstab_tolerance=1e-15, inner_rtol=1e-8)


def _krylov():
    return S.BiCgStabParams(max_iterations=20000, tolerance=1e-15)


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _probe_w(s, label):
    w = np.zeros(s.size)
    w[s.node_index(label)] = 1.0
    return w


def test_dc_adjoint_matches_oracle():
    ckt = ck.diode_mesh(10, 10, seed=2)
    s = mna.compile_circuit(ckt)
    comps = S.ComponentTable(ckt, s)
    x, _ = newton_ref.newton(s)
    w = _probe_w(s, 2 + 99)
    ref, lam_ref = adjoint_ref.dc_adjoint(s, comps, x, w)
    import torch
    plan = S.NewtonPlan(s)
    try:
        xd = torch.from_numpy(x).cuda()
        g, lam, info = S.adjoint_dc(plan, xd.data_ptr(), w, comps, _krylov())
    finally:
        plan.close()
    assert _rel(lam, lam_ref) < 1e-9
    assert _rel(g["R"], ref["R"]) < 1e-8
    assert _rel(g["Is"], ref["Is"]) < 1e-8
    assert info["output"] == pytest.approx(x[s.node_index(101)], rel=1e-14)


def _transient_case():
    ckt = ck.rc_diode_mesh(6, 6, seed=4, diode_frac=0.2)
    s = mna.compile_circuit(ckt)
    return ckt, s, S.ComponentTable(ckt, s), 2 + 35       # probe: the corner opposite the drive


def _gpu_transient_adjoint(s, comps, x0, n_steps, w, checkpoint_every):
    import torch
    plan = S.NewtonPlan(s)
    tr = S.Transient(plan, [])
    try:
        xd = torch.from_numpy(x0).cuda()
        g, info = tr.adjoint(xd.data_ptr(), 0.0, H, n_steps, w, comps, _newton(), checkpoint_every, _krylov())
        assert np.array_equal(xd.cpu().numpy(), x0)              # x0 left unchanged
        return g, info
    finally:
        tr.close()
        plan.close()


def test_transient_adjoint_matches_oracle_and_forward_sensitivity():
    ckt, s, comps, probe = _transient_case()
    x0, _ = newton_ref.newton(s)
    n_steps = 30
    w = _probe_w(s, probe)
    g, info = _gpu_transient_adjoint(s, comps, x0, n_steps, w, 7)
    states = adjoint_ref.transient_states(s, x0, 0.0, H, n_steps)
    ref = adjoint_ref.transient_adjoint(s, comps, states, H, w)
    for k in ("R", "C", "Is"):
        assert _rel(g[k], ref[k]) < 1e-8, k
    assert info["output"] == pytest.approx(states[-1][s.node_index(probe)], rel=1e-10)
    # the DC start solve is skipped when x0 is zero (every DC term vanishes)
    assert info["steps"] == n_steps and info["linear_solves"] == n_steps + (1 if np.any(x0) else 0)
    assert info["recompute_launches"] == 5                     # ceil(30 / 7) segments
    for kind, j in (("R", 4), ("C", 9), ("Is", 2)):
        fs = adjoint_ref.forward_sensitivity(s, comps, states, H, w, kind, j)
        assert abs(g[kind][j] - fs) <= 1e-8 * max(abs(fs), np.max(np.abs(g[kind]))), (kind, j)


def test_transient_adjoint_matches_central_differences():
    """Central differences (relative step 1e-6) of the oracle's transient on
    a few resistors and capacitors, within 1e-6 relative."""
    ckt, s, comps, probe = _transient_case()
    x0, _ = newton_ref.newton(s)
    n_steps = 20
    w = _probe_w(s, probe)
    g, _ = _gpu_transient_adjoint(s, comps, x0, n_steps, w, 20)

    def output(c2):
        s2 = mna.compile_circuit(c2)
        x2, _ = newton_ref.newton(s2)
        return adjoint_ref.transient_states(s2, x2, 0.0, H, n_steps)[-1][s2.node_index(probe)]

    scale = {k: np.max(np.abs(g[k])) for k in ("R", "C")}
    for kind, j in (("R", 0), ("R", 17), ("R", 40), ("C", 3), ("C", 20), ("C", 35)):
        idx = (comps.r_index if kind == "R" else comps.c_index)[j]
        v = ckt.value[idx]
        outs = []
        for sign in (1, -1):
            c2 = copy.deepcopy(ckt)
            c2.value[idx] = v * (1 + sign * 1e-6)
            outs.append(output(c2))
        fd = (outs[0] - outs[1]) / (2e-6 * v)
        assert abs(g[kind][j] - fd) <= 1e-6 * max(abs(fd), 1e-3 * scale[kind]), (kind, j, g[kind][j], fd)


def test_checkpoint_interval_does_not_change_gradients():
    """Recomputing segments from checkpoints reproduces the forward states
    exactly, so every interval gives bit-identical gradients, the same as
    keeping every state (checkpoint_every = 0)."""
    _, s, comps, probe = _transient_case()
    x0, _ = newton_ref.newton(s)
    w = _probe_w(s, probe)
    gs = [_gpu_transient_adjoint(s, comps, x0, 24, w, k)[0] for k in (0, 1, 5, 24)]
    for g in gs[1:]:
        for k in ("R", "C", "Is"):
            np.testing.assert_array_equal(g[k], gs[0][k])


def test_torch_autograd_wrapper():
    """A thin torch.autograd.Function over the C ABI: forward runs the DC
    point and the transient through the adjoint entry point (which returns
    the output and its gradient together), backward scales the saved
    gradient.  Checked against the adjoint entry point and against central
    differences of the oracle's transient."""
    import torch

    base_ckt, _, _, probe = _transient_case()
    r_idx = np.flatnonzero(base_ckt.kind == ck.R)
    c_idx = np.flatnonzero(base_ckt.kind == ck.C)
    n_steps = 15

    def solve(r_vals, c_vals):
        c2 = copy.deepcopy(base_ckt)
        c2.value[r_idx] = r_vals
        c2.value[c_idx] = c_vals
        s2 = mna.compile_circuit(c2)
        comps = S.ComponentTable(c2, s2)
        plan = S.NewtonPlan(s2)
        tr = S.Transient(plan, [])
        try:
            x = torch.zeros(s2.size, dtype=torch.float64, device="cuda")
            plan.newton_device(x.data_ptr(), _newton())
            g, info = tr.adjoint(x.data_ptr(), 0.0, H, n_steps, _probe_w(s2, probe), comps, _newton(), 8, _krylov())
        finally:
            tr.close()
            plan.close()
        return info["output"], g

    class TransientOutput(torch.autograd.Function):
        @staticmethod
        def forward(ctx, r, c):
            out, g = solve(r.detach().cpu().numpy(), c.detach().cpu().numpy())
            ctx.save_for_backward(torch.from_numpy(g["R"]), torch.from_numpy(g["C"]))
            return torch.tensor(out, dtype=torch.float64)

        @staticmethod
        def backward(ctx, grad_out):
            gr, gc = ctx.saved_tensors
            return grad_out * gr, grad_out * gc

    r = torch.tensor(base_ckt.value[r_idx], dtype=torch.float64, requires_grad=True)
    c = torch.tensor(base_ckt.value[c_idx], dtype=torch.float64, requires_grad=True)
    loss = 3.0 * TransientOutput.apply(r, c)
    loss.backward()
    _, g = solve(base_ckt.value[r_idx], base_ckt.value[c_idx])
    np.testing.assert_allclose(r.grad.numpy(), 3.0 * g["R"], rtol=1e-12, atol=0)
    np.testing.assert_allclose(c.grad.numpy(), 3.0 * g["C"], rtol=1e-12, atol=0)

    def oracle_output(r_vals, c_vals):
        c2 = copy.deepcopy(base_ckt)
        c2.value[r_idx] = r_vals
        c2.value[c_idx] = c_vals
        s2 = mna.compile_circuit(c2)
        x2, _ = newton_ref.newton(s2)
        return adjoint_ref.transient_states(s2, x2, 0.0, H, n_steps)[-1][s2.node_index(probe)]

    rv, cv = base_ckt.value[r_idx].copy(), base_ckt.value[c_idx].copy()
    for j in (2, 30):
        rp, rm = rv.copy(), rv.copy()
        rp[j] *= 1 + 1e-6
        rm[j] *= 1 - 1e-6
        fd = 3.0 * (oracle_output(rp, cv) - oracle_output(rm, cv)) / (2e-6 * rv[j])
        assert abs(float(r.grad[j]) - fd) <= 1e-6 * max(abs(fd), 1e-3 * float(r.grad.abs().max())), (j, fd)


# ---- MOSFET |VTO| and KP (descriptor values; KP carries W/L) ----

def _chain_case(stages, vin):
    from tests.test_oracle_adjoint import analog_chain
    ckt = analog_chain(stages=stages, vin=vin)
    s = mna.compile_circuit(ckt)
    return ckt, s, S.ComponentTable(ckt, s)


def test_dc_adjoint_mosfet_gradients():
    """Inverter chain with its first stage on its transfer curve (input
    0.82 V): the GPU's d V(out_1) / d(|VTO|, KP) of every MOSFET against the
    oracle's LU adjoint
    and forward sensitivities (1e-8) and against central differences of the
    oracle's Newton on the f32 descriptor values (1e-6)."""
    import torch
    from tests.test_oracle_adjoint import _fd
    ckt, s, comps = _chain_case(4, 0.82)
    x, _ = newton_ref.newton(s)
    probe = s.node_index(2 + 1)
    w = np.zeros(s.size)
    w[probe] = 1.0
    ref, _ = adjoint_ref.dc_adjoint(s, comps, x, w)
    plan = S.NewtonPlan(s)
    try:
        xd = torch.from_numpy(x).cuda()
        g, _, _ = S.adjoint_dc(plan, xd.data_ptr(), w, comps, _krylov())
    finally:
        plan.close()
    for kind in ("VTO", "KP"):
        scale = np.max(np.abs(ref[kind]))
        assert scale > 0.0
        assert np.max(np.abs(g[kind] - ref[kind])) <= 1e-8 * scale, kind
        for j in range(len(s.mosfet_descriptors)):
            fs = adjoint_ref.forward_sensitivity(s, comps, [x], 1.0, w, kind, j)
            assert abs(g[kind][j] - fs) <= 1e-8 * max(abs(fs), scale), (kind, j)
        for j in (0, 1):
            fd = _fd(s, kind, j, lambda s2: newton_ref.newton(s2, x0=x)[0][probe])
            assert abs(g[kind][j] - fd) <= 1e-6 * max(abs(fd), 1e-3 * scale), (kind, j, g[kind][j], fd)


def test_transient_adjoint_mosfet_gradients():
    """Backward Euler through the input's rising edge (12 steps of 5 ps,
    checkpoints every 5): d V(out_1) / d(|VTO|, KP) against the oracle's LU
    adjoint and forward sensitivities (1e-8); the gradient flows through a
    torch.autograd.Function over the C ABI."""
    import torch
    hh = 5e-12
    ckt, s, comps = _chain_case(3, 0.0)
    x0, _ = newton_ref.dc_operating_point(s)
    probe = s.node_index(2 + 1)
    w = np.zeros(s.size)
    w[probe] = 1.0
    n_steps = 12
    states = adjoint_ref.transient_states(s, x0, 0.0, hh, n_steps)
    ref = adjoint_ref.transient_adjoint(s, comps, states, hh, w)

    def gpu(sysm):
        plan = S.NewtonPlan(sysm)
        tr = S.Transient(plan, [])
        try:
            xd = torch.from_numpy(x0).cuda()
            return tr.adjoint(xd.data_ptr(), 0.0, hh, n_steps, w, comps, _newton(), 5, _krylov())
        finally:
            tr.close()
            plan.close()

    g, info = gpu(s)
    assert info["output"] == pytest.approx(states[-1][probe], rel=1e-10)
    for kind in ("VTO", "KP"):
        scale = np.max(np.abs(ref[kind]))
        assert scale > 0.0
        assert np.max(np.abs(g[kind] - ref[kind])) <= 1e-8 * scale, kind
        for j in (0, 1, 4):
            fs = adjoint_ref.forward_sensitivity(s, comps, states, hh, w, kind, j)
            assert abs(g[kind][j] - fs) <= 1e-8 * max(abs(fs), scale), (kind, j)

    class ChainOutput(torch.autograd.Function):
        """o(|VTO|, KP) of the transient, gradient from the adjoint entry point."""
        @staticmethod
        def forward(ctx, vto, kp):
            s2 = copy.deepcopy(s)
            s2.mosfet_descriptors["vto"] = vto.detach().numpy().astype(np.float32)
            s2.mosfet_descriptors["kp"] = kp.detach().numpy().astype(np.float32)
            g2, info2 = gpu(s2)
            ctx.save_for_backward(torch.from_numpy(g2["VTO"]), torch.from_numpy(g2["KP"]))
            return torch.tensor(info2["output"], dtype=torch.float64)

        @staticmethod
        def backward(ctx, grad_out):
            gv, gk = ctx.saved_tensors
            return grad_out * gv, grad_out * gk

    vto = torch.tensor(s.mosfet_descriptors["vto"].astype(np.float64), requires_grad=True)
    kp = torch.tensor(s.mosfet_descriptors["kp"].astype(np.float64), requires_grad=True)
    (2.0 * ChainOutput.apply(vto, kp)).backward()
    np.testing.assert_allclose(vto.grad.numpy(), 2.0 * g["VTO"], rtol=1e-12, atol=0)
    np.testing.assert_allclose(kp.grad.numpy(), 2.0 * g["KP"], rtol=1e-12, atol=0)
