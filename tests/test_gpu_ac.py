"""GPU: batched AC sweep (one launch, one block per frequency point, complex
FP64 BiCGSTAB on G + j w C formed on the fly) against the oracle's complex
sparse LU per point (src/analysis/ac.rs, src/sparse.rs:149-178)."""
import numpy as np
import pytest

from oracle import ac_ref, newton_ref
from ohmnivore_b200 import circuits as ck
from ohmnivore_b200 import mna
from ohmnivore_b200 import solver as S

pytestmark = pytest.mark.gpu


def _params(**kw):
    """||r|| < 1e-16 ||b||: the reference's unscaled stopping test, taken to
    the FP64 floor, since the RC ladders' high-frequency points have node
    conductances from 1e-4 S to ~1 S in one system."""
    p = S.BiCgStabParams(max_iterations=20000, tolerance=1e-16)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _err(x, ref):
    """Norm-wise relative error per frequency point, worst over points."""
    return float(np.max(np.max(np.abs(x - ref), axis=1) / np.maximum(np.max(np.abs(ref), axis=1), 1e-300)))


def _rc_ladder(sections=40, seed=0):
    rng = np.random.default_rng(seed)
    b = ck.CircuitBuilder()
    b.vsource(1, 0, dc=0.0, ac=(1.0, 0.0), name="VIN")
    nodes = np.arange(1, sections + 2)
    b.resistors(nodes[:-1], nodes[1:], rng.uniform(100.0, 10e3, sections))
    b.capacitors(nodes[1:], 0, rng.uniform(1e-12, 1e-10, sections))
    return b.build()


def _rlc():
    b = ck.CircuitBuilder()
    b.vsource(1, 0, dc=0.0, ac=(1.0, 30.0), name="VIN")
    b.resistors([1, 3, 4], [2, 0, 0], [50.0, 1e3, 200.0])
    b.inductors([2, 3], [3, 4], [1e-6, 4.7e-6])
    b.capacitors([3, 4], [0, 0], [1e-9, 2.2e-10])
    b.isource(0, 4, dc=0.0, ac=(1e-3, -45.0), name="I1")
    return b.build()


@pytest.mark.parametrize("make", [_rc_ladder, _rlc], ids=["rc_ladder", "rlc_inductors"])
def test_ac_sweep_matches_oracle(make):
    s = mna.compile_circuit(make())
    freqs = S.ac_frequencies("dec", 10, 1e3, 1e9)
    assert len(freqs) == 60
    x, infos = S.ac_sweep(s, freqs, _params())
    ref = ac_ref.ac_sweep(s, freqs)
    assert _err(x[:, : s.n_nodes], ref[:, : s.n_nodes]) < 1e-9
    assert _err(x[:, s.n_nodes:], ref[:, s.n_nodes:]) < 1e-9
    assert all(p["krylov_code"] == 1 for p in infos)


def test_small_signal_ac_of_diode_mesh():
    """Linearised at the DC operating point: G replaced by the Jacobian values
    J(x_dc) (device conductances included), then the sweep."""
    import torch
    s = mna.compile_circuit(ck.rc_diode_mesh(12, 12, seed=4))
    x_dc, _ = newton_ref.newton(s)
    plan = S.NewtonPlan(s)
    try:
        jvals, _ = plan.assemble(x_dc)
    finally:
        plan.close()
    b_ac = np.zeros(s.size, dtype=np.complex128)
    b_ac[s.n_nodes] = 1.0                          # 1 V AC on the drive source branch
    s.b_ac = b_ac
    freqs = S.ac_frequencies("oct", 4, 1e6, 1e10)
    x, _ = S.ac_sweep(s, freqs, _params(), g_values=jvals)
    lin = mna.MnaSystem(**{**s.__dict__, "g": mna.Csr(s.g.nrows, s.g.ncols, s.g.row_ptr, s.g.col, jvals)})
    ref = ac_ref.ac_sweep(lin, freqs)
    assert _err(x, ref) < 1e-9


def test_reference_jacobi_without_branch_rows():
    """The reference's Jacobi preconditioner (inverse diagonal) on a current-
    driven RC network, which has no zero-diagonal rows."""
    b = ck.CircuitBuilder()
    rng = np.random.default_rng(3)
    b.isource(0, 1, dc=0.0, ac=(1e-3, 0.0))
    b.resistors(np.arange(1, 30), np.arange(2, 31), rng.uniform(10.0, 1e3, 29))
    b.resistors(np.arange(1, 31), 0, rng.uniform(1e3, 1e5, 30))
    b.capacitors(np.arange(1, 31), 0, rng.uniform(1e-12, 1e-9, 30))
    s = mna.compile_circuit(b.build())
    freqs = S.ac_frequencies("lin", 25, 1e3, 1e8)
    x, _ = S.ac_sweep(s, freqs, _params(precond=1))
    assert _err(x, ac_ref.ac_sweep(s, freqs)) < 1e-9


def test_many_points_one_launch_and_dc_point():
    """Hundreds of points (more than the resident blocks) and f = 0, where the
    system is G x = b_ac."""
    s = mna.compile_circuit(_rc_ladder(25, seed=5))
    freqs = np.concatenate([[0.0], S.ac_frequencies("dec", 100, 1.0, 1e9)])
    x, infos = S.ac_sweep(s, freqs, _params())
    ref = ac_ref.ac_sweep(s, freqs)
    assert len(freqs) == 901
    assert _err(x, ref) < 1e-9


def test_unconverged_point_is_reported():
    s = mna.compile_circuit(_rc_ladder(40, seed=1))
    with pytest.raises(S.SolveError):
        S.ac_sweep(s, [1e3, 1e6], _params(max_iterations=2))


def test_wide_blocks_on_a_large_system():
    """A system of >= 2048 rows swept at fewer points than SMs runs 1024-thread
    blocks, here teams of two per point (the spare SMs join the points);
    same answers as the oracle."""
    ckt = ck.rc_diode_mesh(50, 50, seed=4, diode_frac=0.0)
    src = int(np.flatnonzero(ckt.kind == ck.V)[0])
    ckt.ac[src] = (1.0, 0.0)
    s = mna.compile_circuit(ckt)
    assert s.size >= 2048
    freqs = np.array([1e4, 1e7, 1e9, 3e10, 1e12])
    x, infos = S.ac_sweep(s, freqs, _params(max_iterations=50000))
    assert all(p["krylov_code"] == 1 for p in infos)
    assert _err(x, ac_ref.ac_sweep(s, freqs)) < 1e-9


def test_teams_of_mixed_sizes():
    """60 points on a 4,902-row mesh: every point gets a team of two blocks
    and the lowest frequencies (the slowest) a third, with the dot products
    summed over the members; every point matches the oracle."""
    ckt = ck.rc_diode_mesh(70, 70, seed=4, diode_frac=0.0)
    src = int(np.flatnonzero(ckt.kind == ck.V)[0])
    ckt.ac[src] = (1.0, 0.0)
    s = mna.compile_circuit(ckt)
    freqs = S.ac_frequencies("dec", 6, 1e3, 1e13)[:60]
    assert len(freqs) == 60 and s.size >= 4096
    x, infos = S.ac_sweep(s, freqs, _params(max_iterations=50000))
    assert all(p["krylov_code"] == 1 for p in infos)
    assert _err(x, ac_ref.ac_sweep(s, freqs)) < 1e-9
