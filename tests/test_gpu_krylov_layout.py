"""GPU parity of the single-system solver's two Krylov layouts
(`ohm_ctx_set_krylov_layout`): each block's CSR slice and Krylov state in
shared memory (automatic at these sizes), and global memory for every block
(the path of systems too large for the slices, forced here at test size so
that the parity suite covers it).  Both against the FP64 oracle, and against
each other bit for bit: the layouts differ only in where the data lives."""
import numpy as np
import pytest

from oracle import linear_ref, newton_ref
from ohmnivore_b200 import _lib
from ohmnivore_b200 import circuits as ck
from ohmnivore_b200 import mna
from ohmnivore_b200 import solver as S

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _params(prec):
    return S.NewtonParams(max_iterations=100, abs_tol=1e-10, bicgstab_max_iterations=20000,
                          bicgstab_tolerance=1e-14, precision=prec, inner_rtol=1e-4)


def _hub_circuit(leaves=5000):
    """A hub node fed from a 1 V source through 10 ohm, with a branch of R in
    series with a diode to ground per leaf: the hub's row has one nonzero per
    leaf (a long row, summed in chunks by the whole grid)."""
    rng = np.random.default_rng(11)
    b = ck.CircuitBuilder()
    b.vsource(1, 0, dc=1.0, name="V1")
    b.resistors([1], [2], [10.0])
    leaf = 3 + np.arange(leaves)
    b.resistors(np.full(leaves, 2), leaf, rng.uniform(1e3, 1e4, leaves))
    b.diodes(leaf, 0, is_=1e-14, n=1.0)
    return b.build()


def _newton(ctx, s, prec):
    stats = {}
    x = S.newton_solve(ctx, s.g.val, s.g.col, s.g.row_ptr, s.b_dc, s.diode_descriptors,
                       s.bjt_descriptors, s.mosfet_descriptors, s.size, s.g.nnz, _params(prec), stats)
    return x, stats


@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "mixed"])
@pytest.mark.parametrize("make", [lambda: ck.diode_mesh(40, 40, seed=1), _hub_circuit],
                         ids=["diode_mesh_40", "hub_5000"])
def test_newton_layouts_match_oracle_and_each_other(make, prec):
    s = mna.compile_circuit(make())
    ref, _ = newton_ref.newton(s)
    nn, br = slice(0, s.n_nodes), slice(s.n_nodes, s.size)
    ctx = S.Context(0)
    try:
        out = {}
        for layout in (_lib.KRYLOV_LAYOUT_AUTO, _lib.KRYLOV_LAYOUT_GLOBAL):
            ctx.set_krylov_layout(layout)
            x, stats = _newton(ctx, s, prec)
            assert _rel(x[nn], ref[nn]) < 1e-9, layout
            assert _rel(x[br], ref[br]) < 1e-9, layout
            assert stats["kernel_launches"] == 1, layout
            out[layout] = (x, stats["krylov_iterations"])
        xa, ka = out[_lib.KRYLOV_LAYOUT_AUTO]
        xg, kg = out[_lib.KRYLOV_LAYOUT_GLOBAL]
        np.testing.assert_array_equal(xg, xa)
        assert kg == ka
    finally:
        ctx.close()


def test_linear_layouts_match_direct_solve():
    """A resistor ladder (linear solve with FP64 refinement), both layouts."""
    s = mna.compile_circuit(ck.resistor_ladder(3000, seed=0))
    ref = linear_ref.sparse_lu_solve(s.size, s.g.row_ptr, s.g.col, s.g.val, s.b_dc)
    nn = slice(0, s.n_nodes)
    ctx = S.Context(0)
    try:
        xs = []
        for layout in (_lib.KRYLOV_LAYOUT_AUTO, _lib.KRYLOV_LAYOUT_GLOBAL):
            ctx.set_krylov_layout(layout)
            solver = S.GpuSolver(ctx, S.BiCgStabParams(tolerance=1e-13, max_iterations=50000))
            x = solver.solve_real(s.g, s.b_dc)
            assert _rel(x[nn], ref[nn]) < 1e-9, layout
            xs.append(x)
        np.testing.assert_array_equal(xs[1], xs[0])
    finally:
        ctx.close()


def test_unknown_layout_is_rejected():
    ctx = S.Context(0)
    try:
        with pytest.raises(Exception):
            ctx.set_krylov_layout(7)
    finally:
        ctx.close()
