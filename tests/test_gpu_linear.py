"""GPU parity: linear solves and SolverBackend ops through the C ABI vs the oracle."""
import numpy as np
import pytest

from oracle import linear_ref
from oracle.mna_ref import RefCsr
from ohmnivore_b200 import circuits as ck
from ohmnivore_b200 import mna
from ohmnivore_b200 import solver as S
from tests.golden import known_answers as KA

pytestmark = pytest.mark.gpu


def _mcsr(case):
    a = RefCsr.from_triplets(case["n"], case.get("ncols", case["n"]), case["trip"])
    return mna.Csr(a.nrows, a.ncols, np.array(a.row_pointers, np.int64), np.array(a.col_indices, np.int64),
                   np.array(a.values, np.float64))


@pytest.mark.parametrize("case", KA.REAL_SOLVES, ids=lambda c: c["name"])
def test_solve_real_known_answers(ctx, case):
    a = _mcsr(case)
    solver = S.GpuSolver(ctx, S.BiCgStabParams(tolerance=1e-14))
    x = solver.solve_real(a, case["b"])
    ax = linear_ref.spmv(a.nrows, a.row_ptr, a.col, a.val, x)
    np.testing.assert_allclose(ax, case["b"], atol=1e-10, rtol=0)
    if case["x"] is not None:
        np.testing.assert_allclose(x, case["x"], atol=1e-10, rtol=0)


def test_solve_real_dimension_mismatch(ctx):
    case = KA.REAL_ERRORS[1]
    with pytest.raises(S.SolveError, match="dimension"):
        S.GpuSolver(ctx).solve_real(_mcsr(case), case["b"])


def test_solve_real_empty(ctx):
    a = mna.Csr(0, 0, np.zeros(1, np.int64), np.zeros(0, np.int64), np.zeros(0))
    assert S.GpuSolver(ctx).solve_real(a, []).shape == (0,)


def test_solve_real_zero_rhs(ctx):
    """bicgstab.rs:91-95: b = 0 -> x = 0."""
    case = KA.REAL_SOLVES[1]
    x = S.GpuSolver(ctx).solve_real(_mcsr(case), [0.0, 0.0])
    np.testing.assert_array_equal(x, [0.0, 0.0])


def test_solve_real_bad_params(ctx):
    case = KA.REAL_SOLVES[1]
    with pytest.raises(S.SolveError, match="max_iterations"):
        S.GpuSolver(ctx, S.BiCgStabParams(max_iterations=0)).solve_real(_mcsr(case), case["b"])
    with pytest.raises(S.SolveError, match="tolerance"):
        S.GpuSolver(ctx, S.BiCgStabParams(tolerance=0.0)).solve_real(_mcsr(case), case["b"])


def test_solve_real_maxiter_reported(ctx):
    s = mna.compile_circuit(ck.resistor_ladder(2000, seed=5))
    with pytest.raises(S.SolveError, match="did not converge") as ei:
        S.GpuSolver(ctx, S.BiCgStabParams(max_iterations=1, tolerance=1e-14)).solve_real(s.g, s.b_dc)
    assert ei.value.krylov_code == 2


def test_solve_real_nan_rhs(ctx):
    case = KA.REAL_SOLVES[1]
    with pytest.raises(S.SolveError):
        S.GpuSolver(ctx).solve_real(_mcsr(case), [np.nan, 1.0])


@pytest.mark.parametrize("case", KA.DC_CASES, ids=lambda c: c["name"])
def test_dc_known_answers_gpu(ctx, case):
    """integration_test.rs:48-125 through the GPU BiCGSTAB."""
    ckt = KA.build_circuit(case["comps"])
    s = mna.compile_circuit(ckt)
    x = S.GpuSolver(ctx, S.BiCgStabParams(tolerance=1e-13)).solve_real(s.g, s.b_dc)
    for lbl, v in case["v"].items():
        assert abs(x[s.node_index(lbl)] - v) < case["v_tol"]
    for name, i in case.get("i", {}).items():
        k = [ckt.names[c] for c in s.branch_components].index(name)
        assert abs(x[s.n_nodes + k] - i) < case["i_tol"]


def _rel_err(x, ref, sl):
    return float(np.max(np.abs(x[sl] - ref[sl])) / np.max(np.abs(ref[sl])))


@pytest.mark.parametrize("n_nodes", [200, 2000])
def test_ladder_fp64_vs_dense_oracle(ctx, n_nodes):
    """Resistor ladder (the 10k-node benchmark recipe, smaller): block-Jacobi
    BiCGSTAB vs the dense GE restatement, 1e-9 norm-wise.  The residual
    tolerance is relative to ||b|| = the 10 V source, so the node-current
    residual of tol 1e-12 still leaves ~2e-9 relative voltage error on this
    ladder; 1e-13 meets the 1e-9 bar."""
    s = mna.compile_circuit(ck.resistor_ladder(n_nodes, seed=0))
    ref = linear_ref.dense_solve_real(s.size, s.size, s.g.row_ptr, s.g.col, s.g.val, s.b_dc)
    solver = S.GpuSolver(ctx, S.BiCgStabParams(tolerance=1e-13))
    x = solver.solve_real(s.g, s.b_dc)
    assert _rel_err(x, ref, slice(0, s.n_nodes)) < 1e-9
    assert _rel_err(x, ref, slice(s.n_nodes, s.size)) < 1e-9


@pytest.mark.slow
def test_ladder_10k_fp64_and_mixed(ctx):
    s = mna.compile_circuit(ck.resistor_ladder(10_000, seed=0))
    ref = linear_ref.sparse_lu_solve(s.size, s.g.row_ptr, s.g.col, s.g.val, s.b_dc)
    for prec in (0, 1):
        p = S.BiCgStabParams(tolerance=1e-13, precision=prec, max_refinements=30, max_iterations=20000)
        x = S.GpuSolver(ctx, p).solve_real(s.g, s.b_dc)
        assert _rel_err(x, ref, slice(0, s.n_nodes)) < 1e-9, prec
        assert _rel_err(x, ref, slice(s.n_nodes, s.size)) < 1e-9, prec


def test_mixed_precision_iterative_refinement(ctx):
    """FP32 Krylov inside FP64 iterative refinement reaches the FP64 answer."""
    s = mna.compile_circuit(ck.resistor_ladder(2000, seed=4))
    ref = linear_ref.sparse_lu_solve(s.size, s.g.row_ptr, s.g.col, s.g.val, s.b_dc)
    solver = S.GpuSolver(ctx, S.BiCgStabParams(tolerance=1e-14, precision=1, max_refinements=20))
    x = solver.solve_real(s.g, s.b_dc)
    assert _rel_err(x, ref, slice(0, s.n_nodes)) < 1e-9
    assert _rel_err(x, ref, slice(s.n_nodes, s.size)) < 1e-9
    assert solver.last_info["iterations"] >= 2        # refinement sweeps were used
    assert solver.last_info["final_residual_norm"] < 1e-14 * solver.last_info["b_norm"]


@pytest.mark.parametrize("lengths", ["short", "mixed_long", "dense_rows"])
def test_spmv_row_and_long_row_paths(ctx, lengths):
    """The backend SpMV is bit-identical to a sequential CSR product on rows
    of up to 32 nonzeros (one thread per row, CSR order); longer rows are
    summed by their whole warp, within 1e-13; empty rows give 0."""
    rng = np.random.default_rng({"short": 1, "mixed_long": 2, "dense_rows": 3}[lengths])
    n = 5000
    if lengths == "short":
        cnt = rng.integers(0, 8, n)
    elif lengths == "mixed_long":
        cnt = rng.integers(0, 6, n)
        cnt[rng.choice(n, 40, replace=False)] = rng.integers(200, 3000, 40)
    else:
        cnt = rng.integers(20, 60, n)
    rp = np.concatenate([[0], np.cumsum(cnt)]).astype(np.int64)
    col = np.concatenate([np.sort(rng.choice(n, c, replace=False)) for c in cnt]).astype(np.int64)
    val = rng.standard_normal(len(col))
    a = mna.Csr(n, n, rp, col, val)
    x = rng.standard_normal(n)
    ref = np.zeros(n)
    for i in range(n):                       # sequential CSR order
        acc = 0.0
        for k in range(rp[i], rp[i + 1]):
            acc += val[k] * x[col[k]]
        ref[i] = acc
    be = S.SolverBackend(ctx)
    A = be.upload_matrix(a)
    bx, by = be.new_buffer(n), be.new_buffer(n)
    bx.upload(x)
    be.spmv(A, bx, by)
    got = by.download()
    short = cnt <= 32                        # summed by one thread in CSR order
    assert short.any()
    np.testing.assert_array_equal(got[short], ref[short])
    np.testing.assert_allclose(got, ref, rtol=1e-13, atol=1e-13)


def test_backend_ops(ctx):
    """SolverBackend ops (backend.rs:51-96) vs numpy."""
    s = mna.compile_circuit(ck.diode_mesh(20, 20, seed=3))
    be = S.SolverBackend(ctx)
    rng = np.random.default_rng(0)
    x = rng.standard_normal(s.size)
    y0 = rng.standard_normal(s.size)
    A = be.upload_matrix(s.g)
    bx, by = be.new_buffer(s.size), be.new_buffer(s.size)
    bx.upload(x)
    be.spmv(A, bx, by)
    np.testing.assert_allclose(by.download(), linear_ref.spmv(s.size, s.g.row_ptr, s.g.col, s.g.val, x),
                               rtol=1e-13, atol=1e-13)
    by.upload(y0)
    assert abs(be.dot(bx, by) - float(x @ y0)) < 1e-12 * abs(x).sum() * abs(y0).max()
    # dot_n (backend.rs:60-68): owned entries only
    k = s.size // 3
    assert abs(be.dot_n(bx, by, k) - float(x[:k] @ y0[:k])) < 1e-12 * abs(x[:k]).sum() * abs(y0).max()
    assert be.dot_n(bx, by, 0) == 0.0
    assert be.dot_n(bx, by, s.size) == be.dot(bx, by)
    with pytest.raises(S.InvalidArgument):
        be.dot_n(bx, by, s.size + 1)
    be.axpy(2.5, bx, by)
    np.testing.assert_allclose(by.download(), y0 + 2.5 * x, rtol=0, atol=1e-15)
    be.scale(-3.0, by)
    np.testing.assert_allclose(by.download(), (y0 + 2.5 * x) * -3.0, rtol=0, atol=1e-14)
    be.copy(bx, by)
    np.testing.assert_array_equal(by.download(), x)
    bsol = be.new_buffer(s.size)
    bb = be.new_buffer(s.size)
    bb.upload(s.b_dc)
    info = be.solve_real_device(A, bb, bsol, S.BiCgStabParams(tolerance=1e-13))
    ref = linear_ref.sparse_lu_solve(s.size, s.g.row_ptr, s.g.col, s.g.val, s.b_dc)
    assert _rel_err(bsol.download(), ref, slice(0, s.size)) < 1e-9
    assert info["kernel_launches"] >= 1


# ---- ISAI(1) (src/solver/gpu.rs:139-168: the reference's choice for any zero diagonal) ----
@pytest.mark.parametrize("case", [c for c in KA.REAL_SOLVES if c["name"] != "pivoting_3x3"],
                         ids=lambda c: c["name"])
def test_solve_real_isai_known_answers(ctx, case):
    """ISAI(1) on the reference's known answers.  pivoting_3x3 has a zero
    leading diagonal that needs row pivoting; ILU(0) in natural order cannot
    factor it (MNA matrices order branch rows after node rows, so they can)."""
    a = _mcsr(case)
    x = S.GpuSolver(ctx, S.BiCgStabParams(tolerance=1e-14, precond=2)).solve_real(a, case["b"])
    ax = linear_ref.spmv(a.nrows, a.row_ptr, a.col, a.val, x)
    np.testing.assert_allclose(ax, case["b"], atol=1e-10, rtol=0)


@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "mixed"])
def test_isai_ladder_and_mesh_vs_oracle(ctx, prec):
    for sysm in (mna.compile_circuit(ck.resistor_ladder(2000, seed=0)),
                 mna.compile_circuit(ck.diode_mesh(60, 60, seed=5, diode_frac=0.0))):
        ref = linear_ref.sparse_lu_solve(sysm.size, sysm.g.row_ptr, sysm.g.col, sysm.g.val, sysm.b_dc)
        p = S.BiCgStabParams(tolerance=1e-14, precond=2, precision=prec, max_refinements=20 if prec else 1)
        solver = S.GpuSolver(ctx, p)
        x = solver.solve_real(sysm.g, sysm.b_dc)
        assert _rel_err(x, ref, slice(0, sysm.n_nodes)) < 1e-9


def _isai_apply(ctx, a, r):
    import ctypes
    from ohmnivore_b200 import _lib
    rp = np.ascontiguousarray(a.row_ptr, dtype=np.uint32)
    ci = np.ascontiguousarray(a.col, dtype=np.uint32)
    val = np.ascontiguousarray(a.val, dtype=np.float64)
    r = np.ascontiguousarray(r, dtype=np.float64)
    z = np.zeros_like(r)
    st = ctx.lib.ohm_isai_apply(ctx.handle, a.nrows, len(val), _lib.u32ptr(rp), _lib.u32ptr(ci), _lib.dptr(val),
                                _lib.dptr(r), _lib.dptr(z), r.shape[0])
    assert st == 0, _lib.last_error()
    return z


@pytest.mark.parametrize("make", [lambda: ck.resistor_ladder(60, seed=0),
                                  lambda: ck.diode_mesh(9, 9, seed=5, diode_frac=0.0),
                                  lambda: ck.diode_mesh(3, 40, seed=2, diode_frac=0.0)],
                         ids=["ladder60", "mesh9x9", "mesh3x40"])
def test_isai_apply_matches_oracle(ctx, make):
    """The device ISAI(1) set-up (Chow-Patel ILU(0) + level-1 columns) and its
    apply z = M_U (M_L r) agree with the oracle restatement to rounding."""
    from oracle import isai_ref
    s = mna.compile_circuit(make())
    n = s.size
    ML, MU = isai_ref.isai1_device_ref(n, s.g.row_ptr, s.g.col, s.g.val)
    R = np.random.default_rng(4).standard_normal((3, n))
    Z = _isai_apply(ctx, s.g, R)
    for r, z in zip(R, Z):
        ref = MU @ (ML @ r)
        assert np.max(np.abs(z - ref)) <= 1e-11 * np.max(np.abs(ref))
