"""Pin the oracle and the host compiler against the reference's own known answers."""
import math

import numpy as np
import pytest

from oracle import devices_ref, linear_ref, mna_ref
from oracle.mna_ref import RefCsr
from ohmnivore_b200 import circuits as ck
from ohmnivore_b200 import mna
from tests.golden import known_answers as KA


def _csr(case):
    c = RefCsr.from_triplets(case["n"], case.get("ncols", case["n"]), case["trip"])
    return c


@pytest.mark.parametrize("case", KA.REAL_SOLVES, ids=lambda c: c["name"])
def test_dense_ge_known_answers(case):
    a = _csr(case)
    x = linear_ref.dense_solve_real(a.nrows, a.ncols, a.row_pointers, a.col_indices, a.values, case["b"])
    if case["x"] is not None:
        np.testing.assert_allclose(x, case["x"], atol=case["tol"], rtol=0)
    else:  # verified through spmv (cpu.rs:368-396)
        ax = linear_ref.spmv(a.nrows, a.row_pointers, a.col_indices, a.values, x)
        np.testing.assert_allclose(ax, case["b"], atol=case["tol"], rtol=0)


@pytest.mark.parametrize("case", KA.REAL_SOLVES, ids=lambda c: c["name"])
def test_sparse_lu_known_answers(case):
    a = _csr(case)
    x = linear_ref.sparse_lu_solve(a.nrows, a.row_pointers, a.col_indices, a.values, case["b"])
    ax = linear_ref.spmv(a.nrows, a.row_pointers, a.col_indices, a.values, x)
    np.testing.assert_allclose(ax, case["b"], atol=1e-10, rtol=0)


@pytest.mark.parametrize("case", KA.REAL_ERRORS, ids=lambda c: c["name"])
def test_dense_ge_errors(case):
    a = _csr(case)
    with pytest.raises(linear_ref.SolveError, match=case["err"]):
        linear_ref.dense_solve_real(a.nrows, a.ncols, a.row_pointers, a.col_indices, a.values, case["b"])


def test_dense_ge_empty():
    assert linear_ref.dense_solve_real(0, 0, [0], [], [], []).shape == (0,)


@pytest.mark.parametrize("case", KA.COMPLEX_SOLVES, ids=lambda c: c["name"])
def test_dense_ge_complex_known_answers(case):
    a = RefCsr.from_triplets(case["n"], case["n"], case["trip"])
    x = linear_ref.dense_solve_complex(a.nrows, a.ncols, a.row_pointers, a.col_indices, a.values, case["b"])
    np.testing.assert_allclose(x, case["x"], atol=case["tol"], rtol=0)


@pytest.mark.parametrize("case", KA.COMPLEX_ERRORS, ids=lambda c: c["name"])
def test_dense_ge_complex_errors(case):
    a = RefCsr.from_triplets(case["n"], case["n"], case["trip"])
    with pytest.raises(linear_ref.SolveError):
        linear_ref.dense_solve_complex(a.nrows, a.ncols, a.row_pointers, a.col_indices, a.values, case["b"])


@pytest.mark.parametrize("case", KA.CSR_CASES, ids=lambda c: c["name"])
def test_from_triplets(case):
    a = RefCsr.from_triplets(case["n"], case["n"], case["trip"])
    assert len(a.values) == case["nnz"]
    np.testing.assert_array_equal(a.to_dense(), case["dense"])
    if "row_ptr" in case:
        assert a.row_pointers == case["row_ptr"]


@pytest.mark.parametrize("case", KA.SPMV_CASES, ids=lambda c: c["name"])
def test_spmv(case):
    a = RefCsr.from_triplets(case["n"], case["n"], case["trip"])
    y = linear_ref.spmv(a.nrows, a.row_pointers, a.col_indices, a.values, case["x"])
    np.testing.assert_array_equal(y, case["y"])


def _check_mna(case, got, oracle):
    if case["size"] == 0:
        assert got.size == 0 and oracle["size"] == 0
        return
    gd = got.g.to_dense()
    od = oracle["g"].to_dense()
    for (r, c), v in case.get("g", {}).items():
        assert abs(gd[r, c] - v) < 1e-9, (r, c, gd[r, c], v)
        assert abs(od[r, c] - v) < 1e-9
    for (r, c), v in case.get("c", {}).items():
        assert abs(got.c.to_dense()[r, c] - v) < case.get("c_tol", 1e-9)
    if "b_dc" in case:
        np.testing.assert_allclose(got.b_dc, case["b_dc"], atol=1e-9)
        np.testing.assert_allclose(oracle["b_dc"], case["b_dc"], atol=1e-9)
    for k, v in case.get("b_ac", {}).items():
        assert abs(got.b_ac[k] - v) < 1e-9
        assert abs(oracle["b_ac"][k] - v) < 1e-9
    assert got.size == case["size"] == oracle["size"]
    if "node_labels" in case:
        assert list(got.node_labels) == case["node_labels"] == list(oracle["node_labels"])


@pytest.mark.parametrize("case", KA.MNA_CASES, ids=lambda c: c["name"])
def test_mna_known_answers(case):
    ckt = KA.build_circuit(case["comps"])
    got = mna.compile_circuit(ckt)
    oracle = mna_ref.compile_ref(ckt)
    _check_mna(case, got, oracle)


def test_zero_resistance_rejected():
    """compiler.rs:1114-1123."""
    ckt = KA.build_circuit([("R", "R1", (1, 0), 0.0)])
    with pytest.raises(mna.CompileError, match="zero resistance"):
        mna.compile_circuit(ckt)
    with pytest.raises(ValueError):
        mna_ref.compile_ref(ckt)


def _sent(v):
    return mna.SENTINEL if v == "S" else v


@pytest.mark.parametrize("case", KA.DESCRIPTOR_CASES, ids=lambda c: c["name"])
def test_descriptor_known_answers(case):
    ckt = KA.build_circuit(case["comps"])
    got = mna.compile_circuit(ckt)
    ref = mna_ref.compile_ref(ckt)
    if "diode" in case:
        e = case["diode"]
        d = got.diode_descriptors[0]
        r = ref["diodes"][0]
        assert d["anode"] == _sent(e["anode"]) == r["anode"]
        assert d["cathode"] == _sent(e["cathode"]) == r["cathode"]
        assert [x != mna.SENTINEL for x in d["g_row_col"]] == e["g_valid"]
        assert list(d["g_row_col"]) == r["g_row_col"]
        assert list(d["b_idx"]) == [_sent(v) for v in e["b_idx"]] == r["b_idx"]
        if "is_val" in e:
            assert abs(d["is_val"] - np.float32(e["is_val"])) < 1e-20
            assert abs(d["n_vt"] - np.float32(e["n_vt"])) < 1e-6
        if "g_at_aa" in case:
            assert abs(got.g.val[d["g_row_col"][0]] - case["g_at_aa"]) < 1e-9
    if "bjt" in case:
        e = case["bjt"]
        d = got.bjt_descriptors[0]
        r = ref["bjts"][0]
        for k in ("collector", "base", "emitter"):
            assert d[k] == _sent(e[k]) == r[k]
        assert [x != mna.SENTINEL for x in d["g_row_col"]] == e["g_valid"]
        assert list(d["g_row_col"]) == r["g_row_col"]
        assert list(d["b_idx"]) == [_sent(v) for v in e["b_idx"]] == r["b_idx"]
        assert list(d["node_fixed"]) == r["node_fixed"]
        for k in ("bf", "br", "nf_vt", "nr_vt", "is_val", "polarity"):
            if k in e:
                assert abs(float(d[k]) - e[k]) < 1e-6 * max(1.0, abs(e[k]))
    if "mosfet" in case:
        e = case["mosfet"]
        d = got.mosfet_descriptors[0]
        r = ref["mosfets"][0]
        for k in ("drain", "gate", "source"):
            assert d[k] == _sent(e[k]) == r[k]
        assert [x != mna.SENTINEL for x in d["g_row_col"]] == e["g_valid"]
        assert list(d["g_row_col"]) == r["g_row_col"]
        assert list(d["b_idx"]) == [_sent(v) for v in e["b_idx"]] == r["b_idx"]
        assert d["node_fixed_packed"] == r["node_fixed_packed"]
        for k in ("vto", "kp", "lam", "polarity"):
            if k in e:
                assert abs(float(d[k]) - e[k]) < 1e-6 * max(1.0, abs(e[k]))
    if "counts" in case:
        k = case["counts"]
        assert len(got.diode_descriptors) == k["diodes"]
        assert len(got.bjt_descriptors) == k["bjts"]
        assert len(got.mosfet_descriptors) == k["mosfets"]
        assert got.n_nodes == k["n_nodes"] and got.size == k["size"]


@pytest.mark.parametrize("case", KA.DC_CASES, ids=lambda c: c["name"])
def test_dc_known_answers_oracle(case):
    """integration_test.rs:48-125 through the oracle's compile + dense GE."""
    ckt = KA.build_circuit(case["comps"])
    s = mna.compile_circuit(ckt)
    x = linear_ref.dense_solve_real(s.size, s.size, s.g.row_ptr, s.g.col, s.g.val, s.b_dc)
    for lbl, v in case["v"].items():
        assert abs(x[s.node_index(lbl)] - v) < case["v_tol"]
    for name, i in case.get("i", {}).items():
        k = [ckt.names[c] for c in s.branch_components].index(name)
        assert abs(x[s.n_nodes + k] - i) < case["i_tol"]


def test_mosfet_model_reference_properties():
    """Properties the reference checks on its MOSFET twin formula
    (gpu_shaders.rs:1496-1660): cutoff current ~0, saturation current
    KP/2 * Vov^2 (1 + lambda Vds), continuity across the threshold, and the
    g_m / g_ds partials against central finite differences."""
    md = np.zeros(1, dtype=mna.MOSFET_DTYPE)
    md["drain"], md["gate"], md["source"] = 0, 1, mna.SENTINEL
    md["polarity"], md["vto"], md["kp"], md["lam"] = 1.0, 0.7, 1.1e-4, 0.04
    def ev(vd, vg):
        i, gm, gds = devices_ref.mosfet_eval(md, np.array([vd, vg]))
        return i[0], gm[0], gds[0]
    i, _, _ = ev(1.0, 0.0)
    assert abs(i) < 1e-12                                   # cutoff
    kp = float(np.float32(1.1e-4)); lam = float(np.float32(0.04)); vto = float(np.float32(0.7))
    i, _, _ = ev(3.0, 2.0)
    vov = 2.0 - vto
    assert abs(i - kp / 2 * vov * vov * (1 + lam * 3.0)) < 1e-9 * abs(i)   # saturation
    a, _, _ = ev(1.0, vto - 1e-9); b, _, _ = ev(1.0, vto + 1e-9)
    assert abs(a - b) < 1e-12                               # continuity
    for (vd, vg) in ((0.2, 1.5), (2.0, 1.2), (1.0, 0.75), (0.05, 0.6)):
        h = 1e-6
        _, gm, gds = ev(vd, vg)
        gm_fd = (ev(vd, vg + h)[0] - ev(vd, vg - h)[0]) / (2 * h)
        gds_fd = (ev(vd + h, vg)[0] - ev(vd - h, vg)[0]) / (2 * h)
        assert abs(gm - gm_fd) <= 1e-5 * max(abs(gm), 1e-9)
        assert abs(gds - gds_fd) <= 1e-5 * max(abs(gds), 1e-9)
    md["polarity"] = -1.0                                   # PMOS polarity
    i_p, _, _ = devices_ref.mosfet_eval(md, np.array([-3.0, -2.0]))
    assert i_p[0] < 0


def test_pnjlim_reference_behaviour():
    """Modified pnjlim (ds_nonlinear_shaders.rs:1173-1187)."""
    vt = 0.02585
    vcrit = vt * math.log(vt / (math.sqrt(2) * 1e-14))
    assert devices_ref.pnjlim(0.3, 0.0, vt, vcrit) == 0.3            # below vcrit: unchanged
    v = float(devices_ref.pnjlim(5.0, 0.6, vt, vcrit))
    assert 0.6 < v < 5.0
    assert abs(v - (0.6 + vt * (2 + math.log((1 + 4.4 / vt) - 2)))) < 1e-12
    v2 = float(devices_ref.pnjlim(5.0, -1.0, vt, vcrit))
    assert abs(v2 - vt * math.log(5.0 / vt)) < 1e-12


# ---- ISAI known answers (src/solver/preconditioner.rs:509-820) ----
from oracle import isai_ref  # noqa: E402

_TRI3 = [(0, 0, 4.0), (0, 1, -1.0), (1, 0, -1.0), (1, 1, 4.0), (1, 2, -1.0), (2, 1, -1.0), (2, 2, 4.0)]


def _ref_csr(n, trip):
    a = RefCsr.from_triplets(n, n, trip)
    return a.row_pointers, a.col_indices, a.values


def test_isai_ilu0_reproduces_pa():
    """preconditioner.rs:510-559: L*U == P*A, unit diagonal of L."""
    rp, ci, v = _ref_csr(3, _TRI3)
    L, U, perm = isai_ref.ilu0_ref(3, rp, ci, v)
    A = RefCsr.from_triplets(3, 3, _TRI3).to_dense()
    np.testing.assert_allclose(L @ U, A[perm], atol=1e-10)
    np.testing.assert_allclose(np.diag(L), 1.0, atol=1e-14)


def test_isai0_exact_for_diagonal():
    """preconditioner.rs:561-606."""
    rp, ci, v = _ref_csr(3, [(0, 0, 2.0), (1, 1, 4.0), (2, 2, 5.0)])
    ML, MU, L, U, _ = isai_ref.compute_isai_ref(3, rp, ci, v, level=0)
    np.testing.assert_allclose(ML @ L, np.eye(3), atol=1e-10)
    np.testing.assert_allclose(MU @ U, np.eye(3), atol=1e-10)


def test_isai1_tridiagonal_exact():
    """preconditioner.rs:608-644: M_L * L = I with the L^2 pattern."""
    rp, ci, v = _ref_csr(3, _TRI3)
    ML, _, L, _, _ = isai_ref.compute_isai_ref(3, rp, ci, v, level=1)
    np.testing.assert_allclose(ML @ L, np.eye(3), atol=1e-10)


def test_isai_zero_diagonal_mna_finite():
    """preconditioner.rs:706-736."""
    g1, g2 = 0.001, 0.002
    trip = [(0, 0, g1 + g2), (0, 1, -g2), (0, 2, 1.0), (1, 0, -g2), (1, 1, g2), (2, 0, 1.0)]
    rp, ci, v = _ref_csr(3, trip)
    ML, MU, _, _, _ = isai_ref.compute_isai_ref(3, rp, ci, v, level=0)
    assert np.all(np.isfinite(ML)) and np.all(np.isfinite(MU))


def test_isai_level1_better_than_level0():
    """preconditioner.rs:738-791."""
    trip = [(0, 0, 4.0), (0, 1, -1.0), (1, 0, -1.0), (1, 1, 4.0), (1, 2, -1.0), (2, 1, -1.0), (2, 2, 4.0),
            (2, 3, -1.0), (3, 2, -1.0), (3, 3, 4.0)]
    rp, ci, v = _ref_csr(4, trip)
    ML0, _, L, _, _ = isai_ref.compute_isai_ref(4, rp, ci, v, level=0)
    ML1, _, _, _, _ = isai_ref.compute_isai_ref(4, rp, ci, v, level=1)
    e0 = np.sum((ML0 @ L - np.eye(4)) ** 2)
    e1 = np.sum((ML1 @ L - np.eye(4)) ** 2)
    assert e1 <= e0 + 1e-14


def test_isai1_ill_conditioned_mna():
    """preconditioner.rs:793-819: ISAI(1) closer to A^-1 than ISAI(0)."""
    trip = [(0, 0, 1e-3 + 1e-12), (0, 1, -1e-3), (0, 3, 1.0), (1, 0, -1e-3), (1, 1, 1e-3 + 1e-12),
            (2, 2, 1e-12), (2, 3, -1.0), (3, 0, 1.0), (3, 2, -1.0)]
    rp, ci, v = _ref_csr(4, trip)
    A = RefCsr.from_triplets(4, 4, trip).to_dense()
    ML0, MU0, _, _, _ = isai_ref.compute_isai_ref(4, rp, ci, v, level=0)
    ML1, MU1, _, _, _ = isai_ref.compute_isai_ref(4, rp, ci, v, level=1)
    e0 = np.linalg.norm(MU0 @ ML0 @ A - np.eye(4))
    e1 = np.linalg.norm(MU1 @ ML1 @ A - np.eye(4))
    assert e1 < e0


def test_ilu0_augmented_matches_lu_on_tridiagonal():
    """The device factor (ILU(0) on A + diagonal) equals the exact LU when
    there is no fill (tridiagonal) and gives a nonzero pivot on an MNA branch row."""
    rp, ci, v = _ref_csr(3, _TRI3)
    L, U = isai_ref.ilu0_augmented(3, rp, ci, v)
    A = RefCsr.from_triplets(3, 3, _TRI3).to_dense()
    np.testing.assert_allclose(L @ U, A, atol=1e-12)
    g1, g2 = 0.001, 0.002
    trip = [(0, 0, g1 + g2), (0, 1, -g2), (0, 2, 1.0), (1, 0, -g2), (1, 1, g2), (2, 0, 1.0)]
    rp, ci, v = _ref_csr(3, trip)
    L, U = isai_ref.ilu0_augmented(3, rp, ci, v)
    assert abs(U[2, 2] - (-1.0 / (g1 + g2))) < 1e-9


def test_chow_patel_converges_to_ilu0():
    """Enough Chow-Patel sweeps reach the exact ILU(0) factor of the augmented
    pattern (the fixed point), on a small MNA mesh with a source branch row."""
    s = mna.compile_circuit(ck.diode_mesh(4, 4, seed=2, diode_frac=0.0))
    L, U, _ = isai_ref.chow_patel_ref(s.size, s.g.row_ptr, s.g.col, s.g.val, sweeps=2 * s.size)
    Le, Ue = isai_ref.ilu0_augmented(s.size, s.g.row_ptr, s.g.col, s.g.val)
    np.testing.assert_allclose(L, Le, atol=1e-12 * np.abs(Le).max())
    np.testing.assert_allclose(U, Ue, atol=1e-12 * np.abs(Ue).max())


def test_isai1_device_variant_exact_when_pattern_is_full():
    """With no fill beyond L^2 (a tridiagonal of size 3) and converged sweeps,
    M_L = L^-1 and M_U = U^-1."""
    rp, ci, v = _ref_csr(3, _TRI3)
    ML, MU = isai_ref.isai1_device_ref(3, rp, ci, v, sweeps=8)
    L, U, _ = isai_ref.chow_patel_ref(3, rp, ci, v, sweeps=8)
    np.testing.assert_allclose(ML @ L, np.eye(3), atol=1e-12)
    np.testing.assert_allclose(MU @ U, np.eye(3), atol=1e-12)


# ---- transient source functions: known answers of src/analysis/transient_source.rs tests ----
from oracle import transient_ref as tref  # noqa: E402

_SOURCE_CASES = [
    # (kind, params, t, expected, tol)
    (tref.PULSE, (0.0, 5.0, 1.0, 0.1, 0.1, 1.0, 3.0), 0.5, 0.0, 1e-12),     # before delay
    (tref.PULSE, (0.0, 5.0, 0.0, 1.0, 1.0, 2.0, 6.0), 0.5, 2.5, 1e-12),     # during rise
    (tref.PULSE, (0.0, 5.0, 0.0, 1.0, 1.0, 2.0, 6.0), 2.0, 5.0, 1e-12),     # at peak
    (tref.PULSE, (0.0, 5.0, 0.0, 1.0, 1.0, 2.0, 6.0), 3.5, 2.5, 1e-12),     # during fall
    (tref.PULSE, (0.0, 5.0, 0.0, 1.0, 1.0, 2.0, 6.0), 5.0, 0.0, 1e-12),     # between pulses
    (tref.PULSE, (0.0, 5.0, 0.0, 0.0, 0.0, 1.0, 2.0), 2.5, 5.0, 1e-12),     # period wrap, high
    (tref.PULSE, (0.0, 5.0, 0.0, 0.0, 0.0, 1.0, 2.0), 3.5, 0.0, 1e-12),     # period wrap, low
    (tref.SIN, (1.0, 2.0, 1.0, 1.0, 0.0), 0.5, 1.0, 1e-12),                 # before delay
    (tref.SIN, (0.0, 1.0, 1.0, 0.0, 0.0), 0.25, 1.0, 1e-12),                # quarter period
    (tref.SIN, (0.0, 1.0, 1.0, 0.0, 0.0), 0.5, 0.0, 1e-12),                 # half period
    (tref.SIN, (0.0, 1.0, 1.0, 0.0, 1.0), 0.25, math.exp(-0.25), 1e-12),    # damping
    (tref.SIN, (2.5, 1.0, 1.0, 0.0, 0.0), 0.25, 3.5, 1e-12),                # offset
    (tref.PWL, ((1.0, 0.0), (2.0, 5.0)), 0.0, 0.0, 1e-12),                  # before first
    (tref.PWL, ((1.0, 0.0), (2.0, 5.0)), 3.0, 5.0, 1e-12),                  # after last
    (tref.PWL, ((0.0, 0.0), (1.0, 10.0), (2.0, 10.0), (3.0, 0.0)), 0.5, 5.0, 1e-12),
    (tref.PWL, ((0.0, 0.0), (1.0, 10.0), (2.0, 10.0), (3.0, 0.0)), 1.5, 10.0, 1e-12),
    (tref.PWL, ((0.0, 0.0), (1.0, 10.0), (2.0, 10.0), (3.0, 0.0)), 2.5, 5.0, 1e-12),
    (tref.PWL, ((0.0, 0.0), (1.0, 5.0), (2.0, 3.0)), 1.0, 5.0, 1e-12),      # at breakpoint
    (tref.EXP, (0.0, 5.0, 1.0, 1.0, 3.0, 1.0), 0.5, 0.0, 1e-12),            # before td1
    (tref.EXP, (0.0, 5.0, 0.0, 1.0, 10.0, 1.0), 1.0, 5.0 * (1.0 - math.exp(-1.0)), 1e-10),
    (tref.EXP, (0.0, 5.0, 0.0, 1.0, 5.0, 1.0), 6.0,
     5.0 * (1.0 - math.exp(-6.0)) - 5.0 * (1.0 - math.exp(-1.0)), 1e-10),
]


@pytest.mark.parametrize("case", _SOURCE_CASES, ids=lambda c: f"{c[0]}-{c[2]}")
def test_source_functions_known_answers(case):
    kind, params, t, expected, tol = case
    assert abs(tref.eval_source(kind, params, t) - expected) < tol


def test_be_companion_of_rc_step():
    """One BE step of an RC charged through R from a 1 V step: the oracle's
    companion system gives v = (v0 + h/(RC) * 1) / (1 + h/(RC)) (exact BE)."""
    b = ck.CircuitBuilder()
    b.vsource(1, 0, dc=0.0, name="V1", tran=(ck.TRAN_PULSE, (0.0, 1.0, 0.0, 0.0, 0.0, 1.0, 2.0)))
    b.resistors([1], [2], [1000.0])
    b.capacitors([2], [0], [1e-9])
    s = mna.compile_circuit(b.build())
    x0 = np.zeros(s.size)
    h = 1e-7
    x, wave, _ = tref.be_transient(s, x0, 0.0, h, 3, [s.node_index(2)])
    r = h / (1000.0 * 1e-9)
    v = 0.0
    for k in range(3):
        v = (v + r * 1.0) / (1.0 + r)
        assert abs(wave[k, 0] - v) < 1e-9 * max(1.0, abs(v))


@pytest.mark.parametrize("grid", [("dec", 10, 1e3, 1e9), ("oct", 4, 1e6, 1e10), ("lin", 25, 1e3, 1e8),
                                  ("lin", 1, 5.0, 9.0)])
def test_ac_frequency_grid(grid):
    """Host-side frequency generation equals the restatement of
    generate_frequencies (src/analysis/ac.rs:80-109)."""
    from oracle import ac_ref
    from ohmnivore_b200 import solver as S
    np.testing.assert_array_equal(S.ac_frequencies(*grid), np.array(ac_ref.generate_frequencies(*grid)))


# ---- adjoint oracle: LU adjoint = forward sensitivity = central finite differences ----
def _fd_output(ckt, mutate, h, n_steps, probe_label):
    """o = V(probe) after n_steps BE steps from the DC point, for a circuit
    changed by `mutate(ckt_copy, sysm)` (returns the new system)."""
    from oracle import newton_ref
    s = mutate()
    x0, _ = newton_ref.newton(s)
    states = __import__("oracle.adjoint_ref", fromlist=["x"]).transient_states(s, x0, 0.0, h, n_steps)
    return states[-1][s.node_index(probe_label)]


def test_adjoint_oracle_agrees_with_forward_sensitivity_and_fd():
    import copy
    from oracle import adjoint_ref, newton_ref
    from ohmnivore_b200 import solver as S
    ckt = ck.rc_diode_mesh(4, 4, seed=4, diode_frac=0.25)
    s = mna.compile_circuit(ckt)
    comps = S.ComponentTable(ckt, s)
    h, n_steps = 2e-12, 12
    probe = 2 + 15                                  # opposite corner of the 4x4 mesh
    x0, _ = newton_ref.newton(s)
    states = adjoint_ref.transient_states(s, x0, 0.0, h, n_steps)
    w = np.zeros(s.size)
    w[s.node_index(probe)] = 1.0
    g = adjoint_ref.transient_adjoint(s, comps, states, h, w)
    rel = lambda a, b: abs(a - b) / max(abs(b), 1e-300)  # noqa: E731
    for kind, j in (("R", 3), ("R", 11), ("C", 5), ("C", 15), ("Is", 0)):
        fs = adjoint_ref.forward_sensitivity(s, comps, states, h, w, kind, j)
        assert rel(g[kind][j], fs) < 1e-8, (kind, j)
    # central differences, relative step 1e-6, on R and C
    for kind, idx in (("R", comps.r_index[3]), ("C", comps.c_index[5])):
        v = ckt.value[idx]
        outs = []
        for sign in (1, -1):
            c2 = copy.deepcopy(ckt)
            c2.value[idx] = v * (1 + sign * 1e-6)
            outs.append(_fd_output(c2, lambda c2=c2: mna.compile_circuit(c2), h, n_steps, probe))
        fd = (outs[0] - outs[1]) / (2e-6 * v)
        j = 3 if kind == "R" else 5
        assert rel(g[kind][j], fd) < 1e-6, (kind, g[kind][j], fd)
