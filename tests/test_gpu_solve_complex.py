"""GPU: LinearSolver::solve_complex through ohm_solve_complex (the AC path's
complex BiCGSTAB on one point with w = 1) against the reference's complex
known answers (src/solver/cpu.rs:281-366) and the oracle's complex LU."""
import numpy as np
import pytest

from oracle import linear_ref
from oracle.mna_ref import RefCsr
from ohmnivore_b200 import mna
from ohmnivore_b200 import solver as S
from tests.golden import known_answers as KA

pytestmark = pytest.mark.gpu


def _ccsr(case):
    a = RefCsr.from_triplets(case["n"], case["n"], case["trip"])
    return mna.Csr(a.nrows, a.ncols, np.array(a.row_pointers, np.int64), np.array(a.col_indices, np.int64),
                   np.array(a.values, np.complex128))


def _params(**kw):
    p = S.BiCgStabParams(max_iterations=2000, tolerance=1e-15)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


@pytest.mark.parametrize("case", KA.COMPLEX_SOLVES, ids=lambda c: c["name"])
def test_complex_known_answers(ctx, case):
    x = S.GpuSolver(ctx, _params()).solve_complex(_ccsr(case), case["b"])
    np.testing.assert_allclose(x, case["x"], atol=1e-10, rtol=0)


def test_complex_singular_is_an_error(ctx):
    case = KA.COMPLEX_ERRORS[0]
    with pytest.raises(S.SolveError):
        S.GpuSolver(ctx, _params(max_iterations=200)).solve_complex(_ccsr(case), case["b"])


def test_complex_ladder_matches_lu(ctx):
    """A 300-node RC ladder's admittance matrix at 10 MHz as one complex
    system, against the oracle's dense complex solve."""
    rng = np.random.default_rng(5)
    n = 300
    g = rng.uniform(1e-4, 1e-2, n - 1)
    c = rng.uniform(1e-12, 1e-10, n)
    w = 2 * np.pi * 1e7
    trip = []
    for i in range(n - 1):
        trip += [(i, i, g[i]), (i + 1, i + 1, g[i]), (i, i + 1, -g[i]), (i + 1, i, -g[i])]
    trip += [(i, i, 1j * w * c[i] + 1e-3 * (i == 0)) for i in range(n)]
    a = RefCsr.from_triplets(n, n, trip)
    b = np.zeros(n, dtype=np.complex128)
    b[0] = 1e-3
    ref = linear_ref.dense_solve_complex(n, n, a.row_pointers, a.col_indices, a.values, b)
    m = mna.Csr(n, n, np.array(a.row_pointers, np.int64), np.array(a.col_indices, np.int64),
                np.array(a.values, np.complex128))
    x = S.GpuSolver(ctx, _params(max_iterations=20000, tolerance=1e-16)).solve_complex(m, b)
    assert float(np.max(np.abs(x - ref)) / np.max(np.abs(ref))) < 1e-9
