"""Skewed and large LPs (power-law column counts).

Columns far longer than the rest are moved to the front of the device
numbering and stepped with wide lane groups; the renumbering must be invisible
to the caller.  Checked on a 20,000 x 80,000 power-law LP (column counts 2 to
2,000, mean 10, 1% of rows scaled by 1e3): the single-LP engine and the packed
engine agree on the optimum to 1e-6 relative, and the returned x is
feasible for the original rows and bounds (independent numpy check).
"""
import numpy as np
import pytest

import golden_cases as GC
from mipx_b200 import generators as G
from mipx_b200.pdlp import PdlpOptions, PdlpSolver, Status, batch_solve

pytestmark = pytest.mark.gpu

TOL = 1e-6


def _feasibility(lp, x):
    a = lp.matrix
    rows = np.repeat(np.arange(lp.num_rows), np.diff(a.row_starts))
    ax = np.bincount(rows, weights=a.values * x[a.col_indices], minlength=lp.num_rows)
    viol = np.maximum(lp.row_lower - ax, 0) + np.maximum(ax - lp.row_upper, 0)
    b = np.r_[lp.row_lower[np.isfinite(lp.row_lower)], lp.row_upper[np.isfinite(lp.row_upper)]]
    return np.linalg.norm(viol) / (1 + np.linalg.norm(b))


def test_powerlaw_lp_single_and_batch_agree():
    lp, _ = G.powerlaw_lp(20000, 80000, 2, 2000, 10.0, 0.01, 1e3, 5)
    counts = np.bincount(lp.matrix.col_indices, minlength=lp.num_cols)
    assert counts.max() > 8 * counts.mean()  # the case has long columns
    o = PdlpOptions(verbose=False, primal_tol=TOL, dual_tol=TOL, optimality_tol=TOL, max_solve_seconds=240)
    s = PdlpSolver()
    s.setOptions(o)
    s.load(lp)
    r = s.solve()
    assert r.status == Status.Optimal, r
    x = s.getPrimalValues()
    assert np.all(x >= lp.col_lower - 1e-9) and np.all(x <= lp.col_upper + 1e-9)
    assert _feasibility(lp, x) <= 2 * TOL
    (q, u, _), = batch_solve([lp], o)
    assert q.status == Status.Optimal
    assert GC.rel_err(r.objective, q.objective) <= GC.OBJ_TOL, (r.objective, q.objective)


def _transposed(lp, seed):
    """An LP over A^T of `lp` (its long columns become long rows): columns in
    [0, 10], rows within 1 of A^T x0 for a random x0 in the box, so it has an
    optimum."""
    from scipy.sparse import csr_matrix
    from mipx_b200.pdlp import LpProblem, SparseMatrix
    a = csr_matrix((lp.matrix.values, lp.matrix.col_indices, lp.matrix.row_starts), shape=(lp.num_rows, lp.num_cols))
    t = a.T.tocsr()
    t.sort_indices()
    rng = np.random.default_rng(seed)
    x0 = rng.uniform(0, 10, lp.num_rows)
    ax = t @ x0
    return LpProblem(num_cols=lp.num_rows, obj=rng.normal(size=lp.num_rows), col_lower=np.zeros(lp.num_rows),
                     col_upper=np.full(lp.num_rows, 10.0), num_rows=lp.num_cols, row_lower=ax - 1.0,
                     row_upper=ax + 1.0,
                     matrix=SparseMatrix(lp.num_cols, lp.num_rows, values=t.data.astype(np.float64),
                                         col_indices=t.indices.astype(np.int32),
                                         row_starts=t.indptr.astype(np.int32)))


@pytest.mark.parametrize("side", ["dual", "primal"])
@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_hot_prefix_in_shared_memory_gives_same_bits(side, precision):
    """The hot-prefix kernels (gathers of the other side's longest rows served
    from a shared-memory copy) compute what the plain sliced-ELL kernels
    compute, bit for bit: same iterations, objective, x and y.  'dual':
    power-law columns (the dual step's x gathers); 'primal': the transposed LP,
    whose long rows are the primal step's y gathers."""
    from mipx_b200.pdlp import Precision
    lp, _ = G.powerlaw_lp(20000, 80000, 2, 2000, 10.0, 0.01, 1e3, 5)
    if side == "primal":
        lp = _transposed(lp, 9)
    prec = Precision.Mixed if precision == "mixed" else Precision.FP64
    out = []
    for hot in (0, 64):
        s = PdlpSolver()
        s.setOptions(PdlpOptions(verbose=False, precision=prec, primal_tol=TOL, dual_tol=TOL, optimality_tol=TOL,
                                 max_iter=4000, hot_cache=hot))
        s.load(lp)
        r = s.solve()
        out.append((r, s.getPrimalValues(), s.getDualValues(), s.hotPrefix(prec)))
    (r0, x0, y0, h0), (r1, x1, y1, h1) = out
    assert h0 == {"primal": 0, "dual": 0}
    assert h1[side] > 0 and h1["primal" if side == "dual" else "dual"] == 0, h1  # the hot kernel ran
    assert r0.iterations == r1.iterations and r0.objective == r1.objective
    np.testing.assert_array_equal(x0, x1)
    np.testing.assert_array_equal(y0, y1)


def test_long_column_tiles_match_csr_launch():
    """The mixed-mode primal step of the long columns in row chunks (FP32 y in
    shared memory, per-chunk partial sums added in chunk order) against the
    CSR launch of the same columns: the sums differ only in FP64 association,
    so after 400 iterations (two restart cycles) the iterates agree to 1e-9
    relative, and full solves reach the same optimum to 1e-6."""
    lp, _ = G.powerlaw_lp(100000, 400000, 2, 2000, 10.0, 0.01, 1e3, 11)
    out = []
    for tiles in (0, 1):
        s = PdlpSolver()
        s.setOptions(PdlpOptions(verbose=False, primal_tol=TOL, dual_tol=TOL, optimality_tol=TOL, max_iter=400,
                                 long_tiles=tiles))
        s.load(lp)
        r = s.solve()
        out.append((r, s.getPrimalValues(), s.getDualValues()))
    (r0, x0, y0), (r1, x1, y1) = out
    assert r0.iterations == r1.iterations == 400
    np.testing.assert_allclose(x1, x0, rtol=1e-9, atol=1e-9 * max(1.0, np.abs(x0).max()))
    np.testing.assert_allclose(y1, y0, rtol=1e-9, atol=1e-9 * max(1.0, np.abs(y0).max()))
    full = []
    for tiles in (0, 1):
        s = PdlpSolver()
        s.setOptions(PdlpOptions(verbose=False, primal_tol=TOL, dual_tol=TOL, optimality_tol=TOL,
                                 max_solve_seconds=120, long_tiles=tiles))
        s.load(lp)
        full.append(s.solve())
    assert full[0].status == full[1].status == Status.Optimal
    assert GC.rel_err(full[1].objective, full[0].objective) <= GC.OBJ_TOL


def _duality_certificate(lp, x, y):
    """Independent FP64 optimality certificate of (x, y) for a minimisation LP
    with boxed columns.  The returned duals price A x the other way round (a
    '<=' row's dual is >= 0), so u = -y; u projected onto the sign its rows
    allow is dual feasible, and b-support(u) + bound-support(c - A^T u) is a
    lower bound on the optimum (weak duality).  Returns (relative primal
    residual, |c x - that bound| / max(1, |c x|))."""
    a = lp.matrix
    rows = np.repeat(np.arange(lp.num_rows), np.diff(a.row_starts))
    u = -np.asarray(y, dtype=np.float64)
    yp = np.where(np.isfinite(lp.row_lower), u, np.minimum(u, 0.0))
    yp = np.where(np.isfinite(lp.row_upper), yp, np.maximum(yp, 0.0))
    aty = np.bincount(a.col_indices, weights=a.values * yp[rows], minlength=lp.num_cols)
    rc = lp.obj - aty
    assert np.all(np.isfinite(lp.col_lower)) and np.all(np.isfinite(lp.col_upper))
    row_part = np.where(yp > 0, lp.row_lower, lp.row_upper) * yp
    row_part = np.where(yp == 0, 0.0, row_part)
    dual_bound = row_part.sum() + np.where(rc > 0, lp.col_lower, lp.col_upper) @ rc + lp.obj_offset
    primal = lp.obj @ x + lp.obj_offset
    return _feasibility(lp, x), abs(primal - dual_bound) / max(1.0, abs(primal))


def test_powerlaw_full_size_certificate():
    """The 500,000 x 2,000,000 power-law LP (20.1M nonzeros), mixed precision,
    to 1e-6 relative KKT: no FP64 oracle finishes it here, so the returned
    (x, y) is checked by an independent numpy certificate -- primal residual
    <= 1e-6 and the objective within 2e-6 relative of a weak-duality lower
    bound, hence of the optimum."""
    lp, _ = G.powerlaw_lp(500000, 2000000, 2, 2000, 10.0, 0.01, 1e3, 11)
    s = PdlpSolver()
    s.setOptions(PdlpOptions(verbose=False, primal_tol=TOL, dual_tol=TOL, optimality_tol=TOL,
                             max_solve_seconds=120))
    s.load(lp)
    r = s.solve()
    assert r.status == Status.Optimal, r
    x, y = s.getPrimalValues(), s.getDualValues()
    assert np.all(x >= lp.col_lower - 1e-9) and np.all(x <= lp.col_upper + 1e-9)
    rp, gap = _duality_certificate(lp, x, y)
    assert rp <= 1e-6 and gap <= 2e-6, (rp, gap, r.objective)


def test_sell_window_changes_only_the_numbering():
    """sell_window limits the length sort of the sliced-ELL rows to windows;
    the numbering is undone on read back, so both orders reach the same optimum
    (to 1e-6 relative) with x and y in the caller's numbering."""
    lp, _ = G.powerlaw_lp(20000, 80000, 2, 2000, 10.0, 0.01, 1e3, 5)
    out = []
    for w in (0, 4096):
        s = PdlpSolver()
        s.setOptions(PdlpOptions(verbose=False, primal_tol=TOL, dual_tol=TOL, optimality_tol=TOL,
                                 max_solve_seconds=120, sell_window=w))
        s.load(lp)
        r = s.solve()
        assert r.status == Status.Optimal, (w, r)
        x = s.getPrimalValues()
        assert _feasibility(lp, x) <= 2 * TOL
        out.append(r.objective)
    assert GC.rel_err(out[0], out[1]) <= GC.OBJ_TOL, out
