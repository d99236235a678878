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
