"""The oracle restatement is pinned to the reference: on every golden case it
must reproduce the compiled reference's status, iteration count, objective and
solution vectors exactly (same FP64 operation order, same compiler flags)."""
import numpy as np
import pytest

import golden_cases as GC
import lp_fixtures as F
from mipx_b200.pdlp import PdlpOptions, Status
from oracle import oracle as O


@pytest.mark.parametrize("name", GC.NAMES)
def test_oracle_matches_reference_golden(name):
    e = GC.INDEX[name]
    res, x, y = O.oracle_solve(GC.problem(name), GC.options(name))
    assert int(res.status) == e["status"]
    assert res.iterations == e["iterations"]
    assert res.objective == e["objective"]
    xr, yr = GC.vectors(name)
    if e["status"] == Status.Optimal:
        np.testing.assert_array_equal(x, xr)
        np.testing.assert_array_equal(y, yr)
    if e["status"] == Status.Optimal and name not in ("infeasible", "infeasible_eq", "unbounded_constrained"):
        assert res.work_units == e["work_units"]


@pytest.mark.parametrize("name", [k for k in GC.NAMES if "highs_objective" in GC.INDEX[k]])
def test_reference_objective_matches_highs(name):
    e = GC.INDEX[name]
    ref, hi = e["objective"], e["highs_objective"]
    assert abs(ref - hi) <= 1e-5 * (1.0 + abs(hi))


@pytest.mark.parametrize("name,lp_builder,expected,tol,where", [
    (k, b, v, t, w) for k, (b, v, t, w) in F.KNOWN_ANSWERS.items()])
def test_oracle_known_answers(name, lp_builder, expected, tol, where):
    res, _, _ = O.oracle_solve(lp_builder(), PdlpOptions(verbose=False, use_gpu=False, max_iter=100000))
    assert res.status == Status.Optimal
    assert abs(res.objective - expected) <= tol, where


def test_oracle_statuses():
    o = PdlpOptions(verbose=False, use_gpu=False, max_iter=100000)
    assert O.oracle_solve(F.infeasible_lp(), o)[0].status == Status.Infeasible
    assert O.oracle_solve(F.infeasible_eq_lp(), o)[0].status == Status.Infeasible
    assert O.oracle_solve(F.unbounded_constrained_lp(), o)[0].status == Status.Unbounded
    assert O.oracle_solve(F.unbounded_bounds_only_lp(), o)[0].status == Status.Unbounded
    tl = PdlpOptions(verbose=False, use_gpu=False, max_solve_seconds=0.0)
    assert O.oracle_solve(F.simple_lp(), tl)[0].status == Status.TimeLimit


def test_oracle_farkas_sign():
    """Farkas certificate sign check of test_pdlp.cpp:445-496 on the oracle's dual ray."""
    res, _, y = O.oracle_solve(F.infeasible_lp(), PdlpOptions(verbose=False, use_gpu=False, max_iter=100000))
    assert res.status == Status.Infeasible
    ray = y[0] / abs(y[0])
    assert ray >= -1e-6
    assert ray * (-1.0) - ray * 1.0 < -1e-6


@pytest.mark.skipif(not O.ref_available(), reason="reference build not present (only where its sources exist)")
@pytest.mark.parametrize("seed", [21, 22])
def test_oracle_matches_live_reference(seed):
    from mipx_b200 import generators as G
    lp, _ = G.random_lp(150, 380, 3, 9, seed)
    o = PdlpOptions(verbose=False, use_gpu=False, max_iter=200000, primal_tol=1e-6, dual_tol=1e-6,
                    optimality_tol=1e-6)
    a, xa, ya = O.oracle_solve(lp, o)
    b, xb, yb = O.ref_solve(lp, o)
    assert (a.status, a.iterations, a.objective) == (b.status, b.iterations, b.objective)
    np.testing.assert_array_equal(xa, xb)
    np.testing.assert_array_equal(ya, yb)
