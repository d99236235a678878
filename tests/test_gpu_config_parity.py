"""Parity of the engine on the benchmark configurations against FP64 oracles,
at the north-star bound: objective within 1e-6 relative (to max(1, |oracle|))
and every relative KKT term <= 1e-6.

* transportation LP 1,000 x 1,000: the HiGHS optimum stored by
  tests/golden/make_golden.py;
* 16 LPs of the batched workload (one pdlpx_batch_solve call): the reference's
  own CPU PdlpSolver at 1e-6 relative KKT and the HiGHS optimum;
* 8 node LPs of the serving workload (1-5% of the integer columns fixed, 0-50
  cuts), warm-started through the request server: the reference's CPU
  PdlpSolver at 1e-8 relative KKT on the node LP with its fixed columns
  substituted out;
* the power-law LP at a fifth of the headline size (100,000 x 400,000, 4M
  nonzeros): the reference's CPU PdlpSolver at 1e-7 relative KKT;
the latter three from tests/golden/config_pins.json
(tests/golden/make_config_pins.py).

Also here: the device power iteration against the oracle's spectral norm
(pdlp.cpp:748-795), the removeRows / setObjective edits against fresh oracle
solves (pdlp.cpp:2855-2907), and the reference-compatible fixed-column switch.
"""
import numpy as np
import pytest

import golden_cases as GC
import lp_fixtures as F
from mipx_b200 import generators as G
from mipx_b200.pdlp import LpProblem, PdlpOptions, PdlpSolver, Precision, Server, SparseMatrix, Status, batch_solve
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TIGHT = dict(primal_tol=1e-6, dual_tol=1e-6, optimality_tol=1e-6)


def _kkt_ok(r):
    return r.rel_primal_resid <= 1e-6 and r.rel_dual_resid <= 1e-6 and r.rel_gap <= 1e-6


def test_transport_against_highs():
    """1M-variable transportation LP: 1e-6 relative KKT and the HiGHS optimum to 1e-6."""
    lp, _ = G.transport_lp(1000, 1000, 7)
    s = PdlpSolver()
    s.setOptions(PdlpOptions(verbose=False, **TIGHT))
    s.load(lp)
    r = s.solve()
    assert r.status == Status.Optimal and _kkt_ok(r), r
    hi = GC.INDEX["transport_1000x1000"]["highs_objective"]
    assert GC.rel_err(r.objective, hi) <= GC.OBJ_TOL, (r.objective, hi)


def test_batch_sample_against_reference_and_highs():
    pins = GC.config_pins()["batch_sample"]
    sizes = G.batch_sizes(512, seed=5)
    lps = [G.random_lp(sizes[p["k"]][0], sizes[p["k"]][1], 4, 12, p["seed"])[0] for p in pins]
    out = batch_solve(lps, PdlpOptions(verbose=False, **TIGHT))
    for p, (r, _, _) in zip(pins, out):
        assert p["reference_status"] == 0 and r.status == Status.Optimal and _kkt_ok(r), (p["k"], r)
        assert GC.rel_err(r.objective, p["reference_objective"]) <= GC.OBJ_TOL, (p, r.objective)
        if p["highs_objective"] is not None:
            assert GC.rel_err(r.objective, p["highs_objective"]) <= GC.OBJ_TOL, (p, r.objective)


def test_serving_nodes_against_reference():
    """Node LPs carry fixed columns (lb == ub), which the engine's check treats as
    free of dual residual; the reference's check cannot converge on them, so its
    pin solves the same LP with the fixed columns substituted out."""
    pins = GC.config_pins()["nodes"]
    base, x0 = G.random_lp(20000, 50000, 4, 12, 101)
    ints = G.integer_marks(base.num_cols)
    with Server(PdlpOptions(verbose=False, **TIGHT), max_packs=2, max_pack_lps=32, batch_window_ms=200) as srv:
        tb = srv.submit(base)
        srv.wait(tb)
        tickets = [srv.submit(G.node_lp(base, x0, ints, p["seed"]), warm=tb) for p in pins]
        res = [srv.wait(t)[0] for t in tickets]
    for p, r in zip(pins, res):
        assert p["fixed_columns"] > 0 and p["reference_status"] == 0
        assert r.status == Status.Optimal and _kkt_ok(r), (p["k"], r)
        assert GC.rel_err(r.objective, p["reference_objective"]) <= GC.OBJ_TOL, (p, r.objective)


@pytest.mark.parametrize("precision", [Precision.Mixed, Precision.FP64])
def test_powerlaw_fifth_scale_against_reference(precision):
    pins = GC.config_pins()
    if "powerlaw_100000x400000" not in pins:
        pytest.skip("the reference pin of the 100k x 400k LP is not in tests/golden/config_pins.json")
    p = pins["powerlaw_100000x400000"]
    lp, _ = G.powerlaw_lp(p["m"], p["n"], 2, 2000, 10.0, 0.01, 1e3, p["seed"])
    assert lp.matrix.numNonzeros() == p["nnz"]
    s = PdlpSolver()
    s.setOptions(PdlpOptions(verbose=False, precision=precision, max_solve_seconds=300, **TIGHT))
    s.load(lp)
    r = s.solve()
    assert p["reference_status"] == 0
    assert r.status == Status.Optimal and _kkt_ok(r), r
    assert GC.rel_err(r.objective, p["reference_objective"]) <= GC.OBJ_TOL, (r.objective, p["reference_objective"])


@pytest.mark.parametrize("name", ["medium", "rand_500x1250", "rand_2000x5000"])
@pytest.mark.parametrize("precision", [Precision.FP64, Precision.Mixed])
def test_device_spectral_norm_matches_oracle(name, precision):
    """The step size 0.998 / ||A||_2 from the device power iteration (mt19937(42)
    normal start, pdlp.cpp:748-795) against the oracle's power iteration on the
    same scaled matrix: 1e-9 relative in FP64 mode; 1e-5 with the FP32 matrix
    values the mixed mode iterates with."""
    lp = GC.problem(name)
    s = PdlpSolver()
    s.setOptions(GC.options(name, precision=precision, max_iter=200))
    s.load(lp)
    r = s.solve()
    sigma = O.oracle_spectral_norm(lp, GC.options(name, use_gpu=False))
    step_ref = 0.998 / sigma
    tol = 1e-9 if precision == Precision.FP64 else 1e-5
    assert abs(r.step_size - step_ref) <= tol * step_ref, (r.step_size, step_ref)


def _rebuild(lp, keep_rows, obj=None):
    a = lp.matrix
    trips = []
    for new, i in enumerate(keep_rows):
        for k in range(a.row_starts[i], a.row_starts[i + 1]):
            trips.append((new, int(a.col_indices[k]), float(a.values[k])))
    return LpProblem(num_cols=lp.num_cols, num_rows=len(keep_rows),
                     obj=np.array(obj if obj is not None else lp.obj, dtype=np.float64),
                     col_lower=lp.col_lower.copy(), col_upper=lp.col_upper.copy(),
                     row_lower=lp.row_lower[keep_rows].copy(), row_upper=lp.row_upper[keep_rows].copy(),
                     matrix=SparseMatrix(len(keep_rows), lp.num_cols, trips), sense=lp.sense,
                     obj_offset=lp.obj_offset)


@pytest.mark.parametrize("precision", [Precision.FP64, Precision.Mixed])
def test_remove_rows_and_set_objective_match_fresh_oracle_solves(precision):
    """removeRows then setObjective on a loaded solver (pdlp.cpp:2855-2907: each edit
    changes the original problem and rebuilds the scaled one) give the solution of
    a fresh load of the edited LP (oracle restatement of the reference)."""
    lp = F.medium_lp()
    s = PdlpSolver()
    s.setOptions(PdlpOptions(verbose=False, precision=precision, max_iter=500000, **TIGHT))
    s.load(lp)
    s.solve()
    drop = [1, 4, 7]
    s.removeRows(drop)
    r1 = s.solve()
    keep = [i for i in range(lp.num_rows) if i not in drop]
    ref1, _, _ = O.oracle_solve(_rebuild(lp, keep), PdlpOptions(verbose=False, use_gpu=False, max_iter=500000, **TIGHT))
    assert r1.status == ref1.status == Status.Optimal
    assert GC.rel_err(r1.objective, ref1.objective) <= GC.OBJ_TOL, (r1.objective, ref1.objective)
    c2 = lp.obj * 0.5 + np.linspace(-0.2, 0.2, lp.num_cols)
    s.setObjective(c2)
    r2 = s.solve()
    ref2, _, _ = O.oracle_solve(_rebuild(lp, keep, obj=c2),
                                PdlpOptions(verbose=False, use_gpu=False, max_iter=500000, **TIGHT))
    assert r2.status == ref2.status
    if ref2.status == Status.Optimal:
        assert GC.rel_err(r2.objective, ref2.objective) <= GC.OBJ_TOL, (r2.objective, ref2.objective)


def _fixed_column_lp():
    """min -2 x1 - x2  s.t.  x1 + x2 <= 1.5,  x1 fixed at 1,  0 <= x2 <= 10: optimum
    (1, 0.5), objective -2.5, and the fixed column's reduced cost is negative."""
    return LpProblem(num_cols=2, obj=np.array([-2.0, -1.0]), col_lower=np.array([1.0, 0.0]),
                     col_upper=np.array([1.0, 10.0]), num_rows=1, row_lower=np.array([-np.inf]),
                     row_upper=np.array([1.5]),
                     matrix=SparseMatrix(1, 2, values=np.array([1.0, 1.0]), col_indices=np.array([0, 1], np.int32),
                                         row_starts=np.array([0, 2], np.int32)))


def test_reference_fixed_column_switch():
    """reference_fixed_columns = 1 counts a fixed column's negative reduced cost as
    dual residual, exactly as the reference's check does: on this LP the reference
    (compiled from its sources) and the engine with the switch both end at the
    iteration cap; without the switch the engine converges to the optimum."""
    lp = _fixed_column_lp()
    cap = dict(max_iter=20000, **TIGHT)
    ref, _, _ = O.ref_solve(lp, PdlpOptions(verbose=False, use_gpu=False, **cap))
    assert ref.status == Status.IterLimit
    for prec in (Precision.FP64, Precision.Mixed):
        s = PdlpSolver()
        s.setOptions(PdlpOptions(verbose=False, precision=prec, reference_fixed_columns=True, **cap))
        s.load(lp)
        assert s.solve().status == Status.IterLimit
        s.setOptions(PdlpOptions(verbose=False, precision=prec, **cap))
        r = s.solve()
        assert r.status == Status.Optimal and abs(r.objective + 2.5) <= 1e-5
    (q, _, _), = batch_solve([lp], PdlpOptions(verbose=False, reference_fixed_columns=True, **cap))
    assert q.status == Status.IterLimit


@pytest.mark.parametrize("name", [k for k in GC.NAMES if GC.INDEX[k]["options"]["primal_tol"] <= 1e-6])
def test_reference_fixed_column_switch_keeps_golden_results(name):
    """No golden LP has a fixed column, so the switch changes nothing on them:
    same status and objective within 1e-6 relative of the reference."""
    e = GC.INDEX[name]
    s = PdlpSolver()
    s.setOptions(GC.options(name, precision=Precision.FP64, reference_fixed_columns=True))
    s.load(GC.problem(name))
    r = s.solve()
    assert int(r.status) == e["status"]
    if e["status"] == Status.Optimal:
        assert GC.rel_err(r.objective, e["objective"]) <= GC.OBJ_TOL, (r.objective, e["objective"])
