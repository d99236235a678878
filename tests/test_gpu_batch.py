"""Batched solve (pdlpx_batch_solve: many LPs packed into one device image,
one graph launch per restart cycle for the whole pack).

* parity: a mixed batch of the reference's golden cases (optimal, infeasible,
  unbounded, trivial) reproduces the reference's statuses, and objectives within
  1e-6 relative (to max(1, |obj|)) for LPs solved to 1e-6 relative KKT, within
  the mipx GPU-vs-CPU bounds otherwise;
* batch invariance: an LP's result is bit-identical when solved alone, inside a
  batch of other LPs, split across several packs, and with or without the
  compaction of finished LPs (tiles, launch shape and reduction order depend on
  the LP alone);
* the FP64 mode solves the same LPs.
"""
import numpy as np
import pytest

import golden_cases as GC
from mipx_b200 import generators as G
from mipx_b200.pdlp import PdlpOptions, Precision, Status, batch_solve

pytestmark = pytest.mark.gpu

TIGHT = dict(primal_tol=1e-6, dual_tol=1e-6, optimality_tol=1e-6)


def _check_against_golden(name, r):
    e = GC.INDEX[name]
    assert int(r.status) == e["status"], (name, r.status)
    if e["status"] != Status.Optimal:
        return
    ref = e["objective"]
    tol = e["options"]["optimality_tol"]
    if e["options"]["primal_tol"] <= 1e-6:
        assert GC.rel_err(r.objective, ref) <= GC.OBJ_TOL, (name, r.objective, ref)
    else:
        bound = 1e-4 if name in ("medium", "simple") else 1e-3 * max(1.0, abs(ref))
        assert abs(r.objective - ref) <= max(bound, 2e-4 * abs(ref)), (name, r.objective, ref)


# golden cases that share one option set can go into one batch
DEFAULT_CASES = ["simple", "col_bound_binding", "maximize", "medium", "bounds_only", "empty",
                 "unbounded_bounds_only"]
TIGHT_CASES = ["medium_tight", "ranged", "rand_60x150", "rand_200x500", "rand_500x1250", "rand_2000x5000"]


@pytest.mark.parametrize("precision", [Precision.Mixed, Precision.FP64])
def test_batch_golden_tight(precision):
    probs = [GC.problem(k) for k in TIGHT_CASES]
    o = PdlpOptions(verbose=False, max_iter=500000, precision=precision, **TIGHT)
    out = batch_solve(probs, o)
    for name, (r, x, y) in zip(TIGHT_CASES, out):
        _check_against_golden(name, r)
        assert r.used_gpu and r.kernel_launches > 0


def test_batch_golden_default_options_with_trivial_lps():
    probs = [GC.problem(k) for k in DEFAULT_CASES]
    o = PdlpOptions(verbose=False, max_iter=500000)
    out = batch_solve(probs, o)
    for name, (r, x, y) in zip(DEFAULT_CASES, out):
        _check_against_golden(name, r)


def test_batch_statuses():
    names = ["infeasible", "infeasible_eq", "unbounded_constrained"]
    out = batch_solve([GC.problem(k) for k in names], PdlpOptions(verbose=False, max_iter=100000))
    for name, (r, _, _) in zip(names, out):
        assert int(r.status) == GC.INDEX[name]["status"], name


def test_batch_invariance_alone_and_in_mix():
    target, _ = G.random_lp(700, 1750, 4, 12, 77)
    others = [G.random_lp(m, int(2.5 * m), 4, 12, 500 + k)[0] for k, m in enumerate(
        [200, 3000, 450, 1200, 900, 2500, 300, 1600] * 5)]
    o = PdlpOptions(verbose=False, **TIGHT)
    alone = batch_solve([target], o)[0]
    mix = batch_solve(others[:20] + [target] + others[20:], o)[20]
    assert alone[0].status == Status.Optimal
    assert alone[0].iterations == mix[0].iterations
    assert alone[0].objective == mix[0].objective
    np.testing.assert_array_equal(alone[1], mix[1])
    np.testing.assert_array_equal(alone[2], mix[2])


def _mix(seed0, sizes):
    return [G.random_lp(m, int(2.5 * m), 4, 12, seed0 + k)[0] for k, m in enumerate(sizes)]


def _same(a, b):
    for (r, x, y), (q, u, v) in zip(a, b):
        assert r.status == q.status and r.iterations == q.iterations and r.objective == q.objective
        np.testing.assert_array_equal(x, u)
        np.testing.assert_array_equal(y, v)


def test_batch_split_into_packs_matches_one_pack():
    lps = _mix(1300, (150, 700, 1600, 3000, 400, 2200))
    o = dict(verbose=False, **TIGHT)
    one = batch_solve(lps, PdlpOptions(**o))
    split = batch_solve(lps, PdlpOptions(batch_pack_mb=2, **o))  # about one LP per pack
    assert all(r.status == Status.Optimal for r, _, _ in one)
    _same(one, split)


def test_batch_compaction_does_not_change_results():
    lps = _mix(1400, (200, 2500, 300, 600, 1800, 250, 900, 3500))
    o = dict(verbose=False, **TIGHT)
    _same(batch_solve(lps, PdlpOptions(batch_compact=True, **o)),
          batch_solve(lps, PdlpOptions(batch_compact=False, **o)))


def test_batch_matches_single_lp_solves():
    """Packed and single-LP solves of the same LPs agree to the tolerance."""
    from mipx_b200.pdlp import PdlpSolver
    lps = _mix(1500, (300, 1000, 2200))
    out = batch_solve(lps, PdlpOptions(verbose=False, **TIGHT))
    for lp, (r, _, _) in zip(lps, out):
        s = PdlpSolver()
        s.setOptions(PdlpOptions(verbose=False, **TIGHT))
        s.load(lp)
        q = s.solve()
        assert r.status == q.status == Status.Optimal
        assert GC.rel_err(r.objective, q.objective) <= GC.OBJ_TOL, (r.objective, q.objective)


def test_batch_sliced_ell_matches_csr():
    """The sliced-ELL storage (rows renumbered by length inside each tile) and
    the CSR storage of the same LPs reach the same answers, and the renumbering
    is undone in the returned x and y."""
    lps = _mix(1600, (150, 700, 1600, 3000))
    o = dict(verbose=False, **TIGHT)
    sell = batch_solve(lps, PdlpOptions(batch_sell=True, **o))
    csr = batch_solve(lps, PdlpOptions(batch_sell=False, **o))
    for lp, (r, x, y), (q, u, v) in zip(lps, sell, csr):
        assert r.status == q.status == Status.Optimal
        assert GC.rel_err(r.objective, q.objective) <= GC.OBJ_TOL, (r.objective, q.objective)
        a = lp.matrix
        ax = np.array([a.values[a.row_starts[i]:a.row_starts[i + 1]] @ x[a.col_indices[a.row_starts[i]:a.row_starts[i + 1]]]
                       for i in range(lp.num_rows)])
        viol = np.maximum(lp.row_lower - ax, 0) + np.maximum(ax - lp.row_upper, 0)
        assert np.linalg.norm(viol) <= 1e-5 * (1 + np.linalg.norm(np.r_[lp.row_lower[np.isfinite(lp.row_lower)],
                                                                          lp.row_upper[np.isfinite(lp.row_upper)]]))
        # a renumbering left in place would move entries by O(1); both solves
        # approximate the same (nondegenerate) primal-dual pair
        assert np.linalg.norm(x - u) <= 1e-2 * (1 + np.linalg.norm(u))
        assert np.linalg.norm(y - v) <= 1e-2 * (1 + np.linalg.norm(v))


def test_fixed_column_with_negative_reduced_cost_converges():
    """min -2 x1 - x2  s.t.  x1 + x2 <= 1.5,  x1 fixed at 1,  0 <= x2 <= 10:  x = (1, 0.5),
    objective -2.5; the fixed column's reduced cost is negative at the optimum, which
    must not count as dual residual (single-LP engine and batch)."""
    from mipx_b200.pdlp import LpProblem, PdlpSolver, SparseMatrix
    lp = LpProblem(num_cols=2, obj=np.array([-2.0, -1.0]), col_lower=np.array([1.0, 0.0]),
                   col_upper=np.array([1.0, 10.0]), num_rows=1, row_lower=np.array([-np.inf]),
                   row_upper=np.array([1.5]),
                   matrix=SparseMatrix(1, 2, values=np.array([1.0, 1.0]), col_indices=np.array([0, 1], np.int32),
                                       row_starts=np.array([0, 2], np.int32)))
    o = PdlpOptions(max_iter=200000, **TIGHT)
    s = PdlpSolver()
    s.setOptions(o)
    s.load(lp)
    r = s.solve()
    assert r.status == Status.Optimal and abs(r.objective + 2.5) <= 1e-5, r
    (q, x, _), = batch_solve([lp], o)
    assert q.status == Status.Optimal and abs(q.objective + 2.5) <= 1e-5, q
    np.testing.assert_allclose(x, [1.0, 0.5], atol=1e-5)


def test_autotuned_pack_gives_identical_results():
    """The pack autotuner only picks how many sliced-ELL entries a thread loads
    per round; every variant sums a row in entry order, so results are
    bit-identical with and without it."""
    sizes = G.batch_sizes(24, seed=13)
    lps = [G.random_lp(m, n, 4, 12, 300 + k)[0] for k, (m, n) in enumerate(sizes)]
    base = dict(verbose=False, primal_tol=1e-6, dual_tol=1e-6, optimality_tol=1e-6)
    a = batch_solve(lps, PdlpOptions(**base))
    b = batch_solve(lps, PdlpOptions(autotune=True, **base))
    for (r, x, y), (q, u, v) in zip(a, b):
        assert (r.status, r.iterations, r.objective) == (q.status, q.iterations, q.objective)
        np.testing.assert_array_equal(x, u)
        np.testing.assert_array_equal(y, v)


def test_batch_over_devices_identical_to_one_device():
    """pdlpx_batch_solve_devices: the LPs sharded over a device list (here GPU 0
    twice: two host threads with their own streams and packs side by side) give
    results bit-identical to one pdlpx_batch_solve call (batch invariance), and
    the sharding splits the LPs between both entries of the list."""
    from mipx_b200.pdlp import shard_lps
    lps = _mix(900, [250, 1800, 600, 3200, 400, 1100, 750, 2400, 520, 1500])
    o = PdlpOptions(verbose=False, **TIGHT)
    one = batch_solve(lps, o)
    two = batch_solve(lps, o, devices=[0, 0])
    _same(one, two)
    d = shard_lps([lp.matrix.numNonzeros() + lp.num_rows + lp.num_cols for lp in lps], 2)
    assert set(d.tolist()) == {0, 1}


def test_device_ruiz_in_batch_and_server_is_bit_identical():
    """scale_on_device = 1 runs the Ruiz passes of every LP's preparation on the
    GPU (scaling.cu); the scaled data equal the host loop's to the last bit, so
    the batch and server results are identical with 1 and with 0."""
    from mipx_b200.pdlp import Server
    lps = _mix(1300, [400, 1500, 900])
    res = {}
    for dev in (0, 1):
        o = PdlpOptions(verbose=False, scale_on_device=dev, **TIGHT)
        res[("batch", dev)] = batch_solve(lps, o)
        with Server(o, max_packs=2, max_pack_lps=8, batch_window_ms=0) as srv:
            tickets = [srv.submit(lp) for lp in lps]
            res[("server", dev)] = [srv.wait(t) for t in tickets]
    _same(res[("batch", 0)], res[("batch", 1)])
    _same(res[("server", 0)], res[("server", 1)])
    assert all(r.status == Status.Optimal for r, _, _ in res[("batch", 1)])


def test_server_over_device_list():
    """A server over the device list [0, 0] places its packs on both entries and
    returns the results a one-device server gives."""
    from mipx_b200.pdlp import Server
    lps = _mix(1400, [300, 900, 1200, 500])
    o = PdlpOptions(verbose=False, **TIGHT)
    out = {}
    for devs in (None, [0, 0]):
        with Server(o, max_packs=1, max_pack_lps=1, batch_window_ms=0, devices=devs) as srv:
            tickets = [srv.submit(lp) for lp in lps]
            out[str(devs)] = [srv.wait(t) for t in tickets]
    _same(out["None"], out["[0, 0]"])


def test_persistent_cycle_gives_identical_results():
    """batch_persistent runs the N steps of each restart cycle as one cooperative
    launch over every sliced-ELL tile (grid barriers between the steps) with the
    same per-thread work as the per-class launches: every LP's result, with and
    without the compaction of finished LPs, is bit-identical to the graph's."""
    lps = [G.random_lp(m, int(2.5 * m), 4, 12, 3100 + k)[0] for k, m in enumerate((300, 1800, 700, 2600, 450, 1200))]
    for compact in (True, False):
        o = dict(verbose=False, batch_compact=compact, **TIGHT)
        graph = batch_solve(lps, PdlpOptions(**o))
        pers = batch_solve(lps, PdlpOptions(batch_persistent=True, **o))
        for (r, x, y), (q, u, v) in zip(graph, pers):
            assert r.status == q.status == Status.Optimal
            assert r.iterations == q.iterations and r.objective == q.objective
            np.testing.assert_array_equal(x, u)
            np.testing.assert_array_equal(y, v)
        # the persistent launch replaces the per-class step launches of every cycle
        assert pers[0][0].kernel_launches < graph[0][0].kernel_launches


def test_grid_barrier_wait_is_bounded():
    """The persistent cycle's grid barrier waits a bounded time: with the arrival
    count preloaded so that no barrier completes (a flag nothing sets), every
    block runs out of polls, the call returns PDLPX_E_TIMEOUT with the error word
    set, and the context stays usable for the next launch."""
    import ctypes as C

    from mipx_b200 import _capi
    lib = _capi.load()
    err, sec = C.c_int32(-1), C.c_double(-1.0)
    assert lib.pdlpx_grid_barrier_check(0, 148, 1000, 0, C.byref(err), C.byref(sec)) == 0, lib.pdlpx_last_error(None)
    assert err.value == 0 and 0.0 < sec.value < 5.0
    err, sec = C.c_int32(-1), C.c_double(-1.0)
    assert lib.pdlpx_grid_barrier_check(0, 4, 3, 1, C.byref(err), C.byref(sec)) == 6  # PDLPX_E_TIMEOUT
    assert err.value == 1 and 0.0 < sec.value < 30.0
    assert b"ran out" in lib.pdlpx_last_error(None)
    err = C.c_int32(-1)
    assert lib.pdlpx_grid_barrier_check(0, 148, 10, 0, C.byref(err), None) == 0
    assert err.value == 0
