"""Request server (pdlpx_server_*: LP solves as they arrive, continuously batched).

* same result alone and in the mix: every request's result through the server
  -- packed with whatever else was waiting, with several packs running at once
  -- is bit-identical to the same LP solved alone by pdlpx_batch_solve;
* requests submitted while packs run are admitted and finished, several packs
  overlap, and latency statistics are reported;
* node LPs (fixed integer columns, appended cuts) warm-started from a finished
  base request reach the same optimum as cold solves (PDLP warm starts do not
  reliably save iterations, so only the optimum is compared);
* trivial LPs, invalid LPs, unknown tickets, timeouts and shutdown with work in
  flight come back as error codes or statuses, never as hangs.
"""
import threading
import time

import numpy as np
import pytest

import golden_cases as GC
from mipx_b200 import generators as G
from mipx_b200._capi import PdlpxError
from mipx_b200.pdlp import LpProblem, PdlpOptions, Server, SparseMatrix, Status, batch_solve

pytestmark = pytest.mark.gpu

TIGHT = dict(primal_tol=1e-6, dual_tol=1e-6, optimality_tol=1e-6, verbose=False)


def _lps(seed0, sizes):
    return [G.random_lp(m, int(2.5 * m), 4, 12, seed0 + k)[0] for k, m in enumerate(sizes)]


def test_server_results_equal_alone_solves():
    lps = _lps(2100, (300, 1200, 500, 2000, 800, 250, 1500, 600, 400, 1000))
    o = PdlpOptions(**TIGHT)
    alone = [batch_solve([lp], o)[0] for lp in lps]
    with Server(o, max_packs=3, max_pack_lps=4) as srv:
        tickets = [srv.submit(lp) for lp in lps]
        got = [srv.wait(t, timeout=300) for t in tickets]
        st = srv.stats()
    for (r, x, y), (q, u, v) in zip(got, alone):
        assert r.status == q.status == Status.Optimal
        assert r.iterations == q.iterations and r.objective == q.objective
        np.testing.assert_array_equal(x, u)
        np.testing.assert_array_equal(y, v)
    assert st["completed"] == len(lps) and st["submitted"] == len(lps)
    assert 0 < st["p50_latency_s"] <= st["p99_latency_s"] <= st["max_latency_s"]
    assert st["lps_per_sec"] > 0


def test_server_admits_requests_while_packs_run():
    lps = _lps(2200, [700, 1500, 400, 2500, 900, 1200] * 3)
    o = PdlpOptions(**TIGHT)
    seen_packs = []
    with Server(o, max_packs=4, max_pack_lps=3) as srv:
        tickets = []
        for lp in lps:  # arrivals spread over the solve
            tickets.append(srv.submit(lp))
            seen_packs.append(srv.stats()["packs_running"])
            time.sleep(0.01)
        for t in tickets:
            r, x, _ = srv.wait(t, timeout=300)
            assert r.status == Status.Optimal
        st = srv.stats()
    assert st["completed"] == len(lps)
    assert max(seen_packs) >= 2, seen_packs  # packs overlapped on the device


def test_server_node_lps_warm_started_from_base_ticket():
    base, x0 = G.random_lp(2000, 5000, 4, 12, 31)
    ints = G.integer_marks(base.num_cols)
    nodes = [G.node_lp(base, x0, ints, seed) for seed in range(4)]
    o = PdlpOptions(**TIGHT)
    with Server(o, max_packs=2, max_pack_lps=8) as srv:
        tb = srv.submit(base)
        rb, xb, yb = srv.wait(tb, timeout=300)
        assert rb.status == Status.Optimal
        warm = [srv.submit(nd, warm=tb) for nd in nodes]
        cold = [srv.submit(nd) for nd in nodes]
        for tw, tc in zip(warm, cold):
            rw, _, _ = srv.wait(tw, timeout=300)
            rc, _, _ = srv.wait(tc, timeout=300)
            assert rw.status == rc.status
            if rc.status == Status.Optimal:
                assert GC.rel_err(rw.objective, rc.objective) <= GC.OBJ_TOL, (rw.objective, rc.objective)


def test_server_trivial_invalid_and_unknown_tickets():
    o = PdlpOptions(**TIGHT)
    empty = LpProblem(num_cols=0, num_rows=0, obj_offset=42.0)
    bounds_only = LpProblem(num_cols=1, obj=np.array([1.0]), col_lower=np.array([1.0]), col_upper=np.array([4.0]),
                            num_rows=0, matrix=SparseMatrix(0, 1))
    bad = LpProblem(num_cols=2, obj=np.zeros(2), col_lower=np.zeros(2), col_upper=np.ones(2), num_rows=1,
                    row_lower=np.zeros(1), row_upper=np.ones(1),
                    matrix=SparseMatrix(1, 2, values=np.array([1.0]), col_indices=np.array([7], np.int32),
                                        row_starts=np.array([0, 1], np.int32)))
    with Server(o, max_packs=1) as srv:
        r, _, _ = srv.wait(srv.submit(empty), timeout=60)
        assert r.status == Status.Optimal and r.objective == 42.0
        r, x, _ = srv.wait(srv.submit(bounds_only), timeout=60)
        assert r.status == Status.Optimal and abs(x[0] - 1.0) < 1e-12
        t = srv.submit(bad)
        with pytest.raises(PdlpxError):
            srv.wait(t, timeout=60)
        with pytest.raises(PdlpxError):
            srv.wait(987654321, timeout=1)
        with pytest.raises(PdlpxError):
            srv.submit(bounds_only, warm=987654321)


def test_server_wait_timeout_and_shutdown_with_work_in_flight():
    big, _ = G.random_lp(20000, 50000, 4, 12, 41)
    o = PdlpOptions(**TIGHT)
    srv = Server(o, max_packs=1)
    t = srv.submit(big)
    with pytest.raises(PdlpxError) as e:
        srv.wait(t, timeout=0.05)
    assert e.value.code == 6  # PDLPX_E_TIMEOUT
    done = threading.Event()

    def closer():
        srv.close()
        done.set()

    th = threading.Thread(target=closer)
    th.start()
    th.join(timeout=120)
    assert done.is_set(), "server shutdown did not return"


def test_server_release_while_pack_still_runs():
    """Finished requests are released at once while the rest of their pack keeps
    iterating; the pack still finishes every other request."""
    lps = _lps(2300, (200, 3000, 300, 2500, 250, 2000))
    o = PdlpOptions(**TIGHT)
    with Server(o, max_packs=1, max_pack_lps=8) as srv:
        tickets = [srv.submit(lp) for lp in lps]
        pending = set(tickets)
        t_end = time.time() + 300
        while pending and time.time() < t_end:
            for t in list(pending):
                if srv.done(t):
                    r, _, _ = srv.wait(t, timeout=1)
                    assert r.status == Status.Optimal
                    srv.release(t)
                    pending.discard(t)
            time.sleep(0.002)
        assert not pending


# ---------------------------------------------------------------------------
# Family packs: node LPs warm-started from a base ticket share its rows
# ---------------------------------------------------------------------------
def _family(seed=51, count=8, m=2000, n=5000):
    base, x0 = G.random_lp(m, n, 4, 12, seed)
    ints = G.integer_marks(base.num_cols)
    return base, [G.node_lp(base, x0, ints, 100 + k) for k in range(count)]


def _solve_nodes(base, nodes, opts, **cfg):
    with Server(opts, **cfg) as srv:
        tb = srv.submit(base)
        srv.wait(tb, timeout=300)
        tickets = [srv.submit(nd, warm=tb) for nd in nodes]
        return [srv.wait(t, timeout=300) for t in tickets]


def test_family_results_same_alone_and_in_mix():
    """A node LP's family-pack result is bit-identical in a family of one and
    packed with seven other nodes of the same base (one lane per LP, lane
    arithmetic independent of the other lanes)."""
    base, nodes = _family()
    o = PdlpOptions(**TIGHT)
    mix = _solve_nodes(base, nodes, o, max_packs=1, max_pack_lps=32, batch_window_ms=500)
    for k in (0, 3, 7):
        alone = _solve_nodes(base, [nodes[k]], o, max_packs=1)[0]
        (r, x, y), (q, u, v) = mix[k], alone
        assert r.status == q.status == Status.Optimal
        assert r.iterations == q.iterations and r.objective == q.objective
        np.testing.assert_array_equal(x, u)
        np.testing.assert_array_equal(y, v)
        assert r.fp64_iterations == r.iterations  # family packs iterate in FP64


def test_family_matches_single_lp_fp64():
    """Family results against the single-LP FP64 engine on the same node LPs:
    same status, objectives within 1e-6 relative (both at 1e-6 relative KKT),
    primal feasibility of the returned x within the tolerance."""
    from mipx_b200.pdlp import PdlpSolver, Precision
    base, nodes = _family(seed=52, count=6)
    o = PdlpOptions(**TIGHT)
    fam = _solve_nodes(base, nodes, o, max_packs=1, batch_window_ms=500)
    for nd, (r, x, _) in zip(nodes, fam):
        s = PdlpSolver()
        s.setOptions(PdlpOptions(precision=Precision.FP64, **TIGHT))
        s.load(nd)
        q = s.solve()
        assert r.status == q.status
        if q.status != Status.Optimal:
            continue
        assert GC.rel_err(r.objective, q.objective) <= GC.OBJ_TOL, (r.objective, q.objective)
        assert np.all(x >= nd.col_lower - 1e-9) and np.all(x <= nd.col_upper + 1e-9)
        assert r.rel_primal_resid <= 1e-6 and r.rel_dual_resid <= 1e-6


def test_family_member_check_and_regular_fallback():
    """An LP linked to the ticket whose base rows differ (one value changed) or
    whose columns differ is solved in a regular pack and still reaches the optimum;
    a family pack and the regular packs run side by side."""
    base, nodes = _family(seed=53, count=3)
    changed = G.node_lp(base, np.zeros(base.num_cols), G.integer_marks(base.num_cols), 7)
    changed.matrix.values[5] *= 1.5
    o = PdlpOptions(**TIGHT)
    with Server(o, max_packs=3) as srv:
        tb = srv.submit(base)
        srv.wait(tb, timeout=300)
        tickets = [srv.submit(nd, warm=tb) for nd in nodes + [changed]]
        res = [srv.wait(t, timeout=300) for t in tickets]
    for r, _, _ in res:
        assert r.status == Status.Optimal
    assert res[-1][0].fp64_iterations < res[-1][0].iterations  # regular mixed-precision pack


def test_family_off_uses_regular_packs():
    base, nodes = _family(seed=54, count=2)
    o = PdlpOptions(**TIGHT)
    res = _solve_nodes(base, nodes, o, families=False)
    for r, _, _ in res:
        assert r.status == Status.Optimal
        assert r.fp64_iterations < r.iterations


def test_family_lane_admission_joins_running_pack():
    """Continuous admission at lane granularity: with one pack stream, nodes that
    arrive while a family pack runs take its free lanes between restart cycles
    instead of waiting for it to end; each admitted node's result is
    bit-identical to the same node solved in a family of one (a lane's
    arithmetic depends on its LP alone, whenever it joins)."""
    base, nodes = _family(seed=61, count=5, m=20000, n=50000)
    o = PdlpOptions(**TIGHT)
    with Server(o, max_packs=1, max_pack_lps=32, batch_window_ms=0) as srv:
        tb = srv.submit(base)
        srv.wait(tb, timeout=300)
        first = srv.submit(nodes[0], warm=tb)  # starts a pack of one at once
        time.sleep(0.05)
        later = [srv.submit(nd, warm=tb) for nd in nodes[1:]]
        res = [srv.wait(t, timeout=300) for t in [first] + later]
        st = srv.stats()
    assert st["admitted"] >= 1, st
    for k in (0, 1, len(nodes) - 1):
        alone = _solve_nodes(base, [nodes[k]], o, max_packs=1, lane_admission=False)[0]
        (r, x, y), (q, u, v) = res[k], alone
        assert r.status == q.status == Status.Optimal
        assert r.iterations == q.iterations and r.objective == q.objective
        np.testing.assert_array_equal(x, u)
        np.testing.assert_array_equal(y, v)
