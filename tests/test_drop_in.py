"""The drop-in proof: mipx's own PdlpSolver class (src/lp/pdlp.cpp compiled
from the reference's sources) with the pdlpx binding as the body of its
solveGpu (include/pdlpx_solvegpu.inc, built by `make -C oracle ref_bound`).

With use_gpu on, the reference class's own dispatch (pdlp.cpp:862-868) sends
every solve to the B200 engine: mipx's known answers (tests/test_pdlp.cpp) and
the golden cases come out as the reference's CPU path gives them, and the
concurrent-root race pattern of mipx (mip_solver.cpp:4470-4605) -- two arms
sharing a std::atomic<bool> through PdlpOptions::stop_flag -- stops the losing
arm on the device.  The race wiring itself is checked on the CPU path too.
"""
import pytest

import golden_cases as GC
import lp_fixtures as F
from mipx_b200 import generators as G
from mipx_b200.pdlp import PdlpOptions, Status
from oracle import oracle as O

GPU = dict(use_gpu=True, gpu_min_rows=0, gpu_min_nnz=0)


def _race_lp():
    return G.random_lp(300, 750, 4, 12, 21)[0]


def test_race_pattern_on_the_reference_cpu_path():
    """Two CPU arms of the reference class: the loose arm wins, the tight arm is
    stopped by the shared flag (IterLimit) or finishes."""
    if not O.ref_available():
        pytest.skip("reference library not built")
    lp = _race_lp()
    fast = PdlpOptions(verbose=False, use_gpu=False, primal_tol=1e-3, dual_tol=1e-3, optimality_tol=1e-3)
    slow = PdlpOptions(verbose=False, use_gpu=False, max_iter=4_000_000, primal_tol=1e-12, dual_tol=1e-12,
                       optimality_tol=1e-12)
    r0, r1, w = O.ref_race(lp, fast, slow)
    assert w == 0 and r0.status == Status.Optimal
    assert r1.status in (Status.IterLimit, Status.Optimal)


def _bound_or_skip():
    if not O.REF_BOUND_LIB.exists():
        pytest.skip("bound reference library not built (needs the reference tree at build time)")


@pytest.mark.gpu
def test_known_answers_through_the_reference_class():
    _bound_or_skip()
    for name, (builder, expected, tol, where) in F.KNOWN_ANSWERS.items():
        lp = builder()
        r, x, _ = O.ref_solve(lp, PdlpOptions(verbose=False, max_iter=100000, **GPU), bound=True)
        # LPs without rows are closed form in the reference's solve() before its GPU dispatch
        assert r.used_gpu == (lp.num_rows > 0 and lp.num_cols > 0), name
        assert r.status == Status.Optimal and abs(r.objective - expected) <= tol, (name, r.objective, expected)


@pytest.mark.gpu
@pytest.mark.parametrize("name", [k for k in GC.NAMES if k not in ("empty", "bounds_only", "unbounded_bounds_only")])
def test_golden_cases_through_the_reference_class(name):
    _bound_or_skip()
    e = GC.INDEX[name]
    r, x, y = O.ref_solve(GC.problem(name), GC.options(name, **GPU), bound=True)
    assert r.used_gpu
    assert int(r.status) == e["status"], (name, r.status)
    if e["status"] == Status.Optimal:
        if e["options"]["primal_tol"] <= 1e-6:
            assert GC.rel_err(r.objective, e["objective"]) <= GC.OBJ_TOL, (name, r.objective, e["objective"])
        else:
            bound = 1e-4 if name in ("medium", "simple") else 1e-3 * max(1.0, abs(e["objective"]))
            assert abs(r.objective - e["objective"]) <= max(bound, 2e-4 * abs(e["objective"]))
        gx, _ = GC.vectors(name)
        assert x.shape == gx.shape


@pytest.mark.gpu
def test_race_on_the_device_through_the_reference_class():
    _bound_or_skip()
    lp = _race_lp()
    fast = PdlpOptions(verbose=False, primal_tol=1e-4, dual_tol=1e-4, optimality_tol=1e-4, **GPU)
    slow = PdlpOptions(verbose=False, max_iter=4_000_000, primal_tol=1e-12, dual_tol=1e-12, optimality_tol=1e-12,
                       **GPU)
    r0, r1, w = O.ref_race(lp, fast, slow, bound=True)
    assert r0.used_gpu and r1.used_gpu
    assert w == 0 and r0.status == Status.Optimal
    assert r1.status in (Status.IterLimit, Status.Optimal)
    ref, _, _ = O.ref_solve(lp, PdlpOptions(verbose=False, use_gpu=False, primal_tol=1e-4, dual_tol=1e-4,
                                            optimality_tol=1e-4))
    assert abs(r0.objective - ref.objective) <= 1e-3 * max(1.0, abs(ref.objective))
