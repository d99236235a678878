"""Regenerate the golden fixtures of the PDLP path (run in a container that has
the reference tree and has built oracle/_ref with ``make -C oracle``).

For every case the reference's own PdlpSolver (compiled from its sources into
oracle/_ref/libmipx_pdlp_ref.so) is run with the options of the corresponding
mipx test, and its status, objective, iteration count, work units and primal /
dual vectors are stored.  For the generated LPs the HiGHS optimum (scipy, FP64
dual simplex / IPM) is stored too as an independent objective check.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import lp_fixtures as F  # noqa: E402
from mipx_b200 import generators as G  # noqa: E402
from mipx_b200.pdlp import PdlpOptimalityNorm, PdlpOptions  # noqa: E402
from oracle import oracle as O  # noqa: E402


def quiet(**kw) -> PdlpOptions:
    o = PdlpOptions(verbose=False, use_gpu=False)
    for k, v in kw.items():
        setattr(o, k, v)
    return o


TIGHT = dict(primal_tol=1e-6, dual_tol=1e-6, optimality_tol=1e-6)
# Launch-shape and batching knobs of the device engine: no meaning for the
# reference, left at their defaults when the cases are replayed.
ENGINE_ONLY = {"autotune", "shape_primal", "shape_dual", "batch_pack_mb", "batch_compact", "batch_sell",
               "scale_on_device"}

CASES = {
    # name: (problem builder, options) -- options follow the mipx test that uses the LP
    "simple": (F.simple_lp, quiet(max_iter=10000)),
    "simple_linf": (F.simple_lp, quiet(max_iter=10000, optimality_norm=PdlpOptimalityNorm.LInf)),
    "simple_norescale": (F.simple_lp, quiet(max_iter=50000, do_bound_obj_rescaling=False)),
    "simple_nopolish": (F.simple_lp, quiet(max_iter=50000, enable_polishing=False)),
    "simple_precond": (F.simple_lp, quiet(max_iter=10000, preconditioner_refresh=True)),
    "simple_adaptive": (F.simple_lp, quiet(max_iter=50000, adaptive_step=True)),
    "bounds_only": (F.bounds_only_lp, quiet()),
    "empty": (F.empty_lp, quiet()),
    "unbounded_bounds_only": (F.unbounded_bounds_only_lp, quiet()),
    "infeasible": (F.infeasible_lp, quiet(max_iter=100000)),
    "infeasible_eq": (F.infeasible_eq_lp, quiet(max_iter=100000)),
    "unbounded_constrained": (F.unbounded_constrained_lp, quiet(max_iter=100000)),
    "col_bound_binding": (F.col_bound_binding_lp, quiet(max_iter=50000)),
    "large_rhs": (F.large_rhs_lp, quiet(max_iter=100000)),
    "equality": (F.equality_lp, quiet(max_iter=100000)),
    "equality_polish": (F.equality_lp, quiet(max_iter=100000, polish_primal_tol=1e-7, polish_dual_tol=1e-7)),
    "filter": (F.filter_lp, quiet(max_iter=50000, do_bound_obj_rescaling=False, matrix_zero_tol=1e-10)),
    "maximize": (F.maximize_lp, quiet(max_iter=50000)),
    "ranged": (F.ranged_lp, quiet(max_iter=100000, **TIGHT)),
    "medium": (F.medium_lp, quiet(max_iter=500000)),
    "medium_tight": (F.medium_lp, quiet(max_iter=500000, **TIGHT)),
    "medium_norescale": (F.medium_lp, quiet(max_iter=500000, do_bound_obj_rescaling=False)),
    "medium_polish7": (F.medium_lp, quiet(max_iter=500000, polish_primal_tol=1e-7, polish_dual_tol=1e-7)),
    # Anderson acceleration at restarts (test_pdlp.cpp:1204-1310)
    "simple_anderson": (F.simple_lp, quiet(max_iter=50000, anderson_acceleration=True, anderson_window_size=5)),
    "simple_anderson_w2": (F.simple_lp, quiet(max_iter=50000, anderson_acceleration=True, anderson_window_size=2)),
    "equality_anderson": (F.equality_lp, quiet(max_iter=100000, anderson_acceleration=True, anderson_window_size=5)),
    "medium_anderson": (F.medium_lp, quiet(max_iter=500000, anderson_acceleration=True, anderson_window_size=5)),
}
GENERATED = {
    # name: (m, n, lo, hi, seed)
    "rand_60x150": (60, 150, 4, 12, 3),
    "rand_200x500": (200, 500, 4, 12, 4),
    "rand_500x1250": (500, 1250, 4, 12, 5),
    "rand_2000x5000": (2000, 5000, 4, 12, 1),
}
# Generated LPs solved with Anderson acceleration (window 5), same tolerances.
GENERATED_AA = {
    "rand_500x1250_anderson": (500, 1250, 4, 12, 5),
}

# LPs too large for the reference's CPU PDLP in a test budget: HiGHS optimum only.
HIGHS_ONLY = {
    "transport_1000x1000": (1000, 1000, 7),
}


def highs_objective(lp) -> float:
    from scipy.optimize import linprog
    from scipy.sparse import csr_matrix
    A = csr_matrix((lp.matrix.values, lp.matrix.col_indices, lp.matrix.row_starts), shape=(lp.num_rows, lp.num_cols))
    eq = lp.row_lower == lp.row_upper
    le = ~eq & np.isfinite(lp.row_upper)
    ge = ~eq & np.isfinite(lp.row_lower)
    A_ub = __import__("scipy.sparse", fromlist=["vstack"]).vstack([A[le], -A[ge]])
    b_ub = np.concatenate([lp.row_upper[le], -lp.row_lower[ge]])
    r = linprog(lp.obj, A_ub=A_ub, b_ub=b_ub, A_eq=A[eq], b_eq=lp.row_lower[eq],
                bounds=list(zip(lp.col_lower, lp.col_upper)), method="highs",
                options={"primal_feasibility_tolerance": 1e-10, "dual_feasibility_tolerance": 1e-10})
    assert r.status == 0, r.message
    return float(r.fun) + lp.obj_offset


def main() -> None:
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libmipx_pdlp_ref.so missing: run `make -C oracle` where the reference exists")
    index = {}
    arrays = {}
    todo = [(k, b(), o) for k, (b, o) in CASES.items()]
    for name, (m, n, lo, hi, seed) in GENERATED.items():
        todo.append((name, G.random_lp(m, n, lo, hi, seed)[0], quiet(max_iter=500000, **TIGHT)))
    for name, (m, n, lo, hi, seed) in GENERATED_AA.items():
        todo.append((name, G.random_lp(m, n, lo, hi, seed)[0],
                     quiet(max_iter=500000, anderson_acceleration=True, anderson_window_size=5, **TIGHT)))
    for name, lp, opts in todo:
        res, x, y = O.ref_solve(lp, opts)
        entry = {
            "status": int(res.status), "objective": res.objective, "iterations": res.iterations,
            "work_units": res.work_units, "m": lp.num_rows, "n": lp.num_cols,
            "options": {k: (int(v) if isinstance(v, bool) else v) for k, v in vars(opts).items()
                        if k != "stop_flag" and k not in ENGINE_ONLY and not isinstance(v, object.__class__)},
        }
        entry["options"] = {k: (v if not hasattr(v, "value") else int(v)) for k, v in entry["options"].items()}
        if name in GENERATED or name in GENERATED_AA:
            gen = GENERATED.get(name) or GENERATED_AA[name]
            entry["generator"] = dict(zip(("m", "n", "nnz_lo", "nnz_hi", "seed"), gen))
            entry["highs_objective"] = highs_objective(lp)
        index[name] = entry
        arrays[f"{name}__x"] = x
        arrays[f"{name}__y"] = y
        print(f"{name:24s} status={int(res.status)} obj={res.objective:.12g} iters={res.iterations}", flush=True)
    for name, (s_, d_, seed) in HIGHS_ONLY.items():
        lp, _ = G.transport_lp(s_, d_, seed)
        index[name] = {"generator": {"kind": "transport", "supplies": s_, "demands": d_, "seed": seed},
                       "highs_objective": highs_objective(lp), "m": lp.num_rows, "n": lp.num_cols}
        print(f"{name:24s} highs={index[name]['highs_objective']:.12g}", flush=True)
    (HERE / "ref_pdlp.json").write_text(json.dumps(index, indent=1, sort_keys=True))
    np.savez_compressed(HERE / "ref_pdlp_vectors.npz", **arrays)


if __name__ == "__main__":
    main()
