"""Regenerate tests/golden/config_pins.json: FP64 objective pins of the
benchmark configurations (run where oracle/_ref was built with the reference
tree present; HiGHS through scipy).

* ``batch_sample``  -- the first 16 LPs of the batched workload (lognormal
  sizes, seeds 1000 + k): the reference's own CPU PdlpSolver at 1e-6 relative
  KKT (status, objective, iterations) and the HiGHS dual-simplex optimum.
* ``nodes``         -- 8 branch-and-bound node LPs of the serving workload's
  20,000 x 50,000 base LP (node seeds 1000 + k): the reference's CPU
  PdlpSolver at 1e-8 relative KKT on the same LP with its fixed columns
  (lb == ub) substituted out -- the reference's check counts a fixed column's
  reduced cost as dual residual and cannot converge on the node LP itself --
  plus the number of fixed columns each node carries.
* ``powerlaw_100000x400000`` -- the power-law LP at a fifth of the headline
  size (seed 11): the reference's CPU PdlpSolver at 1e-7 relative KKT.

HiGHS (dual simplex, interior point) does not finish the 20,000 x 50,000 node
LPs or the 100,000 x 400,000 power-law LP within an hour here, so the
reference's FP64 PDLP at a tolerance tighter than the tests' is the pin there.

    python tests/golden/make_config_pins.py
"""
from __future__ import annotations

import json
import multiprocessing as mp
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

BATCH_SAMPLE = 16
NODES = 8
POWERLAW_ROWS = 100_000
WORKERS = 5


def _highs(lp, time_limit: float = 900.0):
    """HiGHS dual simplex optimum (None when it does not finish in time_limit)."""
    from scipy.optimize import linprog
    from scipy.sparse import csr_matrix, vstack
    A = csr_matrix((lp.matrix.values, lp.matrix.col_indices, lp.matrix.row_starts), shape=(lp.num_rows, lp.num_cols))
    eq = lp.row_lower == lp.row_upper
    le = ~eq & np.isfinite(lp.row_upper)
    ge = ~eq & np.isfinite(lp.row_lower)
    t0 = time.perf_counter()
    r = linprog(lp.obj, A_ub=vstack([A[le], -A[ge]]), b_ub=np.concatenate([lp.row_upper[le], -lp.row_lower[ge]]),
                A_eq=A[eq], b_eq=lp.row_lower[eq], bounds=np.stack([lp.col_lower, lp.col_upper], 1),
                method="highs-ds", options={"primal_feasibility_tolerance": 1e-10,
                                           "dual_feasibility_tolerance": 1e-10, "time_limit": time_limit})
    dt = time.perf_counter() - t0
    return (float(r.fun) + lp.obj_offset if r.status == 0 else None), dt


def _ref(lp, tol: float, max_iter: int = 2_000_000):
    from mipx_b200.pdlp import PdlpOptions
    from oracle import oracle as O
    o = PdlpOptions(verbose=False, use_gpu=False, primal_tol=tol, dual_tol=tol, optimality_tol=tol,
                    max_iter=max_iter)
    t0 = time.perf_counter()
    r, _, _ = O.ref_solve(lp, o)
    return r, time.perf_counter() - t0


def substitute_fixed(lp):
    """The same LP with every fixed column (lb == ub) replaced by its value: its
    terms move into the row bounds and the objective offset.  Optimal
    objectives of the two LPs are equal."""
    from mipx_b200.pdlp import LpProblem, SparseMatrix
    fixed = lp.col_lower == lp.col_upper
    keep = np.flatnonzero(~fixed)
    newcol = -np.ones(lp.num_cols, dtype=np.int64)
    newcol[keep] = np.arange(keep.size)
    v = np.where(fixed, lp.col_lower, 0.0)
    a = lp.matrix
    rows = np.repeat(np.arange(lp.num_rows), np.diff(a.row_starts))
    shift = np.bincount(rows, weights=a.values * v[a.col_indices], minlength=lp.num_rows)
    live = ~fixed[a.col_indices]
    starts = np.concatenate([[0], np.cumsum(np.bincount(rows[live], minlength=lp.num_rows))]).astype(np.int32)
    mat = SparseMatrix(lp.num_rows, keep.size, values=a.values[live].copy(),
                       col_indices=newcol[a.col_indices[live]].astype(np.int32), row_starts=starts)
    return LpProblem(num_cols=keep.size, obj=lp.obj[keep].copy(), col_lower=lp.col_lower[keep].copy(),
                     col_upper=lp.col_upper[keep].copy(), num_rows=lp.num_rows, row_lower=lp.row_lower - shift,
                     row_upper=lp.row_upper - shift, matrix=mat, sense=lp.sense,
                     obj_offset=lp.obj_offset + float(np.dot(lp.obj[fixed], lp.col_lower[fixed])))


def batch_job(k: int) -> dict:
    from mipx_b200 import generators as G
    m, n = G.batch_sizes(512, seed=5)[k]
    lp, _ = G.random_lp(m, n, 4, 12, 1000 + k)
    r, tr = _ref(lp, 1e-6, 500_000)
    hi, th = _highs(lp)
    return {"k": k, "m": m, "n": n, "seed": 1000 + k, "reference_status": int(r.status),
            "reference_objective": r.objective, "reference_iterations": r.iterations, "reference_seconds": tr,
            "highs_objective": hi, "highs_seconds": th}


def node_job(k: int) -> dict:
    from mipx_b200 import generators as G
    base, x0 = G.random_lp(20000, 50000, 4, 12, 101)
    ints = G.integer_marks(base.num_cols)
    nd = G.node_lp(base, x0, ints, 1000 + k)
    r, tr = _ref(substitute_fixed(nd), 1e-8)
    return {"k": k, "seed": 1000 + k, "m": nd.num_rows, "n": nd.num_cols,
            "fixed_columns": int(np.sum(nd.col_lower == nd.col_upper)), "cuts": nd.num_rows - base.num_rows,
            "reference_status": int(r.status), "reference_objective": r.objective,
            "reference_iterations": r.iterations, "reference_seconds": tr, "reference_tol": 1e-8}


def powerlaw_job(m: int) -> dict:
    from mipx_b200 import generators as G
    lp, _ = G.powerlaw_lp(m, 4 * m, 2, 2000, 10.0, 0.01, 1e3, 11)
    r, tr = _ref(lp, 1e-7)
    return {"m": m, "n": 4 * m, "nnz": lp.matrix.numNonzeros(), "seed": 11, "reference_status": int(r.status),
            "reference_objective": r.objective, "reference_iterations": r.iterations, "reference_seconds": tr,
            "reference_tol": 1e-7}


def main() -> None:
    ctx = mp.get_context("spawn")
    with ctx.Pool(WORKERS) as pool:
        big = pool.apply_async(powerlaw_job, (POWERLAW_ROWS,))
        nodes = pool.map_async(node_job, range(NODES), chunksize=1)
        batch = pool.map_async(batch_job, range(BATCH_SAMPLE), chunksize=1)
        out = {"batch_sample": batch.get(), "nodes": nodes.get(),
               f"powerlaw_{POWERLAW_ROWS}x{4 * POWERLAW_ROWS}": big.get()}
    (HERE / "config_pins.json").write_text(json.dumps(out, indent=1, sort_keys=True))
    print(json.dumps(out, indent=1)[:4000])


if __name__ == "__main__":
    main()
