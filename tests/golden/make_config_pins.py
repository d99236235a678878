"""Regenerate tests/golden/config_pins.json: FP64 objective pins of the
benchmark configurations (run where oracle/_ref was built with the reference
tree present; HiGHS through scipy).

* ``batch_sample``  -- the first 16 LPs of the batched workload (lognormal
  sizes, seeds 1000 + k): the reference's own CPU PdlpSolver at 1e-6 relative
  KKT (status, objective, iterations) and the HiGHS optimum.
* ``nodes``         -- 8 branch-and-bound node LPs of the serving workload's
  20,000 x 50,000 base LP (node seeds 1000 + k): the HiGHS optimum and the
  number of fixed columns (lb == ub) each node carries.
* ``powerlaw_100000x400000`` -- the power-law LP at a fifth of the headline
  size (seed 11): the HiGHS optimum.

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


def _highs(lp) -> tuple[float, float]:
    sys.path.insert(0, str(HERE))
    from make_golden import highs_objective
    t0 = time.perf_counter()
    return highs_objective(lp), time.perf_counter() - t0


def batch_job(k: int) -> dict:
    from mipx_b200 import generators as G
    from mipx_b200.pdlp import PdlpOptions
    from oracle import oracle as O
    m, n = G.batch_sizes(512, seed=5)[k]
    lp, _ = G.random_lp(m, n, 4, 12, 1000 + k)
    o = PdlpOptions(verbose=False, use_gpu=False, primal_tol=1e-6, dual_tol=1e-6, optimality_tol=1e-6,
                    max_iter=500000)
    r, _, _ = O.ref_solve(lp, o)
    hi, th = _highs(lp)
    return {"k": k, "m": m, "n": n, "seed": 1000 + k, "reference_status": int(r.status),
            "reference_objective": r.objective, "reference_iterations": r.iterations, "highs_objective": hi,
            "highs_seconds": th}


def node_job(k: int) -> dict:
    from mipx_b200 import generators as G
    base, x0 = G.random_lp(20000, 50000, 4, 12, 101)
    ints = G.integer_marks(base.num_cols)
    nd = G.node_lp(base, x0, ints, 1000 + k)
    hi, th = _highs(nd)
    return {"k": k, "seed": 1000 + k, "m": nd.num_rows, "n": nd.num_cols,
            "fixed_columns": int(np.sum(nd.col_lower == nd.col_upper)), "cuts": nd.num_rows - base.num_rows,
            "highs_objective": hi, "highs_seconds": th}


def powerlaw_job(m: int) -> dict:
    from mipx_b200 import generators as G
    lp, _ = G.powerlaw_lp(m, 4 * m, 2, 2000, 10.0, 0.01, 1e3, 11)
    hi, th = _highs(lp)
    return {"m": m, "n": 4 * m, "nnz": lp.matrix.numNonzeros(), "seed": 11, "highs_objective": hi,
            "highs_seconds": th}


def main() -> None:
    ctx = mp.get_context("spawn")
    with ctx.Pool(8) as pool:
        big = pool.apply_async(powerlaw_job, (POWERLAW_ROWS,))
        nodes = pool.map_async(node_job, range(NODES))
        batch = pool.map_async(batch_job, range(BATCH_SAMPLE))
        out = {"batch_sample": batch.get(), "nodes": nodes.get(),
               f"powerlaw_{POWERLAW_ROWS}x{4 * POWERLAW_ROWS}": big.get()}
    (HERE / "config_pins.json").write_text(json.dumps(out, indent=1, sort_keys=True))
    print(json.dumps(out, indent=1)[:4000])


if __name__ == "__main__":
    main()
