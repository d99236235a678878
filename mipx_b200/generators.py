"""Seeded synthetic LPs of the benchmark workloads (C generators in libpdlpx).

* ``random_lp``      -- random sparse LP: columns with U{lo..hi} nonzeros at
  uniform rows, N(0,1) values, x0~U[0,10], rows alternating '=' / '<=' with
  b = A x0 (+U[0,1] slack), 0 <= x <= 10, c~N(0,1).  2,000 x 5,000 with 4-12
  nonzeros per column is the single-LP CPU-sized case.
* ``transport_lp``   -- s x d transportation problem (1,000 x 1,000: 1M
  variables, 2,000 rows, 2M unit nonzeros).
* ``powerlaw_lp``    -- large LP with power-law column counts (500,000 x
  2,000,000, counts in [2, 2000] with mean 10, 1% of rows scaled by 1e3).
* ``batch_sizes``    -- row counts of the 512-LP batch, lognormal(median 1,500,
  sigma 0.8) clipped to [200, 20,000], n = 2.5 m.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from .pdlp import LpProblem, Sense, SparseMatrix


def _take(g: _capi.GenLp) -> tuple[LpProblem, np.ndarray]:
    m, n, nnz = g.m, g.n, g.nnz
    arr = lambda p, k, dt: np.ctypeslib.as_array(p, shape=(k,)).astype(dt, copy=True) if k > 0 else np.zeros(0, dt)
    rp = arr(g.row_ptr, m + 1, np.int32)
    ci = arr(g.col_idx, nnz, np.int32)
    v = arr(g.val, nnz, np.float64)
    lp = LpProblem(
        name="generated", sense=Sense.Minimize, num_cols=n, num_rows=m,
        obj=arr(g.obj, n, np.float64), col_lower=arr(g.col_lb, n, np.float64), col_upper=arr(g.col_ub, n, np.float64),
        row_lower=arr(g.row_lb, m, np.float64), row_upper=arr(g.row_ub, m, np.float64),
        matrix=SparseMatrix(m, n, values=v, col_indices=ci, row_starts=rp))
    x0 = arr(g.x0, n, np.float64)
    _capi.load().pdlpx_free_lp(C.byref(g))
    return lp, x0


def random_lp(m: int = 2000, n: int = 5000, nnz_lo: int = 4, nnz_hi: int = 12, seed: int = 1):
    g = _capi.GenLp()
    _capi.check(_capi.load().pdlpx_gen_random(m, n, nnz_lo, nnz_hi, seed, C.byref(g)))
    lp, x0 = _take(g)
    lp.name = f"random_{m}x{n}_s{seed}"
    return lp, x0


def transport_lp(supplies: int = 1000, demands: int = 1000, seed: int = 7):
    g = _capi.GenLp()
    _capi.check(_capi.load().pdlpx_gen_transport(supplies, demands, seed, C.byref(g)))
    lp, x0 = _take(g)
    lp.name = f"transport_{supplies}x{demands}_s{seed}"
    return lp, x0


def powerlaw_lp(m: int = 500_000, n: int = 2_000_000, kmin: int = 2, kmax: int = 2000, kmean: float = 10.0,
                big_frac: float = 0.01, big_scale: float = 1e3, seed: int = 11):
    g = _capi.GenLp()
    _capi.check(_capi.load().pdlpx_gen_powerlaw(m, n, kmin, kmax, kmean, big_frac, big_scale, seed, C.byref(g)))
    lp, x0 = _take(g)
    lp.name = f"powerlaw_{m}x{n}_s{seed}"
    return lp, x0


def batch_sizes(count: int = 512, median: float = 1500.0, sigma: float = 0.8, lo: int = 200, hi: int = 20000,
                seed: int = 5) -> list[tuple[int, int]]:
    rng = np.random.default_rng(seed)
    ms = np.clip(np.round(np.exp(np.log(median) + sigma * rng.standard_normal(count))), lo, hi).astype(int)
    return [(int(m), int(round(2.5 * m))) for m in ms]


def batch_lps(count: int = 512, seed: int = 5, **kw) -> list[LpProblem]:
    return [random_lp(m, n, 4, 12, seed * 100003 + k)[0] for k, (m, n) in enumerate(batch_sizes(count, seed=seed, **kw))]
