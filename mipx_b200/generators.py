"""Seeded synthetic LPs of the benchmark workloads (C generators in libpdlpx).

Every generator takes ``lib``: the loaded library whose ``pdlpx_gen_*`` entry
points build the LP (default: the engine's libpdlpx.so).  Any library built
from the same generator source gives the same arrays, which is how a caller
that must not load the engine (a CPU baseline) builds the identical workload.

* ``random_lp``      -- random sparse LP: columns with U{lo..hi} nonzeros at
  uniform rows, N(0,1) values, x0~U[0,10], rows alternating '=' / '<=' with
  b = A x0 (+U[0,1] slack), 0 <= x <= 10, c~N(0,1).  2,000 x 5,000 with 4-12
  nonzeros per column is the single-LP CPU-sized case.
* ``transport_lp``   -- s x d transportation problem (1,000 x 1,000: 1M
  variables, 2,000 rows, 2M unit nonzeros).
* ``powerlaw_lp``    -- large LP with power-law column counts (500,000 x
  2,000,000, counts in [2, 2000] with mean 10, 1% of rows scaled by 1e3).
* ``node_lp``        -- branch-and-bound node LP of a base LP: integer-marked
  columns fixed to floor/ceil of x0 and random cuts appended (serving workload).
* ``batch_sizes``    -- row counts of the 512-LP batch, lognormal(median 1,500,
  sigma 0.8) clipped to [200, 20,000], n = 2.5 m.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from .pdlp import LpProblem, Sense, SparseMatrix


def _take(g: _capi.GenLp, lib) -> tuple[LpProblem, np.ndarray]:
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
    lib.pdlpx_free_lp(C.byref(g))
    return lp, x0


def _check(lib, code: int) -> None:
    if code != 0:
        raise _capi.PdlpxError(code, "generator rejected its arguments")


def random_lp(m: int = 2000, n: int = 5000, nnz_lo: int = 4, nnz_hi: int = 12, seed: int = 1, lib=None):
    lib = lib or _capi.load()
    g = _capi.GenLp()
    _check(lib, lib.pdlpx_gen_random(m, n, nnz_lo, nnz_hi, seed, C.byref(g)))
    lp, x0 = _take(g, lib)
    lp.name = f"random_{m}x{n}_s{seed}"
    return lp, x0


def transport_lp(supplies: int = 1000, demands: int = 1000, seed: int = 7, lib=None):
    lib = lib or _capi.load()
    g = _capi.GenLp()
    _check(lib, lib.pdlpx_gen_transport(supplies, demands, seed, C.byref(g)))
    lp, x0 = _take(g, lib)
    lp.name = f"transport_{supplies}x{demands}_s{seed}"
    return lp, x0


def powerlaw_lp(m: int = 500_000, n: int = 2_000_000, kmin: int = 2, kmax: int = 2000, kmean: float = 10.0,
                big_frac: float = 0.01, big_scale: float = 1e3, seed: int = 11, lib=None):
    lib = lib or _capi.load()
    g = _capi.GenLp()
    _check(lib, lib.pdlpx_gen_powerlaw(m, n, kmin, kmax, kmean, big_frac, big_scale, seed, C.byref(g)))
    lp, x0 = _take(g, lib)
    lp.name = f"powerlaw_{m}x{n}_s{seed}"
    return lp, x0


def batch_sizes(count: int = 512, median: float = 1500.0, sigma: float = 0.8, lo: int = 200, hi: int = 20000,
                seed: int = 5) -> list[tuple[int, int]]:
    rng = np.random.default_rng(seed)
    ms = np.clip(np.round(np.exp(np.log(median) + sigma * rng.standard_normal(count))), lo, hi).astype(int)
    return [(int(m), int(round(2.5 * m))) for m in ms]


def batch_lps(count: int = 512, seed: int = 5, lib=None, **kw) -> list[LpProblem]:
    return [random_lp(m, n, 4, 12, seed * 100003 + k, lib=lib)[0]
            for k, (m, n) in enumerate(batch_sizes(count, seed=seed, **kw))]


def integer_marks(n: int, frac: float = 0.3, seed: int = 3) -> np.ndarray:
    """Integrality marks of the serving workload's base LP: a seeded 30% of the columns."""
    return np.random.default_rng(seed).random(n) < frac


def node_lp(base: LpProblem, x0: np.ndarray, is_int: np.ndarray, seed: int, fix_lo: float = 0.01,
            fix_hi: float = 0.05, cuts_max: int = 50, cut_nnz: tuple[int, int] = (20, 200)) -> LpProblem:
    """A branch-and-bound node LP of `base`: a random 1-5% of the integer-marked
    columns fixed to floor or ceil of x0, then 0-50 random cuts a x <= a x0 +
    U[0,1] with 20-200 N(0,1) entries each, appended after the base rows (so a
    parent's duals warm-start the first rows)."""
    rng = np.random.default_rng(seed)
    ints = np.flatnonzero(is_int)
    lo, hi = max(1, int(round(fix_lo * ints.size))), max(1, int(round(fix_hi * ints.size)))
    fix = rng.choice(ints, size=int(rng.integers(lo, hi + 1)), replace=False)
    val = np.where(rng.random(fix.size) < 0.5, np.floor(x0[fix]), np.ceil(x0[fix]))
    cl, cu = base.col_lower.copy(), base.col_upper.copy()
    cl[fix] = np.clip(val, cl[fix], cu[fix])
    cu[fix] = cl[fix]
    a = base.matrix
    rows, starts, idx, vals, rl, ru = [], [a.row_starts], [a.col_indices], [a.values], [base.row_lower], [base.row_upper]
    ncut = int(rng.integers(0, cuts_max + 1))
    nnz = int(a.values.size)
    cut_ptr = []
    for _ in range(ncut):
        k = int(rng.integers(cut_nnz[0], cut_nnz[1] + 1))
        cols = np.sort(rng.choice(base.num_cols, size=k, replace=False)).astype(np.int32)
        v = rng.standard_normal(k)
        idx.append(cols)
        vals.append(v)
        nnz += k
        cut_ptr.append(nnz)
        rl.append(np.array([-np.inf]))
        ru.append(np.array([float(v @ x0[cols]) + float(rng.random())]))
    rp = np.concatenate([a.row_starts, np.array(cut_ptr, dtype=np.int32)]).astype(np.int32)
    m = base.num_rows + ncut
    mat = SparseMatrix(m, base.num_cols, values=np.concatenate(vals), col_indices=np.concatenate(idx).astype(np.int32),
                       row_starts=rp)
    return LpProblem(name=f"{base.name}_node{seed}", sense=base.sense, num_cols=base.num_cols, num_rows=m,
                     obj=base.obj.copy(), col_lower=cl, col_upper=cu, row_lower=np.concatenate(rl),
                     row_upper=np.concatenate(ru), matrix=mat, obj_offset=base.obj_offset)
