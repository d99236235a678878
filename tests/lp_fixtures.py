"""The LPs of mipx's own PDLP tests (tests/test_pdlp.cpp), rebuilt in Python.

Each builder names the reference test builder it follows.  ``medium_lp``
reproduces ``buildMediumLp`` exactly: std::mt19937(123) is numpy's MT19937
with legacy (init_genrand) seeding, and libstdc++'s
uniform_real_distribution<double>(0, 1) draws (r1 + r2 * 2^32) / 2^64 from two
32-bit outputs.
"""
from __future__ import annotations

import numpy as np

from mipx_b200.pdlp import LpProblem, Sense, SparseMatrix, kInf


def _lp(obj, cl, cu, rl, ru, trips, m, n, sense=Sense.Minimize, offset=0.0, name=""):
    return LpProblem(name=name, sense=sense, num_cols=n, obj=np.array(obj, float), col_lower=np.array(cl, float),
                     col_upper=np.array(cu, float), num_rows=m, row_lower=np.array(rl, float),
                     row_upper=np.array(ru, float), matrix=SparseMatrix(m, n, trips), obj_offset=offset)


def simple_lp():
    """buildSimpleLp (test_pdlp.cpp:19-41): min -x-y s.t. x+y<=4, x,y>=0 -> -4."""
    return _lp([-1, -1], [0, 0], [kInf, kInf], [-kInf], [4.0], [(0, 0, 1.0), (0, 1, 1.0)], 1, 2, name="pdlp_simple")


def bounds_only_lp():
    """buildBoundsOnlyLp (test_pdlp.cpp:43-56): min x, 1<=x<=3 -> 1."""
    return _lp([1.0], [1.0], [3.0], [], [], [], 0, 1, name="pdlp_bounds")


def empty_lp():
    """Empty problem with offset 42 (test_pdlp.cpp:303-322)."""
    return _lp([], [], [], [], [], [], 0, 0, offset=42.0, name="pdlp_empty")


def unbounded_bounds_only_lp():
    """min -x, x>=0, no rows -> Unbounded (test_pdlp.cpp:324-345)."""
    return _lp([-1.0], [0.0], [kInf], [], [], [], 0, 1, name="pdlp_unbounded")


def infeasible_lp():
    """min x s.t. x<=-1, x>=1 -> Infeasible (test_pdlp.cpp:347-376, Farkas 445-496)."""
    return _lp([1.0], [1.0], [kInf], [-kInf], [-1.0], [(0, 0, 1.0)], 1, 1, name="pdlp_infeasible")


def infeasible_eq_lp():
    """x+y=5 and x+y=3 -> Infeasible (test_pdlp.cpp:378-412)."""
    return _lp([1, 1], [0, 0], [kInf, kInf], [5.0, 3.0], [5.0, 3.0],
               [(0, 0, 1.0), (0, 1, 1.0), (1, 0, 1.0), (1, 1, 1.0)], 2, 2, name="pdlp_infeasible_eq")


def unbounded_constrained_lp():
    """min -x s.t. x-y<=0 -> Unbounded (test_pdlp.cpp:414-443)."""
    return _lp([-1, 0], [0, 0], [kInf, kInf], [-kInf], [0.0], [(0, 0, 1.0), (0, 1, -1.0)], 1, 2,
               name="pdlp_unbounded_constrained")


def col_bound_binding_lp():
    """min -x-2y s.t. x+y<=100, 0<=x<=3, 0<=y<=5 -> -13 (test_pdlp.cpp:639-663)."""
    return _lp([-1, -2], [0, 0], [3, 5], [-kInf], [100.0], [(0, 0, 1.0), (0, 1, 1.0)], 1, 2)


def large_rhs_lp():
    """min -x-y s.t. x<=1000, y<=2 -> -1002 (test_pdlp.cpp:665-690)."""
    return _lp([-1, -1], [0, 0], [kInf, kInf], [-kInf, -kInf], [1000.0, 2.0], [(0, 0, 1.0), (1, 1, 1.0)], 2, 2)


def equality_lp():
    """min x+2y s.t. x+y=10 -> 10 (test_pdlp.cpp:692-716)."""
    return _lp([1, 2], [0, 0], [kInf, kInf], [10.0], [10.0], [(0, 0, 1.0), (0, 1, 1.0)], 1, 2)


def filter_lp():
    """x+y+1e-15 z<=4 (test_pdlp.cpp:897-940)."""
    return _lp([-1, -1, 0], [0, 0, 0], [kInf] * 3, [-kInf], [4.0], [(0, 0, 1.0), (0, 1, 1.0), (0, 2, 1e-15)], 1, 3)


def maximize_lp():
    """max x+y s.t. x+y<=4 (sense handling, objective 4)."""
    return _lp([1, 1], [0, 0], [kInf, kInf], [-kInf], [4.0], [(0, 0, 1.0), (0, 1, 1.0)], 1, 2, sense=Sense.Maximize)


def ranged_lp():
    """min -x+y s.t. 1 <= x+y <= 3 (ranged row), x-y >= -1, 0<=x,y<=5."""
    return _lp([-1, 1], [0, 0], [5, 5], [1.0, -1.0], [3.0, kInf], [(0, 0, 1.0), (0, 1, 1.0), (1, 0, 1.0),
                                                                  (1, 1, -1.0)], 2, 2)


class _StdMt:
    """std::mt19937 + libstdc++ uniform_real_distribution<double>(0,1)."""

    def __init__(self, seed: int):
        self.bg = np.random.MT19937(0)
        self.bg._legacy_seeding(seed)

    def uniform(self) -> float:
        r = self.bg.random_raw(2)
        v = (float(r[0]) + float(r[1]) * 4294967296.0) / 18446744073709551616.0
        return v if v < 1.0 else np.nextafter(1.0, 0.0)


def medium_lp():
    """buildMediumLp (test_pdlp.cpp:260-299): 50 x 80, ~60% dense, mt19937(123)."""
    rows, cols = 50, 80
    obj = [(1.0 + 0.1 * j) if j % 2 == 0 else -(0.5 + 0.05 * j) for j in range(cols)]
    rng = _StdMt(123)
    trips = []
    for i in range(rows):
        for j in range(cols):
            if rng.uniform() < 0.6:
                trips.append((i, j, 0.1 + rng.uniform() * 2.0))
    return _lp(obj, [0.0] * cols, [100.0] * cols, [-kInf] * rows, [50.0 + 2.0 * i for i in range(rows)], trips,
               rows, cols, name="gpu_vs_cpu_medium")


KNOWN_ANSWERS = {
    # name: (builder, expected objective, abs tolerance, reference test lines)
    "simple": (simple_lp, -4.0, 1e-4, "test_pdlp.cpp:88-107"),
    "bounds_only": (bounds_only_lp, 1.0, 1e-6, "test_pdlp.cpp:109-124"),
    "empty": (empty_lp, 42.0, 1e-9, "test_pdlp.cpp:303-322"),
    "col_bound_binding": (col_bound_binding_lp, -13.0, 1e-3, "test_pdlp.cpp:639-663"),
    "large_rhs": (large_rhs_lp, -1002.0, 1.0, "test_pdlp.cpp:665-690"),
    "equality": (equality_lp, 10.0, 0.1, "test_pdlp.cpp:692-716"),
}
