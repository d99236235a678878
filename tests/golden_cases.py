"""Access to the committed golden fixtures (tests/golden/ref_pdlp*.{json,npz})
produced by tests/golden/make_golden.py from the reference compiled from source."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

import lp_fixtures as F
from mipx_b200 import generators as G
from mipx_b200.pdlp import PdlpOptimalityNorm, PdlpOptions, Precision

GOLDEN = Path(__file__).resolve().parent / "golden"
INDEX = json.loads((GOLDEN / "ref_pdlp.json").read_text())
_VEC = None

BUILDERS = {
    "simple": F.simple_lp, "simple_linf": F.simple_lp, "simple_norescale": F.simple_lp,
    "simple_nopolish": F.simple_lp, "simple_precond": F.simple_lp, "simple_adaptive": F.simple_lp,
    "bounds_only": F.bounds_only_lp, "empty": F.empty_lp, "unbounded_bounds_only": F.unbounded_bounds_only_lp,
    "infeasible": F.infeasible_lp, "infeasible_eq": F.infeasible_eq_lp,
    "unbounded_constrained": F.unbounded_constrained_lp, "col_bound_binding": F.col_bound_binding_lp,
    "large_rhs": F.large_rhs_lp, "equality": F.equality_lp, "equality_polish": F.equality_lp,
    "filter": F.filter_lp, "maximize": F.maximize_lp, "ranged": F.ranged_lp, "medium": F.medium_lp,
    "medium_tight": F.medium_lp, "medium_norescale": F.medium_lp, "medium_polish7": F.medium_lp,
    "simple_anderson": F.simple_lp, "simple_anderson_w2": F.simple_lp, "equality_anderson": F.equality_lp,
    "medium_anderson": F.medium_lp,
}


def vectors(name: str):
    global _VEC
    if _VEC is None:
        _VEC = np.load(GOLDEN / "ref_pdlp_vectors.npz")
    return _VEC[f"{name}__x"], _VEC[f"{name}__y"]


def problem(name: str):
    e = INDEX[name]
    if "generator" in e:
        g = e["generator"]
        return G.random_lp(g["m"], g["n"], g["nnz_lo"], g["nnz_hi"], g["seed"])[0]
    return BUILDERS[name]()


def options(name: str, **over) -> PdlpOptions:
    o = PdlpOptions()
    for k, v in INDEX[name]["options"].items():
        if hasattr(o, k) and k not in ("precision",):
            cur = getattr(o, k)
            if isinstance(cur, PdlpOptimalityNorm):
                v = PdlpOptimalityNorm(v)
            elif isinstance(cur, bool):
                v = bool(v)
            setattr(o, k, v)
    o.verbose = False
    for k, v in over.items():
        setattr(o, k, v)
    return o


NAMES = sorted(k for k in INDEX if "objective" in INDEX[k])
HIGHS_ONLY = sorted(k for k in INDEX if "objective" not in INDEX[k])

# Objective parity bound of the north-star workloads: results within 1e-6
# relative of an FP64 oracle, relative to max(1, |oracle|) so objectives near
# zero are held to 1e-6 absolute.
OBJ_TOL = 1e-6


def rel_err(value: float, oracle: float) -> float:
    return abs(value - oracle) / max(1.0, abs(oracle))


def config_pins() -> dict:
    """FP64 objective pins of the benchmark configurations (tests/golden/make_config_pins.py)."""
    return json.loads((GOLDEN / "config_pins.json").read_text())
