"""MPS reader (pdlpx_read_mps) and the command-line front end (pdlpx_cli).

The reader gives every MPS section the meaning mipx's reader gives it
(src/io/mps_reader.cpp:432-813); the fixtures below spell out each rule.  The
CLI prints mipx's `--pdlp` summary lines (src/cli/main.cpp:553-607), which the
reference's benchmark scripts parse."""
import gzip
import math
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from mipx_b200 import build as B, generators as G
from mipx_b200._capi import PdlpxError
from mipx_b200.pdlp import read_mps

INF = math.inf
from oracle.oracle import reference_dir

_REF_DIR = reference_dir()
REF_TINY = (_REF_DIR / "tests" / "data" / "tiny.mps") if _REF_DIR is not None else Path("tiny.mps.absent")

RULES = """NAME          rules
* comment line
ROWS
 N  cost
 L  lim
 G  need
 E  bal
 E  band
 L  cap
COLUMNS
    a         cost   2.0   lim   1.0
    a         need   1.0   lim   0.5   $ trailing comment, duplicate summed
    MARKER    'MARKER'   'INTORG'
    b         cost  -1.0   bal   1.0
    b         cap    0.0
    MARKER    'MARKER'   'INTEND'
    c         band   3.0   need  2.0
    d         cost   1.5   cap   1.0
RHS
    rhs       cost  -7.5   lim   4.0
    rhs       need   1.0   bal   2.0
    rhs       band   6.0   cap   9.0
RANGES
    rng       lim   -1.5   need  2.0
    rng       bal    3.0   band -4.0
BOUNDS
 UP bnd       a      3.0
 MI bnd       b
 UP bnd       b      5.0
 FX bnd       c      1.25
 FR bnd       d
 LI bnd       e      2.0
 UI bnd       e      7.0
ENDATA
"""


def _check_rules(lp):
    assert (lp.num_rows, lp.num_cols) == (5, 5)  # e exists only in BOUNDS
    np.testing.assert_array_equal(lp.obj, [2.0, -1.0, 0.0, 1.5, 0.0])
    assert lp.obj_offset == 7.5
    np.testing.assert_array_equal(lp.col_lower, [0.0, -INF, 1.25, -INF, 2.0])
    np.testing.assert_array_equal(lp.col_upper, [3.0, 5.0, 1.25, INF, 7.0])
    assert lp.col_type == ["C", "I", "C", "C", "I"]
    # L with range -1.5 -> [4 - 1.5, 4]; G with 2 -> [1, 3]; E with 3 -> [2, 5];
    # E with -4 -> [2, 6]; L without range -> [-inf, 9]
    np.testing.assert_array_equal(lp.row_lower, [2.5, 1.0, 2.0, 2.0, -INF])
    np.testing.assert_array_equal(lp.row_upper, [4.0, 3.0, 5.0, 6.0, 9.0])
    m = lp.matrix
    np.testing.assert_array_equal(m.row_starts, [0, 1, 3, 4, 5, 6])
    np.testing.assert_array_equal(m.col_indices, [0, 0, 2, 1, 2, 3])  # b's zero on cap dropped
    np.testing.assert_array_equal(m.values, [1.5, 1.0, 2.0, 1.0, 3.0, 1.0])


def test_mps_rules(tmp_path):
    p = tmp_path / "rules.mps"
    p.write_text(RULES)
    _check_rules(read_mps(p))


def test_mps_gzip(tmp_path):
    p = tmp_path / "rules.mps.gz"
    p.write_bytes(gzip.compress(RULES.encode()))
    _check_rules(read_mps(p))


def test_mps_errors(tmp_path):
    with pytest.raises(PdlpxError):
        read_mps(tmp_path / "missing.mps")
    bad = tmp_path / "bad.mps"
    bad.write_text("ROWS\n N  c\nCOLUMNS\n    x  nosuchrow  1.0\nENDATA\n")
    with pytest.raises(PdlpxError, match="unknown row"):
        read_mps(bad)


def _write_mps(lp, path):
    """Column-wise MPS of an LP (test helper; repr of a float round-trips it)."""
    f = lambda x: repr(float(x))
    m = lp.matrix
    rs, ci, v = np.asarray(m.row_starts), np.asarray(m.col_indices), np.asarray(m.values)
    cols = [[] for _ in range(lp.num_cols)]
    for i in range(lp.num_rows):
        for k in range(rs[i], rs[i + 1]):
            cols[ci[k]].append((i, v[k]))
    out = ["NAME t", "ROWS", " N obj"]
    for i in range(lp.num_rows):
        lo, up = lp.row_lower[i], lp.row_upper[i]
        out.append(f" {'E' if lo == up else ('L' if lo == -INF else ('G' if up == INF else 'L'))} r{i}")
    out.append("COLUMNS")
    for j in range(lp.num_cols):
        out.append(f"    x{j} obj {f(lp.obj[j])}")
        for i, a in cols[j]:
            out.append(f"    x{j} r{i} {f(a)}")
    out.append("RHS")
    for i in range(lp.num_rows):
        lo, up = lp.row_lower[i], lp.row_upper[i]
        out.append(f"    rhs r{i} {f(up if up != INF else lo)}")
    out.append("RANGES")
    for i in range(lp.num_rows):
        lo, up = lp.row_lower[i], lp.row_upper[i]
        if lo != up and lo != -INF and up != INF:
            out.append(f"    rng r{i} {f(up - lo)}")
    out.append("BOUNDS")
    for j in range(lp.num_cols):
        if lp.col_lower[j] != 0.0:
            out.append(f" LO bnd x{j} {f(lp.col_lower[j])}")
        if lp.col_upper[j] != INF:
            out.append(f" UP bnd x{j} {f(lp.col_upper[j])}")
    out.append("ENDATA")
    path.write_text("\n".join(out) + "\n")


def test_mps_round_trip_of_generated_lp(tmp_path):
    lp, _ = G.random_lp(60, 150, 4, 12, 3)
    p = tmp_path / "r.mps"
    _write_mps(lp, p)
    got = read_mps(p)
    for f in ("obj", "col_lower", "col_upper", "row_lower", "row_upper"):
        np.testing.assert_array_equal(getattr(got, f), getattr(lp, f))
    for f in ("row_starts", "col_indices", "values"):
        np.testing.assert_array_equal(getattr(got.matrix, f), getattr(lp.matrix, f))


@pytest.mark.skipif(not REF_TINY.exists(), reason="the reference's test data is not present")
def test_reference_tiny_mps():
    """The reference's own fixture with the values its test asserts (test_lp_problem.cpp:50-103)."""
    lp = read_mps(REF_TINY)
    assert (lp.num_rows, lp.num_cols) == (3, 3)
    np.testing.assert_array_equal(lp.obj, [1.0, 3.0, 2.0])
    np.testing.assert_array_equal(lp.col_lower, [0.0, 0.0, 1.0])
    np.testing.assert_array_equal(lp.col_upper, [8.0, 1.0, 5.0])
    assert lp.col_type[0] == "C" and lp.col_type[1] == "I" and lp.col_type[2] == "C"
    np.testing.assert_array_equal(lp.row_lower, [-INF, 5.0, 7.0])
    np.testing.assert_array_equal(lp.row_upper, [10.0, INF, 7.0])
    dense = np.zeros((3, 3))
    m = lp.matrix
    for i in range(3):
        for k in range(m.row_starts[i], m.row_starts[i + 1]):
            dense[i, m.col_indices[k]] = m.values[k]
    np.testing.assert_array_equal(dense, [[2.0, 1.0, 0.0], [1.0, 0.0, 1.0], [0.0, 1.0, 1.0]])


def _cli(*args):
    B.build()
    return subprocess.run([str(B.CLI), *map(str, args)], capture_output=True, text=True, timeout=600)


def _summary(out):
    get = lambda k: re.search(rf"^{k}:\s*(\S.*)$", out, re.MULTILINE).group(1).strip()
    return {"status": get("Status"), "objective": float(get("Objective")), "iterations": int(get("Iterations")),
            "work": float(get("Work units")), "time": float(get("Time").rstrip("s"))}


def test_cli_summary_lines_without_rows(tmp_path):
    """An LP with no rows is solved in closed form on the host: the CLI prints
    mipx's summary lines (min 2a - b, a in [1, 3], b in [-inf, 4] -> 2 - 4 = -2)."""
    p = tmp_path / "bounds.mps"
    p.write_text("NAME b\nROWS\n N obj\nCOLUMNS\n    a obj 2.0\n    b obj -1.0\nBOUNDS\n LO bnd a 1.0\n"
                 " UP bnd a 3.0\n MI bnd b\n UP bnd b 4.0\nENDATA\n")
    r = _cli(p, "--pdlp", "--quiet", "--print-backend", "--threads", "4", "--no-presolve")
    assert r.returncode == 0, r.stderr
    s = _summary(r.stdout)
    assert s["status"] == "Optimal" and s["objective"] == -2.0 and s["iterations"] == 0
    assert "Optimal: -2.0000000000e+00 (0 iterations)" in r.stdout
    assert _cli(tmp_path / "missing.mps").returncode == 1
    assert _cli().returncode == 1


@pytest.mark.gpu
def test_cli_solves_mps_on_device(tmp_path):
    """CLI solve of a generated LP written as MPS against the Python API on the
    same LP: same status, objectives within 1e-6 relative at 1e-6 KKT."""
    from mipx_b200.pdlp import PdlpOptions, PdlpSolver
    lp, _ = G.random_lp(500, 1250, 4, 12, 5)
    p = tmp_path / "r.mps.gz"
    plain = tmp_path / "r.mps"
    _write_mps(lp, plain)
    p.write_bytes(gzip.compress(plain.read_bytes()))
    r = _cli(p, "--pdlp", "--print-backend", "--tol", "1e-6", "--time-limit", "300")
    assert r.returncode == 0, r.stderr
    assert "PDLP backend: GPU" in r.stdout
    s = _summary(r.stdout)
    q = PdlpSolver()
    q.setOptions(PdlpOptions(verbose=False, primal_tol=1e-6, dual_tol=1e-6, optimality_tol=1e-6))
    q.load(read_mps(p))
    res = q.solve()
    assert s["status"] == "Optimal" and int(res.status) == 0
    assert abs(s["objective"] - res.objective) <= 1e-6 * max(1.0, abs(res.objective))
    assert s["iterations"] > 0 and s["work"] > 0


def test_mps_edge_rules(tmp_path):
    """RANGES and RHS on the objective row, unknown rows in RHS / RANGES and a
    bound on a column that only BOUNDS names: as mipx's reader treats them
    (objective RHS sets the constant, objective ranges and unknown rows are
    skipped, the new column gets cost 0 and the default lower bound)."""
    p = tmp_path / "edge.mps"
    p.write_text("NAME e\nROWS\n N obj\n E r\nCOLUMNS\n    x obj 1.0 r 1.0\nRHS\n    rhs obj 3.0 nosuch 9.0\n"
                 "    rhs r 2.0\nRANGES\n    rng obj 5.0 nosuch 1.0\nBOUNDS\n UP bnd y 4.0\nENDATA\n")
    lp = read_mps(p)
    assert lp.obj_offset == -3.0
    assert (lp.num_rows, lp.num_cols) == (1, 2)
    np.testing.assert_array_equal(lp.obj, [1.0, 0.0])
    np.testing.assert_array_equal(lp.col_lower, [0.0, 0.0])
    np.testing.assert_array_equal(lp.col_upper, [INF, 4.0])
    np.testing.assert_array_equal(lp.row_lower, [2.0])
    np.testing.assert_array_equal(lp.row_upper, [2.0])


@pytest.mark.gpu
def test_solve_mps_entry_point(tmp_path):
    """mipx_b200.solve_mps: read + PDLP solve in one call, as mipx's Python
    solve_mps does for its models; same result as reading and solving through
    PdlpSolver, and time_limit / verbose reach the options."""
    from mipx_b200 import solve_mps
    from mipx_b200.pdlp import PdlpOptions, PdlpSolver
    lp, _ = G.random_lp(300, 750, 4, 12, 8)
    p = tmp_path / "r.mps"
    _write_mps(lp, p)
    tight = PdlpOptions(primal_tol=1e-6, dual_tol=1e-6, optimality_tol=1e-6)
    r, x, y = solve_mps(p, time_limit=300.0, options=tight)
    q = PdlpSolver()
    q.setOptions(PdlpOptions(verbose=False, primal_tol=1e-6, dual_tol=1e-6, optimality_tol=1e-6,
                             max_solve_seconds=300.0))
    q.load(read_mps(p))
    res = q.solve()
    assert int(r.status) == int(res.status) == 0
    assert r.objective == res.objective and r.iterations == res.iterations
    np.testing.assert_array_equal(x, q.getPrimalValues())
    np.testing.assert_array_equal(y, q.getDualValues())
    assert x.size == 750 and y.size == 300
    r0, _, _ = solve_mps(p, time_limit=0.0, options=tight)
    assert int(r0.status) == 4  # TimeLimit: the limit reached the solver
