"""ORACLE -- TEST INFRASTRUCTURE ONLY.

ctypes access to the CPU checkers of the PDLP path:
  * ``liboracle_pdlp.so``        -- FP64 restatement of mipx's CPU PDLP (pdlp_oracle.cpp);
  * ``_ref/libmipx_pdlp_ref.so`` -- the reference's own PdlpSolver compiled from its
    sources (present only where the reference tree was available at build time).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs use this
module; the engine (mipx_b200/) never imports it.  The oracle library also
carries the workload generators, so the CPU-baseline legs build their inputs
without loading the engine library.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "liboracle_pdlp.so"
REF_LIB = HERE / "_ref" / "libmipx_pdlp_ref.so"
REF_GPU_LIB = HERE / "_ref" / "libmipx_pdlp_ref_gpu.so"
# the reference's PdlpSolver with the pdlpx binding as its solveGpu body (make ref_bound)
REF_BOUND_LIB = HERE / "_ref" / "libmipx_pdlp_bound.so"

_libs: dict = {}


def reference_dir() -> Path | None:
    """The mipx source tree the reference libraries are compiled from:
    $MIPX_REFERENCE_DIR, else the checkout the oracle's Makefile recipe reads
    (/root/reference); None where neither exists (a machine that only runs the
    libraries built beforehand)."""
    for cand in (os.environ.get("MIPX_REFERENCE_DIR"), "/root/reference"):
        if cand and (Path(cand) / "src" / "lp" / "pdlp.cpp").exists():
            return Path(cand)
    return None


def build(ref: bool = True) -> None:
    """Compile the oracle (and, when the reference tree exists, the reference's
    CPU and FP64 GPU PDLP behind the shim)."""
    targets = ["liboracle_pdlp.so"]
    rd = reference_dir()
    if ref and rd is not None:
        targets += ["ref", "ref_gpu", "ref_bound", f"REF={rd}"]
    subprocess.run(["make", "-s", "-C", str(HERE), *targets], check=True)


def _load(path: Path):
    if path not in _libs:
        if not path.exists():
            if path == ORACLE_LIB:
                build(ref=False)
            else:
                raise FileNotFoundError(f"{path} not built (reference sources needed at build time)")
        from mipx_b200 import _capi  # struct layouts only
        lib = C.CDLL(str(path))
        sig = [C.POINTER(_capi.Lp), C.POINTER(_capi.Options), C.POINTER(_capi.Result), _capi.P_f64, _capi.P_f64]
        for name in ("oracle_pdlp_solve", "ref_pdlp_solve"):
            if hasattr(lib, name):
                getattr(lib, name).argtypes = sig
                getattr(lib, name).restype = C.c_int
        if hasattr(lib, "ref_pdlp_solve_rc"):
            lib.ref_pdlp_solve_rc.argtypes = sig[:3] + [_capi.P_f64]
        for name, res, args in _capi.SIGNATURES:  # the workload generators built into the oracle library
            if name.startswith("pdlpx_gen_") or name == "pdlpx_free_lp":
                if hasattr(lib, name):
                    getattr(lib, name).restype = res
                    getattr(lib, name).argtypes = args
        if hasattr(lib, "ref_pdlp_open"):
            lib.ref_pdlp_open.argtypes = sig[:2]
            lib.ref_pdlp_open.restype = C.c_void_p
            lib.ref_pdlp_run.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(_capi.Result)]
            lib.ref_pdlp_run.restype = C.c_int
            lib.ref_pdlp_close.argtypes = [C.c_void_p]
            lib.ref_pdlp_close.restype = None
        if hasattr(lib, "ref_pdlp_race"):
            lib.ref_pdlp_race.argtypes = [C.POINTER(_capi.Lp), C.POINTER(_capi.Options), C.POINTER(_capi.Options),
                                          C.POINTER(_capi.Result), C.POINTER(_capi.Result), C.POINTER(C.c_int)]
            lib.ref_pdlp_race.restype = C.c_int
        if hasattr(lib, "oracle_scaling"):
            lib.oracle_scaling.argtypes = [C.POINTER(_capi.Lp), C.POINTER(_capi.Options)] + [_capi.P_f64] * 11
            lib.oracle_spectral_norm.argtypes = [C.POINTER(_capi.Lp), C.POINTER(_capi.Options)]
            lib.oracle_spectral_norm.restype = C.c_double
            for name in ("oracle_csr_multiply", "oracle_csr_multiply_transpose"):
                getattr(lib, name).argtypes = [C.c_int, C.c_int, _capi.P_i32, _capi.P_i32, _capi.P_f64, _capi.P_f64,
                                               _capi.P_f64]
        _libs[path] = lib
    return _libs[path]


def ref_available() -> bool:
    return REF_LIB.exists()


def gen_lib():
    """The oracle library as a generator source for mipx_b200.generators
    (``lib=``): the same generator code as the engine's, without loading the
    engine library."""
    return _load(ORACLE_LIB)


def _solve(fn, problem, options, warm=None):
    from mipx_b200.pdlp import LpResult
    keep: list = []
    wx, wy = warm if warm is not None else (None, None)
    lp = problem.to_c(keep, wx, wy)
    res = __import__("mipx_b200._capi", fromlist=["Result"]).Result()
    x = np.zeros(problem.num_cols)
    y = np.zeros(problem.num_rows)
    o = options.to_c()
    rc = fn(C.byref(lp), C.byref(o), C.byref(res), x.ctypes.data_as(C.POINTER(C.c_double)),
            y.ctypes.data_as(C.POINTER(C.c_double)))
    if rc != 0:
        raise RuntimeError(f"oracle call failed ({rc})")
    return LpResult.from_c(res), x, y


def oracle_solve(problem, options, warm=None):
    """FP64 CPU restatement of the reference PDLP: (LpResult, x, y)."""
    return _solve(_load(ORACLE_LIB).oracle_pdlp_solve, problem, options, warm)


def _ref_lib(gpu: bool = False, bound: bool = False):
    return _load(REF_BOUND_LIB if bound else (REF_GPU_LIB if gpu else REF_LIB))


def ref_solve(problem, options, warm=None, gpu: bool = False, bound: bool = False):
    """The reference's own PdlpSolver (compiled from source): (LpResult, x, y).
    gpu: its cuSPARSE FP64 GPU path; bound: its class with the pdlpx binding as
    the solveGpu body (the drop-in build)."""
    return _solve(_ref_lib(gpu, bound).ref_pdlp_solve, problem, options, warm)


def ref_race(problem, arm0, arm1, bound: bool = False):
    """mipx's concurrent-root race pattern over the reference's PdlpSolver: two
    arms with a shared std::atomic<bool> stop flag.  Returns (r0, r1, winner)."""
    from mipx_b200.pdlp import LpResult
    from mipx_b200 import _capi
    keep: list = []
    lp = problem.to_c(keep)
    r0, r1, w = _capi.Result(), _capi.Result(), C.c_int(-1)
    rc = _ref_lib(bound=bound).ref_pdlp_race(C.byref(lp), C.byref(arm0.to_c()), C.byref(arm1.to_c()), C.byref(r0),
                                             C.byref(r1), C.byref(w))
    if rc != 0:
        raise RuntimeError(f"race failed ({rc})")
    return LpResult.from_c(r0), LpResult.from_c(r1), w.value


class RefSession:
    """The reference's PdlpSolver loaded once (its scaling pipeline runs in
    load), then solved repeatedly with new caps: ``run(max_iter, sv_max_iter)``
    returns (LpResult, wall seconds of the reference's solve()).  Used to time
    the reference's iteration rate without paying its load for every sample."""

    def __init__(self, problem, options, gpu: bool = False):
        self._lib = _ref_lib(gpu)
        keep: list = []
        lp = problem.to_c(keep)
        self._h = self._lib.ref_pdlp_open(C.byref(lp), C.byref(options.to_c()))
        if not self._h:
            raise RuntimeError("reference solver could not be created")

    def run(self, max_iter: int, sv_max_iter: int):
        from mipx_b200.pdlp import LpResult
        from mipx_b200 import _capi
        res = _capi.Result()
        if self._lib.ref_pdlp_run(self._h, int(max_iter), int(sv_max_iter), C.byref(res)) != 0:
            raise RuntimeError("reference run failed")
        return LpResult.from_c(res), res.solve_seconds

    def close(self):
        if self._h:
            self._lib.ref_pdlp_close(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def ref_reduced_costs(problem, options):
    from mipx_b200 import _capi
    keep: list = []
    lp = problem.to_c(keep)
    res = _capi.Result()
    rc = np.zeros(problem.num_cols)
    _load(REF_LIB).ref_pdlp_solve_rc(C.byref(lp), C.byref(options.to_c()), C.byref(res),
                                     rc.ctypes.data_as(C.POINTER(C.c_double)))
    return rc


def oracle_scaling(problem, options) -> dict:
    lib = _load(ORACLE_LIB)
    keep: list = []
    lp = problem.to_c(keep)
    m, n = problem.num_rows, problem.num_cols
    out = {k: np.zeros(n) for k in ("col_scale", "cscaled", "col_lower", "tau_base", "col_upper")}
    out.update({k: np.zeros(m) for k in ("row_scale", "row_lower", "row_upper", "sigma_base")})
    osc, csc = C.c_double(), C.c_double()
    p = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    lib.oracle_scaling(C.byref(lp), C.byref(options.to_c()), p(out["col_scale"]), p(out["cscaled"]),
                       p(out["col_lower"]), p(out["row_scale"]), p(out["row_lower"]), p(out["row_upper"]),
                       p(out["tau_base"]), p(out["sigma_base"]), p(out["col_upper"]), C.byref(osc), C.byref(csc))
    out["objective_scale"] = osc.value
    out["constraint_scale"] = csc.value
    return out


def oracle_spectral_norm(problem, options) -> float:
    keep: list = []
    lp = problem.to_c(keep)
    return _load(ORACLE_LIB).oracle_spectral_norm(C.byref(lp), C.byref(options.to_c()))


def oracle_spmv(matrix, x, transpose: bool = False) -> np.ndarray:
    lib = _load(ORACLE_LIB)
    rp = np.ascontiguousarray(matrix.row_starts, dtype=np.int32)
    ci = np.ascontiguousarray(matrix.col_indices, dtype=np.int32)
    v = np.ascontiguousarray(matrix.values, dtype=np.float64)
    xa = np.ascontiguousarray(x, dtype=np.float64)
    y = np.zeros(matrix.cols if transpose else matrix.rows)
    fn = lib.oracle_csr_multiply_transpose if transpose else lib.oracle_csr_multiply
    pi = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
    pd = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    fn(matrix.rows, matrix.cols, pi(rp), pi(ci), pd(v), pd(xa), pd(y))
    return y
