"""Python mirror of mipx's PDLP plugin interface over the engine's C ABI.

Names, argument meaning and error behaviour follow the reference:
``PdlpOptions`` (include/mipx/pdlp.h:19-87), ``PdlpSolver`` (pdlp.h:89-174,
the ``LpSolver`` plugin interface of include/mipx/lp_solver.h:26-60),
``LpResult`` (lp_solver.h:11-16), ``Status`` (core.h:11-19), ``LpProblem``
(lp_problem.h:14-64) with a CSR ``SparseMatrix`` (sparse_matrix.h).  Every
solve runs on the GPU through ``libpdlpx.so``; there is no CPU path here.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import enum
import math
from dataclasses import dataclass, field, fields
from typing import Optional, Sequence

import numpy as np

from . import _capi

kInf = math.inf


class Status(enum.IntEnum):
    Optimal = 0
    Infeasible = 1
    Unbounded = 2
    IterLimit = 3
    TimeLimit = 4
    NodeLimit = 5
    Error = 6


class Sense(enum.IntEnum):
    Minimize = 0
    Maximize = 1


class PdlpOptimalityNorm(enum.IntEnum):
    L2 = 0
    LInf = 1


class Precision(enum.IntEnum):
    Mixed = 0  # FP32 matrix/iterates/SpMV, FP64 checks, restarts and polish
    FP64 = 1   # FP64 throughout


class BasisStatus(enum.IntEnum):
    Basic = 0
    AtLower = 1
    AtUpper = 2
    Fixed = 3
    Free = 4


class StopFlag:
    """Cooperative cancel word (the reference's ``const std::atomic<bool>* stop_flag``)."""

    def __init__(self) -> None:
        self._v = C.c_int32(0)

    def set(self) -> None:
        self._v.value = 1

    def clear(self) -> None:
        self._v.value = 0

    def load(self) -> bool:
        return self._v.value != 0

    @property
    def ptr(self):
        return C.pointer(self._v)


@dataclass
class PdlpOptions:
    max_iter: int = 4000000
    optimality_tol: float = 5e-5
    primal_tol: float = 5e-5
    dual_tol: float = 5e-5
    max_solve_seconds: float = -1.0
    optimality_norm: PdlpOptimalityNorm = PdlpOptimalityNorm.L2
    sv_max_iter: int = 5000
    sv_tol: float = 1e-4
    adaptive_step: bool = False
    adaptive_step_down: float = 0.7
    adaptive_step_up: float = 1.0
    adaptive_step_min: float = 1e-6
    adaptive_step_max: float = 1e3
    primal_weight: float = 1.0
    update_primal_weight: bool = True
    pid_kp: float = 0.99
    pid_ki: float = 0.01
    pid_kd: float = 0.0
    pid_i_smooth: float = 0.3
    restart_sufficient_decay: float = 0.2
    restart_necessary_decay: float = 0.5
    restart_artificial_fraction: float = 0.36
    termination_eval_frequency: int = 200
    matrix_zero_tol: float = 0.0
    enable_polishing: bool = True
    polish_primal_tol: float = 1e-6
    polish_dual_tol: float = 1e-6
    polish_max_iter: int = 500000
    do_ruiz_scaling: bool = True
    ruiz_iterations: int = 10
    do_pock_chambolle_scaling: bool = True
    do_bound_obj_rescaling: bool = True
    preconditioner_refresh: bool = False
    preconditioner_refresh_ratio: float = 10.0
    anderson_acceleration: bool = False
    anderson_window_size: int = 5
    anderson_regularization: float = 1e-10
    use_gpu: bool = True
    gpu_min_rows: int = 512
    gpu_min_nnz: int = 10000
    verbose: bool = True
    stop_flag: Optional[StopFlag] = None
    # engine knobs (no counterpart in the reference)
    precision: Precision = Precision.Mixed
    device: int = 0
    fp64_switch: bool = True
    spmv_group_a: int = 0
    spmv_group_at: int = 0
    autotune: bool = False
    shape_primal: int = 0
    shape_dual: int = 0
    batch_pack_mb: int = 0
    batch_compact: bool = True
    batch_sell: bool = True
    scale_on_device: int = -1
    sell: int = -1
    reference_fixed_columns: bool = False
    hot_cache: int = 0
    long_tiles: int = -1
    batch_persistent: bool = False
    sell_window: int = 0

    def to_c(self) -> _capi.Options:
        # every field of pdlpx_options but `reserved` (zero) is set here, so
        # no library call is needed to build the struct
        o = _capi.Options()
        for f in fields(self):
            if f.name == "stop_flag":
                continue
            v = getattr(self, f.name)
            setattr(o, f.name, int(v) if isinstance(v, (bool, enum.IntEnum)) else v)
        return o


@dataclass
class LpResult:
    status: Status = Status.Error
    objective: float = 0.0
    iterations: int = 0
    work_units: float = 0.0
    # engine diagnostics
    rel_primal_resid: float = 0.0
    rel_dual_resid: float = 0.0
    rel_gap: float = 0.0
    primal_objective: float = 0.0
    dual_objective: float = 0.0
    fp64_iterations: int = 0
    restarts: int = 0
    step_size: float = 0.0
    primal_weight: float = 0.0
    solve_seconds: float = 0.0
    device_seconds: float = 0.0
    used_gpu: bool = False
    kernel_launches: int = 0

    @classmethod
    def from_c(cls, r: _capi.Result) -> "LpResult":
        out = cls()
        for f in fields(cls):
            v = getattr(r, f.name)
            if f.name == "status":
                v = Status(v)
            elif f.name == "used_gpu":
                v = bool(v)
            setattr(out, f.name, v)
        return out


class SparseMatrix:
    """CSR matrix with mipx::SparseMatrix semantics (duplicates summed, zeros dropped)."""

    def __init__(self, rows: int, cols: int, triplets: Sequence[tuple] | None = None, *,
                 values=None, col_indices=None, row_starts=None):
        self.rows = int(rows)
        self.cols = int(cols)
        if values is not None:
            self.values = np.ascontiguousarray(values, dtype=np.float64)
            self.col_indices = np.ascontiguousarray(col_indices, dtype=np.int32)
            self.row_starts = np.ascontiguousarray(row_starts, dtype=np.int32)
            return
        trips = list(triplets or [])
        acc: dict[tuple[int, int], float] = {}
        order: list[tuple[int, int]] = []
        for (r, c, v) in trips:
            key = (int(r), int(c))
            if key not in acc:
                acc[key] = 0.0
                order.append(key)
            acc[key] += float(v)
        keys = sorted(k for k in order if acc[k] != 0.0)
        self.row_starts = np.zeros(self.rows + 1, dtype=np.int32)
        for r, _ in keys:
            self.row_starts[r + 1] += 1
        self.row_starts = np.cumsum(self.row_starts, dtype=np.int64).astype(np.int32)
        self.col_indices = np.array([c for _, c in keys], dtype=np.int32)
        self.values = np.array([acc[k] for k in keys], dtype=np.float64)

    def numRows(self) -> int:
        return self.rows

    def numCols(self) -> int:
        return self.cols

    def numNonzeros(self) -> int:
        return int(self.values.size)

    def csr_values(self):
        return self.values

    def csr_col_indices(self):
        return self.col_indices

    def csr_row_starts(self):
        return self.row_starts

    def multiply(self, x):
        x = np.asarray(x, dtype=np.float64)
        y = np.zeros(self.rows)
        for i in range(self.rows):
            b, e = self.row_starts[i], self.row_starts[i + 1]
            y[i] = float(np.dot(self.values[b:e], x[self.col_indices[b:e]]))
        return y


@dataclass
class LpProblem:
    name: str = ""
    sense: Sense = Sense.Minimize
    num_cols: int = 0
    obj: np.ndarray = field(default_factory=lambda: np.zeros(0))
    col_lower: np.ndarray = field(default_factory=lambda: np.zeros(0))
    col_upper: np.ndarray = field(default_factory=lambda: np.zeros(0))
    num_rows: int = 0
    matrix: SparseMatrix = field(default_factory=lambda: SparseMatrix(0, 0))
    row_lower: np.ndarray = field(default_factory=lambda: np.zeros(0))
    row_upper: np.ndarray = field(default_factory=lambda: np.zeros(0))
    obj_offset: float = 0.0
    col_type: list = field(default_factory=list)

    def arrays(self):
        """Contiguous float64/int32 arrays in the C ABI's layout."""
        f = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.float64))
        return (np.ascontiguousarray(self.matrix.row_starts, dtype=np.int32),
                np.ascontiguousarray(self.matrix.col_indices, dtype=np.int32),
                f(self.matrix.values), f(self.obj), f(self.col_lower), f(self.col_upper),
                f(self.row_lower), f(self.row_upper))

    def to_c(self, keep: list, warm_x=None, warm_y=None) -> _capi.Lp:
        rp, ci, v, c, cl, cu, rl, ru = self.arrays()
        keep.extend([rp, ci, v, c, cl, cu, rl, ru])
        lp = _capi.Lp()
        lp.m, lp.n, lp.nnz = self.num_rows, self.num_cols, int(v.size)
        lp.row_ptr, lp.col_idx = _pi(rp), _pi(ci)
        lp.val, lp.obj, lp.col_lb, lp.col_ub, lp.row_lb, lp.row_ub = map(_pd, (v, c, cl, cu, rl, ru))
        lp.sense = int(self.sense)
        lp.obj_offset = float(self.obj_offset)
        if warm_x is not None and warm_y is not None:
            wx = np.ascontiguousarray(warm_x, dtype=np.float64)
            wy = np.ascontiguousarray(warm_y, dtype=np.float64)
            keep.extend([wx, wy])
            lp.warm_x, lp.warm_y = _pd(wx), _pd(wy)
        return lp


def _pd(a: np.ndarray):
    return a.ctypes.data_as(_capi.P_f64)


def _pi(a: np.ndarray):
    return a.ctypes.data_as(_capi.P_i32)


class PdlpSolver:
    """PdlpSolver : LpSolver on the B200 engine (one device solve per ``solve()``)."""

    def __init__(self) -> None:
        self._lib = _capi.load()
        self._h = C.c_void_p()
        self._options = PdlpOptions()
        _capi.check(self._lib.pdlpx_create(C.byref(self._options.to_c()), C.byref(self._h)))
        self._m = 0
        self._n = 0

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.pdlpx_destroy(h)
            self._h = C.c_void_p()

    # -- options
    def setOptions(self, options: PdlpOptions) -> None:
        self._options = options
        _capi.check(self._lib.pdlpx_set_options(self._h, C.byref(options.to_c())), self._h)

    def options(self) -> PdlpOptions:
        return self._options

    # -- LpSolver
    def load(self, problem: LpProblem) -> None:
        rp, ci, v, c, cl, cu, rl, ru = problem.arrays()
        _capi.check(self._lib.pdlpx_load_csr(
            self._h, problem.num_rows, problem.num_cols, int(v.size), _pi(rp), _pi(ci), _pd(v), _pd(c),
            _pd(cl), _pd(cu), _pd(rl), _pd(ru), int(problem.sense), float(problem.obj_offset)), self._h)
        self._m, self._n = problem.num_rows, problem.num_cols

    def solve(self) -> LpResult:
        flag = self._options.stop_flag
        self._lib.pdlpx_set_stop_flag(self._h, flag.ptr if flag is not None else None)
        r = _capi.Result()
        code = self._lib.pdlpx_solve(self._h, C.byref(r))
        if code == 2:  # not loaded: the reference returns Status::Error (pdlp.cpp:802-805)
            return LpResult(status=Status.Error)
        _capi.check(code, self._h)
        return LpResult.from_c(r)

    def getStatus(self) -> Status:
        s = C.c_int32()
        _capi.check(self._lib.pdlpx_get_status(self._h, C.byref(s)), self._h)
        return Status(s.value)

    def getObjective(self) -> float:
        v = C.c_double()
        _capi.check(self._lib.pdlpx_get_objective(self._h, C.byref(v)), self._h)
        return v.value

    def _dims(self):
        m, n, nnz = C.c_int32(), C.c_int32(), C.c_int32()
        self._lib.pdlpx_get_dims(self._h, C.byref(m), C.byref(n), C.byref(nnz))
        return m.value, n.value

    def getPrimalValues(self) -> np.ndarray:
        _, n = self._dims()
        x = np.zeros(n)
        code = self._lib.pdlpx_get_primal(self._h, _pd(x), n)
        if code != 0:  # trivial n == 0 path keeps an empty primal
            return np.zeros(0)
        return x

    def getDualValues(self) -> np.ndarray:
        m, _ = self._dims()
        y = np.zeros(m)
        _capi.check(self._lib.pdlpx_get_dual(self._h, _pd(y), m), self._h)
        return y

    def getReducedCosts(self) -> np.ndarray:
        _, n = self._dims()
        rc = np.zeros(n)
        _capi.check(self._lib.pdlpx_get_reduced_costs(self._h, _pd(rc), n), self._h)
        return rc

    def getBasis(self) -> list:
        return []  # PDLP has no basis (pdlp.cpp:2821-2823)

    def setBasis(self, basis) -> None:
        return None  # no-op (pdlp.cpp:2825-2827)

    def addRows(self, starts, indices, values, lower, upper) -> None:
        st = np.ascontiguousarray(starts, dtype=np.int32)
        ix = np.ascontiguousarray(indices, dtype=np.int32)
        va = np.ascontiguousarray(values, dtype=np.float64)
        lo = np.ascontiguousarray(lower, dtype=np.float64)
        up = np.ascontiguousarray(upper, dtype=np.float64)
        if st.size == 0 or lo.size != up.size or st.size != lo.size + 1 or ix.size != va.size:
            return  # ignored silently like pdlp.cpp:2838-2845
        _capi.check(self._lib.pdlpx_add_rows(self._h, int(lo.size), _pi(st), _pi(ix), _pd(va), int(va.size),
                                             _pd(lo), _pd(up)), self._h)

    def removeRows(self, rows) -> None:
        r = np.ascontiguousarray(rows, dtype=np.int32)
        _capi.check(self._lib.pdlpx_remove_rows(self._h, _pi(r), int(r.size)), self._h)

    def setColBounds(self, col: int, lower: float, upper: float) -> None:
        _capi.check(self._lib.pdlpx_set_col_bounds(self._h, int(col), float(lower), float(upper)), self._h)

    def setObjective(self, obj) -> None:
        o = np.ascontiguousarray(obj, dtype=np.float64)
        _capi.check(self._lib.pdlpx_set_objective(self._h, _pd(o), int(o.size)), self._h)

    # -- PDLP extras
    def setWarmStart(self, x, y) -> None:
        xa = np.ascontiguousarray(x, dtype=np.float64)
        ya = np.ascontiguousarray(y, dtype=np.float64)
        _capi.check(self._lib.pdlpx_set_warm_start(self._h, _pd(xa), int(xa.size), _pd(ya), int(ya.size)),
                    self._h)

    def clearWarmStart(self) -> None:
        _capi.check(self._lib.pdlpx_clear_warm_start(self._h), self._h)

    def usedGpu(self) -> bool:
        u = C.c_int32()
        _capi.check(self._lib.pdlpx_used_gpu(self._h, C.byref(u)), self._h)
        return bool(u.value)

    def timeKernels(self, reps: int = 20, precision: int = -1, flush_bytes: int = 0) -> dict:
        """Average device ms per launch of the primal step, dual step (run as
        `reps` interleaved PDHG iterations in `precision`: Precision.Mixed = the
        FP32 kernels, Precision.FP64, -1 = the precision the solve ended in,
        after an L2-evicting write of flush_bytes) and check pass."""
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        _capi.check(self._lib.pdlpx_time_kernels(self._h, int(precision), int(reps), int(flush_bytes), C.byref(a),
                                                 C.byref(b), C.byref(c)), self._h)
        return {"primal_ms": a.value, "dual_ms": b.value, "check_ms": c.value}

    def stepTimes(self, precision: int) -> dict:
        """Mean device ms of the primal and dual step measured inside the last
        solve (one iteration per restart cycle), for Precision.Mixed (FP32
        kernels) or Precision.FP64; samples = cycles measured."""
        a, b, k = C.c_double(), C.c_double(), C.c_int32()
        _capi.check(self._lib.pdlpx_get_step_times(self._h, int(precision), C.byref(a), C.byref(b), C.byref(k)),
                    self._h)
        return {"primal_ms": a.value, "dual_ms": b.value, "samples": k.value}

    def launchConfig(self) -> dict:
        ga, gat, bp, bd = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        _capi.check(self._lib.pdlpx_get_launch_config(self._h, C.byref(ga), C.byref(gat), C.byref(bp), C.byref(bd)),
                    self._h)
        return {"group_a": ga.value, "group_at": gat.value, "blocks_primal": bp.value, "blocks_dual": bd.value}

    def hotPrefix(self, precision: "Precision" = None) -> dict:
        """Hot-prefix lengths (option hot_cache) of the primal / dual step's
        gathers at `precision` (default: the loaded starting precision)."""
        if precision is None:
            precision = Precision.FP64 if self._options.precision == Precision.FP64 else Precision.Mixed
        p, d = C.c_int32(), C.c_int32()
        _capi.check(self._lib.pdlpx_get_hot_prefix(self._h, int(precision), C.byref(p), C.byref(d)), self._h)
        return {"primal": p.value, "dual": d.value}

    def longTiles(self) -> dict:
        """Row chunks and column groups of the tiled long-column primal step
        (option long_tiles); 0 chunks where the CSR launch runs."""
        c, g = C.c_int32(), C.c_int32()
        _capi.check(self._lib.pdlpx_get_long_tiles(self._h, C.byref(c), C.byref(g)), self._h)
        return {"chunks": c.value, "groups": g.value}

    def scaling(self) -> dict:
        """Scaled-problem arrays of the last load (parity of pdlp.cpp:469-669)."""
        m, n = self._dims()
        out = {k: np.zeros(n) for k in ("col_scale", "cscaled", "col_lower", "tau_base", "col_upper")}
        out.update({k: np.zeros(m) for k in ("row_scale", "row_lower", "row_upper", "sigma_base")})
        osc, csc = C.c_double(), C.c_double()
        _capi.check(self._lib.pdlpx_get_scaling(
            self._h, _pd(out["col_scale"]), _pd(out["cscaled"]), _pd(out["col_lower"]), _pd(out["row_scale"]),
            _pd(out["row_lower"]), _pd(out["row_upper"]), _pd(out["tau_base"]), _pd(out["sigma_base"]),
            _pd(out["col_upper"]), C.byref(osc), C.byref(csc)), self._h)
        out["objective_scale"] = osc.value
        out["constraint_scale"] = csc.value
        return out


def batch_solve(problems: Sequence[LpProblem], options: PdlpOptions, warm: Sequence | None = None,
                devices: Sequence[int] | None = None):
    """Solve many independent LPs in one call; returns [(LpResult, x, y)].
    ``devices``: CUDA ordinals to shard the LPs over (pdlpx_batch_solve_devices;
    one host thread per device, no data between devices); None = options.device."""
    lib = _capi.load()
    keep: list = []
    arr = (_capi.Lp * len(problems))()
    for k, p in enumerate(problems):
        wx, wy = (warm[k] if warm is not None and warm[k] is not None else (None, None))
        arr[k] = p.to_c(keep, wx, wy)
    res = (_capi.Result * len(problems))()
    xs = [np.zeros(p.num_cols) for p in problems]
    ys = [np.zeros(p.num_rows) for p in problems]
    xp = (_capi.P_f64 * len(problems))(*[_pd(x) for x in xs])
    yp = (_capi.P_f64 * len(problems))(*[_pd(y) for y in ys])
    if devices is None:
        _capi.check(lib.pdlpx_batch_solve(len(problems), arr, C.byref(options.to_c()), res, xp, yp))
    else:
        dv = np.ascontiguousarray(devices, dtype=np.int32)
        _capi.check(lib.pdlpx_batch_solve_devices(len(problems), arr, C.byref(options.to_c()), _pi(dv), int(dv.size),
                                                  res, xp, yp))
    return [(LpResult.from_c(res[k]), xs[k], ys[k]) for k in range(len(problems))]


def shard_lps(weights: Sequence[int], ndev: int) -> np.ndarray:
    """Device index of each LP under the engine's deterministic
    longest-processing-time sharding (pdlpx_shard_lps)."""
    lib = _capi.load()
    w = np.ascontiguousarray(weights, dtype=np.int64)
    out = np.zeros(w.size, dtype=np.int32)
    _capi.check(lib.pdlpx_shard_lps(int(w.size), w.ctypes.data_as(C.POINTER(C.c_int64)), int(ndev), _pi(out)))
    return out


def read_mps(path) -> LpProblem:
    """Read a free-format MPS file (plain or .gz) as mipx's ``readMps`` does
    (src/io/mps_reader.cpp:432-813) through the engine library's reader."""
    lib = _capi.load()
    g = _capi.GenLp()
    rc = lib.pdlpx_read_mps(str(path).encode(), C.byref(g))
    if rc != 0:
        raise _capi.PdlpxError(rc, f"{lib.pdlpx_error_string(rc).decode()}: {lib.pdlpx_last_error(None).decode()}")
    try:
        m, n, nnz = g.m, g.n, g.nnz
        arr = lambda p, k, dt: (np.ctypeslib.as_array(p, shape=(k,)).astype(dt, copy=True) if k > 0
                                else np.zeros(0, dt))
        rp = arr(g.row_ptr, m + 1, np.int32)
        lp = LpProblem(
            name=str(path), sense=Sense.Minimize, num_cols=n, num_rows=m,
            obj=arr(g.obj, n, np.float64), col_lower=arr(g.col_lb, n, np.float64),
            col_upper=arr(g.col_ub, n, np.float64), row_lower=arr(g.row_lb, m, np.float64),
            row_upper=arr(g.row_ub, m, np.float64), obj_offset=float(g.obj_offset),
            matrix=SparseMatrix(m, n, values=arr(g.val, nnz, np.float64), col_indices=arr(g.col_idx, nnz, np.int32),
                                row_starts=rp),
            col_type=["I" if k else "C" for k in arr(g.is_int, n, np.int32)])
    finally:
        lib.pdlpx_free_lp(C.byref(g))
    return lp


def solve_mps(filename, time_limit: float = 3600.0, verbose: bool = False,
              options: PdlpOptions | None = None):
    """Read an MPS file (plain or .gz) and solve it with PDLP on the GPU.

    The PDLP path's counterpart of mipx's Python ``solve_mps``
    (python/src/bindings.cpp:169-205: ``readMps`` then a solve with default
    settings): the model is read as mipx's reader reads it and its LP -- integer
    marks ignored, as the CLI's ``--pdlp`` LP mode does (src/cli/main.cpp:509-522)
    -- is solved by ``PdlpSolver``.  ``time_limit`` and ``verbose`` override the
    corresponding fields of ``options`` (default PdlpOptions()).  Returns
    ``(LpResult, x, y)`` with x, y in the model's original space."""
    opts = options if options is not None else PdlpOptions()
    opts = dataclasses.replace(opts, max_solve_seconds=float(time_limit), verbose=bool(verbose))
    s = PdlpSolver()
    s.setOptions(opts)
    s.load(read_mps(filename))
    r = s.solve()
    return r, s.getPrimalValues(), s.getDualValues()


class Server:
    """LP solves as they arrive (``pdlpx_server_*``): submitted LPs are packed
    with whatever else is waiting and solved several packs at a time on the
    device; each result is available as soon as it is finished.

    ``devices``: CUDA ordinals the packs are placed on (the listed device with
    a free stream and the fewest bytes in flight); None = options.device.
    ``submit(lp, warm=None)`` returns a ticket; ``warm`` is an ``(x, y)`` pair or
    the ticket of a finished request.  ``wait(ticket)`` returns
    ``(LpResult, x, y)``.  ``stats()`` reports p50/p99 latency and LPs/s.
    With ``families`` on, requests warm-started from a ticket whose rows they
    keep unchanged (branch-and-bound nodes of that LP) run in family packs."""

    def __init__(self, options: PdlpOptions, budget_bytes: float = 0.0, max_packs: int = 4,
                 max_pack_lps: int = 32, prep_threads: int = 0, queue_limit: int = 100000,
                 batch_window_ms: int = 50, families: bool = True, devices: Sequence[int] | None = None,
                 lane_admission: bool = True):
        self._lib = _capi.load()
        cfg = _capi.ServerConfig()
        self._lib.pdlpx_server_config_default(C.byref(cfg))
        cfg.budget_bytes = float(budget_bytes)
        cfg.max_packs = int(max_packs)
        cfg.max_pack_lps = int(max_pack_lps)
        cfg.prep_threads = int(prep_threads)
        cfg.queue_limit = int(queue_limit)
        cfg.batch_window_ms = int(batch_window_ms)
        cfg.families = int(bool(families))
        cfg.lane_admission = int(bool(lane_admission))
        if devices is not None and len(devices) > 1:
            if len(devices) > len(cfg.devices):
                raise ValueError(f"at most {len(cfg.devices)} devices")
            cfg.num_devices = len(devices)
            for k, d in enumerate(devices):
                cfg.devices[k] = int(d)
        self._h = C.c_void_p()
        _capi.check(self._lib.pdlpx_server_create(C.byref(options.to_c()), C.byref(cfg), C.byref(self._h)))
        self._dims: dict[int, tuple[int, int]] = {}

    def _check(self, code: int) -> None:
        if code != 0:
            raise _capi.PdlpxError(code, self._lib.pdlpx_server_last_error(self._h).decode())

    def submit(self, lp: LpProblem, warm=None) -> int:
        keep: list = []
        t = C.c_int64()
        if isinstance(warm, (int, np.integer)):
            c_lp = lp.to_c(keep, None, None)
            self._check(self._lib.pdlpx_server_submit_warm(self._h, C.byref(c_lp), int(warm), C.byref(t)))
        else:
            wx, wy = warm if warm is not None else (None, None)
            c_lp = lp.to_c(keep, wx, wy)
            self._check(self._lib.pdlpx_server_submit(self._h, C.byref(c_lp), C.byref(t)))
        self._dims[t.value] = (lp.num_cols, lp.num_rows)
        return t.value

    def done(self, ticket: int) -> bool:
        d = C.c_int32()
        self._check(self._lib.pdlpx_server_poll(self._h, int(ticket), C.byref(d)))
        return bool(d.value)

    def wait(self, ticket: int, timeout: float = -1.0):
        r = _capi.Result()
        self._check(self._lib.pdlpx_server_wait(self._h, int(ticket), float(timeout), C.byref(r)))
        n, m = self._dims[ticket]
        x, y = np.zeros(n), np.zeros(m)
        self._check(self._lib.pdlpx_server_get_solution(self._h, int(ticket), _pd(x), n, _pd(y), m))
        return LpResult.from_c(r), x, y

    def release(self, ticket: int) -> None:
        self._check(self._lib.pdlpx_server_release(self._h, int(ticket)))
        self._dims.pop(ticket, None)

    def stats(self) -> dict:
        s = _capi.ServerStats()
        self._check(self._lib.pdlpx_server_get_stats(self._h, C.byref(s)))
        return {name: getattr(s, name) for name, _ in s._fields_ if not name.startswith("reserved")}

    def close(self) -> None:
        if self._h:
            self._lib.pdlpx_server_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def csr_spmv(matrix: SparseMatrix, x, precision: Precision = Precision.Mixed, group: int = 0) -> np.ndarray:
    """y = A x with the engine's device SpMV kernel (parity entry point)."""
    lib = _capi.load()
    xa = np.ascontiguousarray(x, dtype=np.float64)
    y = np.zeros(matrix.rows)
    rp = np.ascontiguousarray(matrix.row_starts, dtype=np.int32)
    ci = np.ascontiguousarray(matrix.col_indices, dtype=np.int32)
    v = np.ascontiguousarray(matrix.values, dtype=np.float64)
    _capi.check(lib.pdlpx_csr_spmv(matrix.rows, matrix.cols, int(v.size), _pi(rp), _pi(ci), _pd(v), _pd(xa),
                                   _pd(y), int(precision), int(group)))
    return y


def row_violation(matrix: SparseMatrix, x, row_lower, row_upper) -> tuple[float, float]:
    """(sum_i v_i^2, max_i |v_i|) with v = A x - clamp(A x, row_lower, row_upper), FP64 on the device."""
    lib = _capi.load()
    xa = np.ascontiguousarray(x, dtype=np.float64)
    rl = np.ascontiguousarray(row_lower, dtype=np.float64)
    ru = np.ascontiguousarray(row_upper, dtype=np.float64)
    rp = np.ascontiguousarray(matrix.row_starts, dtype=np.int32)
    ci = np.ascontiguousarray(matrix.col_indices, dtype=np.int32)
    v = np.ascontiguousarray(matrix.values, dtype=np.float64)
    s, mx = C.c_double(), C.c_double()
    _capi.check(lib.pdlpx_row_violation(matrix.rows, matrix.cols, int(v.size), _pi(rp), _pi(ci), _pd(v), _pd(xa),
                                        _pd(rl), _pd(ru), C.byref(s), C.byref(mx)))
    return s.value, mx.value
