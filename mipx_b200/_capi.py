"""ctypes binding of ``include/pdlpx.h`` (the engine's C ABI).

The structure layouts below mirror the header field for field; ``check_layout``
compares their sizes with the sizes the library was compiled with
(pdlpx_struct_sizes).
Loading fails loudly when the library is missing: there is no Python or CPU
stand-in for the device engine.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

from . import build as _build

i32 = C.c_int32
f64 = C.c_double
P_i32 = C.POINTER(C.c_int32)
P_f64 = C.POINTER(C.c_double)
# pdlpx_stop_poll: int32_t (*)(void* ctx); a Python function wrapped in it can be
# passed to pdlpx_set_stop_callback (keep the wrapper alive while it is set).
STOP_POLL = C.CFUNCTYPE(C.c_int32, C.c_void_p)


class Options(C.Structure):
    _fields_ = [
        ("max_iter", i32), ("optimality_tol", f64), ("primal_tol", f64), ("dual_tol", f64),
        ("max_solve_seconds", f64), ("optimality_norm", i32), ("sv_max_iter", i32), ("sv_tol", f64),
        ("adaptive_step", i32), ("adaptive_step_down", f64), ("adaptive_step_up", f64),
        ("adaptive_step_min", f64), ("adaptive_step_max", f64), ("primal_weight", f64),
        ("update_primal_weight", i32), ("pid_kp", f64), ("pid_ki", f64), ("pid_kd", f64),
        ("pid_i_smooth", f64), ("restart_sufficient_decay", f64), ("restart_necessary_decay", f64),
        ("restart_artificial_fraction", f64), ("termination_eval_frequency", i32),
        ("matrix_zero_tol", f64), ("enable_polishing", i32), ("polish_primal_tol", f64),
        ("polish_dual_tol", f64), ("polish_max_iter", i32), ("do_ruiz_scaling", i32),
        ("ruiz_iterations", i32), ("do_pock_chambolle_scaling", i32), ("do_bound_obj_rescaling", i32),
        ("preconditioner_refresh", i32), ("preconditioner_refresh_ratio", f64),
        ("anderson_acceleration", i32), ("anderson_window_size", i32), ("anderson_regularization", f64),
        ("use_gpu", i32), ("gpu_min_rows", i32), ("gpu_min_nnz", i32), ("verbose", i32),
        ("precision", i32), ("device", i32), ("fp64_switch", i32), ("spmv_group_a", i32),
        ("spmv_group_at", i32), ("autotune", i32), ("shape_primal", i32), ("shape_dual", i32), ("batch_pack_mb", i32),
        ("batch_compact", i32), ("batch_sell", i32), ("scale_on_device", i32), ("sell", i32),
        ("reference_fixed_columns", i32), ("hot_cache", i32),
        ("long_tiles", i32), ("batch_persistent", i32), ("sell_window", i32), ("reserved", i32 * 1),
    ]


class Result(C.Structure):
    _fields_ = [
        ("status", i32), ("objective", f64), ("iterations", i32), ("work_units", f64),
        ("rel_primal_resid", f64), ("rel_dual_resid", f64), ("rel_gap", f64),
        ("primal_objective", f64), ("dual_objective", f64), ("fp64_iterations", i32),
        ("restarts", i32), ("step_size", f64), ("primal_weight", f64), ("solve_seconds", f64),
        ("device_seconds", f64), ("used_gpu", i32), ("kernel_launches", i32),
    ]


class Lp(C.Structure):
    _fields_ = [
        ("m", i32), ("n", i32), ("nnz", i32), ("row_ptr", P_i32), ("col_idx", P_i32), ("val", P_f64),
        ("obj", P_f64), ("col_lb", P_f64), ("col_ub", P_f64), ("row_lb", P_f64), ("row_ub", P_f64),
        ("sense", i32), ("obj_offset", f64), ("warm_x", P_f64), ("warm_y", P_f64),
    ]


class GenLp(C.Structure):
    _fields_ = [
        ("m", i32), ("n", i32), ("nnz", i32), ("row_ptr", P_i32), ("col_idx", P_i32), ("val", P_f64),
        ("obj", P_f64), ("col_lb", P_f64), ("col_ub", P_f64), ("row_lb", P_f64), ("row_ub", P_f64),
        ("x0", P_f64), ("is_int", P_i32), ("obj_offset", f64),
    ]


# (name, restype, argtypes) of every entry point declared in include/pdlpx.h
class ServerConfig(C.Structure):
    _fields_ = [("budget_bytes", f64), ("max_packs", i32), ("max_pack_lps", i32), ("prep_threads", i32),
                ("queue_limit", i32), ("batch_window_ms", i32), ("families", i32), ("num_devices", i32),
                ("lane_admission", i32), ("devices", i32 * 16)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("waiting", C.c_int64), ("running", C.c_int64),
                ("packs_running", i32), ("reserved0", i32), ("p50_latency_s", f64), ("p99_latency_s", f64),
                ("mean_latency_s", f64), ("max_latency_s", f64), ("lps_per_sec", f64), ("bytes_in_flight", f64),
                ("admitted", C.c_int64)]


SIGNATURES = [
    ("pdlpx_options_default", None, [C.POINTER(Options)]),
    ("pdlpx_error_string", C.c_char_p, [i32]),
    ("pdlpx_last_error", C.c_char_p, [C.c_void_p]),
    ("pdlpx_device_count", i32, []),
    ("pdlpx_version", C.c_char_p, []),
    ("pdlpx_struct_sizes", None, [P_i32]),
    ("pdlpx_create", i32, [C.POINTER(Options), C.POINTER(C.c_void_p)]),
    ("pdlpx_destroy", i32, [C.c_void_p]),
    ("pdlpx_set_options", i32, [C.c_void_p, C.POINTER(Options)]),
    ("pdlpx_get_options", i32, [C.c_void_p, C.POINTER(Options)]),
    ("pdlpx_load_csr", i32, [C.c_void_p, i32, i32, i32, P_i32, P_i32, P_f64, P_f64, P_f64, P_f64, P_f64,
                             P_f64, i32, f64]),
    ("pdlpx_set_warm_start", i32, [C.c_void_p, P_f64, i32, P_f64, i32]),
    ("pdlpx_clear_warm_start", i32, [C.c_void_p]),
    ("pdlpx_set_stop_flag", i32, [C.c_void_p, P_i32]),
    ("pdlpx_set_stop_callback", i32, [C.c_void_p, C.c_void_p, C.c_void_p]),  # poll: STOP_POLL or None
    ("pdlpx_solve", i32, [C.c_void_p, C.POINTER(Result)]),
    ("pdlpx_get_status", i32, [C.c_void_p, P_i32]),
    ("pdlpx_get_objective", i32, [C.c_void_p, P_f64]),
    ("pdlpx_get_primal", i32, [C.c_void_p, P_f64, i32]),
    ("pdlpx_get_dual", i32, [C.c_void_p, P_f64, i32]),
    ("pdlpx_get_reduced_costs", i32, [C.c_void_p, P_f64, i32]),
    ("pdlpx_used_gpu", i32, [C.c_void_p, P_i32]),
    ("pdlpx_get_dims", i32, [C.c_void_p, P_i32, P_i32, P_i32]),
    ("pdlpx_add_rows", i32, [C.c_void_p, i32, P_i32, P_i32, P_f64, i32, P_f64, P_f64]),
    ("pdlpx_remove_rows", i32, [C.c_void_p, P_i32, i32]),
    ("pdlpx_set_col_bounds", i32, [C.c_void_p, i32, f64, f64]),
    ("pdlpx_set_objective", i32, [C.c_void_p, P_f64, i32]),
    ("pdlpx_get_scaling", i32, [C.c_void_p] + [P_f64] * 11),
    ("pdlpx_time_kernels", i32, [C.c_void_p, i32, i32, C.c_int64, P_f64, P_f64, P_f64]),
    ("pdlpx_get_step_times", i32, [C.c_void_p, i32, P_f64, P_f64, P_i32]),
    ("pdlpx_get_launch_config", i32, [C.c_void_p, P_i32, P_i32, P_i32, P_i32]),
    ("pdlpx_get_hot_prefix", i32, [C.c_void_p, i32, P_i32, P_i32]),
    ("pdlpx_get_long_tiles", i32, [C.c_void_p, P_i32, P_i32]),
    ("pdlpx_shard_lps", i32, [i32, C.POINTER(C.c_int64), i32, P_i32]),
    ("pdlpx_grid_barrier_check", i32, [i32, i32, i32, i32, P_i32, P_f64]),
    ("pdlpx_batch_solve_devices", i32, [i32, C.POINTER(Lp), C.POINTER(Options), P_i32, i32, C.POINTER(Result),
                                        C.POINTER(P_f64), C.POINTER(P_f64)]),
    ("pdlpx_batch_solve", i32, [i32, C.POINTER(Lp), C.POINTER(Options), C.POINTER(Result),
                                C.POINTER(P_f64), C.POINTER(P_f64)]),
    ("pdlpx_server_config_default", None, [C.POINTER(ServerConfig)]),
    ("pdlpx_server_create", i32, [C.POINTER(Options), C.POINTER(ServerConfig), C.POINTER(C.c_void_p)]),
    ("pdlpx_server_destroy", i32, [C.c_void_p]),
    ("pdlpx_server_submit", i32, [C.c_void_p, C.POINTER(Lp), C.POINTER(C.c_int64)]),
    ("pdlpx_server_submit_warm", i32, [C.c_void_p, C.POINTER(Lp), C.c_int64, C.POINTER(C.c_int64)]),
    ("pdlpx_server_poll", i32, [C.c_void_p, C.c_int64, P_i32]),
    ("pdlpx_server_wait", i32, [C.c_void_p, C.c_int64, f64, C.POINTER(Result)]),
    ("pdlpx_server_get_solution", i32, [C.c_void_p, C.c_int64, P_f64, i32, P_f64, i32]),
    ("pdlpx_server_release", i32, [C.c_void_p, C.c_int64]),
    ("pdlpx_server_get_stats", i32, [C.c_void_p, C.POINTER(ServerStats)]),
    ("pdlpx_server_last_error", C.c_char_p, [C.c_void_p]),
    ("pdlpx_csr_spmv", i32, [i32, i32, i32, P_i32, P_i32, P_f64, P_f64, P_f64, i32, i32]),
    ("pdlpx_row_violation", i32, [i32, i32, i32, P_i32, P_i32, P_f64, P_f64, P_f64, P_f64, P_f64, P_f64]),
    ("pdlpx_row_violation_noalloc", i32, [i32, i32, i32] + [C.c_void_p] * 8),
    ("pdlpx_gen_random", i32, [i32, i32, i32, i32, C.c_uint64, C.POINTER(GenLp)]),
    ("pdlpx_gen_transport", i32, [i32, i32, C.c_uint64, C.POINTER(GenLp)]),
    ("pdlpx_gen_powerlaw", i32, [i32, i32, i32, i32, f64, f64, f64, C.c_uint64, C.POINTER(GenLp)]),
    ("pdlpx_free_lp", None, [C.POINTER(GenLp)]),
    ("pdlpx_read_mps", i32, [C.c_char_p, C.POINTER(GenLp)]),
]

_lib = None


def lib_path() -> Path:
    return _build.LIB


def load(build_if_missing: bool = True) -> C.CDLL:
    """Load libpdlpx.so (building it first when it is absent and nvcc exists)."""
    global _lib
    if _lib is not None:
        return _lib
    path = lib_path()
    if not path.exists():
        if not build_if_missing:
            raise RuntimeError(f"engine library missing: {path}")
        _build.build()
    lib = C.CDLL(str(path), mode=os.RTLD_NOW | getattr(os, "RTLD_GLOBAL", 0))
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    check_layout()
    return lib


def check_layout() -> None:
    """Raise when a ctypes structure here differs in size from the library's."""
    sizes = (C.c_int32 * 6)()
    load().pdlpx_struct_sizes(sizes)
    ours = [C.sizeof(t) for t in (Options, Result, Lp, GenLp, ServerConfig, ServerStats)]
    if list(sizes) != ours:
        raise RuntimeError(f"ABI structure sizes differ: library {list(sizes)}, binding {ours}")


def default_options() -> Options:
    o = Options()
    load().pdlpx_options_default(C.byref(o))
    return o


class PdlpxError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"pdlpx error {code}: {msg}")
        self.code = code


def check(code: int, handle=None) -> None:
    if code != 0:
        lib = load()
        detail = lib.pdlpx_last_error(handle).decode() if handle is not None else ""
        base = lib.pdlpx_error_string(code).decode()
        raise PdlpxError(code, f"{base}: {detail}" if detail else base)
