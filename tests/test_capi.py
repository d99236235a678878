"""C ABI: the library loads, exports every entry point include/pdlpx.h declares,
reports the reference defaults, and validates input -- all without a GPU."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import lp_fixtures as F
from mipx_b200 import _capi
from mipx_b200.pdlp import PdlpOptions, PdlpSolver, Status

HEADER = Path(__file__).resolve().parents[1] / "include" / "pdlpx.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"\b(pdlpx_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _capi.load()
    names = declared_symbols()
    assert len(names) >= 30
    for name in names:
        assert hasattr(lib, name), name
    bound = {n for n, _, _ in _capi.SIGNATURES}
    assert set(names) == bound


def test_defaults_match_reference_options():
    o = _capi.default_options()
    ref = PdlpOptions()  # field defaults of include/mipx/pdlp.h:19-87
    for name, _ in _capi.Options._fields_:
        if name in ("reserved", "precision", "device", "fp64_switch", "spmv_group_a", "spmv_group_at", "autotune", "shape_primal",
                    "shape_dual", "batch_pack_mb", "batch_compact", "batch_sell", "scale_on_device"):
            continue
        assert getattr(o, name) == pytest.approx(float(getattr(ref, name))), name


def test_error_strings_and_version():
    lib = _capi.load()
    assert lib.pdlpx_error_string(0) == b"ok"
    assert b"sm_100a" in lib.pdlpx_version()
    assert lib.pdlpx_device_count() >= 0


def test_invalid_inputs_rejected():
    lib = _capi.load()
    assert lib.pdlpx_create(None, None) == 1
    h = C.c_void_p()
    assert lib.pdlpx_create(None, C.byref(h)) == 0
    r = _capi.Result()
    assert lib.pdlpx_solve(h, C.byref(r)) == 2  # not loaded
    rp = np.array([0, 2], np.int32)
    ci = np.array([0, 5], np.int32)  # column out of range
    v = np.array([1.0, 1.0])
    z = np.zeros(2)
    pd = lambda a: a.ctypes.data_as(_capi.P_f64)
    pi = lambda a: a.ctypes.data_as(_capi.P_i32)
    code = lib.pdlpx_load_csr(h, 1, 2, 2, pi(rp), pi(ci), pd(v), pd(z), pd(z), pd(z), pd(z[:1]), pd(z[:1]), 0, 0.0)
    assert code == 1
    assert b"CSR" in lib.pdlpx_last_error(h)
    lib.pdlpx_destroy(h)


def test_solve_before_load_is_error_status():
    s = PdlpSolver()
    assert s.solve().status == Status.Error


def test_trivial_problems_on_host_semantics():
    """n == 0 and m == 0 are closed-form in the reference (pdlp.cpp:813-860) and need no device."""
    s = PdlpSolver()
    s.setOptions(PdlpOptions(verbose=False))
    s.load(F.empty_lp())
    r = s.solve()
    assert r.status == Status.Optimal and r.objective == 42.0 and r.iterations == 0
    s.load(F.bounds_only_lp())
    r = s.solve()
    assert r.status == Status.Optimal and abs(r.objective - 1.0) < 1e-12
    assert abs(s.getPrimalValues()[0] - 1.0) < 1e-12
    s.load(F.unbounded_bounds_only_lp())
    assert s.solve().status == Status.Unbounded
    assert not s.usedGpu()


def test_basis_api_is_empty():
    s = PdlpSolver()
    assert s.getBasis() == []
    s.setBasis([])


def test_struct_layout_is_consistent():
    # pdlpx_get_options round-trips every field of the ctypes image
    lib = _capi.load()
    o = _capi.default_options()
    o.max_iter = 1234
    o.pid_kp = 0.5
    o.spmv_group_at = 8
    h = C.c_void_p()
    assert lib.pdlpx_create(C.byref(o), C.byref(h)) == 0
    back = _capi.Options()
    assert lib.pdlpx_get_options(h, C.byref(back)) == 0
    for name, _ in _capi.Options._fields_:
        if name != "reserved":
            assert getattr(back, name) == getattr(o, name), name
    lib.pdlpx_destroy(h)


def test_struct_layouts_match_the_library():
    _capi.check_layout()
    assert C.sizeof(_capi.ServerConfig) == 8 + 4 * (6 + 2 + 16)
