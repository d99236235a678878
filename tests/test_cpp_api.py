"""The C++ mirror of mipx's PDLP interface (include/pdlpx.hpp), compiled with
g++ against the engine library: host-only paths here, device solves under the
gpu marker."""
import shutil
import subprocess
from pathlib import Path

import pytest

from mipx_b200 import _capi

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "cpp" / "pdlpx_api_test.cpp"


def _build(tmp_path) -> Path:
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    lib = _capi.lib_path()
    if not lib.exists():
        _capi.load()
    exe = tmp_path / "pdlpx_api_test"
    subprocess.run(["g++", "-std=c++20", "-O1", "-Wall", "-Wextra", "-Werror", f"-I{ROOT / 'include'}", str(SRC),
                    "-o", str(exe),
                    f"-L{lib.parent}", "-lpdlpx", f"-Wl,-rpath,{lib.parent}"], check=True)
    return exe


def _run(exe, mode):
    p = subprocess.run([str(exe), mode], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    assert "FAIL" not in p.stdout


def test_cpp_mirror_host_paths(tmp_path):
    _run(_build(tmp_path), "host")


@pytest.mark.gpu
def test_cpp_mirror_solves_on_device(tmp_path):
    _run(_build(tmp_path), "gpu")
