"""Build the engine's C-ABI library ``mipx_b200/_lib/libpdlpx.so`` for sm_100a.

Every CUDA translation unit is compiled by nvcc with
``-gencode arch=compute_100a,code=sm_100a -lineinfo``; host C++ files go
through nvcc to g++.  Objects land in ``mipx_b200/_build`` and the shared
library in ``mipx_b200/_lib`` (both git-ignored, both travel with the source
tree).  Rebuilds only when a source or header is newer than the library.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIBDIR = PKG / "_lib"
LIB = LIBDIR / "libpdlpx.so"

SOURCES = ["engine.cu", "batch.cu", "residual.cu", "problem.cpp", "capi.cpp", "server.cpp", "generators.cpp", "mps.cpp", "scaling.cu"]
CLI = LIBDIR / "pdlpx_cli"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the engine needs the CUDA toolkit to build")


def _deps() -> list[Path]:
    files = [CSRC / s for s in SOURCES if (CSRC / s).exists()]
    files += list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "pdlpx.h"]
    return files


def up_to_date() -> bool:
    if not LIB.exists() or not CLI.exists():
        return False
    t = min(LIB.stat().st_mtime, CLI.stat().st_mtime)
    return all(p.stat().st_mtime <= t for p in _deps() + [CSRC / "cli.cpp", ROOT / "include" / "pdlpx.hpp"])


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> Path:
    if not force and up_to_date():
        return LIB
    BUILD.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    cc = nvcc()
    common = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "-I", str(ROOT / "include"),
              "-I", str(CSRC), *ARCH]
    if ptxas_info:
        common += ["-Xptxas", "-v"]

    def compile_one(src: str) -> Path:
        obj = BUILD / (src.rsplit(".", 1)[0] + ".o")
        cmd = [cc, *common, "-c", str(CSRC / src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
        if ptxas_info and r.stderr:
            print(r.stderr, file=sys.stderr)
        return obj

    srcs = [s for s in SOURCES if (CSRC / s).exists()]
    with ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(compile_one, srcs))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [cc, *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart_static", "-lrt", "-lpthread", "-ldl",
           "-lz"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    # command-line front end (mipx's `--pdlp` LP mode and its summary lines) over the library
    cxx = shutil.which("g++") or "g++"
    tmp = CLI.with_suffix(".tmp")
    cmd = [cxx, "-std=c++20", "-O2", "-I", str(ROOT / "include"), str(CSRC / "cli.cpp"), "-o", str(tmp),
           "-L", str(LIBDIR), "-lpdlpx", "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"cli build failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, CLI)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
