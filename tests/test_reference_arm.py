"""bench.py's reference arm (`--impl reference`) times the reference's own CPU
PdlpSolver and maps no library of the engine: the ratio of the two arms holds
only if the reference arm never loads libpdlpx.so (its generator comes from the
oracle library, its option structs are plain ctypes)."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
REF_SO = ROOT / "oracle" / "_ref" / "libmipx_pdlp_ref.so"

CODE = """
import argparse, json, sys
sys.path.insert(0, {root!r})
import bench
bench.run_reference(argparse.Namespace(large_rows=2000, warmup=1, steps=1, gpus=1), 0, None)
libs = sorted({{l.split()[-1] for l in open('/proc/self/maps').read().splitlines()
               if '.so' in l and l.split()[-1].startswith({root!r})}})
print('LIBS ' + json.dumps(libs))
"""


@pytest.mark.skipif(not REF_SO.exists(), reason="the reference library (oracle/_ref) is not built")
def test_reference_arm_maps_only_oracle_libraries():
    out = subprocess.run([sys.executable, "-c", CODE.format(root=str(ROOT))], capture_output=True, text=True,
                         timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-3000:]
    lines = out.stdout.splitlines()
    line = json.loads([s for s in lines if s.startswith("{")][-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "reference"
    assert line["e2e"]["h2d_bytes_per_step"] == 0
    libs = json.loads([s for s in lines if s.startswith("LIBS ")][-1][len("LIBS "):])
    assert any("libmipx_pdlp_ref" in p for p in libs), libs
    assert all("/oracle/" in p for p in libs), libs
    assert not any("libpdlpx" in p for p in libs), libs
