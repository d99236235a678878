import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the engine's kernels")
    config.addinivalue_line("markers", "slow: long-running parity case")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Engine and oracle libraries (built here when missing; a machine without the sources gets them prebuilt)."""
    from mipx_b200 import build as engine_build
    engine_build.build()
    from oracle import oracle
    if not oracle.ORACLE_LIB.exists():
        oracle.build()
    yield
