"""Test configuration.

Markers:
  gpu  -- needs a CUDA device (run with ``-m gpu`` on a B200); everything else
          runs on a CPU-only machine.

The native library and the oracle are built in-tree on first use if they are
missing (``python -m monkeygl_b200.build``, ``make -C oracle``).
"""
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _ensure_built():
    from monkeygl_b200 import build as b
    if not b.library_path().exists():
        b.build()
    if not (ROOT / "oracle" / "lib" / "libmkoracle.so").exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "oracle"], check=True,
                       capture_output=True)


_ensure_built()


@pytest.fixture(scope="session")
def golden_dir():
    return GOLDEN
