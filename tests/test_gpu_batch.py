"""Batch MPR through the C++ API: HelloMonkey::GetBatchData.

MonkeyGL declares GetBatchData and BatchInfo (core/HelloMonkey.cpp:415-419,
core/BatchInfo.h:29-54) but returns false (core/Render.cpp:117-120).  The
check program tests/native/batch_check.cpp, compiled here against the
library's C++ headers, renders (1) a one-plane batch with the axial plane's
geometry, which must equal GetPlaneData(PlaneAxial), and (2) a 5-plane
oblique stack of MIP slabs, each plane equal to mk_render_plane with that
plane's parameters."""
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "native" / "batch_check.cpp"
BUILD = ROOT / "tests" / "native" / "_build"
LIBDIR = ROOT / "monkeygl_b200" / "lib"

pytestmark = pytest.mark.gpu


def _build():
    BUILD.mkdir(parents=True, exist_ok=True)
    exe = BUILD / "batch_check"
    if not exe.exists() or exe.stat().st_mtime < max(SRC.stat().st_mtime,
                                                     (LIBDIR / "libmonkeygl_b200.so").stat().st_mtime):
        subprocess.run(["g++", "-O2", "-std=c++17", f"-I{ROOT / 'include'}", str(SRC), "-o", str(exe),
                        f"-L{LIBDIR}", "-lmonkeygl_b200", f"-Wl,-rpath,{LIBDIR}"], check=True)
    return exe


def test_batch_planes_equal_single_planes():
    exe = _build()
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "batch ok" in r.stdout
