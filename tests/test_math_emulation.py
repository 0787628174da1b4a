"""The FP32 emulation of MonkeyGL's double-precision expressions
(monkeygl_b200/csrc/mk_math.h) against the double expressions themselves.

The kernels keep device arithmetic in FP32; where MonkeyGL's code promotes to
double (core/kernel.cu:197 "0.866", :460 "0.05", :773 accumulator,
:860-862 CPR points) they use error-free float transformations.  These tests
compile the same header for the host and count disagreements over large
random and adversarial input sets."""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "native" / "emul_check.cpp"
BUILD = ROOT / "tests" / "native" / "_build"


@pytest.fixture(scope="module")
def lib():
    BUILD.mkdir(exist_ok=True)
    so = BUILD / "libemul_check.so"
    hdr = ROOT / "monkeygl_b200" / "csrc" / "mk_math.h"
    if not so.exists() or so.stat().st_mtime < max(SRC.stat().st_mtime, hdr.stat().st_mtime):
        subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off",
                        f"-I{hdr.parent}", str(SRC), "-o", str(so)], check=True)
    L = C.CDLL(str(so))
    for f in ("check_ray_fy", "check_ray_fy_exact", "check_add005", "check_cpr", "check_mean"):
        getattr(L, f).restype = C.c_int64
    return L


def p(a):
    return C.c_void_p(a.ctypes.data)


def test_ray_parameter_matches_double(lib):
    rng = np.random.default_rng(1)
    n = 2_000_000
    # accuLength values as produced by the schedule (sums of 1/dim steps) and random ones
    a = np.concatenate([
        np.cumsum(np.full(2700, np.float32(1.0) / np.float32(1559)), dtype=np.float32),
        rng.uniform(0, 1.75, n).astype(np.float32),
        (np.float32(0.866) + rng.integers(-64, 64, 10000).astype(np.float32) * np.float32(6e-8)).astype(np.float32),
    ])
    scale = np.where(rng.random(a.size) < 0.5, 1.0, rng.uniform(0.2, 4.0, a.size)).astype(np.float32)
    e = np.empty_like(a)
    r = np.empty_like(a)
    bad = lib.check_ray_fy(p(a), p(scale), a.size, p(e), p(r))
    assert bad == 0, bad


def test_ray_parameter_double_rounding_cases(lib):
    # inputs whose product lies next to a float rounding midpoint, where
    # MonkeyGL's two roundings (to double, then to float) differ from one
    # correct rounding; found by an exhaustive search over all floats in
    # [2^-12, 1.732] at these scales
    cases = [(0x3e79999b, 1.3), (0x3db851e5, 0.8), (0x3db851ef, 0.8), (0x3d449242, 0.4321),
             (0x3e179e87, 0.4321), (0x39b5c183, 1.1), (0x3a3adf4d, 1.1)]
    a = np.array([c[0] for c in cases], np.uint32).view(np.float32)
    scale = np.array([c[1] for c in cases], np.float32)
    e = np.empty_like(a)
    r = np.empty_like(a)
    assert lib.check_ray_fy(p(a), p(scale), a.size, p(e), p(r)) == 0, list(zip(e, r))


def test_ray_parameter_integer_route_matches_double(lib):
    rng = np.random.default_rng(5)
    a = np.concatenate([[0.0], rng.uniform(2.0 ** -30, 1.75, 1_000_000)]).astype(np.float32)
    scale = np.exp(rng.uniform(-3, 3, a.size)).astype(np.float32)
    e = np.empty_like(a)
    r = np.empty_like(a)
    assert lib.check_ray_fy_exact(p(a), p(scale), a.size, p(e), p(r)) == 0


def test_surface_offset_matches_double(lib):
    rng = np.random.default_rng(2)
    x = rng.uniform(-1, 1, 1_000_000).astype(np.float32)
    e = np.empty_like(x)
    r = np.empty_like(x)
    assert lib.check_add005(p(x), x.size, p(e), p(r)) == 0


def test_cpr_coordinate_matches_double(lib):
    rng = np.random.default_rng(3)
    n = 1_000_000
    pt = rng.uniform(-50, 1600, n)
    d = rng.standard_normal(n)
    x = rng.integers(0, 1024, n).astype(np.int32)
    dim = rng.choice([96, 128, 361, 512, 1559], n).astype(np.int32)
    e = np.empty(n, np.float32)
    r = np.empty(n, np.float32)
    bad = lib.check_cpr(p(pt), p(d), p(x), p(dim), n, p(e), p(r))
    assert bad <= 2, bad


def test_slab_mean_matches_double(lib):
    rng = np.random.default_rng(4)
    for k in (1, 2, 3, 5, 8, 17):
        rows = 200_000
        base = rng.integers(-1024, 3072, rows * k).astype(np.float64)
        v = (base * (32768.0 / 32767.0)).astype(np.float32)          # nearest texel values
        v[::7] = np.float32(-32768.0)                                   # out-of-volume samples
        v = v + rng.uniform(-0.5, 0.5, v.size).astype(np.float32) * (rng.random(v.size) < 0.5)
        e = np.empty(rows, np.int16)
        r = np.empty(rows, np.int16)
        bad = lib.check_mean(p(np.ascontiguousarray(v, np.float32)), rows, k, p(e), p(r))
        assert bad == 0, (k, bad)
