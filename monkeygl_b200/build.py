"""Build the native library in-tree for sm_100a.

Produces ``monkeygl_b200/lib/libmonkeygl_b200.so`` (CUDA kernels, volume
residency, host geometry and the C ABI of ``include/monkeygl_b200.h``).
Objects are compiled in parallel and rebuilt only when a source or header is
newer than the library.  Run ``python -m monkeygl_b200.build``.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIBDIR = PKG / "lib"
OBJDIR = PKG / "lib" / "obj"
LIBNAME = "libmonkeygl_b200.so"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-O3", f"-I{ROOT / 'include'}", f"-I{CSRC}",
]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fopenmp",
             f"-I{ROOT / 'include'}", f"-I{CSRC}", "-I/usr/local/cuda/include"]


def _sources():
    cu = sorted(p for p in CSRC.glob("*.cu"))
    cpp = sorted(p for p in CSRC.glob("*.cpp") if not p.name.startswith("py"))
    return cu, cpp


def _headers():
    return list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list((ROOT / "include").rglob("*.h"))


def _newest(paths):
    return max((p.stat().st_mtime for p in paths), default=0.0)


def _compile(src: Path, obj: Path, verbose: bool):
    if src.suffix == ".cu":
        cmd = [NVCC] + NVCC_FLAGS + ["-c", str(src), "-o", str(obj)]
    else:
        cmd = ["g++"] + CXX_FLAGS + ["-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {src.name}\n{r.stdout}\n{r.stderr}")
    return r.stderr


def library_path() -> Path:
    return LIBDIR / LIBNAME


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile and link the native library; return its path."""
    cu, cpp = _sources()
    LIBDIR.mkdir(parents=True, exist_ok=True)
    OBJDIR.mkdir(parents=True, exist_ok=True)
    lib = library_path()
    hdr_time = _newest(_headers())
    jobs = []
    objs = []
    for src in cu + cpp:
        obj = OBJDIR / (src.name + ".o")
        objs.append(obj)
        if force or not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, hdr_time):
            jobs.append((src, obj))
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            futs = [ex.submit(_compile, s, o, verbose) for s, o in jobs]
            for f in futs:
                f.result()
    if force or jobs or not lib.exists() or lib.stat().st_mtime < _newest(objs):
        tmp = lib.with_suffix(".so.tmp")
        cmd = [NVCC] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", str(tmp)] + \
              [str(o) for o in objs] + ["-lcudart_static", "-lrt", "-lpthread", "-ldl", "-lz", "-lgomp"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, lib)
    return lib


def build_python_module(force: bool = False, verbose: bool = False) -> Path:
    """Build the pyMonkeyGL extension (pybind11) next to the library."""
    import sysconfig
    import pybind11

    src = CSRC / "pymonkeygl.cpp"
    suffix = sysconfig.get_config_var("EXT_SUFFIX")
    out = LIBDIR / f"pyMonkeyGL{suffix}"
    lib = library_path()
    deps = [src, lib] + _headers() + list(CSRC.glob("host_*.cpp"))
    if not force and out.exists() and out.stat().st_mtime >= _newest(deps):
        return out
    inc = sysconfig.get_paths()["include"]
    cmd = ["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-ffp-contract=off",
           f"-I{pybind11.get_include()}", f"-I{inc}", f"-I{ROOT / 'include'}", f"-I{CSRC}",
           str(src), "-o", str(out), f"-L{LIBDIR}", "-lmonkeygl_b200",
           "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"pyMonkeyGL build failed\n{r.stdout}\n{r.stderr}")
    return out


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    force = "--force" in argv
    verbose = "-v" in argv or "--verbose" in argv
    lib = build(force=force, verbose=verbose)
    print(lib)
    if (CSRC / "pymonkeygl.cpp").exists():
        print(build_python_module(force=force, verbose=verbose))


if __name__ == "__main__":
    main()
