"""TEST INFRASTRUCTURE -- the parity oracle for MonkeyGL's ray-casting path.

Only tests/, __graft_entry__.smoke() and bench.py (CPU baseline and reference
arm) import this package.  The product library never does.

* ``cpu``      -- ctypes wrapper of lib/libmkoracle.so, the C restatement in
                  mk_oracle.c (texture-emulating FP32 and exact FP64 modes).
* ``RefGPU``   -- MonkeyGL's own CUDA kernels (_ref/libmkref_gpu.so, built from
                  the unmodified core/kernel.cu and core/CuDataManager.cu).
* ``RefHost``  -- MonkeyGL's own host library with kernel-argument capture
                  (_ref/libmkref_host.so), used to generate golden vectors.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
CPU_LIB = HERE / "lib" / "libmkoracle.so"
REF_GPU_LIB = HERE / "_ref" / "libmkref_gpu.so"
REF_HOST_LIB = HERE / "_ref" / "libmkref_host.so"
LABELS = 65
VR_FLOATS = 32 + 3 * LABELS

TEX32, EXACT64 = 0, 1


def _vp(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


class _MkoVolume(C.Structure):
    _fields_ = [("vox", C.c_void_p), ("dim", C.c_int * 3), ("mask", C.c_void_p),
                ("lut", C.c_void_p * LABELS), ("lut_len", C.c_int * LABELS)]


_cpu = None


def cpu():
    global _cpu
    if _cpu is None:
        if not CPU_LIB.exists():
            raise FileNotFoundError(f"{CPU_LIB} missing; run `make -C oracle oracle`")
        L = C.CDLL(str(CPU_LIB))
        L.mko_render_vr.argtypes = [C.POINTER(_MkoVolume), C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int,
                                    C.c_int, C.c_void_p, C.POINTER(C.c_uint64)]
        L.mko_render_vr_rows.argtypes = [C.POINTER(_MkoVolume), C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int,
                                         C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.POINTER(C.c_uint64)]
        L.mko_render_plane.argtypes = [C.POINTER(_MkoVolume), C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int,
                                       C.c_int, C.c_int, C.c_void_p]
        L.mko_render_cpr.argtypes = [C.POINTER(_MkoVolume), C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int,
                                     C.c_int, C.c_int, C.c_void_p]
        L.mko_tex3d_linear.argtypes = [C.POINTER(_MkoVolume), C.c_float, C.c_float, C.c_float]
        L.mko_tex3d_linear.restype = C.c_float
        L.mko_tex3d_point.argtypes = [C.POINTER(_MkoVolume), C.c_float, C.c_float, C.c_float]
        L.mko_tex3d_point.restype = C.c_float
        L.mko_tex1d_lut.argtypes = [C.c_void_p, C.c_int, C.c_float, C.c_void_p]
        L.mko_set_weight_mode.argtypes = [C.c_int]
        _cpu = L
    return _cpu


class CpuVolume:
    """A volume for the CPU oracle (keeps its numpy buffers alive)."""

    def __init__(self, voxels, labels=None):
        self.vox = np.ascontiguousarray(voxels, dtype=np.int16)
        self.mask = None if labels is None else np.ascontiguousarray(labels, dtype=np.uint8)
        self.luts = [None] * LABELS
        self.s = _MkoVolume()
        self.s.vox = self.vox.ctypes.data
        dz, dy, dx = self.vox.shape
        self.s.dim[0], self.s.dim[1], self.s.dim[2] = dx, dy, dz
        self.s.mask = self.mask.ctypes.data if self.mask is not None else None

    def set_lut(self, label, lut):
        if lut is None:
            self.luts[label] = None
            self.s.lut[label] = None
            self.s.lut_len[label] = 0
            return
        t = np.ascontiguousarray(lut, dtype=np.float32).reshape(-1, 4)
        self.luts[label] = t
        self.s.lut[label] = t.ctypes.data
        self.s.lut_len[label] = t.shape[0]

    def render_vr(self, w, h, rtype, flat_params, precision=TEX32, threads=0, with_samples=False):
        out = np.zeros((h, w, 3), np.uint8)
        n = C.c_uint64(0)
        p = np.ascontiguousarray(flat_params, dtype=np.float32)
        rc = cpu().mko_render_vr(C.byref(self.s), w, h, rtype, _vp(p), precision, threads, _vp(out), C.byref(n))
        if rc:
            raise RuntimeError(f"mko_render_vr failed: {rc}")
        return (out, n.value) if with_samples else out

    def render_vr_rows(self, w, h, rtype, flat_params, row0, row_step, nrows, precision=TEX32, threads=0):
        out = np.zeros((nrows, w, 3), np.uint8)
        n = C.c_uint64(0)
        p = np.ascontiguousarray(flat_params, dtype=np.float32)
        rc = cpu().mko_render_vr_rows(C.byref(self.s), w, h, rtype, _vp(p), precision, threads, row0, row_step,
                                      nrows, _vp(out), C.byref(n))
        if rc:
            raise RuntimeError(f"mko_render_vr_rows failed: {rc}")
        return out, n.value

    def render_plane(self, w, h, flat_params, mpr_type, nearest, precision=TEX32, threads=0):
        out = np.zeros((h, w), np.int16)
        p = np.ascontiguousarray(flat_params, dtype=np.float32)
        rc = cpu().mko_render_plane(C.byref(self.s), w, h, _vp(p), mpr_type, int(nearest), precision, threads,
                                    _vp(out))
        if rc:
            raise RuntimeError(f"mko_render_plane failed: {rc}")
        return out

    def render_cpr(self, w, pts, dirs, invert_z, precision=TEX32, threads=0):
        pts = np.ascontiguousarray(pts, np.float64).reshape(-1, 3)
        dirs = np.ascontiguousarray(dirs, np.float64).reshape(-1, 3)
        h = pts.shape[0]
        out = np.zeros((h, w), np.int16)
        rc = cpu().mko_render_cpr(C.byref(self.s), w, h, _vp(pts), _vp(dirs), int(bool(invert_z)), precision,
                                  threads, _vp(out))
        if rc:
            raise RuntimeError(f"mko_render_cpr failed: {rc}")
        return out

    def tex3d_linear(self, x, y, z):
        return cpu().mko_tex3d_linear(C.byref(self.s), x, y, z)

    def tex3d_point(self, x, y, z):
        return cpu().mko_tex3d_point(C.byref(self.s), x, y, z)


def set_weight_mode(mode: int):
    cpu().mko_set_weight_mode(mode)


def ref_gpu_available() -> bool:
    return REF_GPU_LIB.exists()


class RefGPU:
    """MonkeyGL's own CUDA path (one global volume, as in MonkeyGL)."""

    _L = None

    def __init__(self):
        if RefGPU._L is None:
            if not REF_GPU_LIB.exists():
                raise FileNotFoundError(f"{REF_GPU_LIB} missing; run `make -C oracle ref-gpu`")
            L = C.CDLL(str(REF_GPU_LIB))
            L.mkref_volume.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int]
            L.mkref_mask.argtypes = [C.c_void_p]
            L.mkref_tf.argtypes = [C.c_int, C.c_void_p, C.c_int]
            L.mkref_render.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int]
            L.mkref_render_kernel_ms.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int]
            L.mkref_render_kernel_ms.restype = C.c_double
            L.mkref_plane.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int]
            L.mkref_cpr.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int]
            L.mkref_select.argtypes = [C.c_int]
            RefGPU._L = L
        self.L = RefGPU._L

    def device_count(self):
        return self.L.mkref_device_count()

    def select(self, slot):
        """Make resident volume slot 0..7 the one later calls use (slot 0
        by default); each slot keeps its own volume, mask and LUTs."""
        assert self.L.mkref_select(slot) == 0

    def set_volume(self, vox):
        self.vox = np.ascontiguousarray(vox, dtype=np.int16)
        dz, dy, dx = self.vox.shape
        assert self.L.mkref_volume(_vp(self.vox), dx, dy, dz) == 0

    def set_mask(self, labels):
        if labels is None:
            assert self.L.mkref_mask(None) == 0
        else:
            m = np.ascontiguousarray(labels, dtype=np.uint8)
            assert self.L.mkref_mask(_vp(m)) == 0

    def clear_tfs(self):
        self.L.mkref_clear_tfs()

    def set_lut(self, label, lut):
        t = np.ascontiguousarray(lut, dtype=np.float32).reshape(-1, 4)
        assert self.L.mkref_tf(label, _vp(t), t.shape[0]) == 0

    def render(self, w, h, rtype, flat_params):
        out = np.zeros((h, w, 3), np.uint8)
        p = np.ascontiguousarray(flat_params, dtype=np.float32)
        assert self.L.mkref_render(_vp(out), w, h, _vp(p), rtype) == 0
        return out

    def render_into(self, out, w, h, rtype, p):
        return self.L.mkref_render(_vp(out), w, h, _vp(p), rtype)

    def kernel_ms(self, w, h, rtype, flat_params, reps=5):
        p = np.ascontiguousarray(flat_params, dtype=np.float32)
        return self.L.mkref_render_kernel_ms(w, h, _vp(p), rtype, reps)

    def plane(self, w, h, flat_params, mpr_type, nearest):
        out = np.zeros((h, w), np.int16)
        p = np.ascontiguousarray(flat_params, dtype=np.float32)
        assert self.L.mkref_plane(_vp(out), w, h, _vp(p), mpr_type, int(nearest)) == 0
        return out

    def cpr(self, w, pts, dirs, invert_z):
        pts = np.ascontiguousarray(pts, np.float64).reshape(-1, 3)
        dirs = np.ascontiguousarray(dirs, np.float64).reshape(-1, 3)
        h = pts.shape[0]
        out = np.zeros((h, w), np.int16)
        assert self.L.mkref_cpr(_vp(out), w, h, _vp(pts), _vp(dirs), int(bool(invert_z))) == 0
        return out


REF_FULL_LIB = HERE / "_ref" / "libmkref_full.so"


def ref_full_available() -> bool:
    return REF_FULL_LIB.exists() and (HERE / "_ref" / "resources" / "human.stl").exists()


class RefHelloMonkey:
    """MonkeyGL's complete HelloMonkey (its host code and kernels, built
    unmodified into _ref/libmkref_full.so), driven through the mkrh_*
    functions of ref_host_capture.cpp.  MonkeyGL keeps one process-wide
    state, so every instance drives the same singleton."""

    _L = None
    _h = None

    def __init__(self):
        if RefHelloMonkey._L is None:
            if not ref_full_available():
                raise FileNotFoundError(f"{REF_FULL_LIB} missing; run `make -C oracle ref`")
            L = C.CDLL(str(REF_FULL_LIB))
            vp = C.c_void_p
            L.mkrh_create.restype = vp
            L.mkrh_create.argtypes = [C.c_char_p]
            for f, a in {
                "mkrh_set_volume": [vp, vp, C.c_int, C.c_int, C.c_int], "mkrh_set_spacing": [vp, C.c_double,
                                                                                              C.c_double, C.c_double],
                "mkrh_set_direction": [vp, vp], "mkrh_set_wwwl": [vp, C.c_float, C.c_float, C.c_int],
                "mkrh_orientation": [vp, C.c_int], "mkrh_rotate": [vp, C.c_float, C.c_float],
                "mkrh_set_vr_size": [vp, C.c_int, C.c_int], "mkrh_vr_image": [vp, vp, C.c_longlong, vp],
                "mkrh_set_tf": [vp, vp, vp, C.c_int, vp, vp, C.c_int, C.c_int],
                "mkrh_set_cpr_line_voxel": [vp, vp, C.c_int],
            }.items():
                getattr(L, f).argtypes = a
            assert L.mkrh_zero_heap(1) == 1
            RefHelloMonkey._L = L
            RefHelloMonkey._h = L.mkrh_create(str(REF_FULL_LIB.parent).encode())
        self.L, self.h = RefHelloMonkey._L, RefHelloMonkey._h
        self.L.mkrh_set_cpr_line_voxel(self.h, _vp(np.zeros((1, 3))), 0)
        self._img = np.zeros(4096 * 4096 * 3, np.uint8)

    def set_volume(self, vox, spacing, direction=(1, 0, 0, 0, 1, 0, 0, 0, -1)):
        self.vox = np.ascontiguousarray(vox, np.int16)
        Z, Y, X = self.vox.shape
        self.L.mkrh_set_volume(self.h, _vp(self.vox), X, Y, Z)
        self.L.mkrh_set_direction(self.h, _vp(np.asarray(direction, np.float64)))
        self.L.mkrh_set_spacing(self.h, *[float(s) for s in spacing])

    def set_transfer_function(self, points, label=-1):
        """points: {position 0..99: (r, g, b, a)}"""
        pos = np.array(list(points), np.int32)
        val = np.array([points[k] for k in points], np.float32)
        z = np.zeros(1, np.int32)
        return self.L.mkrh_set_tf(self.h, _vp(pos), _vp(val), len(pos), _vp(z), _vp(z.astype(np.float32)), 0, label)

    def set_wwwl(self, ww, wl, label=-1):
        return self.L.mkrh_set_wwwl(self.h, ww, wl, label)

    def orientation(self, which):
        self.L.mkrh_orientation(self.h, which)

    def rotate(self, fx, fy):
        self.L.mkrh_rotate(self.h, fx, fy)

    def set_vr_size(self, w, h):
        return self.L.mkrh_set_vr_size(self.h, w, h)

    def vr_image(self):
        wh = np.zeros(2, np.int32)
        assert self.L.mkrh_vr_image(self.h, _vp(self._img), self._img.size, _vp(wh)) == 1
        w, h = int(wh[0]), int(wh[1])
        return self._img[: w * h * 3].reshape(h, w, 3)
