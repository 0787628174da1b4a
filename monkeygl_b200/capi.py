"""ctypes binding of the C ABI declared in include/monkeygl_b200.h.

The library is the in-tree ``monkeygl_b200/lib/libmonkeygl_b200.so``; there
is no fallback.  If it is missing, loading raises ``MonkeyGLError`` with the
build command.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libmonkeygl_b200.so"
MAX_LABELS = 65

MK_OK = 0
MK_ERR_INVALID_ARGUMENT = 1
MK_ERR_CUDA = 2
MK_ERR_OUT_OF_MEMORY = 3
MK_ERR_NOT_READY = 4
MK_ERR_BUDGET = 5
MK_ERR_TIMEOUT = 6
MK_ERR_NO_DEVICE = 7
MK_ERR_QUEUE_FULL = 8
STATUS = {
    0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "out of device memory", 4: "not ready",
    5: "device memory budget exceeded", 6: "timed out", 7: "no CUDA device", 8: "queue full",
}

RENDER_VR, RENDER_MIP, RENDER_SURFACE = 0, 1, 2
MPR_AVERAGE, MPR_MIP, MPR_MINIP = 0, 1, 2
SAMPLE_LINEAR, SAMPLE_NEAREST = 0, 1
PIXEL_RGB8, PIXEL_RGBA8 = 0, 1
VR_NO_SKIP = 0x1
VR_NO_COOP = 0x2
VR_NO_TAIL = 0x4


class MonkeyGLError(RuntimeError):
    def __init__(self, status, where, detail=""):
        self.status = status
        msg = f"{where}: {STATUS.get(status, status)}"
        if detail:
            msg += f" ({detail})"
        super().__init__(msg)


class VRParams(C.Structure):
    _fields_ = [
        ("width", C.c_int), ("height", C.c_int), ("render_type", C.c_int),
        ("max_len_spacing", C.c_float * 3), ("spacing", C.c_float * 3),
        ("spacing_voxel", C.c_float * 3), ("x_translate", C.c_float),
        ("y_translate", C.c_float), ("scale", C.c_float), ("transform", C.c_float * 9),
        ("invert_z", C.c_int), ("voi", C.c_int * 6), ("background", C.c_float * 4),
        ("pixel_format", C.c_int), ("flags", C.c_int),
    ]


class PlaneParams(C.Structure):
    _fields_ = [
        ("width", C.c_int), ("height", C.c_int), ("mpr_type", C.c_int), ("sampling", C.c_int),
        ("spacing", C.c_float * 3), ("dir_h", C.c_float * 3), ("dir_v", C.c_float * 3),
        ("dir_n", C.c_float * 3), ("left_top", C.c_float * 3), ("pixel_spacing", C.c_float),
        ("invert_z", C.c_int), ("half_num", C.c_float),
    ]



class DVRParams(C.Structure):
    """mk_dvr_params: one view of the differentiable renderer."""
    _fields_ = [
        ("width", C.c_int), ("height", C.c_int), ("dims", C.c_int * 3),
        ("max_len_spacing", C.c_float * 3), ("transform", C.c_float * 9),
        ("scale", C.c_float), ("x_translate", C.c_float), ("y_translate", C.c_float),
        ("step", C.c_float), ("t_min", C.c_float), ("lut_len", C.c_int),
    ]



REQUEST_VR, REQUEST_MIP, REQUEST_SURFACE, REQUEST_MPR = 0, 1, 2, 3


class ServerConfig(C.Structure):
    """mk_server_config."""
    _fields_ = [
        ("device", C.c_int), ("hbm_budget_bytes", C.c_size_t), ("max_slots", C.c_int),
        ("max_pending", C.c_int), ("max_pixels", C.c_int), ("lut_len", C.c_int), ("max_labels", C.c_int),
        ("max_bricks", C.c_int), ("tiles_per_step", C.c_int), ("evict_idle", C.c_int),
    ]


class Request(C.Structure):
    """mk_request."""
    _fields_ = [
        ("volume", C.c_int), ("kind", C.c_int), ("vr", VRParams), ("plane", PlaneParams),
        ("luts", C.c_void_p), ("n_luts", C.c_int), ("label_params", C.c_void_p), ("out", C.c_void_p),
        ("encoded", C.c_void_p), ("encoded_capacity", C.c_size_t),
    ]


class RequestTimes(C.Structure):
    _fields_ = [("submitted_ms", C.c_double), ("started_ms", C.c_double), ("completed_ms", C.c_double),
                ("encoded_length", C.c_size_t)]


class ServerStats(C.Structure):
    _fields_ = [
        ("submitted", C.c_uint64), ("completed", C.c_uint64), ("rejected", C.c_uint64), ("steps", C.c_uint64),
        ("tiles", C.c_uint64), ("evictions", C.c_uint64), ("loads", C.c_uint64),
        ("resident_bytes", C.c_size_t), ("budget_bytes", C.c_size_t),
        ("volumes", C.c_int), ("slots_busy", C.c_int), ("pending", C.c_int),
    ]


_lib = None

_SIGS = {
    "mk_status_string": (C.c_char_p, [C.c_int]),
    "mk_last_error": (C.c_char_p, []),
    "mk_device_count": (C.c_int, [C.POINTER(C.c_int)]),
    "mk_version": (C.c_char_p, []),
    "mk_volume_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int]),
    "mk_volume_destroy": (C.c_int, [C.c_void_p]),
    "mk_volume_device_bytes": (C.c_int, [C.c_void_p, C.POINTER(C.c_size_t)]),
    "mk_volume_dims": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "mk_volume_set_mask": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mk_volume_update_mask": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "mk_volume_brick_maps": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.c_void_p, C.c_void_p,
                                       C.POINTER(C.c_uint64)]),
    "mk_volume_set_transfer_function": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int]),
    "mk_volume_set_label_params": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "mk_render_vr": (C.c_int, [C.c_void_p, C.POINTER(VRParams), C.c_void_p, C.c_int, C.c_void_p]),
    "mk_count_vr_samples": (C.c_int, [C.c_void_p, C.POINTER(VRParams), C.POINTER(C.c_uint64)]),
    "mk_count_vr_footprint": (C.c_int, [C.c_void_p, C.POINTER(VRParams), C.POINTER(C.c_uint64),
                                        C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "mk_render_plane": (C.c_int, [C.c_void_p, C.POINTER(PlaneParams), C.c_void_p, C.c_int, C.c_void_p]),
    "mk_render_plane_u8": (C.c_int, [C.c_void_p, C.POINTER(PlaneParams), C.c_float, C.c_float,
                                     C.c_void_p, C.c_int, C.c_void_p]),
    "mk_render_cpr": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int,
                                C.c_void_p, C.c_int, C.c_void_p]),
    "mk_mesh_load_stl": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "mk_mesh_destroy": (C.c_int, [C.c_void_p]),
    "mk_mesh_facet_count": (C.c_int, [C.c_void_p]),
    "mk_merge_orientation_box": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int]),
    "mk_draw_line_rgb": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float,
                                   C.c_int, C.c_void_p]),
    "mk_encoded_capacity": (C.c_int, [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_size_t)]),
    "mk_encode_png_base64": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_size_t,
                                       C.POINTER(C.c_size_t)]),
    "mk_font_load": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "mk_font_destroy": (C.c_int, [C.c_void_p]),
    "mk_text_size": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "mk_draw_text_rgb": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_char_p, C.c_int, C.c_int,
                                   C.c_int, C.c_int, C.c_void_p]),
    "mk_render_cpr_noalloc": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int,
                                        C.c_void_p, C.c_void_p]),
    "mk_volume_synchronize": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mk_dvr_workspace_floats": (C.c_int, [C.POINTER(DVRParams), C.c_int, C.POINTER(C.c_size_t)]),
    "mk_dvr_forward": (C.c_int, [C.POINTER(DVRParams), C.c_int] + [C.c_void_p] * 6),
    "mk_dvr_backward": (C.c_int, [C.POINTER(DVRParams), C.c_int] + [C.c_void_p] * 7),
    "mk_server_create": (C.c_int, [C.POINTER(ServerConfig), C.POINTER(C.c_void_p)]),
    "mk_server_destroy": (C.c_int, [C.c_void_p]),
    "mk_server_add_volume": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                       C.POINTER(C.c_int)]),
    "mk_server_remove_volume": (C.c_int, [C.c_void_p, C.c_int]),
    "mk_server_submit": (C.c_int, [C.c_void_p, C.POINTER(Request), C.POINTER(C.c_uint64)]),
    "mk_server_wait": (C.c_int, [C.c_void_p, C.c_uint64, C.c_int, C.POINTER(RequestTimes)]),
    "mk_server_get_stats": (C.c_int, [C.c_void_p, C.POINTER(ServerStats)]),
}


def lib():
    """Load the native library (once)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise MonkeyGLError(4, "libmonkeygl_b200.so",
                                f"{LIB_PATH} is missing; build it with `python -m monkeygl_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    return list(_SIGS)


def _check(rc, where):
    if rc != MK_OK:
        detail = lib().mk_last_error().decode(errors="replace")
        raise MonkeyGLError(rc, where, detail)


def device_count() -> int:
    n = C.c_int(0)
    _check(lib().mk_device_count(C.byref(n)), "mk_device_count")
    return n.value


def _ptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)


class Volume:
    """A volume resident on one GPU (owns the mk_volume handle)."""

    def __init__(self, voxels: np.ndarray, device: int = 0):
        vox = np.ascontiguousarray(voxels, dtype=np.int16)
        if vox.ndim != 3:
            raise ValueError("voxels must be (dim_z, dim_y, dim_x)")
        dz, dy, dx = vox.shape
        h = C.c_void_p()
        _check(lib().mk_volume_create(C.byref(h), _ptr(vox), dx, dy, dz, device), "mk_volume_create")
        self.handle = h
        self.dims = (dx, dy, dz)
        self.device = device

    def close(self):
        if getattr(self, "handle", None):
            lib().mk_volume_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def device_bytes(self) -> int:
        n = C.c_size_t(0)
        _check(lib().mk_volume_device_bytes(self.handle, C.byref(n)), "mk_volume_device_bytes")
        return n.value

    def set_mask(self, labels: np.ndarray | None):
        if labels is None:
            _check(lib().mk_volume_set_mask(self.handle, None), "mk_volume_set_mask")
            return
        m = np.ascontiguousarray(labels, dtype=np.uint8)
        if m.shape != self.dims[::-1]:
            raise ValueError("label volume shape differs from the voxels")
        _check(lib().mk_volume_set_mask(self.handle, _ptr(m)), "mk_volume_set_mask")

    def update_mask(self, labels: np.ndarray, box):
        """Re-upload only box = (x0, y0, z0, x1, y1, z1) of the updated label
        volume `labels` (mk_volume_update_mask)."""
        m = np.ascontiguousarray(labels, dtype=np.uint8)
        if m.shape != self.dims[::-1]:
            raise ValueError("label volume shape differs from the voxels")
        b = (C.c_int * 6)(*[int(v) for v in box])
        _check(lib().mk_volume_update_mask(self.handle, _ptr(m), b), "mk_volume_update_mask")

    def brick_maps(self):
        """(minmax (nbz, nby, nbx, 2) int16, labels (nbz, nby, nbx, 3) uint32,
        present labels as a 65-entry bool array) of the occupancy maps."""
        nb = (C.c_int * 3)()
        _check(lib().mk_volume_brick_maps(self.handle, nb, None, None, None), "mk_volume_brick_maps")
        nbx, nby, nbz = nb[0], nb[1], nb[2]
        mm = np.empty((nbz, nby, nbx, 2), np.int16)
        lab = np.empty((nbz, nby, nbx, 3), np.uint32)
        pres = (C.c_uint64 * 2)()
        _check(lib().mk_volume_brick_maps(self.handle, nb, _ptr(mm), _ptr(lab), pres), "mk_volume_brick_maps")
        present = np.array([(pres[l >> 6] >> (l & 63)) & 1 for l in range(MAX_LABELS)], bool)
        return mm, lab, present

    def set_transfer_function(self, label: int, lut: np.ndarray | None):
        if lut is None:
            _check(lib().mk_volume_set_transfer_function(self.handle, label, None, 0),
                   "mk_volume_set_transfer_function")
            return
        t = np.ascontiguousarray(lut, dtype=np.float32).reshape(-1, 4)
        _check(lib().mk_volume_set_transfer_function(self.handle, label, _ptr(t), t.shape[0]),
               "mk_volume_set_transfer_function")

    def set_label_params(self, alpha_ww_wl: np.ndarray):
        p = np.ascontiguousarray(alpha_ww_wl, dtype=np.float32).reshape(-1, 3)
        _check(lib().mk_volume_set_label_params(self.handle, _ptr(p), p.shape[0]),
               "mk_volume_set_label_params")

    def render_vr(self, params: VRParams, out: np.ndarray | None = None) -> np.ndarray:
        ch = 4 if params.pixel_format == PIXEL_RGBA8 else 3
        if out is None:
            out = np.empty((params.height, params.width, ch), dtype=np.uint8)
        _check(lib().mk_render_vr(self.handle, C.byref(params), _ptr(out), 0, None), "mk_render_vr")
        return out

    def render_vr_device(self, params: VRParams, dptr: int, stream: int = 0):
        _check(lib().mk_render_vr(self.handle, C.byref(params), C.c_void_p(dptr), 1,
                                  C.c_void_p(stream) if stream else None), "mk_render_vr")

    def count_samples(self, params: VRParams) -> int:
        n = C.c_uint64(0)
        _check(lib().mk_count_vr_samples(self.handle, C.byref(params), C.byref(n)), "mk_count_vr_samples")
        return n.value

    def count_footprint(self, params: VRParams):
        """(samples, distinct voxels, distinct label voxels) of the reference schedule."""
        a, b, c = C.c_uint64(0), C.c_uint64(0), C.c_uint64(0)
        _check(lib().mk_count_vr_footprint(self.handle, C.byref(params), C.byref(a), C.byref(b), C.byref(c)),
               "mk_count_vr_footprint")
        return a.value, b.value, c.value

    def render_plane(self, params: PlaneParams, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty((params.height, params.width), dtype=np.int16)
        _check(lib().mk_render_plane(self.handle, C.byref(params), _ptr(out), 0, None), "mk_render_plane")
        return out

    def render_plane_device(self, params: PlaneParams, dptr: int, stream: int = 0):
        _check(lib().mk_render_plane(self.handle, C.byref(params), C.c_void_p(dptr), 1,
                                     C.c_void_p(stream) if stream else None), "mk_render_plane")

    def render_plane_u8(self, params: PlaneParams, ww: float, wl: float) -> np.ndarray:
        out = np.empty((params.height, params.width), dtype=np.uint8)
        _check(lib().mk_render_plane_u8(self.handle, C.byref(params), ww, wl, _ptr(out), 0, None),
               "mk_render_plane_u8")
        return out

    def render_cpr(self, width: int, points: np.ndarray, dirs: np.ndarray, invert_z: bool,
                   out: np.ndarray | None = None) -> np.ndarray:
        pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
        drs = np.ascontiguousarray(dirs, dtype=np.float64).reshape(-1, 3)
        h = pts.shape[0]
        if out is None:
            out = np.empty((h, width), dtype=np.int16)
        _check(lib().mk_render_cpr(self.handle, width, h, _ptr(pts), _ptr(drs), int(bool(invert_z)),
                                   _ptr(out), 0, None), "mk_render_cpr")
        return out

    def synchronize(self):
        _check(lib().mk_volume_synchronize(self.handle, None), "mk_volume_synchronize")


def vr_params(width, height, render_type, camera, dims, spacing, invert_z=False, background=(0, 0, 0, 0),
              voi=None, pixel_format=PIXEL_RGB8, flags=0) -> VRParams:
    """Build the cu_render argument block from a camera.Camera and geometry."""
    from .camera import volume_factors

    mls, sv = volume_factors(dims, spacing)
    p = VRParams()
    p.width, p.height, p.render_type = int(width), int(height), int(render_type)
    for k in range(3):
        p.max_len_spacing[k] = mls[k]
        p.spacing[k] = float(np.float32(spacing[k]))
        p.spacing_voxel[k] = sv[k]
    p.x_translate = float(camera.x_translate)
    p.y_translate = float(camera.y_translate)
    p.scale = float(camera.scale)
    for i, m in enumerate(camera.flat()):
        p.transform[i] = m
    p.invert_z = int(bool(invert_z))
    if voi is None:
        voi = (0, dims[0] - 1, 0, dims[1] - 1, 0, dims[2] - 1)
    for i in range(6):
        p.voi[i] = int(voi[i])
    for i in range(4):
        p.background[i] = float(background[i])
    p.pixel_format = int(pixel_format)
    p.flags = int(flags)
    return p


def vr_params_flat(p: VRParams, label_params: np.ndarray) -> np.ndarray:
    """The flat float block (oracle / reference harness layout) for `p`."""
    f = np.zeros(32 + 3 * MAX_LABELS, dtype=np.float32)
    f[0:3] = list(p.max_len_spacing)
    f[3:6] = list(p.spacing)
    f[6:9] = list(p.spacing_voxel)
    f[9], f[10], f[11] = p.x_translate, p.y_translate, p.scale
    f[12:21] = list(p.transform)
    f[21] = p.invert_z
    f[22:28] = list(p.voi)
    f[28:32] = list(p.background)
    lp = np.asarray(label_params, dtype=np.float32).reshape(-1, 3)
    f[32:32 + lp.size] = lp.ravel()
    return f


def plane_params(width, height, mpr_type, sampling, spacing, dir_h, dir_v, dir_n, left_top,
                 pixel_spacing, invert_z, half_num) -> PlaneParams:
    p = PlaneParams()
    p.width, p.height, p.mpr_type, p.sampling = int(width), int(height), int(mpr_type), int(sampling)
    for k in range(3):
        p.spacing[k] = float(spacing[k])
        p.dir_h[k] = float(dir_h[k])
        p.dir_v[k] = float(dir_v[k])
        p.dir_n[k] = float(dir_n[k])
        p.left_top[k] = float(left_top[k])
    p.pixel_spacing = float(pixel_spacing)
    p.invert_z = int(bool(invert_z))
    p.half_num = float(half_num)
    return p


def plane_params_flat(p: PlaneParams) -> np.ndarray:
    f = np.zeros(18, dtype=np.float32)
    f[0:3] = list(p.spacing)
    f[3:6] = list(p.dir_h)
    f[6:9] = list(p.dir_v)
    f[9:12] = list(p.dir_n)
    f[12:15] = list(p.left_top)
    f[15] = p.pixel_spacing
    f[16] = p.invert_z
    f[17] = p.half_num
    return f
