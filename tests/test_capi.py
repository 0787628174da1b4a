"""The C ABI of include/monkeygl_b200.h without a GPU: the library loads,
exports every declared entry point, validates arguments before touching the
device and reports a missing device as MK_ERR_NO_DEVICE instead of exiting
(MonkeyGL's checkCudaErrors exits the process, cuda_common/helper_cuda.h)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from monkeygl_b200 import capi

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "monkeygl_b200.h"


def declared_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:int|const char \*|void)\s+\*?\s*(mk_\w+)\s*\(", text, re.M)))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("mk_volume_create", "mk_render_vr", "mk_render_plane", "mk_render_cpr",
                 "mk_volume_set_mask", "mk_volume_set_transfer_function"):
        assert must in names


def test_library_exports_every_declared_symbol():
    L = capi.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(declared_functions()) <= set(capi.exported_symbols())


def test_header_constants_match_binding():
    # every #define MK_* integer constant that the Python binding mirrors has the header's value
    defines = dict((m.group(1), int(m.group(2), 0)) for m in
                   re.finditer(r"^#define\s+MK_(\w+)\s+(0x[0-9a-fA-F]+|\d+)\b", HEADER.read_text(), re.M))
    for name in ("VR_NO_SKIP", "VR_NO_COOP", "VR_NO_TAIL", "RENDER_VR", "RENDER_MIP", "RENDER_SURFACE"):
        if name in defines and hasattr(capi, name):
            assert getattr(capi, name) == defines[name], name
    assert defines["VR_NO_TAIL"] == capi.VR_NO_TAIL
    flags = [defines[n] for n in ("VR_NO_SKIP", "VR_NO_COOP", "VR_NO_TAIL")]
    assert len(set(flags)) == 3 and all(f & (f - 1) == 0 for f in flags)   # distinct single bits


def test_status_strings():
    L = capi.lib()
    assert L.mk_status_string(0) == b"ok"
    assert L.mk_status_string(7) == b"no CUDA device"
    assert L.mk_status_string(999) == b"unknown status"
    assert L.mk_version().decode().count(".") == 2


def test_device_count_never_fails():
    assert capi.device_count() >= 0


def test_create_validates_before_device():
    L = capi.lib()
    h = C.c_void_p()
    vox = np.zeros(8, np.int16)
    assert L.mk_volume_create(C.byref(h), None, 2, 2, 2, 0) == capi.MK_ERR_INVALID_ARGUMENT
    assert L.mk_volume_create(C.byref(h), C.c_void_p(vox.ctypes.data), 0, 2, 2, 0) == 1
    assert L.mk_volume_create(None, C.c_void_p(vox.ctypes.data), 2, 2, 2, 0) == 1
    assert b"dimension" in L.mk_last_error() or b"null" in L.mk_last_error()


def test_entry_points_reject_null_handles():
    L = capi.lib()
    p = capi.VRParams()
    buf = np.zeros(16, np.uint8)
    assert L.mk_render_vr(None, C.byref(p), C.c_void_p(buf.ctypes.data), 0, None) == 1
    assert L.mk_render_plane(None, C.byref(capi.PlaneParams()), C.c_void_p(buf.ctypes.data), 0, None) == 1
    assert L.mk_render_cpr(None, 4, 4, None, None, 0, None, 0, None) == 1
    assert L.mk_volume_set_mask(None, None) == 1
    box = (C.c_int * 6)(0, 0, 0, 1, 1, 1)
    assert L.mk_volume_update_mask(None, C.c_void_p(buf.ctypes.data), box) == 1
    assert L.mk_volume_update_mask(None, None, None) == 1
    assert L.mk_volume_set_transfer_function(None, 0, None, 0) == 1
    assert L.mk_volume_set_label_params(None, None, 1) == 1
    assert L.mk_volume_destroy(None) == 1
    n = C.c_uint64()
    assert L.mk_count_vr_samples(None, C.byref(p), C.byref(n)) == 1


@pytest.mark.skipif(capi.device_count() > 0, reason="a CUDA device is present")
def test_no_device_is_a_status_not_an_exit():
    with pytest.raises(capi.MonkeyGLError) as ei:
        capi.Volume(np.zeros((4, 4, 4), np.int16))
    assert ei.value.status == 7


def test_dvr_host_validation():
    """mk_dvr_* check their views on the host, before any launch."""
    from monkeygl_b200 import dvr
    from monkeygl_b200.camera import view_camera
    a = dvr.dvr_params(64, 48, view_camera(0.0), (32, 32, 32), (1, 1, 1), 0.5, 0.0, 256)
    b = dvr.dvr_params(64, 48, view_camera(30.0), (32, 32, 32), (1, 1, 1), 0.25, 0.0, 256)
    # checkpoint planes (16 samples apart, 1.74/step + 2 samples), a plane of counts and one of
    # final transmittances
    per = lambda p: (((int(1.74 / p.step) + 2 + 15) // 16) + 2) * 64 * 48
    assert dvr.workspace_floats([a]) == per(a)
    assert dvr.workspace_floats([a, b]) == per(a) + per(b)
    L = dvr._lib()
    n = C.c_size_t(0)
    c = dvr.dvr_params(32, 48, view_camera(0.0), (32, 32, 32), (1, 1, 1))
    for bad in ([a, c],):                                        # differing widths
        arr, nv = dvr.view_array(bad)
        assert L.mk_dvr_workspace_floats(arr, nv, C.byref(n)) == capi.MK_ERR_INVALID_ARGUMENT
    for field, value in (("lut_len", 1), ("lut_len", 2000), ("step", 0.0), ("scale", 0.0), ("width", 0)):
        p = dvr.dvr_params(64, 48, view_camera(0.0), (32, 32, 32), (1, 1, 1))
        setattr(p, field, value)
        arr, nv = dvr.view_array([p])
        assert L.mk_dvr_workspace_floats(arr, nv, C.byref(n)) == capi.MK_ERR_INVALID_ARGUMENT
        assert L.mk_dvr_forward(arr, nv, C.c_void_p(16), C.c_void_p(16), C.c_void_p(16), C.c_void_p(16),
                                None, None) == capi.MK_ERR_INVALID_ARGUMENT
    arr, nv = dvr.view_array([a])
    assert L.mk_dvr_workspace_floats(arr, 0, C.byref(n)) == capi.MK_ERR_INVALID_ARGUMENT
    assert L.mk_dvr_forward(arr, nv, None, C.c_void_p(16), C.c_void_p(16), C.c_void_p(16), None,
                            None) == capi.MK_ERR_INVALID_ARGUMENT
    assert L.mk_dvr_backward(arr, nv, C.c_void_p(16), C.c_void_p(16), None, C.c_void_p(16), C.c_void_p(16),
                             None, None) == capi.MK_ERR_INVALID_ARGUMENT


def test_server_host_validation():
    """mk_server_create validates its configuration before touching a device
    and reports a machine without one as MK_ERR_NO_DEVICE."""
    L = capi.lib()
    h = C.c_void_p()

    def cfg(**kw):
        c = capi.ServerConfig()
        c.device, c.hbm_budget_bytes, c.max_slots, c.max_pending = 0, 0, 8, 16
        c.max_pixels, c.lut_len, c.max_labels, c.max_bricks, c.tiles_per_step = 1 << 20, 256, 8, 0, 0
        for k, v in kw.items():
            setattr(c, k, v)
        return c

    for bad in (dict(max_slots=0), dict(max_slots=257), dict(max_pending=0), dict(lut_len=1), dict(lut_len=5000),
                dict(max_labels=0), dict(max_labels=66), dict(max_pixels=0), dict(tiles_per_step=-1)):
        assert L.mk_server_create(C.byref(cfg(**bad)), C.byref(h)) == capi.MK_ERR_INVALID_ARGUMENT, bad
    assert L.mk_server_create(None, C.byref(h)) == capi.MK_ERR_INVALID_ARGUMENT
    n = C.c_int(-1)
    L.mk_device_count(C.byref(n))
    if n.value == 0:
        assert L.mk_server_create(C.byref(cfg()), C.byref(h)) == capi.MK_ERR_NO_DEVICE
    for fn, args in (("mk_server_destroy", (None,)), ("mk_server_remove_volume", (None, 1)),
                     ("mk_server_get_stats", (None, None)), ("mk_server_wait", (None, 1, 0, None))):
        assert getattr(L, fn)(*args) == capi.MK_ERR_INVALID_ARGUMENT, fn
