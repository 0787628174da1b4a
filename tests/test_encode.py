"""mk_encode_png_base64: the PNG + Base64 output form of MonkeyGL's
GetVRData_pngString / GetPlaneData_pngString (core/HelloMonkey.cpp:212-259,
333-413).  The bytes differ from MonkeyGL's fpng; the decoded pixels must
equal the input for RGB images and for int16 planes packed as W/2 RGBA
pixels, at sizes from 1x1 to 1024x1024 (one band to 64 bands of rows)."""
import ctypes as C

import numpy as np
import pytest

from monkeygl_b200 import capi
from pngcheck import decode_png_base64


def encode(img):
    h, w, ch = img.shape
    cap = C.c_size_t(0)
    assert capi.lib().mk_encoded_capacity(w, h, ch, C.byref(cap)) == capi.MK_OK
    out = np.full(cap.value, 0x55, np.uint8)
    n = C.c_size_t(0)
    rc = capi.lib().mk_encode_png_base64(np.ascontiguousarray(img).ctypes.data, w, h, ch, out.ctypes.data,
                                         cap.value, C.byref(n))
    assert rc == capi.MK_OK, capi.lib().mk_last_error()
    assert out[n.value] == 0 and n.value < cap.value
    return out[:n.value].tobytes().decode("ascii")


@pytest.mark.parametrize("shape", [(1, 1, 3), (2, 5, 4), (31, 17, 3), (32, 64, 4), (33, 100, 3),
                                   (2048, 3, 3), (1024, 1024, 3), (512, 256, 4)])
def test_round_trip(shape):
    rng = np.random.default_rng(sum(shape))
    img = rng.integers(0, 256, shape, dtype=np.uint8)
    img[: shape[0] // 2] //= 64                        # compressible rows too
    assert np.array_equal(decode_png_base64(encode(img)), img)


def test_int16_plane_as_rgba():
    # MonkeyGL hands fpng the int16 plane as W/2 RGBA pixels of its bytes
    rng = np.random.default_rng(5)
    plane = rng.integers(-32768, 32768, (512, 308), dtype=np.int32).astype(np.int16)
    rgba = plane.view(np.uint8).reshape(512, 154, 4)
    dec = decode_png_base64(encode(rgba))
    assert np.array_equal(dec.reshape(512, -1).view(np.int16), plane)


def test_refusals():
    img = np.zeros((4, 4, 3), np.uint8)
    n = C.c_size_t(0)
    out = np.zeros(8, np.uint8)
    assert capi.lib().mk_encode_png_base64(img.ctypes.data, 4, 4, 3, out.ctypes.data, 8, C.byref(n)) != capi.MK_OK
    cap = C.c_size_t(0)
    assert capi.lib().mk_encoded_capacity(4, 4, 2, C.byref(cap)) != capi.MK_OK
    assert capi.lib().mk_encode_png_base64(img.ctypes.data, 0, 4, 3, out.ctypes.data, 8, C.byref(n)) != capi.MK_OK
