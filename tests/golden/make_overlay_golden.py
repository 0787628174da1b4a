"""Generate golden VR overlays from MonkeyGL's own host code.

MonkeyGL's host library (its core/*.cpp built unmodified into
oracle/_ref/libmkref_host.so, kernel launches captured, so its VR image
starts zero-filled) draws the VR provider's overlays over an empty image:

* the orientation box (core/VRImageLayer.cpp:99-194) for a set of camera
  rotations -- each case records RenderInfo's rotate matrix and the
  bottom-right 64x64 pixels of the 512x512 image;
* the CPR line layer (core/CPRLineLayer.cpp:40-65) over a camera view --
  the whole image, with the polyline's end points in image coordinates;
* Methods::DrawLineInImage24Bit (core/Methods.cpp:183-200) for seeded
  segments of several widths and colours.

HelloMonkey's constructor loads ./resources/human.stl, so the library runs
from the directory holding resources/ (the MonkeyGL source tree).

    make -C oracle ref-host && python tests/golden/make_overlay_golden.py [REF_DIR]

Writes tests/golden/overlay.npz.
"""
from __future__ import annotations

import ctypes as C
import os
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
LIB = ROOT / "oracle" / "_ref" / "libmkref_host.so"
OUT = Path(__file__).resolve().parent / "overlay.npz"

# camera sequences: (orientation preset, [(rotate fx, fy), ...])
CAMERAS = [(0, [])] + [(0, [(a, 0.0)]) for a in (10, 33, 45, 90, 137.5, 180, -60, 275)] + \
          [(0, [(30, 10), (-12.5, 40)]), (0, [(0, 75)]), (0, [(20, -35), (5, 5)])] + \
          [(i, [(15, 20)]) for i in range(1, 6)] + [(i, []) for i in range(1, 6)]

CPR_LINE = [[20.0 + 2.5 * i, 30.0 + 9.0 * np.sin(i / 3.0), 5.0 + 4.5 * i] for i in range(20)]


def main(ref_dir=None):
    """ref_dir: the MonkeyGL source tree (argument, else $MONKEYGL_SRC)."""
    ref_dir = ref_dir or os.environ.get("MONKEYGL_SRC")
    if not ref_dir:
        raise SystemExit("give the MonkeyGL source tree as an argument or in MONKEYGL_SRC")
    L = C.CDLL(str(LIB))
    vp = C.c_void_p
    L.mkrh_create.restype = vp
    L.mkrh_create.argtypes = [C.c_char_p]
    for f, args in {
        "mkrh_set_volume": [vp, vp, C.c_int, C.c_int, C.c_int], "mkrh_set_spacing": [vp, C.c_double, C.c_double,
                                                                                      C.c_double],
        "mkrh_set_direction": [vp, vp], "mkrh_orientation": [vp, C.c_int], "mkrh_rotate": [vp, C.c_float, C.c_float],
        "mkrh_vr_image": [vp, vp, C.c_longlong, vp], "mkrh_rotate_matrix": [vp],
        "mkrh_set_cpr_line_voxel": [vp, vp, C.c_int], "mkrh_destroy": [vp],
        "mkrh_draw_line": [vp, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int, C.c_float,
                           C.c_float, C.c_float],
    }.items():
        getattr(L, f).argtypes = args

    def ptr(a):
        return C.c_void_p(a.ctypes.data)

    h = L.mkrh_create(ref_dir.encode())
    X, Y, Z = 96, 80, 120
    vol = np.zeros((Z, Y, X), np.int16)
    L.mkrh_set_volume(h, ptr(vol), X, Y, Z)
    L.mkrh_set_spacing(h, 0.7, 0.7, 1.0)
    L.mkrh_set_direction(h, ptr(np.array([1, 0, 0, 0, 1, 0, 0, 0, -1], np.float64)))
    img = np.zeros(512 * 512 * 3, np.uint8)
    wh = np.zeros(2, np.int32)
    rots, boxes = [], []
    for preset, turns in CAMERAS:
        L.mkrh_orientation(h, preset)
        for fx, fy in turns:
            L.mkrh_rotate(h, fx, fy)
        m = np.zeros(9, np.float32)
        L.mkrh_rotate_matrix(ptr(m))
        img[:] = 0
        assert L.mkrh_vr_image(h, ptr(img), img.size, ptr(wh)) == 1 and tuple(wh) == (512, 512)
        im = img.reshape(512, 512, 3)
        outside = im.copy()
        outside[-64:, -64:] = 0
        assert not outside.any(), "MonkeyGL drew outside the orientation box"
        rots.append(m)
        boxes.append(im[-64:, -64:].copy())

    # CPR line over the anterior view turned by 30 degrees
    L.mkrh_orientation(h, 0)
    L.mkrh_rotate(h, 30.0, 0.0)
    line = np.ascontiguousarray(CPR_LINE, np.float64)
    L.mkrh_set_cpr_line_voxel(h, ptr(line), len(line))
    cpr_rot = np.zeros(9, np.float32)
    L.mkrh_rotate_matrix(ptr(cpr_rot))
    img[:] = 0
    assert L.mkrh_vr_image(h, ptr(img), img.size, ptr(wh)) == 1
    cpr_image = img.reshape(512, 512, 3).copy()
    L.mkrh_destroy(h)

    # line drawing: seeded segments, widths 1-3, on a 160x120 image
    rng = np.random.default_rng(4321)
    segs, line_imgs = [], []
    for i in range(40):
        x0, y0, x1, y1 = (rng.uniform(-20, 180), rng.uniform(-20, 140), rng.uniform(-20, 180), rng.uniform(-20, 140))
        if i % 10 == 0:
            x1, y1 = x0 + 0.3, y0      # short segment
        lw = int(rng.integers(1, 4))
        col = rng.uniform(0, 1, 3).astype(np.float32)
        li = np.zeros((120, 160, 3), np.uint8)
        L.mkrh_draw_line(ptr(li), 160, 120, x0, y0, x1, y1, lw, float(col[0]), float(col[1]), float(col[2]))
        segs.append([x0, y0, x1, y1, lw, col[0], col[1], col[2]])
        line_imgs.append(li)

    np.savez_compressed(OUT, rotations=np.array(rots), boxes=np.array(boxes), cpr_rotation=cpr_rot,
                        cpr_line=line, cpr_image=cpr_image, volume_dims=np.array([X, Y, Z]),
                        volume_spacing=np.array([0.7, 0.7, 1.0]), segments=np.array(segs, np.float32),
                        line_images=np.array(line_imgs))
    print(f"wrote {OUT}: {len(rots)} orientation boxes, {int((np.array(boxes) > 0).any(-1).sum())} box pixels drawn")


if __name__ == "__main__":
    main(*(sys.argv[1:2]))
