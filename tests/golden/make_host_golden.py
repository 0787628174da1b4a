"""Generate golden vectors from MonkeyGL's own host code.

Runs MonkeyGL's HelloMonkey API (its core/*.cpp, built unmodified into
oracle/_ref/libmkref_host.so with kernel-argument capture) through a list of
operation sequences and records the arguments its host code hands to the
CUDA launchers: camera matrix, volume factors, label windows and caps, plane
frames, CPR frames, plus TransferFunction LUTs.  Needs the MonkeyGL source
tree (for building the library and for resources/human.stl, which
HelloMonkey's constructor loads); the outputs are committed so the tests do
not.

    make -C oracle ref-host && python tests/golden/make_host_golden.py [REF_DIR]

Writes tests/golden/host_geometry.json (scenarios and results).
"""
from __future__ import annotations

import ctypes as C
import os
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
LIB = ROOT / "oracle" / "_ref" / "libmkref_host.so"
OUT = Path(__file__).resolve().parent / "host_geometry.json"

# Each scenario: volume dims/spacing/direction, a list of operations, and the
# captures to take (("vr", w, h) or ("plane", plane_type)).
SCENARIOS = []


def scen(name, dims, spacing, ops, captures, direction=(1, 0, 0, 0, 1, 0, 0, 0, -1), masks=0):
    SCENARIOS.append(dict(name=name, dims=list(dims), spacing=list(spacing), direction=list(direction),
                          ops=ops, captures=captures, masks=masks))


SMALL = ((128, 128, 96), (0.35, 0.35, 0.3))
CARD = ((64, 64, 40), (0.351, 0.351, 0.3))
BODY = ((48, 48, 150), (0.7422, 0.7422, 1.0))

# camera sequences
scen("anterior", *SMALL, [["orientation", 0]], [["vr", 512, 512]])
for ang in (0, 45, 90, 30, 137.5, -60):
    scen(f"rot_z_{ang}", *SMALL, [["orientation", 0], ["rotate", ang, 0]], [["vr", 512, 512]])
for i, o in enumerate(["anterior", "posterior", "left", "right", "head", "foot"]):
    scen(f"preset_{o}", *SMALL, [["rotate", 20, 10], ["orientation", i]], [["vr", 512, 512]])
scen("rot_xy", *SMALL, [["orientation", 0], ["rotate", 30, 10], ["rotate", -12.5, 40]], [["vr", 512, 512]])
scen("rot_accum36", *SMALL, [["orientation", 0]] + [["rotate", 10, 0]] * 36, [["vr", 512, 512]])
scen("zoom_pan", *SMALL, [["orientation", 0], ["zoom", 1.5], ["rotate", 30, 10], ["pan", 5, -3],
                          ["zoom", 0.8]], [["vr", 512, 512]])
scen("preset_resets_zoom", *SMALL, [["zoom", 2.0], ["pan", 7, 7], ["orientation", 1]], [["vr", 512, 512]])
for w, h in [(512, 512), (1024, 1024), (2048, 2048), (1000, 999), (777, 300), (1500, 1000)]:
    scen(f"vrsize_{w}x{h}", *SMALL, [["orientation", 0], ["vr_size", w, h]], [["vr", w, h]])
scen("cardiac_view", *CARD, [["orientation", 0], ["rotate", 30, 0]], [["vr", 1024, 1024]])
scen("body_view", *BODY, [["orientation", 0], ["rotate", 45, 0]], [["vr", 1024, 1024]])
scen("invert_z", *SMALL, [["orientation", 0], ["rotate", 45, 0]], [["vr", 512, 512], ["plane", 0], ["plane", 2]],
     direction=(1, 0, 0, 0, 1, 0, 0, 0, 1))
scen("render_types", *SMALL, [["orientation", 0], ["render_type", 1]], [["vr", 512, 512]])
scen("background", *SMALL, [["orientation", 0], ["background", 0.1, 0.2, 0.3, 1.0]], [["vr", 512, 512]])
# label windows and caps
scen("labels_default", *SMALL, [["orientation", 0]], [["vr", 256, 256]], masks=2)
scen("labels_set", *SMALL, [["orientation", 0], ["wwwl", 1700, 650, -1], ["alpha", 0.8, 0], ["alpha", 0.5, 1],
                            ["wwwl", 500, 300, 2], ["wwwl", -3, 10, 1], ["alpha", 1.0, 2]],
     [["vr", 256, 256]], masks=2)
scen("labels_bg04", *BODY, [["orientation", 0], ["alpha", 0.4, 0]], [["vr", 256, 256]], masks=4)
# MPR planes
scen("mpr_default", *CARD, [], [["plane", t] for t in range(6)])
scen("mpr_small", *SMALL, [], [["plane", t] for t in range(6)])
scen("mpr_body", *BODY, [], [["plane", t] for t in range(6)])
scen("mpr_thick_mip", *CARD, [["mpr_type", 1], ["thickness", 2.0, 0], ["thickness", 1.5, 1]],
     [["plane", 0], ["plane", 1], ["plane", 2]])
scen("mpr_update_thick_minip", *CARD, [["mpr_type", 2], ["update_thickness", 3.3]],
     [["plane", t] for t in range(6)])
scen("mpr_browse", *CARD, [["browse", 3.0, 0], ["browse", -2.5, 1], ["browse", 1.0, 2]],
     [["plane", t] for t in range(6)])
scen("mpr_rotate_crosshair", *CARD, [["rotate_crosshair", 30, 3], ["rotate_crosshair", -20, 4]],
     [["plane", t] for t in range(6)])
scen("mpr_pan_crosshair", *CARD, [["pan_crosshair", 10, 12, 0], ["pan_crosshair", 5, 20, 4]],
     [["plane", t] for t in range(6)])
scen("mpr_plane_index", *CARD, [["plane_index", 10, 0], ["plane_index", 40, 1]], [["plane", t] for t in range(3)])
# CPR
CPR_LINE = [[20.0 + 0.5 * i, 30.0 + 6.0 * np.sin(i / 3.0), 5.0 + 1.5 * i] for i in range(20)]
scen("cpr_basic", *CARD, [["cpr_line", CPR_LINE]], [["plane", 7], ["plane", 8]])
scen("cpr_rotated", *CARD, [["cpr_line", CPR_LINE], ["rotate_cpr", 30, 7], ["rotate_cpr", 45, 8],
                            ["rotate_cpr", 15, 8]], [["plane", 7], ["plane", 8]])
scen("cpr_invert", *CARD, [["cpr_line", CPR_LINE]], [["plane", 7], ["plane", 8]],
     direction=(1, 0, 0, 0, 1, 0, 0, 0, 1))

# transfer functions: (rgb points {pos: rgba}, alpha points {pos: a})
TF_CASES = [
    ("default", {5: (0.8, 0.8, 0.8, 0.0), 95: (0.8, 0.8, 0.8, 0.8)}, {}),
    ("four_points", {0: (0.9, 0.3, 0.2, 0.0), 23: (0.95, 0.4, 0.3, 0.0), 50: (0.9, 0.7, 0.5, 0.35),
                     99: (1.0, 0.95, 0.9, 0.85)}, {}),
    ("with_alpha", {10: (1, 0, 0, 0.2), 60: (0, 1, 0, 0.5), 90: (0, 0, 1, 0.9)}, {20: 0.1, 40: 0.6, 70: 0.3}),
    ("out_of_range", {-5: (1, 1, 1, 1), 30: (0.5, 0.5, 0.5, 0.5), 120: (0, 0, 0, 0), 80: (0.2, 0.4, 0.6, 0.8)},
     {150: 0.4, 50: 0.2}),
    ("adjacent", {40: (0, 0, 0, 0), 41: (1, 1, 1, 1)}, {}),
    ("single", {50: (1, 1, 1, 1)}, {}),
]


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
        "mkrh_set_volume": [vp, vp, C.c_int, C.c_int, C.c_int], "mkrh_add_mask": [vp, vp, C.c_int, C.c_int, C.c_int],
        "mkrh_set_spacing": [vp, C.c_double, C.c_double, C.c_double], "mkrh_set_direction": [vp, vp],
        "mkrh_set_background": [vp, C.c_float, C.c_float, C.c_float, C.c_float],
        "mkrh_set_wwwl": [vp, C.c_float, C.c_float, C.c_int], "mkrh_set_alpha": [vp, C.c_float, C.c_int],
        "mkrh_set_render_type": [vp, C.c_int], "mkrh_orientation": [vp, C.c_int],
        "mkrh_rotate": [vp, C.c_float, C.c_float], "mkrh_zoom": [vp, C.c_float], "mkrh_pan": [vp, C.c_float, C.c_float],
        "mkrh_set_vr_size": [vp, C.c_int, C.c_int], "mkrh_set_mpr_type": [vp, C.c_int],
        "mkrh_set_thickness": [vp, C.c_double, C.c_int], "mkrh_update_thickness": [vp, C.c_double],
        "mkrh_browse": [vp, C.c_float, C.c_int], "mkrh_pan_crosshair": [vp, C.c_float, C.c_float, C.c_int],
        "mkrh_rotate_crosshair": [vp, C.c_float, C.c_int], "mkrh_set_plane_index": [vp, C.c_int, C.c_int],
        "mkrh_get_plane_index": [vp, C.c_int], "mkrh_get_plane_number": [vp, C.c_int],
        "mkrh_set_cpr_line_voxel": [vp, vp, C.c_int], "mkrh_rotate_cpr": [vp, C.c_float, C.c_int],
        "mkrh_get_vr": [vp, C.c_int, C.c_int], "mkrh_get_plane": [vp, C.c_int, vp], "mkrh_copy_vr": [vp],
        "mkrh_copy_plane": [vp], "mkrh_copy_cpr": [vp], "mkrh_destroy": [vp], "mkrh_crosshair": [vp, C.c_int, vp],
        "mkrh_direction3d": [vp, C.c_int, vp], "mkrh_pixel_spacing": [vp, C.c_int],
        "mkrh_tf_lut": [vp, vp, C.c_int, vp, vp, C.c_int, vp, C.c_int],
    }.items():
        getattr(L, f).argtypes = args
    L.mkrh_zoom.restype = C.c_float
    L.mkrh_pixel_spacing.restype = C.c_double

    def ptr(a):
        return C.c_void_p(a.ctypes.data)

    results = {}
    h = L.mkrh_create(ref_dir.encode())
    for sc in SCENARIOS:
        dims = sc["dims"]
        X, Y, Z = dims
        vol = np.zeros((Z, Y, X), np.int16)
        L.mkrh_set_volume(h, ptr(vol), X, Y, Z)
        d = np.array(sc["direction"], np.float64)
        L.mkrh_set_direction(h, ptr(d))
        L.mkrh_set_spacing(h, *sc["spacing"])
        # MonkeyGL's singleton keeps camera state across SetVolumeData; start
        # every scenario from the same camera (Anterior) and MPR state (Reset)
        L.mkrh_orientation(h, 0)
        L.mkrh_reset(h) if hasattr(L, "mkrh_reset") else None
        L.mkrh_set_vr_size(h, 512, 512)
        L.mkrh_set_render_type(h, 0)
        L.mkrh_set_mpr_type(h, 0)
        L.mkrh_set_background(h, 0, 0, 0, 0)
        labels = []
        for m in range(sc["masks"]):
            mask = np.zeros((Z, Y, X), np.uint8)
            mask[(m * Z) // max(1, sc["masks"]):((m + 1) * Z) // max(1, sc["masks"]), :, : X // 2] = 1
            labels.append(int(L.mkrh_add_mask(h, ptr(mask), X, Y, Z)))
        for op in sc["ops"]:
            k = op[0]
            if k == "orientation": L.mkrh_orientation(h, op[1])
            elif k == "rotate": L.mkrh_rotate(h, op[1], op[2])
            elif k == "zoom": L.mkrh_zoom(h, op[1])
            elif k == "pan": L.mkrh_pan(h, op[1], op[2])
            elif k == "vr_size": L.mkrh_set_vr_size(h, op[1], op[2])
            elif k == "render_type": L.mkrh_set_render_type(h, op[1])
            elif k == "background": L.mkrh_set_background(h, *op[1:5])
            elif k == "wwwl": L.mkrh_set_wwwl(h, op[1], op[2], op[3])
            elif k == "alpha": L.mkrh_set_alpha(h, op[1], op[2])
            elif k == "mpr_type": L.mkrh_set_mpr_type(h, op[1])
            elif k == "thickness": L.mkrh_set_thickness(h, op[1], op[2])
            elif k == "update_thickness": L.mkrh_update_thickness(h, op[1])
            elif k == "browse": L.mkrh_browse(h, op[1], op[2])
            elif k == "rotate_crosshair": L.mkrh_rotate_crosshair(h, op[1], op[2])
            elif k == "pan_crosshair": L.mkrh_pan_crosshair(h, op[1], op[2], op[3])
            elif k == "plane_index": L.mkrh_set_plane_index(h, op[1], op[2])
            elif k == "cpr_line":
                pts = np.array(op[1], np.float64)
                L.mkrh_set_cpr_line_voxel(h, ptr(pts), len(pts))
            elif k == "rotate_cpr": L.mkrh_rotate_cpr(h, op[1], op[2])
            else:
                raise ValueError(k)
        caps = []
        for cap in sc["captures"]:
            if cap[0] == "vr":
                n = L.mkrh_get_vr(h, cap[1], cap[2])
                buf = np.zeros(n, np.float64)
                L.mkrh_copy_vr(ptr(buf))
                caps.append(dict(kind="vr", args=buf.tolist()))
            else:
                wh = np.zeros(2, np.int32)
                n = L.mkrh_get_plane(h, cap[1], ptr(wh))
                buf = np.zeros(max(n, 0), np.float64)
                if cap[1] >= 7:
                    L.mkrh_copy_cpr(ptr(buf))
                elif n > 0:
                    L.mkrh_copy_plane(ptr(buf))
                extra = {}
                if cap[1] < 6:
                    xy = np.zeros(2, np.float64)
                    L.mkrh_crosshair(h, cap[1], ptr(xy))
                    hv = np.zeros(6, np.float64)
                    L.mkrh_direction3d(h, cap[1], ptr(hv))
                    extra = dict(crosshair=xy.tolist(), dir3d=hv.tolist(),
                                 plane_index=int(L.mkrh_get_plane_index(h, cap[1])),
                                 plane_number=int(L.mkrh_get_plane_number(h, cap[1])),
                                 pixel_spacing=float(L.mkrh_pixel_spacing(h, cap[1])))
                caps.append(dict(kind="plane", plane=cap[1], wh=wh.tolist(), args=buf.tolist(),
                                 mpr_kind=int(L.mkrh_plane_kind()) if hasattr(L, "mkrh_plane_kind") else -1,
                                 **extra))
        results[sc["name"]] = dict(labels=labels, captures=caps)
    L.mkrh_destroy(h)

    tfs = {}
    for name, rgb, alpha in TF_CASES:
        rp = np.array(list(rgb.keys()), np.int32)
        rv = np.array([rgb[k] for k in rgb], np.float32)
        ap = np.array(list(alpha.keys()), np.int32)
        av = np.array([alpha[k] for k in alpha], np.float32)
        out = np.zeros((256, 4), np.float32)
        n = L.mkrh_tf_lut(ptr(rp), ptr(rv), len(rp), ptr(ap) if len(ap) else None,
                          ptr(av) if len(av) else None, len(ap), ptr(out), 256)
        tfs[name] = dict(rgb={str(k): list(v) for k, v in rgb.items()},
                         alpha={str(k): v for k, v in alpha.items()},
                         n=int(n), lut=out[:max(n, 0)].tolist())
    OUT.write_text(json.dumps(dict(source="MonkeyGL core/*.cpp via oracle/_ref/libmkref_host.so",
                                   scenarios=SCENARIOS, results=results, transfer_functions=tfs)))
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes, {len(SCENARIOS)} scenarios, {len(tfs)} TFs)")


if __name__ == "__main__":
    main(*sys.argv[1:])
