"""The MonkeyGL C++ API of this library (pyMonkeyGL over HelloMonkey) against
golden vectors from MonkeyGL's own host code (tests/golden/host_geometry.json).

Each golden scenario is replayed through pyMonkeyGL: the camera matrix,
volume factors, label windows, plane frames, CPR rows and transfer-function
tables our host code would hand to the kernels must equal the arguments
MonkeyGL's host code handed to its kernels, bit for bit (planes and CPR rows
are compared after the same float rounding MonkeyGL applies)."""
import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "monkeygl_b200" / "lib"))
pm = pytest.importorskip("pyMonkeyGL")

GOLD = json.loads((ROOT / "tests" / "golden" / "host_geometry.json").read_text())
SCEN = {s["name"]: s for s in GOLD["scenarios"]}
RES = GOLD["results"]
F32 = np.float32


def replay(sc):
    h = pm.HelloMonkey()
    X, Y, Z = sc["dims"]
    vol = np.zeros((Z, Y, X), np.int16)
    h.SetVolumeArray(vol.swapaxes(2, 0))
    d = sc["direction"]
    h.SetDirection(pm.Direction3d(*d[0:3]), pm.Direction3d(*d[3:6]), pm.Direction3d(*d[6:9]))
    h.SetSpacing(*sc["spacing"])
    h.Anterior()
    h.Reset()
    h.SetVRSize(512, 512)
    h.SetRenderType(pm.RenderTypeVR)
    h.SetMPRType(pm.MPRTypeAverage)
    h.SetColorBackground(pm.RGBA(0, 0, 0, 0))
    labels = []
    n = sc["masks"]
    for m in range(n):
        mask = np.zeros((Z, Y, X), np.uint8)
        mask[(m * Z) // n:((m + 1) * Z) // n, :, : X // 2] = 1
        labels.append(int(h.AddNewObjectMaskArray(mask.swapaxes(2, 0))))
    orient = [h.Anterior, h.Posterior, h.Left, h.Right, h.Head, h.Foot]
    for op in sc["ops"]:
        k = op[0]
        if k == "orientation": orient[op[1]]()
        elif k == "rotate": h.Rotate(op[1], op[2])
        elif k == "zoom": h.Zoom(op[1])
        elif k == "pan": h.Pan(op[1], op[2])
        elif k == "vr_size": h.SetVRSize(op[1], op[2])
        elif k == "render_type": h.SetRenderType(pm.RenderType(op[1]))
        elif k == "background": h.SetColorBackground(pm.RGBA(*op[1:5]))
        elif k == "wwwl":
            h.SetVRWWWL(op[1], op[2]) if op[3] < 0 else h.SetVRWWWL(op[1], op[2], op[3])
        elif k == "alpha":
            h.SetObjectAlpha(op[1]) if op[2] < 0 else h.SetObjectAlpha(op[1], op[2])
        elif k == "mpr_type": h.SetMPRType(pm.MPRType(op[1]))
        elif k == "thickness": h.SetThickness(op[1], pm.PlaneType(op[2]))
        elif k == "update_thickness": h.UpdateThickness(op[1])
        elif k == "browse": h.Browse(op[1], pm.PlaneType(op[2]))
        elif k == "rotate_crosshair": h.RotateCrossHair(op[1], pm.PlaneType(op[2]))
        elif k == "pan_crosshair": h.PanCrossHair(op[1], op[2], pm.PlaneType(op[3]))
        elif k == "plane_index": h.SetPlaneIndex(op[1], pm.PlaneType(op[2]))
        elif k == "cpr_line":
            h.SetCPRLineVoxelArray(np.array(op[1], np.float64))
        elif k == "rotate_cpr": h.RotateCPR(op[1], pm.PlaneType(op[2]))
        else:
            raise ValueError(k)
    return h, labels


def bits(a):
    return np.asarray(a, np.float32).view(np.uint32)


CASES = [(n, i) for n, r in RES.items() for i in range(len(r["captures"]))]


@pytest.mark.parametrize("name,idx", CASES, ids=[f"{n}-{i}" for n, i in CASES])
def test_kernel_arguments_match_monkeygl(name, idx):
    sc = SCEN[name]
    h, labels = replay(sc)
    assert labels == RES[name]["labels"]
    cap = RES[name]["captures"][idx]
    a = np.array(cap["args"])
    if cap["kind"] == "vr":
        p = h.GetVRParams()
        assert (p["width"], p["height"]) == (int(a[0]), int(a[1]))
        assert np.array_equal(bits(p["max_len_spacing"]), bits(a[5:8]))
        assert np.array_equal(bits(p["spacing"]), bits(a[8:11]))
        assert np.array_equal(bits(p["spacing_voxel"]), bits(a[11:14]))
        assert np.array_equal(bits([p["x_translate"], p["y_translate"], p["scale"]]), bits(a[14:17]))
        assert np.array_equal(bits(p["transform"]), bits(a[17:26]))
        assert p["invert_z"] == int(a[26])
        assert p["voi"] == [int(v) for v in a[27:33]]
        assert np.array_equal(bits(p["background"]), bits(a[33:37]))
        assert p["render_type"] == int(a[37])
        assert np.array_equal(bits(h.GetLabelTable().ravel()), bits(a[38:]))
        return
    plane = cap["plane"]
    pt = pm.PlaneType(plane)
    if plane >= 7:
        rows = h.GetCPRRows(pt)
        if not cap["args"]:
            assert rows == ()
            return
        w, hh, P, D = rows
        assert (w, hh) == tuple(cap["wh"])
        H = int(a[1])
        assert (int(a[0]), H) == (w, hh)
        np.testing.assert_array_equal(P.ravel(), a[3:3 + 3 * H])
        np.testing.assert_array_equal(D.ravel(), a[3 + 3 * H:3 + 6 * H])
        return
    p = h.GetPlaneParams(pt)
    assert (p["width"], p["height"]) == tuple(cap["wh"]) == (int(a[0]), int(a[1]))
    assert np.array_equal(bits(p["spacing"]), bits(a[5:8]))
    assert np.array_equal(bits(p["dir_h"]), bits(a[8:11]))
    assert np.array_equal(bits(p["dir_v"]), bits(a[11:14]))
    assert np.array_equal(bits(p["dir_n"]), bits(a[14:17]))
    assert np.array_equal(bits(p["left_top"]), bits(a[17:20]))
    assert np.array_equal(bits([p["pixel_spacing"]]), bits([a[20]]))
    assert p["invert_z"] == int(a[21])
    assert np.array_equal(bits([p["half_num"]]), bits([a[22]]))
    assert p["mpr_type"] == cap["mpr_kind"]
    x, y = h.GetCrossHairPoint(pt).x(), h.GetCrossHairPoint(pt).y()
    assert (x, y) == tuple(cap["crosshair"])
    (hx, hy, hz), (vx, vy, vz) = h.GetDirection3D(pt)
    assert [hx, hy, hz, vx, vy, vz] == cap["dir3d"]
    assert h.GetPlaneIndex(pt) == cap["plane_index"]
    assert h.GetPlaneNumber(pt) == cap["plane_number"]
    assert h.GetPixelSpacing(pt) == cap["pixel_spacing"]


@pytest.mark.parametrize("name", list(GOLD["transfer_functions"]))
def test_transfer_function_tables_match_monkeygl(name):
    tf = GOLD["transfer_functions"][name]
    h = pm.HelloMonkey()
    h.SetVolumeArray(np.zeros((2, 2, 2), np.int16))
    rgb = {int(k): pm.RGBA(*v) for k, v in tf["rgb"].items()}
    alpha = {int(k): float(v) for k, v in tf["alpha"].items()}
    assert h.SetTransferFunc(rgb, alpha, 0)
    lut = h.GetTransferFunctionLUT(0)
    if tf["n"] == 0:
        assert lut is None
        return
    assert np.array_equal(bits(lut.ravel()), bits(np.array(tf["lut"]).ravel()))


def test_transfer_function_file_round_trip(tmp_path):
    h = pm.HelloMonkey()
    h.SetVolumeArray(np.zeros((2, 2, 2), np.int16))
    h.SetTransferFunc({0: pm.RGBA(1, 0, 0, 0), 40: pm.RGBA(0, 1, 0, 0.5), 99: pm.RGBA(0, 0, 1, 1)}, {10: 0.2, 80: 0.9})
    h.SetVRWWWL(800, 120)
    f = tmp_path / "tf.txt"
    assert h.SaveTransferFunction(str(f))
    text = f.read_text().splitlines()
    assert text[0] == "ww: 800" and text[1] == "wl: 120" and text[2] == "idx2rgba: 3"
    g = pm.HelloMonkey()
    g.SetVolumeArray(np.zeros((2, 2, 2), np.int16))
    assert g.LoadTransferFunction(str(f))
    a, b = h.GetTransferFunctionLUT(0), g.GetTransferFunctionLUT(0)
    # loading merges the file's points into the default points 5 and 95 (core/ObjectInfo.h:19-26)
    assert a.shape == b.shape == (100, 4)
    assert np.array_equal(h.GetLabelTable()[0], g.GetLabelTable()[0])


def test_instances_are_independent():
    a, b = pm.HelloMonkey(), pm.HelloMonkey()
    a.SetVolumeArray(np.zeros((8, 8, 8), np.int16))
    b.SetVolumeArray(np.zeros((4, 4, 4), np.int16))
    a.SetSpacing(1, 1, 1)
    b.SetSpacing(2, 2, 2)
    a.Anterior()
    b.Anterior()
    b.Rotate(30, 0)
    assert a.GetVRParams()["transform"] != b.GetVRParams()["transform"]
    assert a.GetVolumeArray().shape == (8, 8, 8) and b.GetVolumeArray().shape == (4, 4, 4)
