"""Host-side geometry against golden vectors captured from MonkeyGL's own
host code (tests/golden/host_geometry.json, written by
tests/golden/make_host_golden.py from MonkeyGL's core/*.cpp).

The VR camera matrix, volume factors, z inversion and image size built here
must equal what MonkeyGL's HelloMonkey hands to cu_render, bit for bit."""
import json
from pathlib import Path

import numpy as np
import pytest

from monkeygl_b200.camera import Camera, need_invert_z, volume_factors

GOLD = json.loads((Path(__file__).resolve().parent / "golden" / "host_geometry.json").read_text())
SCEN = {s["name"]: s for s in GOLD["scenarios"]}
RES = GOLD["results"]

# layout of a captured cu_render argument list (see oracle/ref_host_capture.cpp)
W, H, DIMS, MLS, SP, SV, XT, YT, SCALE, M, INV, VOI, BG, TYPE, LAB = (
    0, 1, slice(2, 5), slice(5, 8), slice(8, 11), slice(11, 14), 14, 15, 16, slice(17, 26), 26,
    slice(27, 33), slice(33, 37), 37, 38)


def vr_size(w, h):
    """RenderInfo::SetVRSize (core/RenderInfo.cpp:52-69): integer area ratio
    against 768^2, then an even width."""
    delta = float((w * h) // (768 * 768))
    if delta > 1:
        w, h = int(w / delta), int(h / delta)
    if w % 2:
        w += 1
    return w, h


def replay_camera(ops):
    cam = Camera()
    cam.anterior()
    size = (512, 512)
    for op in ops:
        k = op[0]
        if k == "orientation":
            [cam.anterior, cam.posterior, cam.left, cam.right, cam.head, cam.foot][op[1]]()
        elif k == "rotate":
            cam.rotate(op[1], op[2])
        elif k == "zoom":
            cam.zoom(op[1])
        elif k == "pan":
            cam.pan(op[1], op[2])
        elif k == "vr_size":
            size = vr_size(op[1], op[2])
    return cam, size


VR_CASES = [(n, i) for n, r in RES.items() for i, c in enumerate(r["captures"]) if c["kind"] == "vr"]


@pytest.mark.parametrize("name,idx", VR_CASES, ids=[f"{n}-{i}" for n, i in VR_CASES])
def test_camera_matrix_bit_exact(name, idx):
    sc = SCEN[name]
    args = np.array(RES[name]["captures"][idx]["args"])
    cam, size = replay_camera(sc["ops"])
    got = np.array(cam.flat(), np.float32)
    want = args[M].astype(np.float32)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (got, want)
    assert np.float32(cam.scale) == np.float32(args[SCALE])
    assert np.float32(cam.x_translate) == np.float32(args[XT])
    assert np.float32(cam.y_translate) == np.float32(args[YT])
    assert (int(args[W]), int(args[H])) == size


@pytest.mark.parametrize("name,idx", VR_CASES, ids=[f"{n}-{i}" for n, i in VR_CASES])
def test_volume_factors_bit_exact(name, idx):
    sc = SCEN[name]
    args = np.array(RES[name]["captures"][idx]["args"])
    mls, sv = volume_factors(sc["dims"], sc["spacing"])
    assert np.array_equal(np.float32(mls), args[MLS].astype(np.float32))
    assert np.array_equal(np.float32(sv), args[SV].astype(np.float32))
    assert np.array_equal(np.float32(sc["spacing"]), args[SP].astype(np.float32))
    d = sc["direction"]
    assert need_invert_z(d[0:3], d[3:6], d[6:9]) == bool(args[INV])
    X, Y, Z = sc["dims"]
    assert list(args[VOI].astype(int)) == [0, X - 1, 0, Y - 1, 0, Z - 1]


def test_default_label_windows():
    # MonkeyGL copies per-label windows into the kernel argument only inside
    # SetVRWWWL / SetObjectAlpha (core/DataManager.cpp:570-611); before the
    # first such call every label reaches the kernel as (0, 0, 0)
    args = np.array(RES["labels_default"]["captures"][0]["args"])
    lab = args[LAB:].reshape(-1, 3)
    assert RES["labels_default"]["labels"] == [1, 2]
    assert (lab == 0).all()
    # after one call, every existing label gets its ObjectInfo defaults
    # (alpha 1, ww 400, wl 40, core/ObjectInfo.h:19-26)
    args = np.array(RES["labels_bg04"]["captures"][0]["args"])
    lab = args[LAB:].reshape(-1, 3)
    assert tuple(lab[0]) == (np.float32(0.4), 400.0, 40.0)
    for l in RES["labels_bg04"]["labels"]:
        assert tuple(lab[l]) == (1.0, 400.0, 40.0)


def test_label_window_updates():
    args = np.array(RES["labels_set"]["captures"][0]["args"])
    lab = args[LAB:].reshape(-1, 3)
    # ops: wwwl on the active label (the last added), caps, ww <= 0 forced to 1
    assert tuple(lab[2]) == (1.0, 500.0, 300.0)
    assert tuple(lab[0]) == (0.800000011920929, 400.0, 40.0)
    assert tuple(lab[1]) == (0.5, 1.0, 10.0)
