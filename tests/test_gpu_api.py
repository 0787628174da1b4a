"""End-to-end parity of the MonkeyGL API on the GPU.

The same operation sequence (volume, spacing, direction, label masks,
transfer-function control points, windows, caps, camera, VR size, MPR type
and thickness, crosshair moves, CPR path and rotation) drives MonkeyGL's own
HelloMonkey (its host code and kernels, built unmodified into
oracle/_ref/libmkref_full.so) and this library's pyMonkeyGL.  VR images,
with MonkeyGL's overlays (the orientation box in the bottom-right 64x64
pixels, drawn from ./resources/human.stl, and the CPR line), planes and CPR
images must match exactly.  Both HelloMonkey objects are constructed in the
directory holding resources/, where MonkeyGL expects its mesh."""
import ctypes as C
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "monkeygl_b200" / "lib"))
pm = pytest.importorskip("pyMonkeyGL")
from monkeygl_b200.phantom import make_phantom  # noqa: E402

pytestmark = pytest.mark.gpu
FULL = ROOT / "oracle" / "_ref" / "libmkref_full.so"


class RefHelloMonkey:
    """MonkeyGL's HelloMonkey through the oracle driver (one process-wide state)."""

    L = None

    def __init__(self):
        if RefHelloMonkey.L is None:
            if not FULL.exists():
                pytest.fail(f"{FULL} missing: run `make -C oracle ref`")
            L = C.CDLL(str(FULL))
            vp = C.c_void_p
            L.mkrh_create.restype = vp
            L.mkrh_create.argtypes = [C.c_char_p]
            sig = {
                "mkrh_set_volume": [vp, vp, C.c_int, C.c_int, C.c_int], "mkrh_add_mask": [vp, vp, C.c_int, C.c_int, C.c_int],
                "mkrh_set_spacing": [vp, C.c_double, C.c_double, C.c_double], "mkrh_set_direction": [vp, vp],
                "mkrh_set_background": [vp, C.c_float, C.c_float, C.c_float, C.c_float],
                "mkrh_set_wwwl": [vp, C.c_float, C.c_float, C.c_int], "mkrh_set_alpha": [vp, C.c_float, C.c_int],
                "mkrh_set_render_type": [vp, C.c_int], "mkrh_orientation": [vp, C.c_int],
                "mkrh_rotate": [vp, C.c_float, C.c_float], "mkrh_zoom": [vp, C.c_float], "mkrh_pan": [vp, C.c_float, C.c_float],
                "mkrh_set_vr_size": [vp, C.c_int, C.c_int], "mkrh_set_mpr_type": [vp, C.c_int],
                "mkrh_set_thickness": [vp, C.c_double, C.c_int], "mkrh_browse": [vp, C.c_float, C.c_int],
                "mkrh_rotate_crosshair": [vp, C.c_float, C.c_int], "mkrh_set_cpr_line_voxel": [vp, vp, C.c_int],
                "mkrh_rotate_cpr": [vp, C.c_float, C.c_int], "mkrh_reset": [vp],
                "mkrh_set_tf": [vp, vp, vp, C.c_int, vp, vp, C.c_int, C.c_int],
                "mkrh_vr_image": [vp, vp, C.c_longlong, vp], "mkrh_plane_image": [vp, C.c_int, vp, C.c_longlong, vp],
                "mkrh_add_annotation": [vp, C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float,
                                        C.c_float, C.c_float],
                "mkrh_remove_annotations": [vp],
            }
            for f, a in sig.items():
                getattr(L, f).argtypes = a
            L.mkrh_mask_max_label.argtypes = [vp]
            # MonkeyGL allocates its label volume uncleared (core/VolumeInfo.cpp:96-104);
            # fresh zero pages keep labels outside the masks at 0
            assert L.mkrh_zero_heap(1) == 1
            RefHelloMonkey.L = L
            RefHelloMonkey.h = L.mkrh_create(str(FULL.parent).encode())
        self.L, self.h = RefHelloMonkey.L, RefHelloMonkey.h


def ptr(a):
    return C.c_void_p(a.ctypes.data)


def run_both(p, ops, masks=None):
    """Apply `ops` to MonkeyGL's HelloMonkey and to pyMonkeyGL; return both."""
    ref = RefHelloMonkey()
    L, h = ref.L, ref.h
    import os
    cwd = os.getcwd()
    os.chdir(FULL.parent)       # ./resources/human.stl, as for MonkeyGL's object
    try:
        mine = pm.HelloMonkey()
    finally:
        os.chdir(cwd)
    X, Y, Z = p.dims
    L.mkrh_set_volume(h, ptr(p.volume), X, Y, Z)
    mine.SetVolumeArray(p.volume.swapaxes(2, 0))
    d = np.array([1, 0, 0, 0, 1, 0, 0, 0, -1], np.float64)
    L.mkrh_set_direction(h, ptr(d))
    # MonkeyGL's process-wide state keeps the last CPR path, whose line
    # layer it draws into every VR image; each test starts without one
    L.mkrh_set_cpr_line_voxel(h, ptr(np.zeros((1, 3), np.float64)), 0)
    mine.SetDirection(pm.Direction3d(1, 0, 0), pm.Direction3d(0, 1, 0), pm.Direction3d(0, 0, -1))
    L.mkrh_set_spacing(h, *p.spacing)
    mine.SetSpacing(*p.spacing)
    for m in masks or []:
        a = L.mkrh_add_mask(h, ptr(m), X, Y, Z)
        b = mine.AddNewObjectMaskArray(m.swapaxes(2, 0))
        assert a == b
    if masks:
        # never hand MonkeyGL's kernel a label beyond its 65-entry tables
        assert 0 <= L.mkrh_mask_max_label(h) <= len(masks)
    orient = [mine.Anterior, mine.Posterior, mine.Left, mine.Right, mine.Head, mine.Foot]
    for op in [("orientation", 0), ("reset",), ("vr_size", 512, 512), ("render_type", 0), ("mpr_type", 0),
               ("background", 0.0, 0.0, 0.0, 0.0)] + list(ops):
        k = op[0]
        if k == "orientation":
            L.mkrh_orientation(h, op[1]); orient[op[1]]()
        elif k == "reset":
            L.mkrh_reset(h); mine.Reset()
        elif k == "vr_size":
            L.mkrh_set_vr_size(h, op[1], op[2]); mine.SetVRSize(op[1], op[2])
        elif k == "render_type":
            L.mkrh_set_render_type(h, op[1]); mine.SetRenderType(pm.RenderType(op[1]))
        elif k == "mpr_type":
            L.mkrh_set_mpr_type(h, op[1]); mine.SetMPRType(pm.MPRType(op[1]))
        elif k == "background":
            L.mkrh_set_background(h, *op[1:5]); mine.SetColorBackground(pm.RGBA(*op[1:5]))
        elif k == "rotate":
            L.mkrh_rotate(h, op[1], op[2]); mine.Rotate(op[1], op[2])
        elif k == "zoom":
            L.mkrh_zoom(h, op[1]); mine.Zoom(op[1])
        elif k == "pan":
            L.mkrh_pan(h, op[1], op[2]); mine.Pan(op[1], op[2])
        elif k == "wwwl":
            L.mkrh_set_wwwl(h, op[1], op[2], op[3])
            mine.SetVRWWWL(op[1], op[2]) if op[3] < 0 else mine.SetVRWWWL(op[1], op[2], op[3])
        elif k == "alpha":
            L.mkrh_set_alpha(h, op[1], op[2])
            mine.SetObjectAlpha(op[1]) if op[2] < 0 else mine.SetObjectAlpha(op[1], op[2])
        elif k == "tf":
            rgb, alpha, label = op[1], op[2], op[3]
            rp = np.array(list(rgb), np.int32)
            rv = np.array([rgb[i] for i in rgb], np.float32)
            ap = np.array(list(alpha) or [0], np.int32)
            av = np.array([alpha[i] for i in alpha] or [0], np.float32)
            L.mkrh_set_tf(h, ptr(rp), ptr(rv), len(rp), ptr(ap), ptr(av), len(alpha), label)
            r2 = {i: pm.RGBA(*rgb[i]) for i in rgb}
            if alpha:
                mine.SetTransferFunc(r2, dict(alpha)) if label < 0 else mine.SetTransferFunc(r2, dict(alpha), label)
            else:
                mine.SetTransferFunc(r2) if label < 0 else mine.SetTransferFunc(r2, label)
        elif k == "thickness":
            L.mkrh_set_thickness(h, op[1], op[2]); mine.SetThickness(op[1], pm.PlaneType(op[2]))
        elif k == "browse":
            L.mkrh_browse(h, op[1], op[2]); mine.Browse(op[1], pm.PlaneType(op[2]))
        elif k == "rotate_crosshair":
            L.mkrh_rotate_crosshair(h, op[1], op[2]); mine.RotateCrossHair(op[1], pm.PlaneType(op[2]))
        elif k == "cpr_line":
            pts = np.ascontiguousarray(op[1], np.float64)
            L.mkrh_set_cpr_line_voxel(h, ptr(pts), len(pts)); mine.SetCPRLineVoxelArray(pts)
        elif k == "rotate_cpr":
            L.mkrh_rotate_cpr(h, op[1], op[2]); mine.RotateCPR(op[1], pm.PlaneType(op[2]))
        elif k == "annotation":
            txt, x, y, fs, fmt, rgba = op[1:]
            L.mkrh_add_annotation(h, txt.encode(), x, y, fs, fmt, *rgba)
            mine.AddAnnotation(pm.PlaneType.PlaneVR, txt, x, y, pm.FontSize(fs), pm.AnnotationFormat(fmt),
                               pm.RGBA(*rgba))
        elif k == "clear_annotations":
            L.mkrh_remove_annotations(h); mine.RemoveAllAnnotations()
        elif k == "add_mask":
            a = L.mkrh_add_mask(h, ptr(op[1]), X, Y, Z)
            b = mine.AddNewObjectMaskArray(op[1].swapaxes(2, 0))
            assert a == b
        elif k == "render_mine":
            mine.GetVRImage()       # the mask goes to the device here; later masks update it in place
        else:
            raise ValueError(k)
    return ref, mine


def ref_vr(ref):
    out = np.zeros(4096 * 4096 * 3, np.uint8)
    wh = np.zeros(2, np.int32)
    assert ref.L.mkrh_vr_image(ref.h, ptr(out), out.size, ptr(wh)) == 1
    w, h = int(wh[0]), int(wh[1])
    return out[: w * h * 3].reshape(h, w, 3)


def ref_plane(ref, plane):
    out = np.zeros(4096 * 4096, np.int16)
    wh = np.zeros(2, np.int32)
    assert ref.L.mkrh_plane_image(ref.h, plane, ptr(out), out.size, ptr(wh)) == 1
    w, h = int(wh[0]), int(wh[1])
    return out[: w * h].reshape(h, w)


def assert_vr_equal(a, b, what):
    assert a.shape == b.shape, (a.shape, b.shape)
    d = np.abs(a.astype(int) - b.astype(int)).max(-1)
    h, w = a.shape[:2]
    box = d[h - 64:, w - 64:] if w > 64 and h > 64 else d[:0]
    assert (d == 0).all(), (f"{what}: {int((d > 0).sum())} pixels differ ({int((box > 0).sum())} in the "
                            f"orientation box), max {int(d.max())}")


@pytest.fixture(scope="module")
def phantom():
    return make_phantom((128, 112, 96), (0.35, 0.35, 0.3), 2024, with_labels=True)


TF4 = {0: (0.9, 0.3, 0.2, 0.0), 22: (0.95, 0.4, 0.3, 0.0), 55: (0.9, 0.7, 0.5, 0.35), 99: (1.0, 0.95, 0.9, 0.85)}


# MonkeyGL keeps one process-wide state: SetVolumeData clears its host-side
# labels but not the device label texture nor the per-label window table of
# the previous volume (core/DataManager.cpp:144-165).  This test needs that
# state fresh, so it runs first; later tests set every window they use.
def test_default_windows_render_background(phantom):
    # before any SetVRWWWL / SetObjectAlpha every label's cap is 0
    ref, mine = run_both(phantom, [("tf", TF4, {}, -1), ("background", 0.2, 0.3, 0.4, 1.0)])
    img = mine.GetVRImage()
    assert_vr_equal(img, ref_vr(ref), "default windows")
    assert (img[:200, :200] == [51, 76, 102]).all()


# Before any label mask exists in MonkeyGL's process-wide state (see above).
def test_cpr_line_layer_in_vr(phantom):
    # the VR image carries the CPR path as a white 1-pixel polyline over the
    # orientation box and the ray-cast image
    line = [[20.0 + 3.0 * i, 30.0 + 8.0 * np.sin(i / 4.0), 10.0 + 2.5 * i] for i in range(30)]
    ops = [("cpr_line", line), ("rotate_cpr", 30, 7), ("tf", TF4, {}, -1), ("wwwl", 1700, 650, -1),
           ("rotate", 40, 0)]
    ref, mine = run_both(phantom, ops)
    img = mine.GetVRImage()
    assert_vr_equal(img, ref_vr(ref), "VR with the CPR line layer")
    assert ((img == 255).all(-1)).sum() >= 100, "no CPR line drawn"


# Before any label mask exists in MonkeyGL's process-wide state (see above).
def test_text_annotations_in_vr(phantom):
    """VR images with MonkeyGL's annotation layer: text of the three font
    sizes and alignments, clipped at the image edges, drawn after the
    orientation box (core/VRProvider.cpp:30-36, core/AnnotationLayer.cpp:41-61).
    Both objects load their glyphs and mesh from oracle/_ref/resources."""
    anns = [("annotation", "MonkeyGL B200 - VR 512x512", 6, 4, 0, 0, (1.0, 1.0, 0.0, 1.0)),
            ("annotation", "WW/WL: 1700/650", 506, 30, 1, 1, (0.2, 0.9, 1.0, 1.0)),
            ("annotation", "Axial {R} [x] ~`!@#$%^&*()", 256, 240, 2, 2, (1.0, 0.5, 0.25, 1.0)),
            ("annotation", "edge clip", 480, 500, 2, 0, (0.9, 0.9, 0.9, 1.0)),
            ("annotation", "left clip", -30, -10, 1, 0, (0.5, 1.0, 0.5, 1.0))]
    ops = [("clear_annotations",), ("tf", TF4, {}, -1), ("wwwl", 1700, 650, -1), ("rotate", 25, 5)] + anns
    try:
        ref, mine = run_both(phantom, ops)
        img = mine.GetVRImage()
        assert_vr_equal(img, ref_vr(ref), "VR with text annotations")
        # the text is there: the same view without annotations differs
        L, h = ref.L, ref.h
        L.mkrh_remove_annotations(h)
        mine.RemoveAllAnnotations()
        plain = mine.GetVRImage()
        assert_vr_equal(plain, ref_vr(ref), "VR after removing the annotations")
        assert int(np.count_nonzero((img != plain).any(-1))) > 500
    finally:
        RefHelloMonkey().L.mkrh_remove_annotations(RefHelloMonkey().h)


@pytest.mark.parametrize("rtype", [0, 1, 2])
def test_vr_through_the_api(phantom, rtype):
    ops = [("tf", TF4, {}, -1), ("wwwl", 1700, 650, -1), ("render_type", rtype), ("rotate", 30, 10),
           ("zoom", 1.3), ("pan", 12, -7)]
    ref, mine = run_both(phantom, ops)
    assert_vr_equal(mine.GetVRImage(), ref_vr(ref), f"VR type {rtype}")


def test_multilabel_vr_through_the_api(phantom):
    labels = phantom.labels
    masks = [(labels == l).astype(np.uint8) for l in (1, 2, 3, 4)]
    ops = [("tf", TF4, {}, 0), ("tf", {0: (1, 0, 0, 0.1), 99: (1, 1, 0, 0.9)}, {}, 1),
           ("tf", {0: (0, 1, 0, 0.0), 50: (0, 1, 1, 0.6), 99: (0, 0, 1, 1)}, {20: 0.0, 70: 0.8}, 2),
           ("wwwl", 1700, 650, 0), ("wwwl", 1200, 400, 1), ("wwwl", 900, 300, 2), ("wwwl", 1700, 650, 3),
           ("wwwl", 1700, 650, 4), ("alpha", 0.4, 0), ("alpha", 0.7, 1), ("alpha", 1.0, 2),
           ("rotate", 60, 0), ("vr_size", 640, 480)]
    ref, mine = run_both(phantom, ops, masks)
    assert_vr_equal(mine.GetVRImage(), ref_vr(ref), "multi-label VR")


def test_incremental_masks_through_the_api(phantom):
    """Masks added after the first render reach the device as an update of
    the box they change (mk_volume_update_mask), MonkeyGL re-uploads its
    whole mask; the images must agree after every addition."""
    labels = phantom.labels
    X, Y, Z = phantom.dims
    first = (labels == 1).astype(np.uint8)
    small = np.zeros_like(first)
    small[40:52, 30:61, 70:77] = 1                  # a box that is not brick-aligned
    edge = np.zeros_like(first)
    edge[Z - 5:, Y - 9:, :17] = 1                   # touching the volume's far faces
    ops = [("tf", TF4, {}, 0), ("tf", {0: (1, 0, 0, 0.1), 99: (1, 1, 0, 0.9)}, {}, 1),
           ("wwwl", 1700, 650, 0), ("wwwl", 1200, 400, 1), ("alpha", 0.4, 0), ("rotate", 35, 15),
           ("render_mine",), ("add_mask", (labels == 2).astype(np.uint8)), ("render_mine",),
           ("add_mask", small), ("render_mine",), ("add_mask", edge),
           ("tf", {0: (0, 1, 0, 0.0), 50: (0, 1, 1, 0.6), 99: (0, 0, 1, 1)}, {}, 4), ("alpha", 0.8, 3)]
    ref, mine = run_both(phantom, ops, [first])
    assert_vr_equal(mine.GetVRImage(), ref_vr(ref), "VR after incremental mask updates")


def test_planes_through_the_api(phantom):
    ops = [("mpr_type", 1), ("thickness", 1.2, 0), ("thickness", 0.9, 1), ("browse", 2.5, 0),
           ("rotate_crosshair", 25, 3), ("rotate_crosshair", -40, 4)]
    ref, mine = run_both(phantom, ops)
    for plane in range(6):
        a = mine.GetPlaneArray(pm.PlaneType(plane))
        b = ref_plane(ref, plane)
        assert a.shape == b.shape and np.array_equal(a, b), f"plane {plane}"


def test_cpr_through_the_api(phantom):
    line = [[20.0 + 3.0 * i, 30.0 + 8.0 * np.sin(i / 4.0), 10.0 + 2.5 * i] for i in range(30)]
    ops = [("cpr_line", line), ("rotate_cpr", 30, 7), ("rotate_cpr", 45, 8)]
    ref, mine = run_both(phantom, ops)
    for plane in (7, 8):
        a = mine.GetPlaneArray(pm.PlaneType(plane))
        b = ref_plane(ref, plane)
        assert a.shape == b.shape and np.array_equal(a, b), f"CPR plane {plane}"


def test_png_strings_decode_to_the_images(phantom):
    import base64
    import zlib
    ref, mine = run_both(phantom, [("tf", TF4, {}, -1), ("wwwl", 1700, 650, -1), ("rotate", 15, 0)])
    png = base64.b64decode(mine.GetVRData_pngString())
    assert png[:8] == b"\x89PNG\r\n\x1a\n"
    # IHDR + single IDAT: inflate and strip the filter bytes
    w = int.from_bytes(png[16:20], "big")
    h = int.from_bytes(png[20:24], "big")
    i = png.index(b"IDAT")
    n = int.from_bytes(png[i - 4:i], "big")
    raw = zlib.decompress(png[i + 4:i + 4 + n])
    img = np.frombuffer(raw, np.uint8).reshape(h, 1 + w * 3)[:, 1:].reshape(h, w, 3)
    assert np.array_equal(img, mine.GetVRImage())

