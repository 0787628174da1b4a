"""VR overlays against MonkeyGL's own host code (no GPU needed).

tests/golden/overlay.npz holds what MonkeyGL's host library drew over an
empty image (tests/golden/make_overlay_golden.py): its orientation box for
22 camera rotations, the CPR line layer over one view, and
Methods::DrawLineInImage24Bit for 40 seeded segments.  The library's
mk_merge_orientation_box and mk_draw_line_rgb must reproduce every pixel.

The orientation mesh is MonkeyGL's resources/human.stl; the oracle build
places it in oracle/_ref/resources/ (it is not part of this repository).
"""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from monkeygl_b200 import capi

ROOT = Path(__file__).resolve().parents[1]
GOLD = ROOT / "tests" / "golden" / "overlay.npz"
MESH = ROOT / "oracle" / "_ref" / "resources" / "human.stl"


def _ptr(a):
    return C.c_void_p(a.ctypes.data)


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


@pytest.fixture(scope="module")
def mesh():
    if not MESH.exists():
        pytest.skip(f"{MESH} not built: run `make -C oracle ref-full` with the MonkeyGL sources")
    h = C.c_void_p()
    assert capi.lib().mk_mesh_load_stl(str(MESH).encode(), C.byref(h)) == capi.MK_OK, capi.lib().mk_last_error()
    yield h
    capi.lib().mk_mesh_destroy(h)


def box(mesh, rot, w=512, h=512):
    img = np.zeros((h, w, 3), np.uint8)
    rot = np.ascontiguousarray(rot, np.float32)
    assert capi.lib().mk_merge_orientation_box(mesh, _ptr(rot), _ptr(img), w, h) == capi.MK_OK
    return img


def test_mesh_loads_every_facet(mesh):
    n = capi.lib().mk_mesh_facet_count(mesh)
    assert n == (MESH.stat().st_size - 84) // 50


def test_orientation_box_matches_monkeygl(gold, mesh):
    bad = []
    for i, (rot, want) in enumerate(zip(gold["rotations"], gold["boxes"])):
        img = box(mesh, rot)
        assert not img[:-64].any() and not img[:, :-64].any(), "drawn outside the box"
        got = img[-64:, -64:]
        if not np.array_equal(got, want):
            bad.append((i, int((got != want).any(-1).sum())))
    assert not bad, f"(case, differing pixels): {bad}"
    assert sum(int(b.any(-1).sum()) for b in gold["boxes"]) > 1000   # the boxes are not empty


def test_orientation_box_placement_and_small_images(gold, mesh):
    rot, want = gold["rotations"][3], gold["boxes"][3]
    img = box(mesh, rot, 300, 200)           # any size above 64: the box sits bottom-right
    assert np.array_equal(img[-64:, -64:], want) and not img[:-64].any()
    assert not box(mesh, rot, 64, 200).any()  # MonkeyGL draws nothing unless both sides exceed 64
    assert not box(mesh, rot, 200, 64).any()


def test_line_drawing_matches_monkeygl(gold):
    for seg, want in zip(gold["segments"], gold["line_images"]):
        x0, y0, x1, y1, lw = (float(v) for v in seg[:5])
        col = np.ascontiguousarray(seg[5:8], np.float32)
        img = np.zeros((120, 160, 3), np.uint8)
        rc = capi.lib().mk_draw_line_rgb(_ptr(img), 160, 120, x0, y0, x1, y1, int(lw), _ptr(col))
        assert rc == capi.MK_OK
        assert np.array_equal(img, want), f"segment {seg[:5]}: {int((img != want).any(-1).sum())} pixels differ"


def test_cpr_line_layer_pixels(gold, mesh):
    # MonkeyGL's full VR overlay for one view: the orientation box plus the
    # CPR path; with the box removed, what remains is the polyline
    img = box(mesh, gold["cpr_rotation"])
    want = gold["cpr_image"]
    line_only = want.copy()
    line_only[img.any(-1)] = 0
    assert line_only.any(), "the golden image holds no CPR line"
    assert np.array_equal(img[-64:, -64:][~line_only[-64:, -64:].any(-1)],
                          want[-64:, -64:][~line_only[-64:, -64:].any(-1)])


def test_invalid_arguments():
    h = C.c_void_p()
    assert capi.lib().mk_mesh_load_stl(b"/nonexistent/human.stl", C.byref(h)) == capi.MK_ERR_INVALID_ARGUMENT
    assert capi.lib().mk_merge_orientation_box(None, None, None, 512, 512) == capi.MK_ERR_INVALID_ARGUMENT
    assert capi.lib().mk_draw_line_rgb(None, 10, 10, 0, 0, 1, 1, 1, None) == capi.MK_ERR_INVALID_ARGUMENT


GLYPHS = ROOT / "oracle" / "_ref" / "resources" / "annotation_glyphs.bin"
REF_HOST = ROOT / "oracle" / "_ref" / "libmkref_host.so"


@pytest.fixture(scope="module")
def font():
    if not GLYPHS.exists() or not REF_HOST.exists():
        pytest.skip("MonkeyGL's glyphs not extracted: run `make -C oracle ref` with the MonkeyGL sources")
    h = C.c_void_p()
    assert capi.lib().mk_font_load(str(GLYPHS).encode(), C.byref(h)) == capi.MK_OK, capi.lib().mk_last_error()
    yield h
    capi.lib().mk_font_destroy(h)


def test_text_matches_monkeygl_textout(font):
    """mk_draw_text_rgb against MonkeyGL's AnnotationUtils::Textout2Image
    (its host library, built from its sources): random printable strings
    with a few bytes that have no glyph, every font size (and an undefined
    one), the three alignments, positions that clip at every edge, random
    colours, several image sizes; plus mk_text_size against GetSize."""
    L = C.CDLL(str(REF_HOST))
    L.mkrh_textout.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float,
                               C.c_void_p, C.c_int, C.c_int]
    rng = np.random.default_rng(77)
    printable = [bytes([c]) for c in range(0x20, 0x7f)]
    extra = ["·".encode(), "é".encode(), b"\t"]
    n = 0
    for case in range(400):
        k = int(rng.integers(0, 14))
        text = b"".join(printable[int(i)] for i in rng.integers(0, len(printable), k))
        if case % 7 == 0:
            text += extra[case % 3] + b"Z"
        w, h = [(512, 512), (97, 41), (10, 10), (300, 64)][case % 4]
        x = int(rng.integers(-60, w + 20))
        y = int(rng.integers(-50, h + 10))
        size = int(rng.integers(-1, 3))
        fmt = int(rng.integers(0, 3))
        col = rng.uniform(0, 1, 3).astype(np.float32)
        if case % 11 == 0:
            col = np.array([1.0, 1.0, 1.0], np.float32)
        mine = rng.integers(0, 256, (h, w, 3), dtype=np.uint8)
        ref = mine.copy()
        rc = capi.lib().mk_draw_text_rgb(font, _ptr(mine), w, h, text, x, y, size, fmt, _ptr(col))
        ok = L.mkrh_textout(text, x, y, size, fmt, float(col[0]), float(col[1]), float(col[2]), _ptr(ref), w, h)
        assert (rc == capi.MK_OK) == (ok == 1)
        diff = int(np.count_nonzero(mine != ref))
        assert diff == 0, f"case {case}: text {text!r} at ({x}, {y}) size {size} format {fmt}: {diff} values differ"
        n += int(np.count_nonzero(mine))
    assert n > 0
    # refused like MonkeyGL: images below 10 pixels, an undefined format
    img = np.zeros((9, 40, 3), np.uint8)
    col = np.ones(3, np.float32)
    assert capi.lib().mk_draw_text_rgb(font, _ptr(img), 40, 9, b"A", 0, 0, 0, 0, _ptr(col)) != capi.MK_OK
    assert capi.lib().mk_draw_text_rgb(font, _ptr(img), 40, 9, b"A", 0, 0, 0, -1, _ptr(col)) != capi.MK_OK
    w, h = C.c_int(), C.c_int()
    assert capi.lib().mk_text_size(font, b"Hello, 3D", 1, C.byref(w), C.byref(h)) == capi.MK_OK
    assert w.value > 0 and h.value == 33
    assert capi.lib().mk_text_size(font, b"a\xc2\xb7", 0, C.byref(w), C.byref(h)) == capi.MK_OK
    assert h.value == -1
