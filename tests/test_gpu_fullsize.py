"""Parity with MonkeyGL's own CUDA kernels at the benchmark configurations'
full sizes.

The other parity tests run on small phantoms; indexing that depends on the
size of the volume, the brick grid, the schedule table or the frame (the
body volume has 1559 slices, a schedule of about 2700 entries, 64x64x195
bricks and a 409 MB label volume) is exercised only here:

* body 512x512x1559 with 4 labelled objects, per-object 256-entry LUTs and
  opacity caps, background cap 0.4 and 0.8, 1024x1024 VR and MIP at views
  0/10/90/190 degrees, with and without the frame-tail hand-off and
  empty-space skipping (core/kernel.cu:133-364);
* cardiac 512x512x361: axial, sagittal and coronal planes plus 8 seeded
  oblique planes at 512x512, nearest and trilinear, one sample and a
  3-sample MIP slab (core/kernel.cu:570-837), and the same planes through
  the display window the reference's HTML client applies (ww 400, wl 40);
* body stretched and straightened CPR of 512x1024 along a 200-point
  Catmull-Rom spline through a vessel centreline (core/kernel.cu:839-918).

Every image must equal MonkeyGL's bit for bit (oracle/_ref/libmkref_gpu.so,
built from its unmodified sources)."""
import numpy as np
import pytest

import oracle
from monkeygl_b200 import capi
from monkeygl_b200 import workloads as wl
from monkeygl_b200.camera import view_camera

pytestmark = pytest.mark.gpu

VIEWS = (0.0, 10.0, 90.0, 190.0)


def assert_same(mine, ref, what):
    d = mine.astype(np.int32) != ref.astype(np.int32)
    n = int(np.count_nonzero(d))
    print(f"{what}: {n} values differ of {d.size}")
    assert n == 0, f"{what}: {n} values differ (max |diff| "\
                   f"{np.abs(mine.astype(np.int32) - ref.astype(np.int32)).max()})"


@pytest.fixture(scope="module")
def ref():
    if not oracle.ref_gpu_available():
        pytest.fail("oracle/_ref/libmkref_gpu.so is missing: run `make -C oracle ref-gpu`")
    return oracle.RefGPU()


@pytest.fixture(scope="module")
def body():
    return wl.make_workload("body", bg_alpha=0.4)


@pytest.fixture(scope="module")
def body_vol(body):
    v = capi.Volume(body.phantom.volume)
    v.set_mask(body.phantom.labels)
    for l, lut in body.luts.items():
        v.set_transfer_function(l, lut)
    v.set_label_params(body.label_params)
    yield v
    v.close()


def _load_ref(ref, w):
    ref.set_volume(w.phantom.volume)
    ref.set_mask(w.phantom.labels)
    ref.clear_tfs()
    for l, lut in w.luts.items():
        ref.set_lut(l, lut)


@pytest.mark.parametrize("bg", [0.4, 0.8])
def test_body_1024_matches_reference(ref, body, body_vol, bg):
    _load_ref(ref, body)
    lp = body.label_params.copy()
    lp[0, 0] = bg
    body_vol.set_label_params(lp)
    try:
        for rtype in (capi.RENDER_VR, capi.RENDER_MIP):
            for ang in VIEWS:
                p = capi.vr_params(1024, 1024, rtype, view_camera(ang), body.dims, body.spacing)
                r = ref.render(1024, 1024, rtype, capi.vr_params_flat(p, lp))
                m = body_vol.render_vr(p)
                assert_same(m, r, f"body bg {bg} type {rtype} {ang:.0f} deg")
                assert m.any()
                for flags in (capi.VR_NO_TAIL, capi.VR_NO_SKIP, capi.VR_NO_TAIL | capi.VR_NO_SKIP):
                    p.flags = flags
                    assert_same(body_vol.render_vr(p), r, f"body bg {bg} type {rtype} {ang:.0f} deg flags {flags}")
    finally:
        body_vol.set_label_params(body.label_params)


@pytest.fixture(scope="module")
def cardiac():
    return wl.make_workload("cardiac")


@pytest.fixture(scope="module")
def cardiac_vol(cardiac):
    v = capi.Volume(cardiac.phantom.volume)
    v.set_transfer_function(0, cardiac.luts[0])
    v.set_label_params(cardiac.label_params)
    yield v
    v.close()


def _plane(pl, mpr_type, sampling, spacing, half):
    return capi.plane_params(pl.width, pl.height, mpr_type, sampling, spacing, pl.dir_h, pl.dir_v,
                             pl.dir_n, pl.left_top, pl.pixel_spacing, False, half)


def test_cardiac_mpr_planes_match_reference(ref, cardiac, cardiac_vol):
    _load_ref(ref, cardiac)
    planes = wl.mpr_planes(cardiac.phantom, size=512, n_oblique=8)
    assert len(planes) == 11
    for pl in planes:
        for sampling in (capi.SAMPLE_LINEAR, capi.SAMPLE_NEAREST):
            for mt, half in ((capi.MPR_AVERAGE, 0.0), (capi.MPR_MIP, 1.0)):
                pp = _plane(pl, mt, sampling, cardiac.spacing, half)
                r = ref.plane(512, 512, capi.plane_params_flat(pp), mt, sampling)
                m = cardiac_vol.render_plane(pp)
                assert_same(m, r, f"cardiac {pl.name} type {mt} sampling {sampling} half {half}")
                assert (m > -32768).any()


def cornerstone_window(plane, ww, wc):
    """The display window of MonkeyGL's HTML client: decodeMPR
    (examples/html/js/utils.js:62-118) gives ww 400 / wc 40 to cornerstone
    0.12.2, whose generateLut (examples/html/js/libs/cornerstone@0.12.2.js:
    688-733) computes ((x - wc) / ww + 0.5) * 255 in double and stores it in
    a Uint8ClampedArray (clamp to [0, 255], round half to even)."""
    v = ((plane.astype(np.float64) - wc) / ww + 0.5) * 255.0
    return np.rint(np.clip(v, 0.0, 255.0)).astype(np.uint8)


def test_window_epilogue_matches_client(ref, cardiac, cardiac_vol):
    """mk_render_plane_u8 on the cardiac planes at W/L 400/40 equals the
    client's window applied to MonkeyGL's int16 plane, value for value."""
    _load_ref(ref, cardiac)
    for pl in wl.mpr_planes(cardiac.phantom, size=512, n_oblique=8):
        for sampling in (capi.SAMPLE_LINEAR, capi.SAMPLE_NEAREST):
            pp = _plane(pl, capi.MPR_AVERAGE, sampling, cardiac.spacing, 0.0)
            r = ref.plane(512, 512, capi.plane_params_flat(pp), capi.MPR_AVERAGE, sampling)
            m = cardiac_vol.render_plane_u8(pp, 400.0, 40.0)
            assert_same(m, cornerstone_window(r, 400.0, 40.0), f"window {pl.name} sampling {sampling}")


def test_window_epilogue_every_int16_value():
    """Every int16 value through the window.  A 256x256x2 volume holds each
    int16 value once per slice; a nearest-sampled axial plane through the
    first slice's voxel centres returns them (scaled as MonkeyGL's
    normalized read scales them), so the windowed plane must be the client's
    window of that plane -- including the values where
    ((x - wc)/ww + 0.5) * 255 is an exact half (x - wc a multiple of 80 at
    ww 400), and other windows (ww 1, ww 4096, a fractional centre)."""
    vals = np.arange(-32768, 32768, dtype=np.int32).astype(np.int16).reshape(256, 256)
    vox = np.stack([vals, vals])
    v = capi.Volume(vox)
    try:
        pp = capi.plane_params(256, 256, capi.MPR_AVERAGE, capi.SAMPLE_NEAREST, (1.0, 1.0, 1.0), (1, 0, 0),
                               (0, 1, 0), (0, 0, 1), (0.5, 0.5, 1.5), 1.0, False, 0.0)
        plane = v.render_plane(pp)
        assert len(np.unique(plane)) > 65000
        for ww, wc in ((400.0, 40.0), (1.0, 0.0), (4096.0, -1024.0), (255.0, 127.5), (3.0, 1.0)):
            m = v.render_plane_u8(pp, ww, wc)
            assert_same(m, cornerstone_window(plane, ww, wc), f"window ww {ww} wc {wc}")
    finally:
        v.close()


def test_body_cpr_512x1024_matches_reference(ref, body, body_vol):
    _load_ref(ref, body)
    path = wl.vessel_path(body.phantom, n_points=200, rows=1024)
    for builder in (wl.cpr_stretched, wl.cpr_straightened):
        pts, dirs = builder(path, 512)
        assert pts.shape == (1024, 3)
        for inv in (False, True):
            r = ref.cpr(512, pts, dirs, inv)
            m = body_vol.render_cpr(512, pts, dirs, inv)
            assert_same(m, r, f"body cpr {builder.__name__} invert {inv}")
            assert (m != -2048).any()
