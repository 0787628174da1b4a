"""Parity of the sm_100a kernels with MonkeyGL's own CUDA kernels.

MonkeyGL's core/kernel.cu and core/CuDataManager.cu, built unmodified for
sm_100a (oracle/_ref/libmkref_gpu.so), render the same volume, transfer
functions, camera and planes; every image must match within the bar:

* VR / MIP / surface and trilinear MPR / CPR: max error <= 2/255 per channel
  (2 HU for int16 planes) and PSNR >= 45 dB;
* nearest-neighbour MPR: bit-exact.

In practice the kernels reproduce MonkeyGL's arithmetic exactly, so the tests
also report the fraction of identical pixels.  A second, looser check runs
against the CPU restatement (oracle/mk_oracle.c), which emulates the texture
unit and so differs slightly."""
import numpy as np
import pytest

import oracle
from monkeygl_b200 import capi
from monkeygl_b200.camera import Camera, view_camera
from monkeygl_b200.phantom import make_phantom, make_tf_control_points, make_tf_lut
from monkeygl_b200 import workloads as wl

pytestmark = pytest.mark.gpu

MAX_ERR = 2          # per channel, out of 255 (or HU for planes)
MIN_PSNR = 45.0


def psnr(a, b, peak=255.0):
    d = a.astype(np.float64) - b.astype(np.float64)
    mse = (d * d).mean()
    return 99.0 if mse == 0 else 10 * np.log10(peak * peak / mse)


def assert_image_parity(mine, ref, what, exact=False):
    d = np.abs(mine.astype(np.int32) - ref.astype(np.int32))
    frac = float((d == 0).mean())
    print(f"{what}: identical {frac:.6f}, max {d.max()}, psnr {psnr(mine, ref):.1f}")
    if exact:
        assert d.max() == 0, f"{what}: {np.count_nonzero(d)} values differ"
    assert d.max() <= MAX_ERR, f"{what}: max error {d.max()}"
    assert psnr(mine, ref) >= MIN_PSNR


@pytest.fixture(scope="module")
def ref():
    if not oracle.ref_gpu_available():
        pytest.fail("oracle/_ref/libmkref_gpu.so is missing: run `make -C oracle ref-gpu`")
    r = oracle.RefGPU()
    assert r.device_count() >= 1
    return r


@pytest.fixture(scope="module")
def small():
    return wl.make_workload("small")


@pytest.fixture(scope="module")
def small_vol(small):
    v = capi.Volume(small.phantom.volume)
    v.set_transfer_function(0, small.luts[0])
    v.set_label_params(small.label_params)
    yield v
    v.close()


def load_ref(ref, w):
    ref.set_volume(w.phantom.volume)
    ref.set_mask(w.phantom.labels)
    ref.clear_tfs()
    for l, lut in w.luts.items():
        ref.set_lut(l, lut)


def params(w, angle, rtype, size=None, **kw):
    size = size or w.width
    return capi.vr_params(size, size, rtype, view_camera(angle), w.dims, w.spacing, **kw)


@pytest.mark.parametrize("rtype", [0, 1, 2], ids=["vr", "mip", "surface"])
@pytest.mark.parametrize("angle", [0.0, 45.0, 90.0])
def test_small_raycast_matches_reference(ref, small, small_vol, rtype, angle):
    load_ref(ref, small)
    p = params(small, angle, rtype)
    r = ref.render(p.width, p.height, rtype, capi.vr_params_flat(p, small.label_params))
    m = small_vol.render_vr(p)
    assert_image_parity(m, r, f"small type {rtype} {angle}", exact=True)
    p.flags = capi.VR_NO_SKIP
    assert np.array_equal(small_vol.render_vr(p), m), "empty-space skipping changed the image"
    p.flags = capi.VR_NO_COOP
    assert np.array_equal(small_vol.render_vr(p), m), "the cooperative tail changed the image"


def test_small_camera_variants(ref, small, small_vol):
    load_ref(ref, small)
    cases = []
    cam = Camera(); cam.anterior(); cam.zoom(1.7); cam.rotate(33.0, 12.0); cam.pan(25, -40)
    cases.append(("zoom-pan", cam, dict()))
    cam = Camera(); cam.head(); cam.rotate(-20.0, 5.0)
    cases.append(("head", cam, dict(background=(0.1, 0.3, 0.5, 1.0))))
    cam = Camera(); cam.foot(); cam.zoom(0.6)
    cases.append(("foot-zoomout", cam, dict(invert_z=True)))
    cam = Camera(); cam.left(); cam.rotate(0.0, 70.0)
    cases.append(("left", cam, dict(voi=(10, 100, 20, 90, 5, 80))))
    for name, cam, kw in cases:
        for rtype in (0, 1, 2):
            p = capi.vr_params(384, 256, rtype, cam, small.dims, small.spacing, **kw)
            r = ref.render(384, 256, rtype, capi.vr_params_flat(p, small.label_params))
            assert_image_parity(small_vol.render_vr(p), r, f"{name} type {rtype}", exact=True)


def test_rgba_output_and_device_output(small, small_vol):
    import torch
    p = params(small, 30.0, 0)
    rgb = small_vol.render_vr(p)
    p.pixel_format = capi.PIXEL_RGBA8
    rgba = small_vol.render_vr(p)
    assert np.array_equal(rgba[..., :3], rgb) and (rgba[..., 3] == 255).all()
    p.pixel_format = capi.PIXEL_RGB8
    dev = torch.empty(p.width * p.height * 3, dtype=torch.uint8, device="cuda")
    s = torch.cuda.Stream()
    small_vol.render_vr_device(p, dev.data_ptr(), s.cuda_stream)
    s.synchronize()
    assert np.array_equal(dev.cpu().numpy().reshape(rgb.shape), rgb)


def test_host_output_paths_agree(labelled):
    """With host output, the image is copied while the hand-off launch runs
    and the handed-over pixels are patched in afterwards from the hand-off
    launch's (pixel, rgb) list.  Pinned and pageable host buffers, RGB and
    RGBA, on the default and on a caller's stream, must equal the device
    output of the same frame, which no patch is involved in."""
    import torch
    w = labelled
    v = capi.Volume(w.phantom.volume)
    v.set_mask(w.phantom.labels)
    for l, lut in w.luts.items():
        v.set_transfer_function(l, lut)
    v.set_label_params(w.label_params)
    for ang in (0.0, 35.0, 250.0):
        p = params(w, ang, 0, size=640)
        dev = torch.empty(p.width * p.height * 3, dtype=torch.uint8, device="cuda")
        s = torch.cuda.Stream()
        v.render_vr_device(p, dev.data_ptr(), s.cuda_stream)
        s.synchronize()
        want = dev.cpu().numpy().reshape(p.height, p.width, 3)
        pageable = v.render_vr(p)
        pinned = torch.empty(p.width * p.height * 3, dtype=torch.uint8, pin_memory=True)
        v.render_vr(p, out=pinned.numpy().reshape(p.height, p.width, 3))
        assert np.array_equal(pageable, want), f"pageable {ang}"
        assert np.array_equal(pinned.numpy().reshape(want.shape), want), f"pinned {ang}"
        p.pixel_format = capi.PIXEL_RGBA8
        rgba = v.render_vr(p)
        assert np.array_equal(rgba[..., :3], want) and (rgba[..., 3] == 255).all(), f"rgba {ang}"
    v.close()


@pytest.mark.parametrize("size", [(77, 33), (333, 45), (1, 1), (2, 511)])
def test_odd_image_sizes(ref, small, small_vol, size):
    load_ref(ref, small)
    w, h = size
    p = capi.vr_params(w, h, 0, view_camera(20.0), small.dims, small.spacing)
    r = ref.render(w, h, 0, capi.vr_params_flat(p, small.label_params))
    assert_image_parity(small_vol.render_vr(p), r, f"size {size}", exact=True)


def test_odd_volume_shapes(ref):
    rng = np.random.default_rng(11)
    for dims in [(17, 9, 5), (8, 8, 8), (3, 40, 2), (31, 1, 13)]:
        X, Y, Z = dims
        vox = rng.integers(-1000, 2000, (Z, Y, X)).astype(np.int16)
        lut = make_tf_lut(make_tf_control_points(rng))
        lp = np.zeros((65, 3), np.float32); lp[:, 1] = 1; lp[0] = (1.0, 1700, 650)
        v = capi.Volume(vox)
        v.set_transfer_function(0, lut)
        v.set_label_params(lp)
        ref.set_volume(vox); ref.set_mask(None); ref.clear_tfs(); ref.set_lut(0, lut)
        spacing = (0.5, 0.7, 1.1)
        for rtype in (0, 1, 2):
            for ang in (0.0, 63.0):
                p = capi.vr_params(96, 80, rtype, view_camera(ang), dims, spacing)
                r = ref.render(96, 80, rtype, capi.vr_params_flat(p, lp))
                assert_image_parity(v.render_vr(p), r, f"{dims} type {rtype} {ang}", exact=True)
        v.close()


@pytest.fixture(scope="module")
def labelled():
    p = make_phantom((96, 80, 120), (0.7422, 0.7422, 1.0), 99, with_labels=True)
    return wl.make_workload("body", bg_alpha=0.4, phantom=p)


@pytest.mark.parametrize("bg", [0.4, 0.8])
def test_multilabel_matches_reference(ref, labelled, bg):
    w = labelled
    lp = w.label_params.copy()
    lp[0, 0] = bg
    v = capi.Volume(w.phantom.volume)
    v.set_mask(w.phantom.labels)
    for l, lut in w.luts.items():
        v.set_transfer_function(l, lut)
    v.set_label_params(lp)
    load_ref(ref, w)
    for rtype in (0, 1):
        for ang in (0.0, 50.0, 130.0):
            p = params(w, ang, rtype, size=256)
            r = ref.render(256, 256, rtype, capi.vr_params_flat(p, lp))
            m = v.render_vr(p)
            assert_image_parity(m, r, f"labels bg {bg} type {rtype} {ang}", exact=True)
            p.flags = capi.VR_NO_SKIP
            assert np.array_equal(v.render_vr(p), m)
            p.flags = capi.VR_NO_COOP
            assert np.array_equal(v.render_vr(p), m)
            p.flags = capi.VR_NO_COOP | capi.VR_NO_SKIP
            assert np.array_equal(v.render_vr(p), m)
    # many capped labels force the local-memory path
    lp2 = lp.copy()
    lp2[:20, 0] = 0.5
    v.set_label_params(lp2)
    p = params(w, 20.0, 0, size=200)
    r = ref.render(200, 200, 0, capi.vr_params_flat(p, lp2))
    assert_image_parity(v.render_vr(p), r, "labels local caps", exact=True)
    v.close()


def test_mip_label_windows_match_reference(ref, labelled):
    """MIP takes a loop without label fetches when every label present is
    visible and all of them share one window with a positive width (the
    window is monotonic, so the maximum of the windowed samples is the
    window of the largest raw sample); per-label windows or a hidden label
    take the general loop (widths are positive: mk_volume_set_label_params
    refuses others).  Every variant equals
    MonkeyGL's image (core/kernel.cu:326-364), with and without skipping."""
    w = labelled
    v = capi.Volume(w.phantom.volume)
    v.set_mask(w.phantom.labels)
    for l, lut in w.luts.items():
        v.set_transfer_function(l, lut)
    load_ref(ref, w)
    base = w.label_params.copy()
    variants = [("uniform", base)]
    lp = base.copy()
    lp[2, 1:] = (900.0, 300.0)
    variants.append(("per-label window", lp))
    lp = base.copy()
    lp[3, 0] = 0.0
    variants.append(("hidden label", lp))
    lp = base.copy()
    lp[0, 0] = 0.0
    variants.append(("hidden background", lp))
    lp = base.copy()
    lp[:5, 1:] = (400.0, 40.0)
    variants.append(("uniform narrow window", lp))
    for name, lp in variants:
        v.set_label_params(lp)
        for ang in (0.0, 70.0, 200.0):
            p = params(w, ang, 1, size=256)
            r = ref.render(256, 256, 1, capi.vr_params_flat(p, lp))
            m = v.render_vr(p)
            assert_image_parity(m, r, f"mip {name} {ang}", exact=True)
            p.flags = capi.VR_NO_SKIP
            assert np.array_equal(v.render_vr(p), m), f"mip {name} {ang} without skipping"
    v.close()


def test_cardiac_frame_matches_reference(ref):
    w = wl.make_workload("cardiac")
    v = capi.Volume(w.phantom.volume)
    v.set_transfer_function(0, w.luts[0])
    v.set_label_params(w.label_params)
    load_ref(ref, w)
    for rtype in (0, 1):
        p = params(w, 40.0, rtype)
        r = ref.render(p.width, p.height, rtype, capi.vr_params_flat(p, w.label_params))
        assert_image_parity(v.render_vr(p), r, f"cardiac type {rtype}", exact=True)
    v.close()


def test_cooperative_tail_matches_reference(ref, labelled):
    """VR warps finish their last rays with several lanes per ray (lanes
    evaluate the samples ahead, then walk MonkeyGL's schedule over them).
    Sparse images -- a small VOI, a zoomed-out camera, thin image strips --
    leave most warps with few rays from the start, so most samples of these
    frames go through that path.  Each image must equal MonkeyGL's and the
    one-lane-per-ray march, with and without empty-space skipping."""
    w = labelled
    lp = w.label_params.copy()
    v = capi.Volume(w.phantom.volume)
    v.set_mask(w.phantom.labels)
    for l, lut in w.luts.items():
        v.set_transfer_function(l, lut)
    v.set_label_params(lp)
    load_ref(ref, w)
    cams = []
    cam = Camera(); cam.anterior(); cam.zoom(0.35); cam.rotate(25.0, 10.0)
    cams.append(("zoomed-out", cam, {}, (256, 256)))
    cam = Camera(); cam.left(); cam.rotate(40.0, -15.0)
    cams.append(("voi", cam, dict(voi=(30, 50, 20, 60, 40, 90)), (256, 192)))
    cam = Camera(); cam.anterior(); cam.zoom(2.5); cam.rotate(70.0, 0.0)
    cams.append(("strip", cam, {}, (509, 3)))
    cam = Camera(); cam.head(); cam.rotate(-35.0, 20.0)
    cams.append(("column", cam, dict(invert_z=True), (5, 300)))
    for name, cam, kw, (W, H) in cams:
        for flags in (0, capi.VR_NO_SKIP):
            p = capi.vr_params(W, H, 0, cam, w.dims, w.spacing, **kw)
            p.flags = flags
            r = ref.render(W, H, 0, capi.vr_params_flat(p, lp))
            m = v.render_vr(p)
            assert_image_parity(m, r, f"coop {name} flags {flags}", exact=True)
            p.flags = flags | capi.VR_NO_COOP
            assert np.array_equal(v.render_vr(p), m), f"coop {name}: differs from the one-lane march"
    v.close()


def test_tail_launch_matches_reference(ref, labelled):
    """Once most tiles of a VR frame have finished, the rays still marching
    are handed (state and opacity caps) to a second launch that finishes
    them with several lanes per ray.  Frames of fewer tiles than the hand-off
    threshold hand over every ray still marching after 16 steps; larger ones
    only the frame's tail.  Every image must equal MonkeyGL's and the frame
    rendered without the hand-off, also when two streams render the same
    volume at once (each stream has its own hand-off list)."""
    import torch
    w = labelled
    lp = w.label_params.copy()
    v = capi.Volume(w.phantom.volume)
    v.set_mask(w.phantom.labels)
    for l, lut in w.luts.items():
        v.set_transfer_function(l, lut)
    v.set_label_params(lp)
    load_ref(ref, w)
    frames = []
    for ang, (W, H) in ((0.0, (1024, 768)), (65.0, (1024, 1024)), (130.0, (256, 256)), (200.0, (640, 360))):
        p = capi.vr_params(W, H, 0, view_camera(ang), w.dims, w.spacing)
        r = ref.render(W, H, 0, capi.vr_params_flat(p, lp))
        m = v.render_vr(p)
        assert_image_parity(m, r, f"tail {ang} {W}x{H}", exact=True)
        p.flags = capi.VR_NO_TAIL
        assert np.array_equal(v.render_vr(p), m), f"tail {ang}: differs from the frame without the hand-off"
        p.flags = 0
        frames.append((p, m))
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    outs = [torch.empty(p.width * p.height * 3, dtype=torch.uint8, device="cuda") for p, _ in frames]
    for rep in range(3):
        for i, (p, _) in enumerate(frames):
            v.render_vr_device(p, outs[i].data_ptr(), streams[i % 2].cuda_stream)
        torch.cuda.synchronize()
        for i, (p, m) in enumerate(frames):
            got = outs[i].cpu().numpy().reshape(p.height, p.width, 3)
            assert np.array_equal(got, m), f"two streams, frame {i} repeat {rep}"
    v.close()


def _plane(pl, mpr_type, sampling, spacing, half):
    return capi.plane_params(pl.width, pl.height, mpr_type, sampling, spacing, pl.dir_h, pl.dir_v,
                             pl.dir_n, pl.left_top, pl.pixel_spacing, False, half)


@pytest.mark.parametrize("half", [0.0, 1.0, 1.5, 2.0])
def test_mpr_matches_reference(ref, small, small_vol, half):
    load_ref(ref, small)
    for pl in wl.mpr_planes(small.phantom, size=256, n_oblique=4):
        for mt in (0, 1, 2):
            for sampling in (0, 1):
                pp = _plane(pl, mt, sampling, small.spacing, half)
                r = ref.plane(pp.width, pp.height, capi.plane_params_flat(pp), mt, sampling)
                m = small_vol.render_plane(pp)
                assert_image_parity(m, r, f"mpr {pl.name} t{mt} s{sampling} h{half}", exact=(sampling == 1))


def test_cpr_matches_reference(ref, small, small_vol):
    load_ref(ref, small)
    path = wl.vessel_path(small.phantom, rows=300)
    for builder in (wl.cpr_straightened, wl.cpr_stretched):
        pts, dirs = builder(path, 128)
        r = ref.cpr(128, pts, dirs, False)
        m = small_vol.render_cpr(128, pts, dirs, False)
        assert_image_parity(m, r, f"cpr {builder.__name__}", exact=True)
        r = ref.cpr(128, pts, dirs, True)
        m = small_vol.render_cpr(128, pts, dirs, True)
        assert_image_parity(m, r, f"cpr {builder.__name__} inverted", exact=True)


def test_against_cpu_oracle(small, small_vol):
    cv = oracle.CpuVolume(small.phantom.volume)
    cv.set_lut(0, small.luts[0])
    for rtype, min_psnr in ((0, 45.0), (1, 55.0)):
        p = params(small, 45.0, rtype)
        c = cv.render_vr(p.width, p.height, rtype, capi.vr_params_flat(p, small.label_params))
        m = small_vol.render_vr(p)
        print(f"cpu oracle type {rtype}: psnr {psnr(m, c):.1f}")
        assert psnr(m, c) >= min_psnr
    pl = wl.mpr_planes(small.phantom, size=256, n_oblique=1)[3]
    pp = _plane(pl, 0, 0, small.spacing, 0.0)
    c = cv.render_plane(256, 256, capi.plane_params_flat(pp), 0, 0)
    m = small_vol.render_plane(pp)
    assert np.abs(c.astype(int) - m).max() <= 16
    assert psnr(m, c, peak=4096.0) >= MIN_PSNR


def test_error_against_fp64_method(small, small_vol):
    """The FP32 path against the same method in FP64 with exact filtering."""
    cv = oracle.CpuVolume(small.phantom.volume)
    cv.set_lut(0, small.luts[0])
    p = params(small, 45.0, 1)
    e = cv.render_vr(p.width, p.height, 1, capi.vr_params_flat(p, small.label_params), precision=oracle.EXACT64)
    m = small_vol.render_vr(p)
    print(f"MIP vs FP64 method: psnr {psnr(m, e):.1f}, max {np.abs(m.astype(int) - e).max()}")
    assert psnr(m, e) >= 40.0


def test_sample_counts(small, small_vol):
    cv = oracle.CpuVolume(small.phantom.volume)
    cv.set_lut(0, small.luts[0])
    for rtype in (0, 1, 2):
        p = params(small, 45.0, rtype)
        n = small_vol.count_samples(p)
        _, nc = cv.render_vr(p.width, p.height, rtype, capi.vr_params_flat(p, small.label_params),
                             with_samples=True)
        assert n > 0 and abs(n - nc) <= 0.01 * nc, (rtype, n, nc)
        s, vox, lab = small_vol.count_footprint(p)
        assert s == n and 0 < vox <= np.prod(small.dims) and lab == 0


def test_invalid_arguments_on_device(small_vol):
    p = capi.vr_params(64, 64, 0, view_camera(0.0), (128, 128, 96), (0.35, 0.35, 0.3))
    p.scale = 0.0
    with pytest.raises(capi.MonkeyGLError) as e:
        small_vol.render_vr(p)
    assert e.value.status == capi.MK_ERR_INVALID_ARGUMENT
    p.scale = 1.0
    p.render_type = 7
    with pytest.raises(capi.MonkeyGLError):
        small_vol.render_vr(p)
    bad = np.zeros((65, 3), np.float32)
    with pytest.raises(capi.MonkeyGLError):
        small_vol.set_label_params(bad)                   # ww = 0
    with pytest.raises(capi.MonkeyGLError):
        small_vol.set_transfer_function(65, np.zeros((4, 4), np.float32))
    with pytest.raises(ValueError):
        small_vol.set_mask(np.zeros((2, 2, 2), np.uint8))
    pp = capi.plane_params(8, 8, 5, 0, (1, 1, 1), (1, 0, 0), (0, 1, 0), (0, 0, 1), (0, 0, 0), 1.0, False, 0.0)
    with pytest.raises(capi.MonkeyGLError):
        small_vol.render_plane(pp)
