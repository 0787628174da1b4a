"""Known-answer tests of the CPU oracle (oracle/mk_oracle.c).

MonkeyGL ships no tests or golden images, so the restatement is pinned two
ways: these hand-derived cases (constant volume, impulse footprint, LUT
ramp, transparent TF, opaque slab, out-of-volume fills, CPR vs MPR, labels),
and, on the GPU, image-for-image comparison with MonkeyGL's own kernels
(tests/test_gpu_parity.py)."""
import numpy as np
import pytest

import oracle
from monkeygl_b200 import capi
from monkeygl_b200.camera import view_camera


def flat_vr(dims, spacing, angle=0.0, bg=(0, 0, 0, 0), label_params=None, w=64, h=64, rtype=0):
    p = capi.vr_params(w, h, rtype, view_camera(angle), dims, spacing, background=bg)
    lp = label_params
    if lp is None:
        lp = np.zeros((65, 3), np.float32)
        lp[:, 1] = 1
        lp[0] = (1.0, 1700.0, 650.0)
    return capi.vr_params_flat(p, lp)


def axial_plane(dims, spacing, z_index, w=None, h=None, mpr_type=0, half=0.0):
    """Axial plane through voxel-centre row z_index (invert_z false flips z)."""
    X, Y, Z = dims
    sx, sy, sz = spacing
    w = w or X
    h = h or Y
    # f_z = (lt_z)/(sz*Z) then flipped: 1 - f_z = (z_index + 0.5)/Z
    lt_z = (1.0 - (z_index + 0.5) / Z) * sz * Z
    pp = capi.plane_params(w, h, mpr_type, 0, spacing, (1, 0, 0), (0, 1, 0), (0, 0, 1),
                           (0.5 * sx, 0.5 * sy, lt_z), sx, False, half)
    return capi.plane_params_flat(pp), pp


def test_constant_volume_gives_constant_plane():
    vol = np.full((12, 10, 8), 100, np.int16)
    cv = oracle.CpuVolume(vol)
    flat, _ = axial_plane((8, 10, 12), (1.0, 1.0, 1.0), 5)
    for mt in (0, 1, 2):
        for nearest in (0, 1):
            out = cv.render_plane(8, 10, flat, mt, nearest)
            assert (out == 100).all(), (mt, nearest, np.unique(out))


def test_normalized_read_and_scale():
    # 32768 * (v / 32767) truncated: v for |v| small, v+1 near the top of the range
    for v, want in [(0, 0), (1, 1), (-1, -1), (1000, 1000), (-1000, -1000), (32766, 32767), (-32768, -32768)]:
        cv = oracle.CpuVolume(np.full((2, 2, 2), v, np.int16))
        flat, _ = axial_plane((2, 2, 2), (1, 1, 1), 0)
        assert cv.render_plane(2, 2, flat, 1, 1)[0, 0] == want, v


def test_impulse_trilinear_footprint():
    vol = np.zeros((8, 8, 8), np.int16)
    vol[4, 4, 4] = 1000
    cv = oracle.CpuVolume(vol)
    # voxel centre
    assert round(cv.tex3d_linear(4.5 / 8, 4.5 / 8, 4.5 / 8) * 32767) == 1000
    # half a voxel off along x: weight exactly 1/2
    assert abs(cv.tex3d_linear(5.0 / 8, 4.5 / 8, 4.5 / 8) * 32767 - 500) < 1e-3
    # half a voxel off on all axes: 1/8
    assert abs(cv.tex3d_linear(5.0 / 8, 5.0 / 8, 5.0 / 8) * 32767 - 125) < 1e-3
    # outside the footprint
    assert cv.tex3d_linear(6.5 / 8, 4.5 / 8, 4.5 / 8) == 0.0
    # nearest: floor(x * N)
    assert round(cv.tex3d_point(4.99 / 8, 4.01 / 8, 4.5 / 8) * 32767) == 1000
    assert cv.tex3d_point(5.01 / 8, 4.5 / 8, 4.5 / 8) == 0.0


def test_weights_are_quantised_to_eighth_bits():
    vol = np.zeros((1, 1, 2), np.int16)
    vol[0, 0, 1] = 25600
    cv = oracle.CpuVolume(vol)
    # texel coordinate 0 + 1/1024: the fraction rounds to 0
    x = (1.0 / 1024 + 0.5) / 2
    assert cv.tex3d_linear(x, 0.5, 0.5) == 0.0
    # fraction 5/1024 rounds to 1/256
    x = (5.0 / 1024 + 0.5) / 2
    assert abs(cv.tex3d_linear(x, 0.5, 0.5) * 32767 - 100.0) < 1e-2


def test_lut_ramp_lookup_at_entry_centres():
    n = 16
    lut = np.repeat((np.arange(n, dtype=np.float32) / (n - 1))[:, None], 4, axis=1)
    out = np.zeros(4, np.float32)
    for i in range(n):
        oracle.cpu().mko_tex1d_lut(oracle._vp(lut), n, np.float32((i + 0.5) / n), oracle._vp(out))
        assert np.allclose(out, i / (n - 1))
    # clamp below 0 and above 1
    oracle.cpu().mko_tex1d_lut(oracle._vp(lut), n, np.float32(-3.0), oracle._vp(out))
    assert np.allclose(out, 0.0)
    oracle.cpu().mko_tex1d_lut(oracle._vp(lut), n, np.float32(1.0), oracle._vp(out))
    assert np.allclose(out, 1.0)


def _slab_volume():
    vol = np.full((16, 32, 32), -1000, np.int16)
    vol[:, 14:20, :] = 1000          # slab across y (the viewing direction at 0 deg)
    return vol


def test_transparent_tf_paints_background():
    vol = _slab_volume()
    cv = oracle.CpuVolume(vol)
    cv.set_lut(0, np.zeros((256, 4), np.float32))
    flat = flat_vr((32, 32, 16), (1, 1, 1), bg=(0.2, 0.4, 0.6, 1.0))
    img = cv.render_vr(64, 64, 0, flat)
    assert (img.reshape(-1, 3) == [51, 102, 153]).all()


def test_opaque_slab_first_hit_colour():
    vol = _slab_volume()
    cv = oracle.CpuVolume(vol)
    lut = np.zeros((256, 4), np.float32)
    lut[:, :3] = (1.0, 0.5, 0.25)
    lut[160:, 3] = 1.0               # t = (HU - 650)/1700 + 0.5 > ~0.63 opaque
    cv.set_lut(0, lut)
    flat = flat_vr((32, 32, 16), (1, 1, 1))
    img = cv.render_vr(64, 64, 0, flat)
    centre = img[24:40, 24:40].reshape(-1, 3)
    # one colour across the flat slab; headlight along the slab normal: 0.35 + 0.8 + 0.16
    assert len(np.unique(centre, axis=0)) == 1
    r, g, b = centre[0]
    assert r == 255 and abs(int(g) - 167) <= 3 and abs(int(b) - 83) <= 3


def test_surface_flat_slab():
    vol = _slab_volume()
    cv = oracle.CpuVolume(vol)
    flat = flat_vr((32, 32, 16), (1, 1, 1), bg=(0, 0, 0, 0))
    img = cv.render_vr(64, 64, 2, flat)
    centre = img[24:40, 24:40].reshape(-1, 3)
    assert (centre == 255).all()      # N.L + 0.05 saturates
    assert (img[:8, :8] == 0).all()   # misses the volume: background


def test_mip_of_a_bright_sphere():
    vol = np.full((32, 32, 32), 0, np.int16)
    zz, yy, xx = np.mgrid[:32, :32, :32]
    vol[(xx - 16) ** 2 + (yy - 16) ** 2 + (zz - 16) ** 2 <= 25] = 300
    cv = oracle.CpuVolume(vol)
    lp = np.zeros((65, 3), np.float32)
    lp[:, 1] = 1
    lp[0] = (1.0, 400.0, 40.0)
    flat = flat_vr((32, 32, 32), (1, 1, 1), label_params=lp)
    img = cv.render_vr(64, 64, 1, flat)
    # (300 * 32768/32767 - 40)/400 + 0.5 = 1.15 -> saturates to 255 at the centre
    assert img[32, 32, 0] == 255
    # elsewhere (0 - 40)/400 + 0.5 = 0.4 -> 102
    assert img[33, 4, 0] == 102


def test_out_of_volume_fill_values():
    vol = np.full((4, 4, 4), 7, np.int16)
    cv = oracle.CpuVolume(vol)
    pp = capi.plane_params(4, 4, 0, 0, (1, 1, 1), (1, 0, 0), (0, 1, 0), (0, 0, 1), (100, 100, 100), 1.0,
                           False, 0.0)
    for mt in (0, 1, 2):
        assert (cv.render_plane(4, 4, capi.plane_params_flat(pp), mt, 0) == -32768).all()
    pts = np.tile([[100.0, 100.0, 100.0]], (3, 1))
    dirs = np.tile([[1.0, 0, 0]], (3, 1))
    assert (cv.render_cpr(4, pts, dirs, False) == -2048).all()


def test_slab_reductions():
    rng = np.random.default_rng(5)
    vol = rng.integers(-500, 500, (16, 16, 16)).astype(np.int16)
    cv = oracle.CpuVolume(vol)
    flat0, _ = axial_plane((16, 16, 16), (1, 1, 1), 8, mpr_type=0, half=0.0)
    flat2, _ = axial_plane((16, 16, 16), (1, 1, 1), 8, mpr_type=0, half=1.0)
    nearest = [cv.render_plane(16, 16, f, 1, 1) for f in (flat0,)]
    mx = cv.render_plane(16, 16, flat2, 1, 1)
    mn = cv.render_plane(16, 16, flat2, 2, 1)
    av = cv.render_plane(16, 16, flat2, 0, 1)
    # nearest slab of 3 axial samples = voxel rows 7, 8, 9 (z flipped by invert_z false)
    zs = [vol[15 - 7], vol[15 - 8], vol[15 - 9]]
    zs = [vol[z] for z in (7, 8, 9)]
    st = np.stack(zs)
    assert (nearest[0] == vol[8]).all()
    assert (mx == st.max(0)).all()
    assert (mn == st.min(0)).all()
    assert (np.abs(av.astype(int) - np.trunc(st.astype(float).mean(0) * (32768 / 32767))) <= 1).all()


def test_cpr_along_x_matches_axial_row():
    rng = np.random.default_rng(6)
    vol = rng.integers(-1000, 2000, (10, 12, 16)).astype(np.int16)
    cv = oracle.CpuVolume(vol)
    z0, y0 = 4.5, 6.5
    pts = np.array([[0.5, y0, z0]])
    dirs = np.array([[1.0, 0.0, 0.0]])
    cpr = cv.render_cpr(15, pts, dirs, True)
    pp = capi.plane_params(15, 1, 0, 0, (1, 1, 1), (1, 0, 0), (0, 1, 0), (0, 0, 1), (0.5, y0, z0), 1.0, True, 0.0)
    mpr = cv.render_plane(15, 1, capi.plane_params_flat(pp), 0, 0)
    assert np.abs(cpr[0].astype(int) - mpr[0]).max() <= 1
    assert (cpr[0] == vol[4, 6, :15]).all()


def test_label_caps_limit_object_opacity():
    vol = np.full((8, 32, 16), 1000, np.int16)
    labels = np.zeros_like(vol, np.uint8)
    labels[:, :16] = 1
    lut = np.zeros((256, 4), np.float32)
    lut[:, :3] = 1.0
    lut[:, 3] = 0.2
    lp = np.zeros((65, 3), np.float32)
    lp[:, 1] = 1
    lp[0] = (1.0, 1700, 650)
    lp[1] = (0.3, 1700, 650)
    cv = oracle.CpuVolume(vol, labels)
    cv.set_lut(0, lut)
    cv.set_lut(1, lut)
    capped = cv.render_vr(32, 32, 0, flat_vr((16, 32, 8), (1, 1, 1), label_params=lp, w=32, h=32))
    lp[1, 0] = 1.0
    free = cv.render_vr(32, 32, 0, flat_vr((16, 32, 8), (1, 1, 1), label_params=lp, w=32, h=32))
    assert capped[16, 16].sum() > 0 and free[16, 16].sum() > 0
    assert not np.array_equal(capped, free)


def test_exact64_mode_close_to_tex32():
    rng = np.random.default_rng(7)
    vol = rng.integers(-1000, 2000, (20, 24, 28)).astype(np.int16)
    cv = oracle.CpuVolume(vol)
    flat, _ = axial_plane((28, 24, 20), (1, 1, 1), 9)
    a = cv.render_plane(28, 24, flat, 0, 0, precision=oracle.TEX32)
    b = cv.render_plane(28, 24, flat, 0, 0, precision=oracle.EXACT64)
    assert np.abs(a.astype(int) - b).max() <= 12   # 8-bit weights on a 3000 HU range
