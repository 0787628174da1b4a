"""Occupancy maps built at upload, read back through mk_volume_brick_maps and
compared with numpy.

* Value bounds: for every 8^3 brick, the minimum and maximum voxel of the
  brick grown by one voxel on every side (clamped to the volume) -- every
  voxel a trilinear tap of a sample the brick owns can touch.  Empty-space
  skipping relies on these bounds, so they must be exact.
* Label sets: the labels (0..64; larger values count as 64) among each
  brick's own voxels, and the labels present anywhere.

The body volume (512x512x1559 with its 4-object label volume) and a volume
whose x, y and z are multiples of no brick size take the row kernels
(rows of whole bricks) and the per-brick kernels respectively; a third
volume has whole bricks across x but ragged y and z."""
import numpy as np
import pytest

from monkeygl_b200 import capi
from monkeygl_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _grown(a, axis, fn):
    """fn-reduction of each 8-long brick along `axis`, grown by one element
    on both sides (clamped at the ends)."""
    a = np.moveaxis(a, axis, -1)
    n = a.shape[-1]
    nb = -(-n // 8)
    a = np.pad(a, [(0, 0)] * (a.ndim - 1) + [(0, nb * 8 - n)], mode="edge")
    own = fn.reduce(a.reshape(a.shape[:-1] + (nb, 8)), axis=-1)
    left = np.concatenate([a[..., :1], a[..., 7:nb * 8 - 1:8]], axis=-1)
    right = np.concatenate([a[..., 8::8], a[..., -1:]], axis=-1)
    return np.moveaxis(fn(fn(own, left), right), -1, axis)


def numpy_minmax(vox):
    lo, hi = vox, vox
    for ax in (2, 1, 0):
        lo = _grown(lo, ax, np.minimum)
        hi = _grown(hi, ax, np.maximum)
    return lo, hi


def numpy_label_sets(lab):
    Z, Y, X = lab.shape
    nbz, nby, nbx = -(-Z // 8), -(-Y // 8), -(-X // 8)
    lab = np.minimum(lab, 64)
    lab = np.pad(lab, [(0, nbz * 8 - Z), (0, nby * 8 - Y), (0, nbx * 8 - X)], mode="edge")
    bricks = lab.reshape(nbz, 8, nby, 8, nbx, 8)
    words = np.zeros((nbz, nby, nbx, 3), np.uint32)
    present = np.zeros(65, bool)
    for l in np.unique(lab):
        has = (bricks == l).any(axis=(1, 3, 5))
        words[..., l // 32] |= np.where(has, np.uint32(1) << np.uint32(l % 32), np.uint32(0))
        present[l] = True
    return words, present


def check_maps(vox, lab, what):
    v = capi.Volume(vox)
    try:
        if lab is not None:
            v.set_mask(lab)
        mm, words, present = v.brick_maps()
        lo, hi = numpy_minmax(vox)
        assert mm.shape[:3] == lo.shape, (mm.shape, lo.shape)
        bad = int(np.count_nonzero(mm[..., 0] != lo) + np.count_nonzero(mm[..., 1] != hi))
        print(f"{what}: {lo.size} bricks, {bad} wrong bounds")
        assert bad == 0
        if lab is None:
            assert (words[..., 0] == 1).all() and (words[..., 1:] == 0).all()
            assert present[0] and not present[1:].any()
        else:
            want, want_present = numpy_label_sets(lab)
            bad = int(np.count_nonzero(words != want))
            print(f"{what}: {bad} wrong label words")
            assert bad == 0
            assert np.array_equal(present, want_present)
    finally:
        v.close()


def test_brick_maps_body():
    w = wl.make_workload("body")
    check_maps(w.phantom.volume, w.phantom.labels, "body")


@pytest.mark.parametrize("dims", [(100, 90, 70), (64, 60, 45), (8, 8, 8), (7, 3, 2), (2048, 16, 9),
                                  (200, 40, 33), (24, 20, 17)])
def test_brick_maps_shapes(dims):
    X, Y, Z = dims
    rng = np.random.default_rng(X * 7 + Y * 3 + Z)
    vox = rng.integers(-32768, 32768, (Z, Y, X), dtype=np.int32).astype(np.int16)
    # smooth regions too, so that bounds differ between neighbours by little
    vox[: Z // 2] = (np.arange(X)[None, None, :] * 37 - 2000).astype(np.int16)
    lab = rng.choice(np.array([0, 0, 0, 1, 2, 5, 33, 64, 70, 200], np.uint8), size=(Z, Y, X))
    lab[:, : Y // 2] = 0
    check_maps(vox, lab, f"{dims}")
    check_maps(vox, None, f"{dims} no labels")


def test_incremental_mask_update_matches_full_upload():
    """mk_volume_update_mask re-uploads and re-bricks only a box: the brick
    label sets must equal numpy's on the final labels, and every render must
    equal a volume given the final labels in one mk_volume_set_mask."""
    from monkeygl_b200.camera import view_camera
    rng = np.random.default_rng(77)
    X, Y, Z = 100, 90, 70                 # rows not whole bricks: the box kernels see partial bricks
    vox = rng.integers(-1000, 2000, (Z, Y, X), dtype=np.int32).astype(np.int16)
    lab = np.zeros((Z, Y, X), np.uint8)
    lab[10:40, 20:60, 30:80] = 1
    a = capi.Volume(vox)
    a.set_mask(lab)
    lut = np.zeros((256, 4), np.float32)
    lut[:, 0] = np.linspace(0, 1, 256)
    lut[:, 1] = 0.5
    lut[:, 2] = np.linspace(1, 0, 256)
    lut[:, 3] = np.linspace(0, 0.3, 256)
    lp = np.zeros((65, 3), np.float32)
    lp[:, 1] = 1.0
    for l in range(4):
        a.set_transfer_function(l, lut)
        lp[l] = (0.9 if l else 0.5, 1700.0, 650.0)
    a.set_label_params(lp)
    p = capi.vr_params(160, 120, 0, view_camera(25.0), (X, Y, Z), (1, 1, 1))
    a.render_vr(p)                        # maps built for the first mask
    boxes = [(33, 17, 5, 47, 29, 21, 2), (0, 0, 0, 8, 8, 8, 3), (91, 83, 61, 100, 90, 70, 2), (5, 3, 50, 97, 88, 69, 0)]
    for x0, y0, z0, x1, y1, z1, val in boxes:
        lab[z0:z1, y0:y1, x0:x1] = val
        a.update_mask(lab, (x0, y0, z0, x1, y1, z1))
        _, words, present = a.brick_maps()
        want, _ = numpy_label_sets(lab)
        assert np.array_equal(words, want), f"label sets after box {(x0, y0, z0, x1, y1, z1)}"
        assert present[val] and present[0]
        b = capi.Volume(vox)
        b.set_mask(lab)
        for l in range(4):
            b.set_transfer_function(l, lut)
        b.set_label_params(lp)
        for ang in (25.0, 140.0):
            q = capi.vr_params(160, 120, 0, view_camera(ang), (X, Y, Z), (1, 1, 1))
            assert np.array_equal(a.render_vr(q), b.render_vr(q)), f"VR {ang} after box {(x0, y0, z0)}"
            q = capi.vr_params(160, 120, 1, view_camera(ang), (X, Y, Z), (1, 1, 1))
            assert np.array_equal(a.render_vr(q), b.render_vr(q)), f"MIP {ang} after box {(x0, y0, z0)}"
        b.close()
    with pytest.raises(capi.MonkeyGLError):
        a.update_mask(lab, (0, 0, 0, X + 1, 4, 4))
    a.close()
