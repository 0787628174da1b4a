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
