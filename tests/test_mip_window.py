"""The MIP loop without label fetches (monkeygl_b200/csrc/mk_raycast_impl.cuh)
applies MonkeyGL's window w(t) = (32768 t - wl) / ww + 0.5 (core/kernel.cu:
337-345) only to a new raw maximum: it relies on w being non-decreasing in t
for ww > 0 when every operation is rounded to float32, so that the maximum of
w over a ray's samples is w of the largest sample.  Checked here in float32
(numpy rounds each operation as the kernel does) on every normalized int16
read value and on random rays.  CPU only."""
import numpy as np


def window(t, wl, ww):
    t = np.asarray(t, np.float32)
    return ((np.float32(32768) * t - np.float32(wl)) / np.float32(ww) + np.float32(0.5)).astype(np.float32)


def test_window_is_monotonic_on_every_int16_read():
    # normalized-float texture reads of int16 are v / 32767 (plus trilinear
    # blends of them); all exact reads, and midpoints between neighbours
    v = np.arange(-32768, 32768, dtype=np.float64)
    t = np.sort(np.concatenate([v / 32767.0, (v[:-1] + 0.5) / 32767.0]).astype(np.float32))
    rng = np.random.default_rng(3)
    for wl, ww in [(650.0, 1700.0), (40.0, 400.0), (-1000.0, 1.0), (300.0, 0.75), (3000.0, 4000.0)] + \
            [(float(rng.uniform(-2000, 3000)), float(rng.uniform(0.5, 5000))) for _ in range(20)]:
        w = window(t, wl, ww)
        assert (np.diff(w) >= 0).all(), (wl, ww)


def test_max_of_window_is_window_of_max():
    rng = np.random.default_rng(11)
    for _ in range(2000):
        n = int(rng.integers(1, 400))
        t = rng.uniform(-1, 1, n).astype(np.float32)
        wl, ww = float(rng.uniform(-2000, 3000)), float(rng.uniform(0.5, 5000))
        assert window(t, wl, ww).max() == window(t.max(), wl, ww)
