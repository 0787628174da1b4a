"""Seeded synthetic CT phantoms, transfer functions, planes and CPR paths.

The MonkeyGL datasets (cardiac.raw, body.raw) are not distributed with it, so
every workload runs on synthetic volumes with the same dimensions and spacing:

* air at -1000 HU;
* a centred ellipsoid body (semi-axes 0.45/0.40/0.45 of the extent) at 40 HU
  plus Gaussian noise (sigma 20 HU);
* 6 spheres of radius U[4, 10] voxels at U[300, 1500] HU;
* 3 tubular vessels of radius U[2, 3] voxels at U[250, 400] HU along
  Catmull-Rom curves through random points inside the body;
* values clipped to [-1024, 3071].

Labels (for multi-object rendering) group the primitives into 4 objects:
spheres 1-3, spheres 4-6, vessel 1, vessels 2-3; where primitives overlap
the later one wins, as MonkeyGL's AddNewObjectMask does for later masks
(core/VolumeInfo.cpp:94-116).

Volumes are returned as numpy arrays of shape (dim_z, dim_y, dim_x), i.e. the
x-fastest memory MonkeyGL's SetVolumeData takes.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

__all__ = [
    "Phantom", "make_phantom", "catmull_rom", "make_tf_lut", "make_tf_control_points",
    "CONFIGS", "config_phantom",
]


@dataclass
class Phantom:
    volume: np.ndarray                 # int16 (z, y, x)
    spacing: tuple                     # (sx, sy, sz) mm
    labels: np.ndarray | None = None   # uint8 (z, y, x), 0 = background
    vessels: list = field(default_factory=list)   # control points (N, 3) in voxel units (x, y, z)
    spheres: list = field(default_factory=list)   # (cx, cy, cz, r, hu)

    @property
    def dims(self):
        z, y, x = self.volume.shape
        return (x, y, z)


def catmull_rom(points: np.ndarray, samples_per_segment: int = 16) -> np.ndarray:
    """Centripetal-free (uniform) Catmull-Rom curve through `points` (N, 3)."""
    p = np.asarray(points, dtype=np.float64)
    if len(p) < 2:
        return p.copy()
    ext = np.vstack([2 * p[0] - p[1], p, 2 * p[-1] - p[-2]])
    out = []
    t = np.linspace(0.0, 1.0, samples_per_segment, endpoint=False)[:, None]
    for i in range(1, len(ext) - 2):
        p0, p1, p2, p3 = ext[i - 1], ext[i], ext[i + 1], ext[i + 2]
        a = 2 * p1
        b = p2 - p0
        c = 2 * p0 - 5 * p1 + 4 * p2 - p3
        d = -p0 + 3 * p1 - 3 * p2 + p3
        out.append(0.5 * (a + b * t + c * t * t + d * t * t * t))
    out.append(p[-1][None, :])
    return np.vstack(out)


def _resample_polyline(curve: np.ndarray, n: int) -> np.ndarray:
    seg = np.linalg.norm(np.diff(curve, axis=0), axis=1)
    s = np.concatenate([[0.0], np.cumsum(seg)])
    target = np.linspace(0.0, s[-1], n)
    return np.stack([np.interp(target, s, curve[:, k]) for k in range(3)], axis=1)


def _paint_ball(vol, lab, center, r, value, label, zyx_shape):
    cx, cy, cz = center
    x0, x1 = int(np.floor(cx - r)), int(np.ceil(cx + r)) + 1
    y0, y1 = int(np.floor(cy - r)), int(np.ceil(cy + r)) + 1
    z0, z1 = int(np.floor(cz - r)), int(np.ceil(cz + r)) + 1
    Z, Y, X = zyx_shape
    x0, y0, z0 = max(x0, 0), max(y0, 0), max(z0, 0)
    x1, y1, z1 = min(x1, X), min(y1, Y), min(z1, Z)
    if x0 >= x1 or y0 >= y1 or z0 >= z1:
        return
    zz, yy, xx = np.ogrid[z0:z1, y0:y1, x0:x1]
    m = (xx - cx) ** 2 + (yy - cy) ** 2 + (zz - cz) ** 2 <= r * r
    sub = vol[z0:z1, y0:y1, x0:x1]
    sub[m] = value
    if lab is not None:
        lab[z0:z1, y0:y1, x0:x1][m] = label


def make_phantom(dims, spacing, seed: int, with_labels: bool = False, slab: int = 32) -> Phantom:
    """Build the CT-like phantom for dims = (dim_x, dim_y, dim_z)."""
    X, Y, Z = (int(d) for d in dims)
    rng = np.random.Generator(np.random.PCG64(seed))
    vol = np.full((Z, Y, X), -1000, dtype=np.int16)
    cx, cy, cz = (X - 1) / 2.0, (Y - 1) / 2.0, (Z - 1) / 2.0
    ax, ay, az = 0.45 * X, 0.40 * Y, 0.45 * Z
    xs = ((np.arange(X) - cx) / ax) ** 2
    ys = ((np.arange(Y) - cy) / ay) ** 2
    inside_xy = xs[None, :] + ys[:, None]                   # (Y, X)
    noise_rng = np.random.Generator(np.random.PCG64(seed + 7919))
    for z0 in range(0, Z, slab):
        z1 = min(Z, z0 + slab)
        zs = ((np.arange(z0, z1) - cz) / az) ** 2
        body = inside_xy[None, :, :] + zs[:, None, None] <= 1.0
        n = noise_rng.standard_normal(body.shape, dtype=np.float32)
        val = np.rint(40.0 + 20.0 * n)
        v = vol[z0:z1]
        v[body] = val[body].astype(np.int16)

    lab = np.zeros((Z, Y, X), dtype=np.uint8) if with_labels else None

    def inside_body(p, margin=0.8):
        return ((p[0] - cx) / ax) ** 2 + ((p[1] - cy) / ay) ** 2 + ((p[2] - cz) / az) ** 2 <= margin

    spheres = []
    for i in range(6):
        r = rng.uniform(4.0, 10.0)
        hu = rng.uniform(300.0, 1500.0)
        for _ in range(100):
            c = np.array([rng.uniform(0, X - 1), rng.uniform(0, Y - 1), rng.uniform(0, Z - 1)])
            if inside_body(c, 0.6):
                break
        spheres.append((float(c[0]), float(c[1]), float(c[2]), float(r), float(hu)))
        _paint_ball(vol, lab, c, r, int(round(hu)), 1 if i < 3 else 2, (Z, Y, X))

    vessels = []
    for j in range(3):
        r = rng.uniform(2.0, 3.0)
        hu = int(round(rng.uniform(250.0, 400.0)))
        pts = []
        while len(pts) < 6:
            c = np.array([rng.uniform(0, X - 1), rng.uniform(0, Y - 1), rng.uniform(0, Z - 1)])
            if inside_body(c, 0.7):
                pts.append(c)
        pts = np.array(pts)
        order = np.argsort(pts[:, 2])                        # run head to foot
        pts = pts[order]
        vessels.append(pts)
        curve = catmull_rom(pts, 32)
        length = np.linalg.norm(np.diff(curve, axis=0), axis=1).sum()
        dense = _resample_polyline(curve, max(2, int(length / 0.5)))
        for p in dense:
            _paint_ball(vol, lab, p, r, hu, 3 if j == 0 else 4, (Z, Y, X))

    np.clip(vol, -1024, 3071, out=vol)
    return Phantom(volume=vol, spacing=tuple(float(s) for s in spacing), labels=lab,
                   vessels=vessels, spheres=spheres)


def make_tf_control_points(rng: np.random.Generator):
    """Four control points (t in [0, 1], RGBA) of a CT-style transfer
    function: transparent below a soft-tissue cut, then two opaque ramps."""
    t1 = rng.uniform(0.18, 0.28)
    t2 = rng.uniform(0.40, 0.60)
    pts = [
        (0.0, (rng.uniform(0.6, 0.9), rng.uniform(0.2, 0.4), rng.uniform(0.1, 0.3), 0.0)),
        (t1, (rng.uniform(0.7, 1.0), rng.uniform(0.3, 0.5), rng.uniform(0.2, 0.4), 0.0)),
        (t2, (rng.uniform(0.8, 1.0), rng.uniform(0.6, 0.8), rng.uniform(0.4, 0.6), rng.uniform(0.2, 0.5))),
        (1.0, (rng.uniform(0.9, 1.0), rng.uniform(0.9, 1.0), rng.uniform(0.8, 1.0), rng.uniform(0.7, 0.95))),
    ]
    return pts


def make_tf_lut(points, n: int = 256) -> np.ndarray:
    """Piecewise-linear RGBA LUT (n, 4) float32 through control points given
    as (t, (r, g, b, a)) with t in [0, 1]; entry i sits at t = i / (n - 1)."""
    ts = np.array([p[0] for p in points], dtype=np.float64)
    cs = np.array([p[1] for p in points], dtype=np.float64)
    x = np.arange(n, dtype=np.float64) / (n - 1)
    lut = np.stack([np.interp(x, ts, cs[:, c]) for c in range(4)], axis=1)
    return lut.astype(np.float32)


# BASELINE configurations: name -> (dims, spacing, seed, labels)
CONFIGS = {
    "small": ((128, 128, 96), (0.35, 0.35, 0.3), 1234, False),
    "cardiac": ((512, 512, 361), (0.351, 0.351, 0.3), 1235, False),
    "body": ((512, 512, 1559), (0.7422, 0.7422, 1.0), 1236, True),
    "diff": ((256, 256, 256), (1.0, 1.0, 1.0), 1237, False),
}


def config_phantom(name: str) -> Phantom:
    dims, spacing, seed, labels = CONFIGS[name]
    return make_phantom(dims, spacing, seed, with_labels=labels)
