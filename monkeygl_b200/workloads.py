"""The benchmark workloads: phantoms with their transfer functions, label
windows, camera views, MPR planes and CPR paths.

* small    128x128x96, spacing 0.35x0.35x0.3, 512^2 VR, views 0/45/90 deg.
* cardiac  512x512x361, spacing 0.351x0.351x0.3, 1024^2 VR and MIP at 36
           views (10 deg steps about z); MPR axial/sagittal/coronal plus 8
           seeded oblique planes at 512^2, window 400/40.
* body     512x512x1559, spacing 0.7422x0.7422x1.0, 4 labelled objects with
           their own 256-entry LUT and opacity cap, background cap 0.4 or
           0.8, 1024^2 VR; stretched and straightened CPR of 512x1024 along a
           Catmull-Rom spline through a vessel centreline.

Transfer functions are 256-entry piecewise-linear LUTs over the window
[-200, 1500] HU (ww 1700, wl 650) through 4 seeded control points.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import camera as cam
from .phantom import Phantom, catmull_rom, config_phantom, make_tf_control_points, make_tf_lut

WW, WL = 1700.0, 650.0


@dataclass
class Workload:
    name: str
    phantom: Phantom
    luts: dict                       # label -> (256, 4) float32
    label_params: np.ndarray         # (65, 3) alpha, ww, wl
    width: int
    height: int
    angles: list = field(default_factory=list)

    @property
    def dims(self):
        return self.phantom.dims

    @property
    def spacing(self):
        return self.phantom.spacing


def _label_params(alphas: dict) -> np.ndarray:
    lp = np.zeros((65, 3), np.float32)
    lp[:, 1] = 1.0
    for l, a in alphas.items():
        lp[l] = (a, WW, WL)
    return lp


def make_workload(name: str, bg_alpha: float = 0.4, phantom: Phantom | None = None) -> Workload:
    p = phantom if phantom is not None else config_phantom(name)
    seed = {"small": 1234, "cardiac": 1235, "body": 1236, "diff": 1237}[name]
    rng = np.random.Generator(np.random.PCG64(seed + 100))
    if name == "body":
        luts = {l: make_tf_lut(make_tf_control_points(rng)) for l in range(5)}
        alphas = {0: bg_alpha}
        for l in range(1, 5):
            alphas[l] = float(np.float32(rng.uniform(0.6, 1.0)))
        lp = _label_params(alphas)
        return Workload(name, p, luts, lp, 1024, 1024, [10.0 * i for i in range(36)])
    luts = {0: make_tf_lut(make_tf_control_points(rng))}
    lp = _label_params({0: 1.0})
    if name == "small":
        return Workload(name, p, luts, lp, 512, 512, [0.0, 45.0, 90.0])
    return Workload(name, p, luts, lp, 1024, 1024, [10.0 * i for i in range(36)])


def view_camera(angle: float) -> cam.Camera:
    return cam.view_camera(angle)


# ----------------------------------------------------------------------
# MPR planes

@dataclass
class Plane:
    name: str
    dir_h: np.ndarray
    dir_v: np.ndarray
    dir_n: np.ndarray
    left_top: np.ndarray
    width: int
    height: int
    pixel_spacing: float


def mpr_planes(p: Phantom, size: int = 512, n_oblique: int = 8, seed: int = 4321) -> list:
    """Axial, sagittal and coronal planes (MonkeyGL's frames,
    core/MPRInfo.cpp:109-135) plus seeded oblique planes (unit normal uniform
    on the sphere, random in-plane rotation, centre within 10% of the volume
    centre), all size x size at the minimum spacing."""
    rng = np.random.Generator(np.random.PCG64(seed))
    ext = np.array(p.dims, np.float64) * np.array(p.spacing, np.float64)
    ps = float(min(p.spacing))
    frames = [("axial", np.array([1.0, 0, 0]), np.array([0, 1.0, 0])),
              ("sagittal", np.array([0, 1.0, 0]), np.array([0, 0, -1.0])),
              ("coronal", np.array([1.0, 0, 0]), np.array([0, 0, -1.0]))]
    for i in range(n_oblique):
        n = rng.standard_normal(3)
        n /= np.linalg.norm(n)
        a = np.cross(n, [1.0, 0, 0] if abs(n[0]) < 0.9 else [0, 1.0, 0])
        a /= np.linalg.norm(a)
        b = np.cross(n, a)
        th = rng.uniform(0, 2 * np.pi)
        h = np.cos(th) * a + np.sin(th) * b
        v = np.cross(n, h)
        frames.append((f"oblique{i}", h, v))
    planes = []
    for k, (name, h, v) in enumerate(frames):
        n = np.cross(h, v)
        c = ext / 2.0
        if k >= 3:
            c = c + rng.uniform(-0.1, 0.1, 3) * ext
        lt = c - h * (0.5 * size * ps) - v * (0.5 * size * ps)
        planes.append(Plane(name, h, v, n, lt, size, size, ps))
    return planes


# ----------------------------------------------------------------------
# CPR paths

def vessel_path(p: Phantom, n_points: int = 200, rows: int = 1024, vessel: int = 0) -> np.ndarray:
    """Centreline of a vessel as a 200-point Catmull-Rom spline (FP64, voxel
    units), resampled by arc length to `rows` points."""
    ctrl = np.asarray(p.vessels[vessel], np.float64)
    dense = catmull_rom(ctrl, 64)
    seg = np.linalg.norm(np.diff(dense, axis=0), axis=1)
    s = np.concatenate([[0.0], np.cumsum(seg)])
    spline = np.stack([np.interp(np.linspace(0, s[-1], n_points), s, dense[:, k]) for k in range(3)], 1)
    seg = np.linalg.norm(np.diff(spline, axis=0), axis=1)
    s = np.concatenate([[0.0], np.cumsum(seg)])
    return np.stack([np.interp(np.linspace(0, s[-1], rows), s, spline[:, k]) for k in range(3)], 1)


def _unit(v):
    return v / np.linalg.norm(v)


def cpr_straightened(path: np.ndarray, width: int) -> tuple:
    """Straightened CPR frames in FP64: rows follow the path; each row's
    direction is carried along the path by the cross-product construction of
    CPRInfo::GetCPRInfoStraightened (core/CPRInfo.cpp:111-160), and the row
    starts width/2 voxels before the centreline."""
    n = len(path)
    d0 = _unit(path[1] - path[0])
    a = np.array([1.0, 0, 0]) if abs(d0[0]) < 0.9 else np.array([0, 1.0, 0])
    first = _unit(np.cross(np.cross(d0, a), d0))
    dirs = np.zeros((n, 3))
    dirs[0] = first
    for i in range(1, n):
        prev = path[i - 1]
        cur = path[i]
        nxt = path[min(i + 1, n - 1)] if i + 1 < n else cur + (cur - prev)
        d1 = dirs[i - 1]
        d2 = _unit(cur - prev)
        d3 = _unit(nxt - cur)
        t = np.cross(d1, d2)
        d = np.cross(d3, t)
        ln = np.linalg.norm(d)
        d = d1 if ln < 0.99 * np.linalg.norm(t) or ln == 0 else d / ln
        if np.dot(d, d1) < 0:
            d = -d
        dirs[i] = d
    half = width / 2.0
    pts = path - dirs * half
    return pts, dirs


def cpr_stretched(path: np.ndarray, width: int) -> tuple:
    """Stretched CPR: one constant in-plane direction perpendicular to the
    chord, as CPRInfo::GetCPRInfoStretched (core/CPRInfo.cpp:81-109)."""
    chord = _unit(path[-1] - path[0])
    a = np.array([1.0, 0, 0]) if abs(chord[0]) < 0.9 else np.array([0, 1.0, 0])
    d = _unit(np.cross(chord, a))
    dirs = np.tile(d, (len(path), 1))
    pts = path - dirs * (width / 2.0)
    return pts, dirs


# ----------------------------------------------------------------------
# Serving trace

# Resident volumes of the serving workload: (dims, spacing, seed, labels).
SERVING_VOLUMES = [
    ((256, 256, 256), (1.0, 1.0, 1.0), 2001, False),
    ((512, 512, 361), (0.351, 0.351, 0.3), 1235, False),
    ((512, 512, 600), (0.7, 0.7, 0.8), 2003, False),
    ((512, 512, 1559), (0.7422, 0.7422, 1.0), 1236, True),
]


@dataclass
class ServingRequest:
    arrival_s: float
    volume: int                      # index into the volume list
    kind: int                        # capi.REQUEST_VR / _MIP / _MPR
    size: int
    vr: object = None                # capi.VRParams
    plane: object = None             # capi.PlaneParams
    luts: np.ndarray | None = None   # (n, 256, 4) float32, labels 0..n-1
    label_params: np.ndarray | None = None   # (n, 3) alpha, ww, wl


def random_plane(dims, spacing, size: int, rng, sampling: int = 0):
    """Oblique plane through the volume centre +-10% of the extent: unit
    normal uniform on the sphere, random in-plane rotation, size x size at
    the minimum spacing, slab of one sample."""
    from . import capi
    ext = np.array(dims, np.float64) * np.array(spacing, np.float64)
    ps = float(min(spacing))
    n = rng.standard_normal(3)
    n /= np.linalg.norm(n)
    a = np.cross(n, [1.0, 0, 0] if abs(n[0]) < 0.9 else [0, 1.0, 0])
    a /= np.linalg.norm(a)
    b = np.cross(n, a)
    th = rng.uniform(0, 2 * np.pi)
    h = np.cos(th) * a + np.sin(th) * b
    v = np.cross(n, h)
    c = ext / 2.0 + rng.uniform(-0.1, 0.1, 3) * ext
    lt = c - h * (0.5 * size * ps) - v * (0.5 * size * ps)
    return capi.plane_params(size, size, capi.MPR_AVERAGE, sampling, spacing, h, v, np.cross(h, v), lt, ps, False, 0.0)


def serving_trace(volumes, n: int, rate: float, seed: int = 77, sizes=(256, 512, 768, 1024),
                  mix=(0.6, 0.2, 0.2)) -> list:
    """n requests with Poisson arrivals at `rate` per second over `volumes`
    (list of (dims, spacing, has_labels)): VR / MIP / MPR in proportions
    `mix`, square images of a size drawn from `sizes`, random cameras
    (rotation about z and x, zoom 0.8-1.5) and random transfer functions
    (one 4-point piecewise-linear LUT per label, opacity caps U(0.6, 1) on
    labelled objects and U(0.3, 1) on the background), random oblique planes
    with trilinear or nearest sampling."""
    from . import capi
    rng = np.random.Generator(np.random.PCG64(seed))
    out, t = [], 0.0
    for _ in range(n):
        t += rng.exponential(1.0 / rate)
        vi = int(rng.integers(len(volumes)))
        dims, spacing, labelled = volumes[vi]
        u = rng.random()
        kind = capi.REQUEST_VR if u < mix[0] else capi.REQUEST_MIP if u < mix[0] + mix[1] else capi.REQUEST_MPR
        size = int(sizes[int(rng.integers(len(sizes)))])
        if kind == capi.REQUEST_MPR:
            plane = random_plane(dims, spacing, size, rng, sampling=int(rng.integers(2)))
            out.append(ServingRequest(t, vi, kind, size, plane=plane))
            continue
        c = cam.Camera()
        c.anterior()
        c.rotate(float(rng.uniform(0.0, 360.0)), float(rng.uniform(-40.0, 40.0)))
        c.zoom(float(rng.uniform(0.8, 1.5)))
        vr = capi.vr_params(size, size, kind, c, dims, spacing)
        nl = 5 if labelled else 1
        luts = np.stack([make_tf_lut(make_tf_control_points(rng)) for _ in range(nl)])
        lp = np.zeros((nl, 3), np.float32)
        lp[:, 1] = WW
        lp[:, 2] = WL
        lp[0, 0] = rng.uniform(0.3, 1.0) if labelled else 1.0
        lp[1:, 0] = rng.uniform(0.6, 1.0, nl - 1)
        out.append(ServingRequest(t, vi, kind, size, vr=vr, luts=luts, label_params=lp))
    return out
