"""Camera and volume-geometry setup for ray casting, in MonkeyGL's FP32
arithmetic.

MonkeyGL keeps the VR camera as a 3x3 float matrix accumulated by
Methods::ComputeTransformMatrix (core/Methods.cpp:52-132): every rotate or
zoom multiplies the current matrix on the right by S(1/scale), Rz(z) and
Rx(x), in float, with each product accumulated left to right.  The
orientation presets (core/RenderInfo.cpp:100-134) reset the matrix, pan and
zoom and then apply one rotation.  Rotate(fx, fy) passes (fy, fx) as
(x-angle, z-angle) (core/RenderInfo.cpp:77-80), so Rotate(a, 0) turns the
view by a degrees about z.  Volume factors follow DataManager::InitCommon
(core/DataManager.h:201-216) and the z inversion test
VolumeInfo::Need2InvertZ (core/VolumeInfo.cpp:142-148).

This module mirrors that arithmetic with numpy float32 scalars so that a
matrix built here is bit-identical to MonkeyGL's; the C++ host library
(HelloMonkey) carries its own implementation of the same steps.
"""
from __future__ import annotations

import math

import numpy as np

F = np.float32
PI = 3.141592654   # MonkeyGL's PI macro (core/Defines.h:33), a double


def _ang(deg) -> float:
    # (fAngle)/180.0f*PI: float division, then a double product
    return float(F(deg) / F(180.0)) * PI


def _matmul(a, b):
    """3x3 float product, each entry accumulated left to right in float
    (core/Methods.cpp:134-153)."""
    out = [[F(0)] * 3 for _ in range(3)]
    for i in range(3):
        for j in range(3):
            t = F(a[i][0] * b[0][j])
            for k in range(1, 3):
                t = F(t + F(a[i][k] * b[k][j]))
            out[i][j] = t
    return out


def _identity():
    return [[F(1) if i == j else F(0) for j in range(3)] for i in range(3)]


class Camera:
    """The VR camera state of MonkeyGL's RenderInfo (transform, zoom, pan)."""

    def __init__(self):
        self.init()

    def init(self):
        self.x_translate = F(0)
        self.y_translate = F(0)
        self.scale = F(1)
        self.matrix = _identity()

    def _compute(self, fx, fz, fscale):
        s = F(F(1.0) / F(fscale))
        S = [[s, F(0), F(0)], [F(0), s, F(0)], [F(0), F(0), s]]
        ax, az = _ang(fx), _ang(fz)
        Rx = _identity()
        Rx[1][1] = F(math.cos(ax))
        Rx[1][2] = F(-math.sin(ax))
        Rx[2][1] = F(math.sin(ax))
        Rx[2][2] = F(math.cos(ax))
        Rz = _identity()
        Rz[0][0] = F(math.cos(az))
        Rz[0][1] = F(math.sin(az))
        Rz[1][0] = F(-math.sin(az))
        Rz[1][1] = F(math.cos(az))
        m = _matmul(self.matrix, S)
        m = _matmul(m, Rz)
        self.matrix = _matmul(m, Rx)

    # RenderInfo::Rotate: (fxRotate, fyRotate) -> Compute(fyRotate, fxRotate, 1)
    def rotate(self, fx, fy):
        self._compute(fy, fx, 1.0)

    def zoom(self, ratio):
        self.scale = F(self.scale * F(ratio))
        self._compute(0.0, 0.0, ratio)
        return self.scale

    def pan(self, dx, dy):
        self.x_translate = F(self.x_translate + F(dx))
        self.y_translate = F(self.y_translate + F(dy))

    def _preset(self, fx, fz):
        self.init()
        self._compute(fx, fz, self.scale)

    def anterior(self):
        self._preset(0.0, 0.0)

    def posterior(self):
        self._preset(0.0, 180.0)

    def left(self):
        self._preset(0.0, -90.0)

    def right(self):
        self._preset(0.0, 90.0)

    def head(self):
        self._preset(90.0, 180.0)

    def foot(self):
        self._preset(-90.0, 0.0)

    def flat(self):
        return [float(self.matrix[i][j]) for i in range(3) for j in range(3)]


def volume_factors(dims, spacing):
    """(maxLenSpacing, spacingVoxel) of DataManager::InitCommon in float."""
    sx, sy, sz = (F(s) for s in spacing)   # InitCommon takes floats
    w, h, d = (F(x) for x in dims)
    ext = [F(w * sx), F(h * sy), F(d * sz)]
    max_len = max(ext[0], max(ext[1], ext[2]))
    mls = [float(F(F(F(1.0) * max_len) / e)) for e in ext]
    sv = [float(F(F(1.0) / x)) for x in (w, h, d)]
    return mls, sv


def need_invert_z(dir_x, dir_y, dir_z) -> bool:
    """VolumeInfo::Need2InvertZ: (dirX x dirY) . dirZ > 0 on normalised directions."""
    def unit(v):
        v = np.asarray(v, dtype=np.float64)
        return v / np.sqrt((v * v).sum())
    a, b, c = unit(dir_x), unit(dir_y), unit(dir_z)
    n = np.cross(a, b)
    n = n / np.sqrt((n * n).sum())
    return float(np.dot(n, c)) > 0


def view_camera(angle_deg: float) -> Camera:
    """Anterior view turned by angle_deg about z (Anterior(); Rotate(a, 0))."""
    cam = Camera()
    cam.anterior()
    if angle_deg:
        cam.rotate(angle_deg, 0.0)
    return cam
