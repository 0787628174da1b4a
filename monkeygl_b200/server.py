"""Serving: continuous batching of VR / MIP / MPR requests over several
resident volumes (mk_server_* in include/monkeygl_b200.h).

    srv = Server(max_slots=32)
    vid = srv.add_volume(voxels, labels)                 # (z, y, x) int16 / uint8
    t = srv.submit_vr(vid, capi.vr_params(...), luts, label_params)
    image, times = srv.wait(t)                           # (H, W, 3) uint8

Requests are queued on the host and rendered by the library's worker thread;
`wait` blocks in the library with the GIL released.  Output arrays are pinned
host memory (torch) when torch is importable, so finished images are copied
straight into them.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi


def _pinned_empty(shape, dtype):
    try:
        import torch
        if torch.cuda.is_available():
            t = torch.empty(int(np.prod(shape)) * np.dtype(dtype).itemsize, dtype=torch.uint8, pin_memory=True)
            return t.numpy().view(dtype).reshape(shape), t
    except (ImportError, RuntimeError):
        pass
    return np.empty(shape, dtype), None


class Server:
    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0, max_slots: int = 32, max_pending: int = 4096,
                 max_pixels: int = 1024 * 1024, lut_len: int = 256, max_labels: int = 8, max_bricks: int = 0,
                 tiles_per_step: int = 0, evict_idle: bool = False):
        cfg = capi.ServerConfig()
        cfg.device, cfg.hbm_budget_bytes, cfg.max_slots, cfg.max_pending = device, hbm_budget_bytes, max_slots, max_pending
        cfg.max_pixels, cfg.lut_len, cfg.max_labels = max_pixels, lut_len, max_labels
        cfg.max_bricks, cfg.tiles_per_step, cfg.evict_idle = max_bricks, tiles_per_step, int(bool(evict_idle))
        self.config = cfg
        h = C.c_void_p()
        capi._check(capi.lib().mk_server_create(C.byref(cfg), C.byref(h)), "mk_server_create")
        self.handle = h
        self._outs = {}
        self._dims = {}

    def close(self):
        if self.handle:
            capi._check(capi.lib().mk_server_destroy(self.handle), "mk_server_destroy")
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def add_volume(self, voxels: np.ndarray, labels: np.ndarray | None = None) -> int:
        v = np.ascontiguousarray(voxels, dtype=np.int16)
        dz, dy, dx = v.shape
        lab = None
        if labels is not None:
            lab = np.ascontiguousarray(labels, dtype=np.uint8)
            assert lab.shape == v.shape
        vid = C.c_int(0)
        capi._check(capi.lib().mk_server_add_volume(self.handle, v.ctypes.data_as(C.c_void_p), dx, dy, dz,
                                                    lab.ctypes.data_as(C.c_void_p) if lab is not None else None,
                                                    C.byref(vid)), "mk_server_add_volume")
        self._dims[vid.value] = (dx, dy, dz)
        return vid.value

    def remove_volume(self, vid: int):
        capi._check(capi.lib().mk_server_remove_volume(self.handle, vid), "mk_server_remove_volume")
        self._dims.pop(vid, None)

    def _submit(self, req: capi.Request, out, keep, encode=None) -> int:
        """encode: None, or (width, height, channels) of the PNG to also produce."""
        t = C.c_uint64(0)
        req.out = out.ctypes.data
        enc = None
        if encode is not None:
            cap = C.c_size_t(0)
            capi._check(capi.lib().mk_encoded_capacity(*encode, C.byref(cap)), "mk_encoded_capacity")
            enc = np.zeros(cap.value, np.uint8)
            req.encoded = enc.ctypes.data
            req.encoded_capacity = cap.value
        capi._check(capi.lib().mk_server_submit(self.handle, C.byref(req), C.byref(t)), "mk_server_submit")
        self._outs[t.value] = (out, (keep, enc))
        return t.value

    def submit_vr(self, vid: int, params: capi.VRParams, luts, label_params, kind: int = capi.REQUEST_VR,
                  out: np.ndarray | None = None, encode: bool = False) -> int:
        """Ray-cast request.  luts: (n, lut_len, 4) float32 for labels 0..n-1;
        label_params: (n, 3) rows of (alpha, ww, wl).  encode: also return
        the image as a Base64 PNG (times["png_base64"] from wait)."""
        lt = np.ascontiguousarray(luts, dtype=np.float32)
        if lt.ndim == 2:
            lt = lt[None]
        lp = np.ascontiguousarray(label_params, dtype=np.float32).reshape(-1, 3)
        if lp.shape[0] < lt.shape[0]:
            raise ValueError("one (alpha, ww, wl) row per LUT")
        lp = np.ascontiguousarray(lp[:lt.shape[0]])
        req = capi.Request()
        req.volume, req.kind, req.vr = vid, kind, params
        req.luts = lt.ctypes.data
        req.n_luts = lt.shape[0]
        req.label_params = lp.ctypes.data
        ch = 4 if params.pixel_format == capi.PIXEL_RGBA8 else 3
        keep = None
        if out is None:
            out, keep = _pinned_empty((params.height, params.width, ch), np.uint8)
        return self._submit(req, out, keep, (params.width, params.height, ch) if encode else None)

    def submit_plane(self, vid: int, params: capi.PlaneParams, out: np.ndarray | None = None,
                     encode: bool = False) -> int:
        """MPR request; encode: also the plane as MonkeyGL's Base64 PNG (W/2
        RGBA pixels, even widths only)."""
        req = capi.Request()
        req.volume, req.kind, req.plane = vid, capi.REQUEST_MPR, params
        keep = None
        if out is None:
            out, keep = _pinned_empty((params.height, params.width), np.int16)
        return self._submit(req, out, keep, (params.width // 2, params.height, 4) if encode else None)

    def wait(self, ticket: int, timeout_ms: int = -1):
        """(image, times) once the request is done; raises MonkeyGLError with
        MK_ERR_TIMEOUT if it is not done within timeout_ms."""
        tm = capi.RequestTimes()
        rc = capi.lib().mk_server_wait(self.handle, C.c_uint64(ticket), int(timeout_ms), C.byref(tm))
        if rc == capi.MK_ERR_TIMEOUT:
            raise capi.MonkeyGLError(rc, "mk_server_wait")
        out, (_, enc) = self._outs.pop(ticket)
        capi._check(rc, "mk_server_wait")
        times = {"submitted_ms": tm.submitted_ms, "started_ms": tm.started_ms, "completed_ms": tm.completed_ms}
        if enc is not None:
            times["png_base64"] = enc[:tm.encoded_length].tobytes().decode("ascii")
        return out, times

    def stats(self) -> dict:
        st = capi.ServerStats()
        capi._check(capi.lib().mk_server_get_stats(self.handle, C.byref(st)), "mk_server_get_stats")
        return {k: getattr(st, k) for k, _ in capi.ServerStats._fields_}


def submit_request(srv: Server, vid: int, req, out: np.ndarray | None = None, encode: bool = False) -> int:
    """Submit a workloads.ServingRequest for volume id `vid`."""
    if req.kind == capi.REQUEST_MPR:
        return srv.submit_plane(vid, req.plane, out=out, encode=encode)
    return srv.submit_vr(vid, req.vr, req.luts, req.label_params, kind=req.kind, out=out, encode=encode)


def render_plain(vol: capi.Volume, req, out: np.ndarray | None = None) -> np.ndarray:
    """The same request through the one-frame entry points, one launch per
    request: the request's LUTs and label parameters are set on the volume,
    then mk_render_vr / mk_render_plane render it synchronously."""
    if req.kind == capi.REQUEST_MPR:
        return vol.render_plane(req.plane, out=out)
    n = req.luts.shape[0]
    for l in range(n):
        vol.set_transfer_function(l, req.luts[l])
    lp = np.zeros((capi.MAX_LABELS, 3), np.float32)
    lp[:, 1] = 1.0
    lp[:n] = req.label_params
    vol.set_label_params(lp)
    return vol.render_vr(req.vr, out=out)
