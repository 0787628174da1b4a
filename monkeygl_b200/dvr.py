"""Differentiable volume rendering on the sm_100a kernels (mk_dvr_* in
include/monkeygl_b200.h), exposed as a torch.autograd.Function.

    views = [dvr_params(256, 256, view_camera(a), dims, spacing) for a in angles]
    images = render(volume, lut, views)          # (V, H, W, 3), differentiable
    loss = ((images - target) ** 2).mean()
    loss.backward()                              # volume.grad, lut.grad

`volume` is a float32 CUDA tensor (dim_z, dim_y, dim_x) with values in [0, 1]
and `lut` a float32 CUDA tensor (n, 4) of RGBA entries.  Torch provides the
device memory and the stream; forward and backward are the library's kernels.
The method (fixed step, exact trilinear, value as LUT coordinate,
front-to-back compositing with termination at t_min) is described in
monkeygl_b200/csrc/mk_dvr.cu.
"""
from __future__ import annotations

import ctypes as C

from . import capi
from .capi import DVRParams
from .camera import volume_factors


def _lib():
    return capi.lib()


def dvr_params(width, height, camera, dims, spacing, step_voxels=0.5, t_min=1e-4, lut_len=256) -> DVRParams:
    """Parameters of one view.  The step is in voxels of the longest axis:
    MonkeyGL's ray parameter advances by 1/dim_z per voxel (core/kernel.cu:169)."""
    mls, _ = volume_factors(dims, spacing)
    p = DVRParams()
    p.width, p.height = int(width), int(height)
    for k in range(3):
        p.dims[k] = int(dims[k])
        p.max_len_spacing[k] = mls[k]
    for i, m in enumerate(camera.flat()):
        p.transform[i] = m
    p.scale = float(camera.scale)
    p.x_translate = float(camera.x_translate)
    p.y_translate = float(camera.y_translate)
    p.step = float(step_voxels) / float(dims[2])
    p.t_min = float(t_min)
    p.lut_len = int(lut_len)
    return p


def params_flat(p: DVRParams):
    """The parameter block of oracle.mko_dvr_forward_d (FP64 restatement)."""
    import numpy as np
    return np.array([p.width, p.height, *p.dims, *p.max_len_spacing, *p.transform, p.scale, p.x_translate,
                     p.y_translate, p.step, p.t_min, p.lut_len], np.float64)


def _check(rc, where):
    if rc != 0:
        raise capi.MonkeyGLError(rc, where, capi.lib().mk_last_error().decode(errors="replace"))


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def view_array(views):
    """The views as a C array of DVRParams (ctypes)."""
    views = list(views)
    return (DVRParams * len(views))(*views), len(views)


def workspace_floats(views) -> int:
    arr, n = view_array(views)
    out = C.c_size_t(0)
    _check(_lib().mk_dvr_workspace_floats(arr, n, C.byref(out)), "mk_dvr_workspace_floats")
    return out.value


def _torch_function():
    import torch

    class VolumeRender(torch.autograd.Function):
        @staticmethod
        def forward(ctx, volume, lut, views):
            if not (volume.is_cuda and lut.is_cuda):
                raise ValueError("volume and lut must be CUDA tensors")
            volume = volume.detach().contiguous().float()
            lut = lut.detach().contiguous().float()
            L = _lib()
            arr, nv = view_array(views)
            p0 = arr[0]
            for p in arr:
                if p.lut_len != lut.shape[0] or tuple(p.dims) != tuple(volume.shape[::-1]):
                    raise ValueError("view parameters do not match the volume or LUT")
                if (p.width, p.height) != (p0.width, p0.height):
                    raise ValueError("the views of one render must share width and height")
            stream = C.c_void_p(torch.cuda.current_stream(volume.device).cuda_stream)
            images = torch.empty((nv, p0.height, p0.width, 3), dtype=torch.float32, device=volume.device)
            trans = torch.empty((nv, p0.height, p0.width), dtype=torch.float32, device=volume.device)
            work = None
            if ctx.needs_input_grad[0] or ctx.needs_input_grad[1]:
                work = torch.empty(workspace_floats(arr), dtype=torch.float32, device=volume.device)
            _check(L.mk_dvr_forward(arr, nv, _ptr(volume), _ptr(lut), _ptr(images), _ptr(trans), _ptr(work),
                                    stream), "mk_dvr_forward")
            ctx.views = arr
            ctx.work = work
            ctx.save_for_backward(volume, lut)
            return images

        @staticmethod
        def backward(ctx, grad_images):
            volume, lut = ctx.saved_tensors
            L = _lib()
            stream = C.c_void_p(torch.cuda.current_stream(volume.device).cuda_stream)
            grad_lut = torch.zeros_like(lut)
            grad_vol = torch.zeros_like(volume) if ctx.needs_input_grad[0] else None
            g = grad_images.contiguous().float()
            _check(L.mk_dvr_backward(ctx.views, len(ctx.views), _ptr(volume), _ptr(lut), _ptr(ctx.work), _ptr(g),
                                     _ptr(grad_lut), _ptr(grad_vol), stream), "mk_dvr_backward")
            return grad_vol, (grad_lut if ctx.needs_input_grad[1] else None), None

    return VolumeRender


_VR = None


def render(volume, lut, views):
    """Differentiable render of `views` (list of DVRParams): (V, H, W, 3)."""
    global _VR
    if _VR is None:
        _VR = _torch_function()
    return _VR.apply(volume, lut, list(views))
