"""mk_render_cpr_noalloc: curved reformation without any device allocation.

Callers such as a viewer running under a fixed, pre-planned device-memory
budget, a framework whose caching allocator already owns the GPU memory, or
a render loop that cannot afford the synchronisation cudaMalloc/cudaFree
may imply, cannot let the library allocate.  This entry point keeps its
per-row table in a fixed device array and writes into the caller's buffer.
Its images must equal those of mk_render_cpr (the CPR tests compare
exactly), on consecutive calls that reuse the shared table with different
path lengths.  The file is named to run last, so a failure here comes after
every other test has run; it also passes on its own in a fresh process."""
import ctypes as C

import numpy as np
import pytest

from monkeygl_b200 import capi
from monkeygl_b200 import workloads as wl

pytestmark = pytest.mark.gpu

MAX_ROWS = 4096


def _noalloc(vol, width, pts, dirs, invert_z, out_dev, stream):
    pts = np.ascontiguousarray(pts, np.float64)
    dirs = np.ascontiguousarray(dirs, np.float64)
    return capi.lib().mk_render_cpr_noalloc(vol.handle, width, pts.shape[0], C.c_void_p(pts.ctypes.data),
                                            C.c_void_p(dirs.ctypes.data), int(invert_z),
                                            C.c_void_p(out_dev.data_ptr()), C.c_void_p(stream.cuda_stream))


def test_noalloc_cpr_matches_allocating_entry_point():
    import torch

    w = wl.make_workload("small")
    vol = capi.Volume(w.phantom.volume)
    path = wl.vessel_path(w.phantom, rows=300)
    straight = wl.cpr_straightened(path, 128)
    stretched = wl.cpr_stretched(path[:200], 96)
    stream = torch.cuda.Stream()
    calls = [(128, straight, False), (96, stretched, True), (128, straight, True)]
    for width, (pts, dirs), inv in calls:
        want = vol.render_cpr(width, pts, dirs, inv)
        out = torch.full((pts.shape[0], width), 12345, dtype=torch.int16, device="cuda")
        # the fill is queued on torch's stream: the call's stream waits for it
        stream.wait_stream(torch.cuda.current_stream())
        rc = _noalloc(vol, width, pts, dirs, inv, out, stream)
        assert rc == capi.MK_OK, capi.lib().mk_last_error()
        stream.synchronize()
        got = out.cpu().numpy()
        assert np.array_equal(got, want), f"{np.count_nonzero(got != want)} pixels differ"
    vol.close()


def test_noalloc_cpr_rejects_paths_beyond_its_table():
    import torch

    w = wl.make_workload("small")
    vol = capi.Volume(w.phantom.volume)
    n = MAX_ROWS + 1
    pts = np.zeros((n, 3))
    dirs = np.tile([1.0, 0.0, 0.0], (n, 1))
    out = torch.empty((n, 8), dtype=torch.int16, device="cuda")
    rc = _noalloc(vol, 8, pts, dirs, False, out, torch.cuda.Stream())
    assert rc == capi.MK_ERR_INVALID_ARGUMENT
    assert b"4096" in capi.lib().mk_last_error()
    vol.close()


def test_noalloc_cpr_leaves_device_memory_unchanged():
    """After a first call on a new volume (which looks up the table's device
    address), further calls of several path lengths must not change the
    device's free memory: the entry point allocates nothing."""
    import torch

    w = wl.make_workload("small")
    vol = capi.Volume(w.phantom.volume)
    path = wl.vessel_path(w.phantom, rows=1000)
    paths = [wl.cpr_straightened(path, 160), wl.cpr_stretched(path[:700], 200),
             wl.cpr_straightened(path[:40], 64)]
    stream = torch.cuda.Stream()
    outs = [torch.zeros((p[0].shape[0], wd), dtype=torch.int16, device="cuda")
            for p, wd in zip(paths, (160, 200, 64))]
    stream.wait_stream(torch.cuda.current_stream())
    assert _noalloc(vol, 160, *paths[0], False, outs[0], stream) == capi.MK_OK
    stream.synchronize()
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for rep in range(3):
        for (pts, dirs), out in zip(paths, outs):
            rc = _noalloc(vol, out.shape[1], pts, dirs, rep == 1, out, stream)
            assert rc == capi.MK_OK, capi.lib().mk_last_error()
    stream.synchronize()
    free_after = torch.cuda.mem_get_info()[0]
    assert free_after >= free_before, f"device free memory fell by {free_before - free_after} bytes"
    vol.close()
