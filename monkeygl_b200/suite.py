"""Per-mode benchmark table of the ray-casting library (``bench.py --suite``).

Rows (synthetic seeded phantoms of monkeygl_b200.phantom):
  * VR and MIP of the cardiac phantom (int16 512x512x361) at 1024^2, 36 views;
  * MIP of the body phantom at 1024^2;
  * VR of the body phantom (int16 512x512x1559, 4 labels) at 1024^2 with
    background opacity caps 0.4 and 0.8;
  * MPR of the cardiac phantom: axial, sagittal, coronal and 8 seeded oblique
    planes of 512^2, trilinear and nearest, slab of 1 sample;
  * CPR of a body vessel (200-point Catmull-Rom centreline), 1024 rows x 512
    columns, stretched and straightened;
  * VR of the body phantom with a dense transfer function (soft tissue
    visible), where empty-space skipping cannot help inside the body;
  * differentiable VR: float32 256^3 volume, 256-entry LUT, 8 views of 256^2,
    step 0.5 voxel -- forward, backward and their ratio;
  * GetVRData through the HelloMonkey API (render, orientation box, copy
    back), 512x512, 36 views, beside MonkeyGL's complete HelloMonkey path;
  * upload of the body volume and its labels (brick maps included).

Device times are CUDA events on the launching stream around each call, L2
flushed (256 MiB write) between calls outside the events, median over the
calls.  "e2e" times are wall clock around the C ABI call with host output.
Where the caller supplies MonkeyGL's own CUDA path, its times for the same
calls are listed beside ours: kernel time for VR/MIP (CUDA events around its
d_render launch), whole-call wall time for MPR and CPR (its launchers
allocate, copy and free device memory on every call).
"""
from __future__ import annotations

import ctypes as C
import json
import statistics
import time

import numpy as np


def _median_ms(fn, reps, stream, flush):
    import torch
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
    with torch.cuda.stream(stream):
        for i in range(reps):
            flush.zero_()
            ev[i][0].record(stream)
            fn(i)
            ev[i][1].record(stream)
    torch.cuda.synchronize()
    return statistics.median(a.elapsed_time(b) for a, b in ev)


def _wall_ms(fn, reps):
    ts = []
    for i in range(reps):
        t0 = time.perf_counter()
        fn(i)
        ts.append((time.perf_counter() - t0) * 1e3)
    return statistics.median(ts)


def _load_ref(ref, w):
    ref.set_volume(w.phantom.volume)
    ref.set_mask(w.phantom.labels)
    ref.clear_tfs()
    for l, lut in w.luts.items():
        ref.set_lut(l, lut)


def _workload(ctx, name, bg=0.4):
    """Workload with the phantom generated once per suite run."""
    from monkeygl_b200.phantom import config_phantom
    from monkeygl_b200.workloads import make_workload
    ph = ctx.setdefault("phantoms", {})
    if name not in ph:
        ph[name] = config_phantom(name)
    return make_workload(name, bg_alpha=bg, phantom=ph[name])


def dense_luts(w):
    """A transfer function with soft tissue visible: alpha rises from 0 at
    -200 HU to 0.03 at about 0 HU (the body's 40 +- 20 HU), 0.12 at 300 HU
    and 0.9 at 1500 HU, so rays composite (and refine their step) all
    through the body and empty-space skipping cannot help inside it.  Same
    colours for every label."""
    from monkeygl_b200.phantom import make_tf_lut
    pts = [(0.0, (0.8, 0.5, 0.4, 0.0)), (0.12, (0.85, 0.55, 0.45, 0.03)), (0.3, (0.9, 0.7, 0.6, 0.12)),
           (1.0, (1.0, 0.95, 0.9, 0.9))]
    lut = make_tf_lut(pts)
    return {l: lut for l in w.luts}


def vr_rows(name, bg, rtypes, ctx, dense=False):
    import torch
    from monkeygl_b200 import capi
    from monkeygl_b200.workloads import view_camera
    w = _workload(ctx, name, bg)
    if dense:
        w.luts = dense_luts(w)
    vol = capi.Volume(w.phantom.volume)
    if w.phantom.labels is not None:
        vol.set_mask(w.phantom.labels)
    for l, lut in w.luts.items():
        vol.set_transfer_function(l, lut)
    vol.set_label_params(w.label_params)
    size = 1024
    out = torch.empty(size * size * 3, dtype=torch.uint8, device="cuda")
    host = np.empty((size, size, 3), np.uint8)
    ref = ctx["ref"]
    if ref is not None:
        _load_ref(ref, w)
    rows = []
    for rt in rtypes:
        params = [capi.vr_params(size, size, rt, view_camera(a), w.dims, w.spacing) for a in w.angles]
        n = len(params)
        stream = ctx["stream"]
        for i in range(3):
            vol.render_vr_device(params[i], out.data_ptr(), stream.cuda_stream)
        ms = _median_ms(lambda i: vol.render_vr_device(params[i % n], out.data_ptr(), stream.cuda_stream),
                        n, stream, ctx["flush"])
        e2e = _wall_ms(lambda i: vol.render_vr(params[i % n], out=host), n)
        row = {"row": f"{'VR' if rt == 0 else 'MIP'} {name}" + (f" bg {bg}" if name == "body" else "") +
                      (" dense TF (soft tissue visible)" if dense else ""),
               "image": f"{size}x{size}", "views": n, "ms": round(ms, 4), "fps": round(1e3 / ms, 1),
               "e2e_ms": round(e2e, 4)}
        if ref is not None:
            flats = [np.ascontiguousarray(capi.vr_params_flat(p, w.label_params)) for p in params]
            pick = sorted({(k * n) // 6 for k in range(6)})
            rms = statistics.median(ref.kernel_ms(size, size, rt, flats[i], 3) for i in pick)
            row["ref_kernel_ms"] = round(rms, 4)
            row["speedup_kernel"] = round(rms / ms, 2)
        rows.append(row)
    vol.close()
    return rows


def mpr_rows(ctx):
    import torch
    from monkeygl_b200 import capi
    from monkeygl_b200.workloads import mpr_planes
    w = _workload(ctx, "cardiac")
    vol = capi.Volume(w.phantom.volume)
    planes = mpr_planes(w.phantom, size=512, n_oblique=8)
    out = torch.empty(512 * 512, dtype=torch.int16, device="cuda")
    ref = ctx["ref"]
    if ref is not None:
        _load_ref(ref, w)
    rows = []
    for sampling, sname in ((0, "trilinear"), (1, "nearest")):
        pp = [capi.plane_params(pl.width, pl.height, 0, sampling, w.spacing, pl.dir_h, pl.dir_v, pl.dir_n,
                                pl.left_top, pl.pixel_spacing, False, 0.0) for pl in planes]
        n = len(pp)
        stream = ctx["stream"]
        for i in range(3):
            vol.render_plane_device(pp[i], out.data_ptr(), stream.cuda_stream)
        ms = _median_ms(lambda i: vol.render_plane_device(pp[i % n], out.data_ptr(), stream.cuda_stream),
                        4 * n, stream, ctx["flush"])
        e2e = _wall_ms(lambda i: vol.render_plane(pp[i % n]), 4 * n)
        row = {"row": f"MPR cardiac {sname}", "image": "512x512", "planes": n, "ms": round(ms, 4),
               "planes_per_s": round(1e3 / ms, 1), "e2e_ms": round(e2e, 4)}
        if ref is not None:
            flats = [capi.plane_params_flat(p) for p in pp]
            rms = _wall_ms(lambda i: ref.plane(512, 512, flats[i % n], 0, sampling), 2 * n)
            row["ref_call_ms"] = round(rms, 4)
            row["speedup_e2e"] = round(rms / e2e, 2)
        rows.append(row)
    vol.close()
    return rows


def cpr_rows(ctx):
    import torch
    from monkeygl_b200 import capi
    from monkeygl_b200.workloads import cpr_straightened, cpr_stretched, vessel_path
    w = _workload(ctx, "body")
    vol = capi.Volume(w.phantom.volume)
    path = vessel_path(w.phantom, n_points=200, rows=1024)
    width = 512
    out = torch.empty(1024 * width, dtype=torch.int16, device="cuda")
    ref = ctx["ref"]
    if ref is not None:
        _load_ref(ref, w)
    L = capi.lib()
    rows = []
    for builder in (cpr_stretched, cpr_straightened):
        pts, dirs = builder(path, width)
        pts = np.ascontiguousarray(pts, np.float64)
        dirs = np.ascontiguousarray(dirs, np.float64)
        h = pts.shape[0]
        stream = ctx["stream"]

        def dev(i):
            capi._check(L.mk_render_cpr(vol.handle, width, h, pts.ctypes.data_as(C.c_void_p),
                                        dirs.ctypes.data_as(C.c_void_p), 0, C.c_void_p(out.data_ptr()), 1,
                                        C.c_void_p(stream.cuda_stream)), "mk_render_cpr")

        for i in range(3):
            dev(i)
        ms = _median_ms(dev, 20, stream, ctx["flush"])
        e2e = _wall_ms(lambda i: vol.render_cpr(width, pts, dirs, False), 20)
        row = {"row": f"CPR body {builder.__name__.split('_')[1]}", "image": f"{width}x{h}", "ms": round(ms, 4),
               "e2e_ms": round(e2e, 4)}
        if ref is not None:
            rms = _wall_ms(lambda i: ref.cpr(width, pts, dirs, False), 10)
            row["ref_call_ms"] = round(rms, 4)
            row["speedup_e2e"] = round(rms / e2e, 2)
        rows.append(row)
    vol.close()
    return rows


def dvr_rows(ctx):
    import torch
    from monkeygl_b200 import dvr
    from monkeygl_b200.camera import view_camera
    from monkeygl_b200.phantom import config_phantom, make_tf_control_points, make_tf_lut
    ph = config_phantom("diff")
    vol = np.clip((ph.volume.astype(np.float32) + 1024.0) / 4095.0, 0.0, 1.0).astype(np.float32)
    rng = np.random.Generator(np.random.PCG64(1337))
    lut = make_tf_lut(make_tf_control_points(rng))
    target_lut = make_tf_lut(make_tf_control_points(rng))
    views = [dvr.dvr_params(256, 256, view_camera(a), (256, 256, 256), (1, 1, 1), 0.5, 1e-4, 256)
             for a in np.arange(8) * 45.0]
    v = torch.tensor(vol, device="cuda", requires_grad=True)
    l = torch.tensor(lut, device="cuda", requires_grad=True)
    stream = ctx["stream"]
    with torch.cuda.stream(stream):
        with torch.no_grad():
            target = dvr.render(v, torch.tensor(target_lut, device="cuda"), views)
        fw, bw = [], []
        for it in range(13):
            v.grad = None
            l.grad = None
            ctx["flush"].zero_()
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record(stream)
            img = dvr.render(v, l, views)
            e1.record(stream)
            loss = ((img - target) ** 2).mean()
            loss.backward()
            e2.record(stream)
            torch.cuda.synchronize()
            if it >= 3:
                fw.append(e0.elapsed_time(e1))
                bw.append(e1.elapsed_time(e2))
    # samples per pass from the forward's sample counts
    work = torch.empty(dvr.workspace_floats(views), dtype=torch.float32, device="cuda")
    imgs = torch.empty((8, 256, 256, 3), device="cuda")
    tr = torch.empty((8, 256, 256), device="cuda")
    arr, nv = dvr.view_array(views)
    L = dvr._lib()
    capi_check = dvr._check
    capi_check(L.mk_dvr_forward(arr, nv, C.c_void_p(v.data_ptr()), C.c_void_p(l.data_ptr()),
                                C.c_void_p(imgs.data_ptr()), C.c_void_p(tr.data_ptr()), C.c_void_p(work.data_ptr()),
                                None), "mk_dvr_forward")
    torch.cuda.synchronize()
    # per view: checkpoint planes, then a plane of sample counts, then one of final transmittances
    per, npix = work.numel() // 8, 256 * 256
    samples = sum(int(work[i * per + per - 2 * npix:i * per + per - npix].view(torch.int32).sum().item())
                  for i in range(8))
    f, b = statistics.median(fw), statistics.median(bw)
    return [{"row": "DVR 256^3, 8 views 256^2 (forward)", "ms": round(f, 4), "samples": samples,
             "gsamples_per_s": round(samples / f / 1e6, 2)},
            {"row": "DVR 256^3, 8 views 256^2 (backward, LUT + volume)", "ms": round(b, 4),
             "bwd_over_fwd": round(b / f, 3), "gsamples_per_s": round(samples / b / 1e6, 2)}]


def api_rows(ctx):
    """GetVRData through the drop-in API (render, orientation box, copy back)
    against MonkeyGL's complete HelloMonkey path on the same calls: the
    cardiac phantom, a 100-entry TF from 4 control points, window 1700/650,
    512x512 VR (MonkeyGL's default size), 36 views 10 degrees apart.  Both
    objects are made in the directory holding resources/human.stl, so both
    draw the orientation box.  Wall time per call, median."""
    import os
    import sys
    from pathlib import Path
    lib = Path(__file__).resolve().parent / "lib"
    if str(lib) not in sys.path:
        sys.path.insert(0, str(lib))
    import pyMonkeyGL as pm
    ref = ctx.get("ref_api")
    w = _workload(ctx, "cardiac")
    vol = w.phantom.volume
    tf = {0: (0.9, 0.3, 0.2, 0.0), 22: (0.95, 0.4, 0.3, 0.0), 55: (0.9, 0.7, 0.5, 0.35), 99: (1.0, 0.95, 0.9, 0.85)}
    cwd = os.getcwd()
    res_dir = ctx.get("resources_dir")
    if res_dir:
        os.chdir(res_dir)
    try:
        mine = pm.HelloMonkey()
    finally:
        os.chdir(cwd)
    mine.SetVolumeArray(vol.swapaxes(2, 0))
    mine.SetDirection(pm.Direction3d(1, 0, 0), pm.Direction3d(0, 1, 0), pm.Direction3d(0, 0, -1))
    mine.SetSpacing(*w.spacing)
    mine.SetTransferFunc({k: pm.RGBA(*v) for k, v in tf.items()})
    mine.SetVRWWWL(1700.0, 650.0)
    mine.SetVRSize(512, 512)
    mine.Anterior()
    times, same = [], True
    if ref is not None:
        ref.set_volume(vol, w.spacing)
        ref.set_transfer_function(tf)
        ref.set_wwwl(1700.0, 650.0)
        ref.set_vr_size(512, 512)
        ref.orientation(0)
    for i in range(3):
        mine.GetVRImage()
        if ref is not None:
            ref.vr_image()
    rtimes = []
    for i in range(36):
        mine.Rotate(10.0, 0.0)
        t0 = time.perf_counter()
        img = mine.GetVRImage()
        times.append((time.perf_counter() - t0) * 1e3)
        if ref is not None:
            ref.rotate(10.0, 0.0)
            t0 = time.perf_counter()
            rimg = ref.vr_image()
            rtimes.append((time.perf_counter() - t0) * 1e3)
            same = same and np.array_equal(img, rimg)
    ms = statistics.median(times)
    row = {"row": "GetVRData cardiac 512^2 (API: render + orientation box + copy)", "image": "512x512",
           "e2e_ms": round(ms, 4), "fps": round(1e3 / ms, 1)}
    if ref is not None:
        rms = statistics.median(rtimes)
        row.update({"ref_call_ms": round(rms, 4), "speedup_e2e": round(rms / ms, 2), "identical_images": same})
    return [row]


def upload_rows(ctx):
    """Upload of the body volume and its labels: mk_volume_create (3D array
    copy, brick min/max, schedule table) + mk_volume_set_mask (mask texture,
    brick label sets), wall clock from host arrays, beside MonkeyGL's
    SetVolumeData + SetMask of the same arrays (its CuDataManager copies the
    volume into a 3D array and the mask into another)."""
    from monkeygl_b200 import capi
    w = _workload(ctx, "body")
    vox, lab = w.phantom.volume, w.phantom.labels

    def ours(_):
        v = capi.Volume(vox)
        v.set_mask(lab)
        v.close()

    ours(0)
    row = {"row": "upload body volume + labels", "image": "x".join(map(str, vox.shape[::-1])),
           "e2e_ms": round(_wall_ms(ours, 5), 2)}
    ref = ctx["ref"]
    if ref is not None:
        def theirs(_):
            ref.set_volume(vox)
            ref.set_mask(lab)
        theirs(0)
        row["ref_call_ms"] = round(_wall_ms(theirs, 5), 2)
        row["speedup_e2e"] = round(row["ref_call_ms"] / row["e2e_ms"], 2)
    # one more object (a 64^3 box) in the resident label volume: this library
    # updates the box, MonkeyGL re-uploads the whole mask
    v = capi.Volume(vox)
    v.set_mask(lab)
    lab2 = lab.copy()
    z0, y0, x0 = (np.array(lab.shape) // 2 - 32).tolist()

    def update(i):
        lab2[z0:z0 + 64, y0:y0 + 64, x0:x0 + 64] = 5 + (i & 1)
        v.update_mask(lab2, (x0, y0, z0, x0 + 64, y0 + 64, z0 + 64))

    update(0)
    row2 = {"row": "add a 64^3 object to the body labels", "image": "64x64x64", "e2e_ms": round(_wall_ms(update, 5), 3)}
    v.close()
    if ref is not None:
        def ref_update(i):
            lab2[z0:z0 + 64, y0:y0 + 64, x0:x0 + 64] = 5 + (i & 1)
            ref.set_mask(lab2)
        ref_update(0)
        row2["ref_call_ms"] = round(_wall_ms(ref_update, 5), 2)
        row2["speedup_e2e"] = round(row2["ref_call_ms"] / row2["e2e_ms"], 1)
    return [row, row2]


def main(args=None, ref=None, ref_api=None, resources_dir=None):
    """Print the table.  `ref` is MonkeyGL's own CUDA path (an object with
    set_volume / set_mask / clear_tfs / set_lut / kernel_ms / plane / cpr),
    `ref_api` its complete HelloMonkey (set_volume / set_transfer_function /
    set_wwwl / set_vr_size / orientation / rotate / vr_image) and
    `resources_dir` the directory holding resources/human.stl, all supplied
    by the caller, or None for no reference columns."""
    import torch
    torch.cuda.init()
    ctx = {"stream": torch.cuda.Stream(), "flush": torch.empty(256 << 20, dtype=torch.uint8, device="cuda"),
           "ref": ref, "ref_api": ref_api, "resources_dir": resources_dir}
    only = {g for g in (getattr(args, "suite_only", "") or "").split(",") if g}
    want = lambda g: not only or g in only
    rows = []
    if want("vr"):
        rows += vr_rows("cardiac", 0.4, (0,), ctx)
        rows += vr_rows("body", 0.4, (0,), ctx)
        rows += vr_rows("body", 0.8, (0,), ctx)
        rows += vr_rows("body", 0.4, (0,), ctx, dense=True)
    if want("mip"):
        rows += vr_rows("cardiac", 0.4, (1,), ctx)
        rows += vr_rows("body", 0.4, (1,), ctx)
    if want("mpr"):
        rows += mpr_rows(ctx)
    if want("cpr"):
        rows += cpr_rows(ctx)
    if want("dvr"):
        rows += dvr_rows(ctx)
    if want("api"):
        rows += api_rows(ctx)
    if want("upload"):
        rows += upload_rows(ctx)
    for r in rows:
        print(json.dumps(r), flush=True)
    keys = ["row", "image", "ms", "e2e_ms", "ref_kernel_ms", "ref_call_ms", "speedup_kernel", "speedup_e2e",
            "bwd_over_fwd", "gsamples_per_s"]
    print("| " + " | ".join(keys) + " |")
    print("|" + "---|" * len(keys))
    for r in rows:
        print("| " + " | ".join(str(r.get(k, "")) for k in keys) + " |")


if __name__ == "__main__":
    main()
