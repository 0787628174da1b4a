#!/usr/bin/env python
"""Benchmark of MonkeyGL-B200's volume ray-casting path.

Headline workload (one "step" = one frame): direct volume rendering of the
body phantom (int16 512x512x1559, spacing 0.7422x0.7422x1.0) with 4 labelled
objects, per-object 256-entry transfer functions and opacity caps,
background cap 0.4, into a 1024x1024 RGB8 image, cycling through 36 views
(10 degree steps about z).  Synthetic seeded data (monkeygl_b200.workloads).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mine|reference]
    python bench.py --suite        # per-mode table (VR/MIP/MPR/CPR, differentiable VR), not the contract line
    python bench.py --serve        # serving: p50/p99 latency and renders/s vs the one-launch-per-request path

`value` is device time of the rendering kernels (CUDA events on the launching
stream, L2 flushed by a 256 MiB write between steps, outside the events);
`e2e` is the same frames through the C ABI call mk_render_vr with a pinned
host output buffer (device->host copy inside the timed region).  With N>1
ranks each GPU holds a replica and renders its own views (replicas only: the
path has no exchange step); the time is the max over ranks.

The reference arm runs MonkeyGL's own CUDA path (core/kernel.cu and
core/CuDataManager.cu built unmodified for sm_100a, oracle/_ref) through its
own launcher cu_render, host buffers, same workload.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "VR fps & Gsamples/s vs ref CUDA on 1xB200; served p50/p99 ms; bwd/fwd time"
MODES = {"vr": 0, "mip": 1, "surface": 2}
WORKLOADS = {
    "body": ("body {mode}: int16 512x512x1559 (0.7422x0.7422x1.0 mm), 4 labelled objects + background "
             "(cap {bg}), 256-entry LUT per label, {size}x{size} RGB8, 36 views about z"),
    "cardiac": ("cardiac {mode}: int16 512x512x361 (0.351x0.351x0.3 mm), one 256-entry LUT, "
                "{size}x{size} RGB8, 36 views about z"),
    "small": ("small {mode}: int16 128x128x96 (0.35x0.35x0.3 mm), one 256-entry LUT, {size}x{size} RGB8, "
              "3 views about z"),
}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1080)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["mine", "reference"], default="mine")
    ap.add_argument("--bg", type=float, default=0.4)
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="body")
    ap.add_argument("--size", type=int, default=1024)
    ap.add_argument("--mode", choices=["vr", "mip", "surface"], default="vr",
                    help="render type of the timed frames (the contract line is VR)")
    ap.add_argument("--suite", action="store_true")
    ap.add_argument("--suite-only", default="", help="comma list of suite groups: vr,mip,mpr,cpr,dvr,api,upload (default all)")
    ap.add_argument("--serve", action="store_true", help="serving benchmark (monkeygl_b200.serve_bench)")
    ap.add_argument("--serve-requests", type=int, default=10000)
    ap.add_argument("--serve-rate", type=float, default=200.0)
    ap.add_argument("--saturation", type=int, default=2000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the serving and differentiable-rendering figures of the contract line")
    ap.add_argument("--extra-requests", type=int, default=1000,
                    help="requests of the contract line's serving trace")
    return ap.parse_args()


# ----------------------------------------------------------------------
# process group (one process per GPU)

def dist_setup(n_gpus, backend="nccl"):
    """Rank, local rank and world size from the torchrun environment; joins
    the process group when there is more than one rank.  `backend` "gloo"
    runs the same host logic without GPUs."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    if backend == "nccl":
        torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        kw = {"device_id": torch.device("cuda", local)} if backend == "nccl" else {}
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120), **kw)
    return rank, local, world


def _reduce_device():
    import torch.distributed as dist
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=_reduce_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rank_views(angles, rank):
    """The views a rank renders, in order: every view, starting 7 views
    further along per rank so the replicas do not render in lockstep."""
    return [angles[(rank * 7 + i) % len(angles)] for i in range(len(angles))]


def sum_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=_reduce_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


# ----------------------------------------------------------------------
# clock sampling during the timed region

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, mx, pw, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
                pw.append(float(parts[3]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "power_w_max": max(pw),
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_from_profile(args):
    """DRAM bytes per frame of the VR launches (tile launch + tail launch)
    from the committed ncu summary of the default workload (body VR, 1024^2,
    background cap 0.4); None for any other workload, which has no capture."""
    if (args.workload, args.mode, args.size, args.bg) != ("body", "vr", 1024, 0.4):
        return None
    p = ROOT / "profiles" / "vr_body_1024_traffic.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return d.get("dram_bytes_per_frame", d.get("dram_bytes_per_launch"))
        except (ValueError, OSError):
            return None
    return None


# ----------------------------------------------------------------------
# my implementation

def bench_config(args, world):
    """The `config` of both arms' lines (identical for the same workload)."""
    return {"workload": WORKLOADS[args.workload].format(bg=args.bg, size=args.size, mode=args.mode.upper()),
            "views": 36 if args.workload != "small" else 3, "image": f"{args.size}x{args.size}",
            "bg_alpha": args.bg, "parallelism": f"replicas{world}" if world > 1 else "single GPU"}


def frames_crc32(render_view, n_views):
    """CRC-32 of the RGB image of each view (rendered again after the timed
    region: an image depends only on its view) and a CRC-32 over those, so
    the two arms' lines show whether they produce the same frames."""
    import zlib
    per = [zlib.crc32(memoryview(np.ascontiguousarray(render_view(i))).cast("B")) for i in range(n_views)]
    allc = zlib.crc32(np.asarray(per, dtype="<u4").tobytes())
    return {"all": f"{allc:08x}", "per_view": [f"{c:08x}" for c in per]}


def setup_volume(w, device):
    from monkeygl_b200 import capi
    vol = capi.Volume(w.phantom.volume, device=device)
    if w.phantom.labels is not None:
        vol.set_mask(w.phantom.labels)
    for l, lut in w.luts.items():
        vol.set_transfer_function(l, lut)
    vol.set_label_params(w.label_params)
    return vol


def frame_params(w, angle, size, render_type=0):
    from monkeygl_b200 import capi
    from monkeygl_b200.workloads import view_camera
    return capi.vr_params(size, size, render_type, view_camera(angle), w.dims, w.spacing, invert_z=False)


def cpu_baseline(w, angle, size, rtype=0):
    """Time the C restatement (oracle, texture-emulating FP32): whole frames
    of consecutive views with OpenMP over rows on every host thread for about
    10 s, and one thread on every 16th row of a frame (scaled to a frame)."""
    import oracle
    from monkeygl_b200 import capi
    cv = oracle.CpuVolume(w.phantom.volume, w.phantom.labels)
    for l, lut in w.luts.items():
        cv.set_lut(l, lut)
    cores = os.cpu_count() or 1
    frames, t0 = 0, time.perf_counter()
    angles = list(w.angles)
    start = angles.index(angle) if angle in angles else 0
    while True:
        a = angles[(start + frames) % len(angles)]
        flat = capi.vr_params_flat(frame_params(w, a, size, rtype), w.label_params)
        cv.render_vr(size, size, rtype, flat, threads=cores)
        frames += 1
        dt = time.perf_counter() - t0
        if dt >= 10.0 or frames >= 2 * len(angles):
            break
    flat = capi.vr_params_flat(frame_params(w, angles[start], size, rtype), w.label_params)
    t1 = time.perf_counter()
    cv.render_vr_rows(size, size, rtype, flat, 0, 16, size // 16, threads=1)
    one = (time.perf_counter() - t1) * 16
    return {"value": round(frames / dt, 4), "unit": "fps", "cores": cores, "kind": "port",
            "single_thread_fps": round(1.0 / one, 5),
            "sample": f"oracle/mk_oracle.c (FP32, texture emulation, OpenMP over rows) rendering {frames} "
                      f"full {size}x{size} frames of consecutive views from {angle:.0f} deg in "
                      f"{dt:.1f} s on {cores} host threads; single thread: every 16th row of one frame, "
                      f"{one:.1f} s per frame"}


def run_mine(args, rank, local, world):
    import torch
    from monkeygl_b200 import capi
    from monkeygl_b200.workloads import make_workload

    w = make_workload(args.workload, bg_alpha=args.bg)
    size = args.size
    vol = setup_volume(w, local)
    angles = w.angles
    views = rank_views(angles, rank)
    rtype = MODES[args.mode]
    params = [frame_params(w, a, size, rtype) for a in views]
    stream = torch.cuda.Stream()
    out = torch.empty(size * size * 3, dtype=torch.uint8, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    K, W = args.steps, max(3, args.warmup)

    with torch.cuda.stream(stream):
        for i in range(W):
            vol.render_vr_device(params[i % len(params)], out.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    with torch.cuda.stream(stream):
        for i in range(K):
            flush.zero_()
            ev0[i].record(stream)
            vol.render_vr_device(params[i % len(params)], out.data_ptr(), stream.cuda_stream)
            ev1[i].record(stream)
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    clk = clocks.stop()
    step_ms = [ev0[i].elapsed_time(ev1[i]) for i in range(K)]
    total_s = sum(step_ms) / 1e3
    total_max = max_over_ranks(total_s, world)
    value = K * world / total_max

    # end to end through the C ABI with a pinned host buffer
    host = torch.empty(size * size * 3, dtype=torch.uint8, pin_memory=True)
    host_np = host.numpy().reshape(size, size, 3)
    for i in range(W):
        vol.render_vr(params[i % len(params)], out=host_np)
    barrier(world)
    Ke = K
    t0 = time.perf_counter()
    for i in range(Ke):
        vol.render_vr(params[i % len(params)], out=host_np)
    e2e_s = time.perf_counter() - t0
    e2e_max = max_over_ranks(e2e_s, world)
    e2e_value = Ke * world / e2e_max

    crc = None
    if rank == 0:
        def mine_view(i):
            vol.render_vr(params[i], out=host_np)
            return host_np
        crc = frames_crc32(mine_view, len(params))

    # reference-schedule samples per frame (all views) and footprint bytes (3 views)
    samples = [vol.count_samples(p) for p in params]
    mean_samples = float(np.mean(samples))
    n = len(params)
    foot = [vol.count_footprint(params[i]) for i in sorted({0, n // 3, (2 * n) // 3})]
    vox = float(np.mean([f[1] for f in foot]))
    lab = float(np.mean([f[2] for f in foot]))
    out_bytes = size * size * 3
    b_alg = 2.0 * vox + lab + out_bytes
    mean_ms = total_s * 1e3 / K
    achieved = b_alg / (mean_ms / 1e3) / 1e9
    peak, peak_kind = measured_peaks()
    gsps = mean_samples * (K / total_s) / 1e9
    # a VR frame is two launches: the tiles, then the rays handed to the tail launch
    tail = args.mode == "vr" and os.environ.get("MONKEYGL_B200_TAIL_TILES", "") != "0"
    launches_per_frame = 2 if tail else 1
    kernel_desc = (f"mk::k_raycast<{args.mode.upper()}> + mk::k_vr_tail (two launches per frame, timed together)"
                   if tail else f"mk::k_raycast<{args.mode.upper()}> (one launch per frame)")

    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "fps", "n_gpus": world, "steps": K,
        "warmup": W, "ms_per_step": round(total_max * 1e3 / K, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": bench_config(args, world),
        "l2": "flushed between steps (256 MiB write, outside the events)",
        "gsamples_per_s": round(gsps * world, 3),
        "samples_per_frame": int(mean_samples),
        "e2e": {"value": round(e2e_value, 3), "unit": "fps", "h2d_bytes_per_step": ctypes.sizeof(capi.VRParams),
                "d2h_bytes_per_step": out_bytes,
                "note": "each step is one mk_render_vr call with a pinned host output buffer: the volume, "
                        "labels and LUTs are resident in HBM (uploaded once, before timing); the per-frame "
                        "input is the mk_vr_params block (camera, size, flags), which reaches the device as "
                        "kernel arguments; the RGB image is copied device to host inside the timed region"},
        "frames_crc32": crc,
        "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic_from_profile(args),
                     "peak_kind": f"{peak_kind} hbm_gbs (burst copy)",
                     "algorithmic_bytes_per_frame": int(b_alg),
                     "kernel": kernel_desc},
        "clocks": {k: clk.get(k) for k in ("sm_mhz", "sm_max_mhz", "reasons", "samples")},
        "gpu_launches": K * launches_per_frame,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(w, views[0], size, rtype)
    vol.close()
    if rank == 0 and world == 1 and not args.no_extras and args.workload == "body":
        line.update(extra_figures(args, w))
    return line


def extra_figures(args, w):
    """The metric's other figures, measured after the timed frames: served
    p50/p99 latency and renders/s of the continuous-batching server against
    this library's one-launch-per-request path (a short serving trace over
    the four resident serving volumes), and the backward/forward time of the
    differentiable renderer (256^3 float volume, 8 views of 256^2)."""
    import torch
    from monkeygl_b200 import serve_bench, suite
    out = {}
    sv = serve_bench.measure(n=args.extra_requests, rate=200.0, nsat=max(1, args.extra_requests // 2),
                             phantoms=serve_bench.serving_phantoms(body=w.phantom), evict=False)
    out["served_p50_ms"] = sv["server"]["p50_ms"]
    out["served_p99_ms"] = sv["server"]["p99_ms"]
    out["served_renders_per_s"] = sv["server"]["saturation_renders_per_s"]
    out["plain_renders_per_s"] = sv["plain"]["saturation_renders_per_s"]
    out["served_renders_per_s_ratio"] = sv["saturation_ratio"]
    out["served_workload"] = (f"{args.extra_requests} requests (seeded Poisson 200/s; VR/MIP/MPR 60/20/20, "
                              "256..1024^2, 4 resident volumes, random cameras and TFs); p50/p99 at the "
                              "arrival rate, renders/s with the first half submitted at once; ratio against "
                              "mk_render_vr/mk_render_plane one request per launch")
    ctx = {"stream": torch.cuda.Stream(), "flush": torch.empty(256 << 20, dtype=torch.uint8, device="cuda")}
    rows = suite.dvr_rows(ctx)
    out["dvr_fwd_ms"] = rows[0]["ms"]
    out["dvr_bwd_ms"] = rows[1]["ms"]
    out["dvr_bwd_fwd_ratio"] = rows[1]["bwd_over_fwd"]
    return out


# ----------------------------------------------------------------------
# reference arm: MonkeyGL's own CUDA path

def run_reference(args, rank, world):
    import oracle
    from monkeygl_b200 import capi
    from monkeygl_b200.workloads import make_workload

    if rank != 0:
        return None
    if not oracle.ref_gpu_available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libmkref_gpu.so was not built"}
    w = make_workload(args.workload, bg_alpha=args.bg)
    size = args.size
    ref = oracle.RefGPU()
    ref.set_volume(w.phantom.volume)
    ref.set_mask(w.phantom.labels)
    ref.clear_tfs()
    for l, lut in w.luts.items():
        ref.set_lut(l, lut)
    flats = []
    for a in w.angles:
        p = frame_params(w, a, size, MODES[args.mode])
        flats.append(np.ascontiguousarray(capi.vr_params_flat(p, w.label_params)))
    K, W = args.steps, max(3, args.warmup)
    out = np.zeros((size, size, 3), np.uint8)
    for i in range(W):
        ref.render_into(out, size, size, MODES[args.mode], flats[i % len(flats)])
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    t0 = time.perf_counter()
    for i in range(K):
        ref.render_into(out, size, size, MODES[args.mode], flats[i % len(flats)])
    dt = time.perf_counter() - t0
    clk = clocks.stop()
    kms = float(np.mean([ref.kernel_ms(size, size, MODES[args.mode], flats[i], 3)
                         for i in sorted({(k * len(flats)) // 4 for k in range(4)})]))

    def ref_view(i):
        ref.render_into(out, size, size, MODES[args.mode], flats[i])
        return out
    crc = frames_crc32(ref_view, len(flats))
    value = K / dt
    extras = {}
    if args.workload == "body" and not args.no_extras:
        from monkeygl_b200 import serve_bench
        sv = serve_bench.measure_monkeygl(ref, n=args.extra_requests, rate=200.0,
                                          nsat=max(1, args.extra_requests // 2),
                                          phantoms=serve_bench.serving_phantoms(body=w.phantom))
        extras = {"served_p50_ms": sv["p50_ms"], "served_p99_ms": sv["p99_ms"],
                  "served_renders_per_s": sv["saturation_renders_per_s"],
                  "served_workload": "the same trace as this line's other arm, one request per launch through "
                                     "MonkeyGL's cu_setTransferFunc + cu_render / cu_renderPlane_* (volumes "
                                     "resident in the harness)"}
    line = {
        "metric": METRIC, "impl": "reference", "value": round(value, 3), "unit": "fps", "n_gpus": 1,
        "steps": K, "warmup": W, "ms_per_step": round(dt * 1e3 / K, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": bench_config(args, 1),
        "l2": "inputs larger than L2 (817 MB volume)",
        "kernel_ms_per_frame": round(kms, 4),
        "frames_crc32": crc,
        "e2e": {"value": round(value, 3), "unit": "fps", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "cpu_baseline": {"value": round(value, 3), "unit": "fps", "cores": 1, "kind": "reference",
                         "sample": "MonkeyGL's own cu_render (core/kernel.cu, unmodified, sm_100a) on this "
                                   f"B200 with host buffers, {K} frames over 36 views; MonkeyGL has no "
                                   "CPU rendering path"},
        "clocks": {k: clk.get(k) for k in ("sm_mhz", "sm_max_mhz", "reasons", "samples")},
    }
    line.update(extras)
    return line


def main():
    args = parse_args()
    if args.suite:
        import oracle
        from monkeygl_b200 import suite
        # MonkeyGL's own kernels built from its sources (oracle/_ref), for the reference columns
        suite.main(args, oracle.RefGPU() if oracle.ref_gpu_available() else None,
                   oracle.RefHelloMonkey() if oracle.ref_full_available() else None,
                   str(oracle.REF_FULL_LIB.parent) if oracle.ref_full_available() else None)
        return
    if args.serve:
        from monkeygl_b200 import serve_bench
        import oracle
        # MonkeyGL's own kernels (oracle/_ref) for the one-launch-per-request comparison
        serve_bench.main(args, oracle.RefGPU() if oracle.ref_gpu_available() else None)
        return
    if args.impl == "reference":
        # MonkeyGL is one process on one GPU: rank 0 runs it, other ranks exit
        rank = int(os.environ.get("RANK", "0"))
        line = run_reference(args, rank, 1)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    rank, local, world = dist_setup(args.gpus)
    try:
        line = run_mine(args, rank, local, world)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
