"""Serving benchmark (``bench.py --serve``).

Four resident int16 phantoms (256^3; 512x512x361; 512x512x600; 512x512x1559
with 4 labelled objects) and a seeded Poisson stream of VR / MIP / MPR
requests (60/20/20) with square images of 256, 512, 768 or 1024 pixels,
random cameras and transfer functions (workloads.serving_trace).  The same
trace runs through

  * the server (mk_server_*): requests submitted at their arrival times by
    one thread, collected by another; latency = completion - arrival;
  * the plain path: one thread renders each request with the one-frame entry
    points (set the request's LUTs and label parameters, mk_render_vr /
    mk_render_plane, synchronous), first come first served; latency =
    completion - arrival, so time spent waiting behind earlier requests
    counts.

Then both run the first `--saturation` requests of the trace all at once
(arrival 0) for the renders/s each path sustains.  Outputs go to pinned host
buffers in both paths.
"""
from __future__ import annotations

import json
import queue
import sys
import threading
import time


def _phase(what, t0=[None]):
    """Progress of the benchmark's phases on stderr (the result line goes
    to stdout at the end)."""
    now = time.perf_counter()
    if t0[0] is None:
        t0[0] = now
    print(f"[serve_bench {now - t0[0]:8.1f} s] {what}", file=sys.stderr, flush=True)

import numpy as np


class _Pool:
    """Pinned output buffers of the largest image, reused once collected."""

    def __init__(self, n, nbytes):
        import torch
        self._t = [torch.empty(nbytes, dtype=torch.uint8, pin_memory=True) for _ in range(n)]
        self._free = queue.Queue()
        for i in range(n):
            self._free.put(i)

    def take(self):
        return self._free.get()

    def give(self, i):
        self._free.put(i)

    def view(self, i, shape, dtype):
        n = int(np.prod(shape)) * np.dtype(dtype).itemsize
        return self._t[i][:n].numpy().view(dtype).reshape(shape)


def _shape(r):
    from . import capi
    if r.kind == capi.REQUEST_MPR:
        return (r.size, r.size), np.int16
    return (r.size, r.size, 3), np.uint8


def _pcts(lat):
    a = np.asarray(lat, np.float64)
    return {"p50_ms": round(float(np.percentile(a, 50)), 3), "p99_ms": round(float(np.percentile(a, 99)), 3),
            "mean_ms": round(float(a.mean()), 3), "max_ms": round(float(a.max()), 3)}


# A request not done this long after the collector starts waiting for it
# ends the run with MK_ERR_TIMEOUT instead of waiting for good.
WAIT_LIMIT_MS = 120_000


def eviction_trace(trace, n, pairs):
    """`n` requests of `trace` in len(pairs) phases of equal length: phase k
    takes, in trace order, the next requests whose volume is in pairs[k] (a
    reader who finishes one pair of studies and opens the next).  Arrival
    gaps are the trace's own, so the rate is unchanged."""
    from dataclasses import replace
    per = -(-n // len(pairs))
    out, t, used = [], 0.0, set()
    gaps = [r.arrival_s - (trace[i - 1].arrival_s if i else 0.0) for i, r in enumerate(trace)]
    for k, pair in enumerate(pairs):
        taken = 0
        for i, r in enumerate(trace):
            if taken == per or len(out) == n:
                break
            if i in used or r.volume not in pair:
                continue
            used.add(i)
            t += gaps[len(out)]
            out.append(replace(r, arrival_s=t))
            taken += 1
    return out


def run_server(srv, vids, trace, pool, open_loop: bool):
    """Submit the trace (at its arrival times if open_loop, else at once);
    returns per-request latencies (ms), wall seconds and the images' tickets order."""
    from . import server as S
    q = queue.Queue()
    t0 = time.perf_counter()

    def submitter():
        for i, r in enumerate(trace):
            if open_loop:
                dt = t0 + r.arrival_s - time.perf_counter()
                if dt > 0:
                    time.sleep(dt)
            b = pool.take()
            shape, dt_ = _shape(r)
            sub_wall = time.perf_counter()
            t = S.submit_request(srv, vids[r.volume], r, out=pool.view(b, shape, dt_))
            q.put((i, t, b, sub_wall))
        q.put(None)

    th = threading.Thread(target=submitter, daemon=True)
    th.start()
    lat = [0.0] * len(trace)
    last = t0
    while True:
        item = q.get()
        if item is None:
            break
        i, t, b, sub_wall = item
        _, tm = srv.wait(t, WAIT_LIMIT_MS)
        pool.give(b)
        late = max(0.0, sub_wall - (t0 + trace[i].arrival_s)) * 1e3 if open_loop else (sub_wall - t0) * 1e3
        lat[i] = late + (tm["completed_ms"] - tm["submitted_ms"])
        last = time.perf_counter()
    th.join()
    return lat, last - t0


def run_plain(vols, trace, pool, open_loop: bool):
    from . import server as S
    b = pool.take()
    lat = []
    t0 = time.perf_counter()
    for r in trace:
        if open_loop:
            dt = t0 + r.arrival_s - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
        shape, dt_ = _shape(r)
        S.render_plain(vols[r.volume], r, out=pool.view(b, shape, dt_))
        lat.append((time.perf_counter() - (t0 + (r.arrival_s if open_loop else 0.0))) * 1e3)
    wall = time.perf_counter() - t0
    pool.give(b)
    return lat, wall


def run_monkeygl(ref, trace, pool, open_loop: bool):
    """The trace through MonkeyGL's own launchers (its core/kernel.cu and
    core/CuDataManager.cu, oracle/_ref), one request per launch as its
    HelloMonkey serves one: the request's LUTs through cu_setTransferFunc
    (an array allocated per table), then cu_render (output allocated, kernel,
    synchronous copy, free) or cu_renderPlane_*.  The volumes stay resident
    in the harness's slots, which MonkeyGL's one-volume singleton cannot do,
    so no upload is counted.  Volume i of the trace is the harness's slot
    i + 1 (slot 0 keeps the volume its caller loaded)."""
    from . import capi
    b = pool.take()
    lat = []
    lp65 = np.zeros((capi.MAX_LABELS, 3), np.float32)
    t0 = time.perf_counter()
    for r in trace:
        if open_loop:
            dt = t0 + r.arrival_s - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
        ref.select(r.volume + 1)
        if r.kind == capi.REQUEST_MPR:
            ref.plane(r.size, r.size, capi.plane_params_flat(r.plane), r.plane.mpr_type, r.plane.sampling)
        else:
            ref.clear_tfs()
            n = r.luts.shape[0]
            for l in range(n):
                ref.set_lut(l, r.luts[l])
            lp65[:] = (0.0, 1.0, 0.0)
            lp65[:n] = r.label_params
            out = pool.view(b, (r.size, r.size, 3), np.uint8)
            ref.render_into(out, r.size, r.size, r.kind, np.ascontiguousarray(capi.vr_params_flat(r.vr, lp65)))
        lat.append((time.perf_counter() - (t0 + (r.arrival_s if open_loop else 0.0))) * 1e3)
    wall = time.perf_counter() - t0
    pool.give(b)
    return lat, wall


def measure(n=10000, rate=200.0, nsat=2000, phantoms=None, ref=None, evict=True):
    """The serving figures as a dict: the trace through the server, through
    this library's one-launch-per-request path and (with `ref`, MonkeyGL's
    kernels) through MonkeyGL's one-launch-per-request path; then an
    eviction run (server with evict_idle under a budget below the four
    volumes) when `evict`.  `phantoms` may pass the four serving phantoms
    (workloads.SERVING_VOLUMES) already built."""
    import torch
    from . import capi
    from . import server as S
    from .workloads import serving_trace

    nsat = min(n, nsat)
    torch.cuda.init()
    _phase("phantoms")
    if phantoms is None:
        phantoms = serving_phantoms()
    specs = [(p.dims, p.spacing, p.labels is not None) for p in phantoms]
    _phase("trace")
    trace = serving_trace(specs, n, rate, seed=2024)
    pool = _Pool(64, 1024 * 1024 * 4)
    _phase("server and volumes")

    srv = S.Server(max_slots=32, max_pending=max(n, 1), max_pixels=1024 * 1024, max_labels=8)
    slot_bytes = srv.stats()["resident_bytes"]
    vids, vol_bytes = [], []
    for p in phantoms:
        before = srv.stats()["resident_bytes"]
        vids.append(srv.add_volume(p.volume, p.labels))
        vol_bytes.append(srv.stats()["resident_bytes"] - before)
    plain_vols = []
    for p in phantoms:
        v = capi.Volume(p.volume)
        if p.labels is not None:
            v.set_mask(p.labels)
        plain_vols.append(v)

    _phase("warm-up")
    # warm-up: every volume and kind once on both paths; spot-check equality
    warm = serving_trace(specs, 64, 1000.0, seed=99)
    bad = []
    for i, r in enumerate(warm):
        shape, dt = _shape(r)
        b1, b2 = pool.take(), pool.take()
        out1, out2 = pool.view(b1, shape, dt), pool.view(b2, shape, dt)
        srv.wait(S.submit_request(srv, vids[r.volume], r, out=out1))
        S.render_plain(plain_vols[r.volume], r, out=out2)
        if not np.array_equal(out1, out2):
            d = np.abs(out1.astype(np.int64) - out2.astype(np.int64))
            bad.append({"request": i, "kind": r.kind, "volume": r.volume, "size": r.size,
                        "pixels_differing": int((d.reshape(r.size, r.size, -1).max(-1) > 0).sum()),
                        "max_diff": int(d.max())})
        pool.give(b1)
        pool.give(b2)
    if bad:
        print(json.dumps({"mismatches": bad}), flush=True)
        raise RuntimeError(f"server and plain path images differ on {len(bad)} of {len(warm)} requests")

    st0 = srv.stats()
    _phase("server, open loop")
    lat_s, wall_s = run_server(srv, vids, trace, pool, open_loop=True)
    st1 = srv.stats()
    _phase("plain path, open loop")
    lat_p, wall_p = run_plain(plain_vols, trace, pool, open_loop=True)
    _phase("server, saturation")
    sat_s_lat, sat_s = run_server(srv, vids, trace[:nsat], pool, open_loop=False)
    _phase("plain path, saturation")
    sat_p_lat, sat_p = run_plain(plain_vols, trace[:nsat], pool, open_loop=False)
    srv.close()
    for v in plain_vols:
        v.close()

    kinds = {0: "VR", 1: "MIP", 3: "MPR"}
    mix = {k: sum(1 for r in trace if r.kind == c) for c, k in kinds.items()}
    line = {
        "metric": "served latency p50/p99 (ms) at the arrival rate, and renders/s at saturation",
        "workload": f"{n} requests, Poisson {rate:g}/s, VR/MIP/MPR {mix}, sizes 256..1024^2, 4 resident volumes "
                    "(256^3, 512^2x361, 512^2x600, 512^2x1559 + labels), random cameras and TFs",
        "server": {**_pcts(lat_s), "renders_per_s": round(n / wall_s, 1),
                   "saturation_renders_per_s": round(nsat / sat_s, 1),
                   "steps": st1["steps"] - st0["steps"], "tiles": st1["tiles"] - st0["tiles"],
                   "resident_mb": round(st1["resident_bytes"] / 2 ** 20, 1)},
        "plain": {**_pcts(lat_p), "renders_per_s": round(n / wall_p, 1),
                  "saturation_renders_per_s": round(nsat / sat_p, 1)},
        "saturation_requests": nsat,
        "saturation_ratio": round((nsat / sat_s) / (nsat / sat_p), 2),
        "p99_target_ms": 20.0,
    }
    line["saturation_latency"] = {"server": _pcts(sat_s_lat), "plain": _pcts(sat_p_lat)}
    if ref is not None:
        for i, p in enumerate(phantoms):
            ref.select(i + 1)
            ref.set_volume(p.volume)
            ref.set_mask(p.labels)
        _phase("MonkeyGL path, open loop")
        lat_m, wall_m = run_monkeygl(ref, trace, pool, open_loop=True)
        _phase("MonkeyGL path, saturation")
        sat_m_lat, sat_m = run_monkeygl(ref, trace[:nsat], pool, open_loop=False)
        ref.select(0)
        line["monkeygl_plain"] = {**_pcts(lat_m), "renders_per_s": round(n / wall_m, 1),
                                  "saturation_renders_per_s": round(nsat / sat_m, 1)}
        line["saturation_ratio_vs_monkeygl"] = round((nsat / sat_s) / (nsat / sat_m), 2)
        line["saturation_latency"]["monkeygl_plain"] = _pcts(sat_m_lat)
    if evict:
        # The budget holds the slots and the two largest volumes, not all
        # four; the requests move between pairs of volumes in phases.  Each
        # phase change evicts the idle volume that the new pair does not use
        # and uploads the one it needs, while requests for the other keep
        # running.  (A budget below the volumes that the requests of any one
        # second use makes every path thrash: each request waits for an upload.)
        big = sorted(range(len(vol_bytes)), key=lambda i: -vol_bytes[i])
        budget = int(slot_bytes + vol_bytes[big[0]] + vol_bytes[big[1]])
        nv = len(phantoms)
        pairs = [(k % nv, (k + 1) % nv) for k in range(nv)]
        ne = min(n, 2000)
        etrace = eviction_trace(trace, ne, pairs)
        _phase("eviction run")
        with S.Server(max_slots=32, max_pending=max(ne, 1), max_pixels=1024 * 1024, max_labels=8,
                      hbm_budget_bytes=budget, evict_idle=True) as es:
            evids = [es.add_volume(p.volume, p.labels) for p in phantoms]
            lat_e, wall_e = run_server(es, evids, etrace, pool, open_loop=True)
            est = es.stats()
        line["eviction"] = {**_pcts(lat_e), "requests": len(etrace), "renders_per_s": round(len(etrace) / wall_e, 1),
                            "phases": [list(p) for p in pairs], "budget_mb": round(budget / 2 ** 20, 1),
                            "volumes_mb": round(sum(vol_bytes) / 2 ** 20, 1),
                            "evictions": est["evictions"], "loads": est["loads"]}
    _phase("done")
    return line


def serving_phantoms(body=None):
    """The four serving phantoms (workloads.SERVING_VOLUMES); `body` may pass
    the 512x512x1559 labelled one (the same seed as the body workload)."""
    from .phantom import make_phantom
    from .workloads import SERVING_VOLUMES
    out = []
    for d, sp, seed, lab in SERVING_VOLUMES:
        if body is not None and tuple(d) == tuple(body.dims) and lab and seed == 1236:
            out.append(body)
        else:
            out.append(make_phantom(d, sp, seed, with_labels=lab))
    return out


def measure_monkeygl(ref, n=1000, rate=200.0, nsat=500, phantoms=None):
    """MonkeyGL's one-launch-per-request path alone on the same trace as
    measure(): p50/p99 at the arrival rate and renders/s at saturation."""
    from .workloads import serving_trace
    if phantoms is None:
        phantoms = serving_phantoms()
    specs = [(p.dims, p.spacing, p.labels is not None) for p in phantoms]
    trace = serving_trace(specs, n, rate, seed=2024)
    nsat = min(n, nsat)
    pool = _Pool(2, 1024 * 1024 * 4)
    for i, p in enumerate(phantoms):
        ref.select(i + 1)
        ref.set_volume(p.volume)
        ref.set_mask(p.labels)
    run_monkeygl(ref, serving_trace(specs, 64, 1000.0, seed=99), pool, open_loop=False)   # warm-up
    lat, wall = run_monkeygl(ref, trace, pool, open_loop=True)
    _, sat = run_monkeygl(ref, trace[:nsat], pool, open_loop=False)
    ref.select(0)
    return {**_pcts(lat), "renders_per_s": round(n / wall, 1), "saturation_renders_per_s": round(nsat / sat, 1),
            "requests": n, "saturation_requests": nsat}


def main(args, ref=None):
    n = getattr(args, "serve_requests", 10000) or 10000
    rate = getattr(args, "serve_rate", 200.0) or 200.0
    nsat = getattr(args, "saturation", 2000) or 2000
    line = measure(n, rate, nsat, ref=ref)
    print(json.dumps(line), flush=True)
    return line
