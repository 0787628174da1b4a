"""Serving (mk_server_*): every request's image is the one the one-frame
entry points produce for it, whether it runs alone or mixed with others
(continuous batching over two volumes, requests spanning several steps),
and the admission limits -- HBM budget, pending queue, volume removal,
wait timeouts, an injected allocation failure -- come back as statuses."""
import os

import numpy as np
import pytest

from monkeygl_b200 import capi
from monkeygl_b200 import server as srvmod
from monkeygl_b200.camera import view_camera
from monkeygl_b200.phantom import make_phantom
from monkeygl_b200.workloads import serving_trace

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def vols():
    return [make_phantom((96, 80, 64), (0.8, 0.8, 1.0), 31, with_labels=True),
            make_phantom((64, 64, 48), (1.0, 1.0, 1.0), 32)]


def specs(vols):
    return [(p.dims, p.spacing, p.labels is not None) for p in vols]


def plain_images(vols, reqs):
    out = []
    handles = []
    for p in vols:
        v = capi.Volume(p.volume)
        if p.labels is not None:
            v.set_mask(p.labels)
        handles.append(v)
    for r in reqs:
        out.append(srvmod.render_plain(handles[r.volume], r).copy())
    for v in handles:
        v.close()
    return out


def test_alone_and_mixed_match_plain_path(vols):
    # odd sizes (not multiples of the 32x8 tile) and a step quota of 24 tiles,
    # so most requests span several steps and steps hold several requests
    reqs = serving_trace(specs(vols), 48, 1000.0, seed=5, sizes=(37, 64, 100, 128))
    assert {r.kind for r in reqs} == {capi.REQUEST_VR, capi.REQUEST_MIP, capi.REQUEST_MPR}
    plain = plain_images(vols, reqs)
    with srvmod.Server(max_slots=6, max_pending=256, max_pixels=128 * 128, max_labels=8, tiles_per_step=24) as srv:
        vids = [srv.add_volume(p.volume, p.labels) for p in vols]
        alone = []
        for r in reqs:
            img, _ = srv.wait(srvmod.submit_request(srv, vids[r.volume], r))
            alone.append(img.copy())
        for i, (a, b) in enumerate(zip(alone, plain)):
            assert np.array_equal(a, b), f"request {i} (kind {reqs[i].kind}) alone differs from the plain path"
        tickets = [srvmod.submit_request(srv, vids[r.volume], r) for r in reqs]
        mixed, times = [], []
        for t in tickets:
            img, tm = srv.wait(t)
            mixed.append(img.copy())
            times.append(tm)
        for i, (a, b) in enumerate(zip(mixed, alone)):
            assert np.array_equal(a, b), f"request {i} differs between alone and mixed"
        # requests overlapped on the device: one started before an earlier one finished
        overlap = sum(1 for i in range(1, len(times)) if times[i]["started_ms"] < times[i - 1]["completed_ms"])
        assert overlap > 0
        st = srv.stats()
        assert st["completed"] == 2 * len(reqs) and st["slots_busy"] == 0 and st["pending"] == 0
        print(f"steps {st['steps']}, tiles {st['tiles']}, overlapping requests {overlap}")


def test_budget_queue_and_removal(vols):
    a, b = vols
    with srvmod.Server(max_slots=2, max_pending=8, max_pixels=256 * 256, max_labels=8) as probe:
        base = probe.stats()["resident_bytes"]
        probe.add_volume(b.volume)
        cost_b = probe.stats()["resident_bytes"] - base
    # room for the slots and the small volume, not for the labelled one beside it
    with srvmod.Server(hbm_budget_bytes=base + cost_b + 4096, max_slots=2, max_pending=8, max_pixels=256 * 256,
                       max_labels=8) as srv:
        vb = srv.add_volume(b.volume)
        with pytest.raises(capi.MonkeyGLError) as e:
            srv.add_volume(a.volume, a.labels)
        assert e.value.status == capi.MK_ERR_BUDGET
        srv.remove_volume(vb)                       # its memory is released and admits again
        assert srv.stats()["resident_bytes"] == base
        srv.add_volume(b.volume)
        assert srv.stats()["volumes"] == 1

    # one slot, two pending places; a heavy first request (2048^2, every
    # sample marched) holds the slot for milliseconds while the checks run
    reqs = serving_trace(specs(vols), 24, 1000.0, seed=9, sizes=(256,))
    small = [r for r in reqs if r.kind != capi.REQUEST_MPR][:3]
    heavy = capi.vr_params(2048, 2048, 0, view_camera(30.0), a.dims, a.spacing, flags=capi.VR_NO_SKIP)
    hl = next(r for r in reqs if r.volume == 0 and r.luts is not None)
    with srvmod.Server(max_slots=1, max_pending=2, max_pixels=2048 * 2048, max_labels=8) as srv:
        vids = [srv.add_volume(p.volume, p.labels) for p in vols]
        th = srv.submit_vr(vids[0], heavy, hl.luts, hl.label_params)
        tq = [srvmod.submit_request(srv, vids[r.volume], r) for r in small[:2]]
        with pytest.raises(capi.MonkeyGLError) as e:
            srvmod.submit_request(srv, vids[small[2].volume], small[2])
        assert e.value.status == capi.MK_ERR_QUEUE_FULL and srv.stats()["rejected"] == 1
        # a volume with requests queued or in flight cannot be removed
        with pytest.raises(capi.MonkeyGLError) as e:
            srv.remove_volume(vids[0])
        assert e.value.status == capi.MK_ERR_NOT_READY
        # the last request waits behind the heavy one: a zero timeout expires
        with pytest.raises(capi.MonkeyGLError) as e:
            srv.wait(tq[-1], timeout_ms=0)
        assert e.value.status == capi.MK_ERR_TIMEOUT
        srv.wait(th)
        plain = plain_images(vols, small[:2])
        for t, ref in zip(tq, plain):
            img, _ = srv.wait(t)
            assert np.array_equal(img, ref)
        for v in vids:
            srv.remove_volume(v)
        assert srv.stats()["volumes"] == 0


def test_allocation_failure_is_a_status():
    """An allocation failure during creation (injected on the host: the
    n-th device allocation reports out of memory) releases what was
    allocated and returns MK_ERR_OUT_OF_MEMORY; the next server works."""
    for n in (1, 5, 9):
        os.environ["MK_SERVER_FAIL_ALLOC"] = str(n)
        try:
            with pytest.raises(capi.MonkeyGLError) as e:
                srvmod.Server(max_slots=2, max_pending=4, max_pixels=64 * 64)
            assert e.value.status == capi.MK_ERR_OUT_OF_MEMORY
        finally:
            del os.environ["MK_SERVER_FAIL_ALLOC"]
    with srvmod.Server(max_slots=2, max_pending=4, max_pixels=64 * 64) as srv:
        assert srv.stats()["volumes"] == 0


def test_bad_requests_are_refused(vols):
    reqs = serving_trace(specs(vols), 64, 1000.0, seed=3, sizes=(64,))
    with srvmod.Server(max_slots=2, max_pending=8, max_pixels=64 * 64, max_labels=2) as srv:
        vid = srv.add_volume(vols[1].volume)
        vr = next(r for r in reqs if r.kind == capi.REQUEST_VR and r.volume == 1)
        with pytest.raises(capi.MonkeyGLError) as e:                     # unknown volume
            srvmod.submit_request(srv, vid + 100, vr)
        assert e.value.status == capi.MK_ERR_INVALID_ARGUMENT
        big = capi.vr_params(128, 128, 0, view_camera(0.0), vols[1].dims, vols[1].spacing)
        with pytest.raises(capi.MonkeyGLError) as e:                     # larger than max_pixels
            srv.submit_vr(vid, big, vr.luts, vr.label_params)
        assert e.value.status == capi.MK_ERR_INVALID_ARGUMENT
        lp = vr.label_params.copy()
        lp[0, 1] = 0.0
        with pytest.raises(capi.MonkeyGLError) as e:                     # ww <= 0
            srv.submit_vr(vid, vr.vr, vr.luts, lp)
        assert e.value.status == capi.MK_ERR_INVALID_ARGUMENT
        with pytest.raises(capi.MonkeyGLError) as e:                     # more LUTs than max_labels
            srv.submit_vr(vid, vr.vr, np.repeat(vr.luts, 3, axis=0), np.repeat(vr.label_params, 3, axis=0))
        assert e.value.status == capi.MK_ERR_INVALID_ARGUMENT
        img, _ = srv.wait(srvmod.submit_request(srv, vid, vr))            # the server still works
        assert img.shape == (64, 64, 3)


def test_eviction_under_a_budget_below_the_volumes(vols):
    """evict_idle: with room for two of three volumes, adding the third
    evicts the least recently used idle one, requests for an evicted volume
    upload it again (evicting another), every image still equals the plain
    path's, and the resident bytes never exceed the budget."""
    third = make_phantom((72, 72, 56), (0.9, 0.9, 1.1), 33)
    allv = [vols[0], vols[1], third]
    with srvmod.Server(max_slots=3, max_pending=64, max_pixels=128 * 128, max_labels=8) as probe:
        base = probe.stats()["resident_bytes"]
        costs = []
        for p in allv:
            before = probe.stats()["resident_bytes"]
            probe.add_volume(p.volume, p.labels)
            costs.append(probe.stats()["resident_bytes"] - before)
    budget = base + costs[0] + max(costs[1], costs[2]) + 4096
    reqs = serving_trace(specs(allv), 36, 1000.0, seed=21, sizes=(48, 96))
    plain = plain_images(allv, reqs)
    with srvmod.Server(hbm_budget_bytes=budget, max_slots=3, max_pending=64, max_pixels=128 * 128, max_labels=8,
                       evict_idle=True) as srv:
        vids = [srv.add_volume(p.volume, p.labels) for p in allv]
        st = srv.stats()
        assert st["volumes"] == 3 and st["evictions"] >= 1 and st["resident_bytes"] <= budget
        for rnd in range(2):
            tickets = [srvmod.submit_request(srv, vids[r.volume], r) for r in reqs]
            for i, t in enumerate(tickets):
                img, _ = srv.wait(t)
                assert np.array_equal(img, plain[i]), f"round {rnd} request {i} (volume {reqs[i].volume}) differs"
                assert srv.stats()["resident_bytes"] <= budget
        st = srv.stats()
        print(f"evictions {st['evictions']}, loads {st['loads']}, resident {st['resident_bytes']} of {budget}")
        assert st["loads"] >= 1 and st["evictions"] >= 2
        # an evicted volume can be removed; one larger than the budget is refused
        for v in vids:
            srv.remove_volume(v)
        assert srv.stats()["volumes"] == 0 and srv.stats()["resident_bytes"] == base
        big = make_phantom((256, 256, 200), (1.0, 1.0, 1.0), 34)
        with pytest.raises(capi.MonkeyGLError) as e:
            srv.add_volume(big.volume)
        assert e.value.status == capi.MK_ERR_BUDGET


def test_encoded_output_decodes_to_the_image(vols):
    """Requests that ask for MonkeyGL's *_pngString form (a Base64 PNG; a
    plane as W/2 RGBA pixels) get it written by the server's encoder thread:
    alone and mixed, it decodes to the request's own image, which equals the
    plain path's."""
    import sys
    sys.path.insert(0, str(__import__("pathlib").Path(__file__).parent))
    from pngcheck import decode_png_base64
    reqs = serving_trace(specs(vols), 24, 1000.0, seed=13, sizes=(64, 96, 128))
    plain = plain_images(vols, reqs)
    with srvmod.Server(max_slots=4, max_pending=64, max_pixels=128 * 128, max_labels=8, tiles_per_step=40) as srv:
        vids = [srv.add_volume(p.volume, p.labels) for p in vols]
        for rnd in range(2):
            if rnd == 0:
                got = [srv.wait(srvmod.submit_request(srv, vids[r.volume], r, encode=True)) for r in reqs]
            else:
                tickets = [srvmod.submit_request(srv, vids[r.volume], r, encode=(i % 2 == 0))
                           for i, r in enumerate(reqs)]
                got = [srv.wait(t) for t in tickets]
            for i, ((img, tm), r) in enumerate(zip(got, reqs)):
                assert np.array_equal(img, plain[i]), f"round {rnd} request {i}"
                if "png_base64" not in tm:
                    assert rnd == 1 and i % 2 == 1
                    continue
                dec = decode_png_base64(tm["png_base64"])
                if r.kind == capi.REQUEST_MPR:
                    dec = dec.reshape(r.size, -1).view(np.int16)
                assert np.array_equal(dec, img), f"round {rnd} request {i}: the encoded form differs"
