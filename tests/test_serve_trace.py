"""The serving benchmark's eviction trace (monkeygl_b200/serve_bench.py):
phases over pairs of volumes drawn from the Poisson trace, in trace order,
with the trace's own arrival gaps.  CPU only."""
import numpy as np

from monkeygl_b200.serve_bench import eviction_trace
from monkeygl_b200.workloads import serving_trace

SPECS = [((64, 64, 64), (1, 1, 1), False), ((64, 64, 48), (1, 1, 1), False),
         ((64, 64, 40), (1, 1, 1), False), ((64, 64, 32), (1, 1, 1), True)]


def test_phases_use_their_pair_in_trace_order():
    trace = serving_trace(SPECS, 2000, 200.0, seed=5)
    pairs = [(0, 1), (1, 2), (2, 3), (3, 0)]
    et = eviction_trace(trace, 400, pairs)
    assert len(et) == 400
    for k, pair in enumerate(pairs):
        phase = et[k * 100:(k + 1) * 100]
        assert {r.volume for r in phase} <= set(pair), (k, {r.volume for r in phase})
    # every request is a request of the trace, none taken twice, in order within a phase
    ids = [next(i for i, r in enumerate(trace) if r is not None and r.size == q.size and r.kind == q.kind
                and r.volume == q.volume and (r.vr is q.vr) and (r.plane is q.plane)) for q in et]
    assert len(set(ids)) == len(ids)
    for k in range(4):
        seg = ids[k * 100:(k + 1) * 100]
        assert seg == sorted(seg)


def test_arrival_gaps_are_the_traces():
    trace = serving_trace(SPECS, 1000, 200.0, seed=9)
    et = eviction_trace(trace, 300, [(0, 1), (2, 3)])
    got = np.diff([0.0] + [r.arrival_s for r in et])
    want = np.diff([0.0] + [r.arrival_s for r in trace[:300]])
    assert np.allclose(got, want)
    assert all(b > a for a, b in zip([r.arrival_s for r in et], [r.arrival_s for r in et][1:]))
