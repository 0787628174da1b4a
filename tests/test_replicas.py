"""bench.py's multi-GPU host logic on two gloo ranks on the CPU.

The path shards as replicas (each rank holds the volume and renders its own
views; there is no data-path exchange), so what N > 1 adds is host logic: the
process group, the barrier around the timed region, the max over ranks of the
device time and the sum of work, the per-rank view order, and the reference
arm, which only rank 0 runs.  NCCL on GPUs runs the same code."""
import argparse
import multiprocessing as mp
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE="2",
                      LOCAL_RANK=str(rank))
    import bench
    import torch.distributed as dist
    try:
        r, local, world = bench.dist_setup(2, backend="gloo")
        bench.barrier(world)
        mx = bench.max_over_ranks(1.5 + r, world)
        sm = bench.sum_over_ranks(1.5 + r, world)
        views = bench.rank_views([10.0 * i for i in range(36)], r)
        args = argparse.Namespace(workload="small", bg=0.4, size=64, steps=3, warmup=3)
        ref = bench.run_reference(args, r, world) if r != 0 else "rank 0 runs the reference"
        bench.barrier(world)
        q.put((r, world, mx, sm, views, ref))
    finally:
        if dist.is_initialized():
            dist.destroy_process_group()


def test_two_rank_replica_logic():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = {}
    for _ in procs:
        r, world, mx, sm, views, ref = q.get(timeout=180)
        results[r] = (world, mx, sm, views, ref)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert set(results) == {0, 1}
    for r, (world, mx, sm, views, ref) in results.items():
        assert world == 2
        assert mx == 2.5 and sm == 4.0               # max and sum over the two ranks
        assert sorted(views) == [10.0 * i for i in range(36)]   # every rank renders every view
    assert results[0][3][0] == 0.0 and results[1][3][0] == 70.0  # ... starting at different views
    assert results[1][4] is None                      # only rank 0 runs the reference arm


def test_single_rank_needs_no_process_group(monkeypatch):
    import bench
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    rank, local, world = bench.dist_setup(1, backend="gloo")
    assert (rank, local, world) == (0, 0, 1)
    assert bench.max_over_ranks(3.0, world) == 3.0 and bench.sum_over_ranks(3.0, world) == 3.0
