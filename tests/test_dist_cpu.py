"""Multi-process plumbing of the replica benchmarks on CPU (gloo, world size
2): every rank reaches the same collectives in the same order, the job time
is the max over ranks, and ranks run different seeded streams (replicas,
no data-path collective).  The GPU runs use the same helpers over NCCL."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _child(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        tmax = bench.dist_max(dist, 1.5 + rank)          # rank r "took" 1.5 + r seconds
        bench.dist_barrier(dist)
        data = bench.make_stream(1 + 7919 * rank, 3)      # the stream bench's per-rank seed
        out.put((rank, tmax, float(np.sum(data["vals"])), int(data["offs"][-1])))
    finally:
        dist.destroy_process_group()


def test_replicas_two_ranks_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_child, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get() for _ in range(2))
    assert [r[1] for r in res] == [2.5, 2.5]              # max over ranks on every rank
    assert res[0][2] != res[1][2]                          # different streams per rank
    assert res[0][3] > 0 and res[1][3] > 0


def _child_reference(rank, world, port, out):
    import argparse
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        import bench
        # a small stream of the same generator, so the CPU reference is quick
        bench.C2.update(I=300, J=200, T=8, total_nnz=4000, median=500, rank=8)
        os.cpu_count = lambda: 2                      # OpenMP threads of the reference run
        args = argparse.Namespace(warmup=3, steps=2, cpu_slices=4, seed=5)
        line = bench.bench_reference(args, world, rank)
        bench.dist_barrier(dist)
        out.put((rank, line))
    finally:
        dist.destroy_process_group()


def test_reference_arm_two_ranks_gloo():
    """`bench.py --impl reference` under two ranks: rank 0 alone runs the
    reference's CPU stream and returns the line (the requested steps after
    at least 3 warm-up slices); the other rank does no work and returns
    nothing; both pass the closing barrier."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_child_reference, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = dict(q.get() for _ in range(2))
    assert res[1] is None
    line = res[0]
    assert line["impl"] == "reference" and line["steps"] == 2 and line["warmup"] == 3
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"]
    assert line["cpu_baseline"]["kind"] in ("reference", "port")
