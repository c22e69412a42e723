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
