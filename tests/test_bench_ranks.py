"""The multi-rank timing of bench.py (replicas, one per GPU): the job time
is the maximum over ranks, taken on the process group (gloo here, two
ranks on the CPU), and every rank gets it."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, values, out):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        out.put((rank, bench.max_over_ranks(values[rank])))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_with_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    values = [12.5, 47.25]
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, values, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = dict(q.get() for _ in range(2))
    assert got == {0: 47.25, 1: 47.25}


def test_max_over_ranks_without_a_group():
    import bench
    assert bench.max_over_ranks(3.5) == 3.5
