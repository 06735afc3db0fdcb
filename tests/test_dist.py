"""The multi-rank plumbing of bench.py on CPU: two gloo ranks, the max-over-ranks timing and the
whole-job rate of replicas (each rank advances its own box; no data-path collective)."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist

    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        my_ms = 10.0 + 5.0 * rank                    # rank 1 is the slow one
        slowest = bench.max_over_ranks_of(my_ms, dist, torch.device("cpu"))
        out[rank] = (slowest, bench.whole_job_mlups(1_000_000, world, slowest))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_time_by_the_slowest_rank():
    import torch.multiprocessing as mp
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0] == res[1]
    slowest, mlups = res[0]
    assert slowest == pytest.approx(15.0)
    assert mlups == pytest.approx(2 * 1_000_000 / 0.015 / 1e6)
