"""The replica path of bench.py under torchrun, on CPU: two gloo ranks run the
same rank helpers the GPU job uses (barrier, max-over-ranks time, units summed
over ranks), with unequal work and times per rank."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(dist)
        units = 1000.0 * (rank + 1)   # rank 0: 1000 updates, rank 1: 2000
        secs = 0.5 + rank * 1.5       # rank 1 is the slowest: 2.0 s
        out[rank] = (bench.allreduce_max(dist, secs), bench.job_rate(dist, units, secs))
        bench.barrier(dist)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_aggregate_as_the_job():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(world):
        t_max, rate = out[r]
        assert t_max == 2.0
        assert rate == pytest.approx(3000.0 / 2.0)


def test_single_process_helpers_need_no_group():
    import bench
    assert bench.allreduce_max(None, 1.5) == 1.5
    assert bench.job_rate(None, 10.0, 2.0) == 5.0
