"""Replica throughput over ranks with the gloo backend on the CPU: each rank
reports its own time; the job rate uses the slowest rank."""
import os

import pytest
import torch.multiprocessing as mp


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from datetime import timedelta
    from imex_sflow2d_v2_b200.replicas import job_rate
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    rate, slowest = job_rate(1.0 + rank, 100.0, dist, "cpu")   # rank r took 1 + r seconds
    out[rank] = (rate, slowest)
    dist.barrier()
    dist.destroy_process_group()


def test_job_rate_uses_slowest_rank():
    world = 2
    port = 29500 + os.getpid() % 1000
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for rank in range(world):
        rate, slowest = res[rank]
        assert slowest == 2.0
        assert rate == pytest.approx(world * 100.0 / 2.0)


def test_single_process_rate():
    from imex_sflow2d_v2_b200.replicas import job_rate
    assert job_rate(2.0, 10.0) == (5.0, 2.0)
