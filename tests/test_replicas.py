"""Multi-process (gloo, world size 2) check of the replica bookkeeping used by
bench.py --gpus N: job throughput = all ranks' updates / slowest rank's time."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from bgk3d_gpu_b200.replicas import job_throughput
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    updates = 1000.0 * (rank + 1)
    seconds = 2.0 if rank == 0 else 5.0
    out[rank] = job_throughput(updates, seconds)
    dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_job_throughput_two_ranks():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for r in range(2):
        total, tmax, rate = out[r]
        assert total == 3000.0 and tmax == 5.0 and rate == 600.0


def test_job_throughput_single_process():
    from bgk3d_gpu_b200.replicas import job_throughput
    assert job_throughput(10.0, 2.0) == (10.0, 2.0, 5.0)
