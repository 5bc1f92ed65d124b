"""Replica timing over ranks (bench.py --gpus N under torchrun), world size 2 on
CPU with gloo: the job's time is the slowest rank's and the work is the sum."""
import os
import socket

import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    from nbodysim_b200.replicas import job_totals
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ms, units = job_totals(dist, "cpu", 10.0 + 5.0 * rank, 1e9 * (rank + 1))
    dist.barrier()
    out[rank] = (ms, units)
    dist.destroy_process_group()


def test_job_totals_two_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        for r in range(2):
            assert out[r] == (15.0, 3e9)


def test_job_totals_single_process():
    from nbodysim_b200.replicas import job_totals
    assert job_totals(None, "cpu", 3.0, 7.0) == (3.0, 7.0)
