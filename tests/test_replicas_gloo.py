"""The N > 1 path of bench.py on CPU: two gloo ranks (the GPU path is replicas only, one process
per GPU, no data-path collective).  Each rank reports its own device time; the job's time is the
maximum over ranks, and the whole-job rate is N x cells x steps / that time."""
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
    import sys

    import torch.distributed as dist

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = [1.0 + rank, 5.0 - rank]  # rank 0 slower end to end, rank 1 slower on the device
        out[rank] = bench.max_over_ranks(mine, "cpu")
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert out[0] == [2.0, 5.0] and out[1] == [2.0, 5.0]


def test_whole_job_rate():
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    assert bench.whole_job_rate(2, 393216, 5, 2.0) == pytest.approx(2 * 393216 * 5 / 2.0)
