"""The N>1 path of bench.py on CPU: two gloo ranks, each timing its own
domain; the reported time is the max over ranks and the value counts every
rank's sites (weak scaling).  No GPU, no NCCL."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    ms = bench.max_over_ranks(10.0 + 5.0 * rank, dist, "cpu")
    val = bench.job_mlups(1_000_000, world, 4, ms)
    out[rank] = (ms, val)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_max_and_weak_scaling_value():
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert out[0][0] == out[1][0] == 15.0
    assert out[0][1] == pytest.approx(1_000_000 * 2 * 4 / 15e-3 / 1e6)


def test_single_process_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5) == 3.5
    assert bench.job_mlups(100, 1, 10, 1000.0) == pytest.approx(1e-3)
