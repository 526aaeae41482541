"""The multi-GPU mode of bench.py is replicas only: each rank advances its own
mesh, and the only collective is the all_reduce(MAX) of the elapsed time that
makes the whole-job figure.  This runs that aggregation on two gloo ranks on
the CPU (127.0.0.1) with different per-rank times."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    local = 100.0 + 37.5 * rank
    ms = bench.max_over_ranks(local, "cpu")
    out[rank] = (ms, bench.replicas_value(1000, 10, world, ms))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_replicas_take_the_slowest_rank():
    world, port = 2, _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    slowest = 100.0 + 37.5 * (world - 1)
    for r in range(world):
        ms, value = res[r]
        assert ms == slowest
        assert value == pytest.approx(1000 * 10 * world / (slowest / 1e3))
