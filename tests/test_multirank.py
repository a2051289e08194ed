"""The N-GPU form of bench.py on CPU: two gloo ranks (the replicas of a
multi-GPU run) agree on the slowest rank's step time and on the whole-job
throughput.  No GPU involved."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, times, out):
    import sys
    sys.path.insert(0, ROOT)
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        ms = bench.max_over_ranks(times[rank], world, "cpu")
        out[rank] = (ms, bench.replica_throughput(320_000_064, world, ms))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("times", [(20.0, 25.0), (31.5, 30.0)])
def test_replicas_take_the_slowest_rank(times):
    world = 2
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()  # both ranks rendezvous on one port
        procs = [ctx.Process(target=_rank, args=(r, world, port, times, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    slow = max(times)
    for r in range(world):
        ms, value = res[r]
        assert ms == slow
        assert value == pytest.approx(2 * 320_000_064 / (slow / 1e3) / 1e9)


def test_single_rank_needs_no_process_group():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(12.5, 1, "cpu") == 12.5
    assert bench.replica_throughput(1_000_000_000, 1, 1000.0) == pytest.approx(1.0)
