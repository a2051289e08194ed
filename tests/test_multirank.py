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


# ---- the sharded count: two ranks, each with its share of the Bloom words and
# of the k-mers, against the single-rank oracle --------------------------------
def _shard_rank(rank, world, port, k, bits, out):
    import sys
    sys.path[:0] = [ROOT, os.path.join(ROOT, "spades-rs_b200"), os.path.join(ROOT, "tests")]
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from helpers import synth_small_packed
        from oracle import ora
        from spk import shard
        data, offs, lens = synth_small_packed()
        num_words = max((bits + 63) // 64, 1)
        K, Cn, seen, twice = shard.count_sharded(
            lambda r, w: ora.shard_bloom(data, offs, lens, k, bits, r, w),
            lambda tw, r, w: ora.shard_count(data, offs, lens, k, bits, tw, r, w),
            num_words)
        out[rank] = (K.tobytes(), Cn.tobytes(), seen.tobytes(), twice.tobytes(), K.shape)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("k,bits", [(31, 1 << 16), (55, 100_003)])
def test_sharded_count_equals_single_rank(world, k, bits):
    """Each rank applies the Bloom inserts that fall in its word range and
    counts the k-mers its hash range owns; the gathered tiers and the merged
    table equal the single-rank twice-tier oracle, bit for bit."""
    import sys
    import numpy as np
    sys.path[:0] = [os.path.join(ROOT, "tests")]
    from helpers import synth_small_packed
    from oracle import ora
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_shard_rank, args=(r, world, port, k, bits, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(300)
            assert p.exitcode == 0
        res = dict(out)
    data, offs, lens = synth_small_packed()
    ref = ora.count(data, offs, lens, k, bits, mode=ora.MODE_TWICE)
    tk, tc = ref.table(1)
    oseen, otwice = ref.bloom()
    for r in range(world):
        kb, cb, sb, twb, shape = res[r]
        np.testing.assert_array_equal(np.frombuffer(kb, np.uint64).reshape(shape), tk)
        np.testing.assert_array_equal(np.frombuffer(cb, np.uint32), tc)
        np.testing.assert_array_equal(np.frombuffer(sb, np.uint64), oseen)
        np.testing.assert_array_equal(np.frombuffer(twb, np.uint64), otwice)


def test_owner_matches_the_oracle_partition(ora):
    """The host's owner() is floor(h * G / 2^64), the partition the oracle's
    rank shares use: every k-mer lands in exactly one rank's table."""
    import sys
    import numpy as np
    sys.path[:0] = [os.path.join(ROOT, "spades-rs_b200")]
    from spk import shard
    rng = np.random.default_rng(1)
    h = rng.integers(0, 2 ** 63, 100_000, dtype=np.int64).astype(np.uint64) * np.uint64(2) + np.uint64(1)
    for world in (1, 2, 3, 8, 7):
        o = shard.owner(h, world)
        want = np.array([(int(x) * world) >> 64 for x in h], dtype=np.int32)
        np.testing.assert_array_equal(o, want)
        assert o.min() >= 0 and o.max() < world
