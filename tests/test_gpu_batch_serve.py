"""Batched counting (spk_count_batch), concurrent multi-k counting and the
serving loop (spk_submit / spk_wait), through the C ABI.

Every job of a batch or of the serving mix must give exactly what spk_count
gives on that job alone: the samples share nothing but the device.  Integer
results, compared bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def spk(spk_lib):
    return spk_lib


@pytest.fixture(scope="module")
def samples():
    """Six read sets of uneven size (genome 20-200 kb, 20-120x, GC 0.35-0.65)."""
    from spk import synth
    plan = [(20_000, 120, 0.5), (200_000, 30, 0.35), (60_000, 80, 0.65), (5_000, 20, 0.5),
            (150_000, 60, 0.45), (90_000, 100, 0.55)]
    return [synth.sample(g, c, seed=7, stream=i, gc=gc, err=(0.005, 0.005)).packed
            for i, (g, c, gc) in enumerate(plan)]


def same_result(a, b, k_count):
    """Two CountResults hold the same lists, edges, tiers and statistics."""
    for ki in range(k_count):
        ia, ib = a.info(ki), b.info(ki)
        for key in ("k", "cutoff", "occurrences", "admitted_occurrences", "n_table", "n_list",
                    "n_solid", "n_edges", "n_singletons", "seen_popcount", "twice_popcount",
                    "n_distinct"):
            assert ia[key] == ib[key], (ki, key)
        ka, ca = a.kmers(ki, 1)
        kb, cb = b.kmers(ki, 1)
        np.testing.assert_array_equal(ka, kb)
        np.testing.assert_array_equal(ca, cb)
        np.testing.assert_array_equal(a.edges(ki), b.edges(ki))
        sa, ta = a.bloom(ki)
        sb, tb = b.bloom(ki)
        np.testing.assert_array_equal(sa, sb)
        np.testing.assert_array_equal(ta, tb)


OPTS = dict(bloom_bits=1 << 22, list_min_count=1)


def test_batch_equals_one_at_a_time(spk, samples):
    ks = [[33], [21, 55], [33], [55], [21], [33, 77]]
    jobs = [spk.Job(p, k, dict(OPTS)) for p, k in zip(samples, ks)]
    batch = spk.count_batch(jobs)
    assert len(batch) == len(jobs)
    for p, k, r in zip(samples, ks, batch):
        same_result(r, spk.count(p, k, **OPTS), len(k))
        r.close()


def test_batch_reports_the_failing_job(spk, samples):
    good = spk.Job(samples[0], [33], dict(OPTS))
    d, o, l = samples[3].data, samples[3].offsets.copy(), samples[3].lengths
    o[-1] = d.size + 100  # the last read points past the packed data
    bad = spk.Job((d, o, l), [33], dict(OPTS))
    with pytest.raises(spk.SpkError) as e:
        spk.count_batch([good, bad, good])
    assert e.value.code == 1 and "job 1" in str(e.value)


def test_empty_batch(spk):
    assert spk.count_batch([]) == []
    assert list(spk.count_batch_iter([])) == []


def test_streamed_batch_equals_one_at_a_time(spk, samples):
    """spk_batch_next hands the results out in job order as they finish; each
    is downloaded while the jobs after it still count, and equals count()
    on its sample alone."""
    ks = [[33], [55], [21, 33], [33], [55], [77]]
    jobs = [spk.Job(p, k, dict(OPTS)) for p, k in zip(samples, ks)]
    seen = []
    for i, r in spk.count_batch_iter(jobs):
        seen.append(i)
        same_result(r, spk.count(samples[i], ks[i], **OPTS), len(ks[i]))
        r.close()
    assert seen == list(range(len(jobs)))


def test_streamed_batch_goes_on_after_a_failed_job(spk, samples):
    """A job that fails raises at its turn; the results handed out before it
    stay valid, and the batch ends cleanly."""
    good = spk.Job(samples[0], [33], dict(OPTS))
    d, o, l = samples[3].data, samples[3].offsets.copy(), samples[3].lengths
    o[-1] = d.size + 100
    bad = spk.Job((d, o, l), [33], dict(OPTS))
    got = []
    with pytest.raises(spk.SpkError) as e:
        for i, r in spk.count_batch_iter([good, bad, good]):
            got.append((i, r))
    assert e.value.code == 1 and "job 1" in str(e.value)
    assert [i for i, _ in got] == [0]
    same_result(got[0][1], spk.count(samples[0], [33], **OPTS), 1)
    got[0][1].close()
    # the context takes a new batch afterwards
    r = spk.count_batch([good])[0]
    same_result(r, spk.count(samples[0], [33], **OPTS), 1)
    r.close()


def test_multik_concurrent_equals_single_k(spk, samples):
    """k values of one call count concurrently; each equals its own call."""
    p = samples[1]
    ks = [21, 33, 55, 77]
    multi = spk.count(p, ks, **OPTS)
    assert len(multi) == 4
    for i, k in enumerate(ks):
        single = spk.count(p, [k], **OPTS)
        a, b = multi.info(i), single.info(0)
        assert a["k"] == k
        ka, ca = multi.kmers(i, 1)
        kb, cb = single.kmers(0, 1)
        np.testing.assert_array_equal(ka, kb)
        np.testing.assert_array_equal(ca, cb)
        np.testing.assert_array_equal(multi.edges(i), single.edges(0))
        assert a["n_solid"] == b["n_solid"] and a["cutoff"] == b["cutoff"]


def test_serving_isolation(spk, samples):
    """Jobs submitted back to back run concurrently (up to 3 in flight) and
    each result equals the job counted alone."""
    srv = spk.Server(hbm_budget_bytes=0, max_inflight=3)
    try:
        ks = [[33], [55], [21, 33], [55], [33], [21]]
        tickets = [srv.submit(spk.Job(p, k, dict(OPTS))) for p, k in zip(samples, ks)]
        lat = []
        for t, p, k in zip(tickets, samples, ks):
            r, ms = srv.wait(t)
            assert ms >= 0
            lat.append(ms)
            same_result(r, spk.count(p, k, **OPTS), len(k))
            r.close()
        assert len(lat) == len(samples)
    finally:
        srv.stop()


def test_serving_admission_by_budget(spk, samples):
    """A job whose estimated HBM need exceeds the whole budget is refused; the
    others still run one at a time under a budget that fits one job."""
    one = spk.Server.estimate(spk.Job(samples[1], [33], dict(OPTS)))
    srv = spk.Server(hbm_budget_bytes=one + (1 << 20), max_inflight=4)
    try:
        big = spk.Job(samples[1], [21, 33, 55], dict(OPTS))
        assert spk.Server.estimate(big) > one + (1 << 20)
        tb = srv.submit(big)
        ts = [srv.submit(spk.Job(p, [33], dict(OPTS))) for p in samples[:3]]
        with pytest.raises(spk.SpkError) as e:
            srv.wait(tb)
        assert e.value.code == 8  # SPK_E_ADMISSION
        for t, p in zip(ts, samples[:3]):
            r, _ = srv.wait(t)
            same_result(r, spk.count(p, [33], **OPTS), 1)
            r.close()
    finally:
        srv.stop()
