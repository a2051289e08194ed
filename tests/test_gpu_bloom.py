"""GPU TwoTierFilter (spk_bloom_*) against the reference's tests and the
serial oracle.  Batched calls must equal per-key calls in array order."""
import hashlib

import numpy as np
import pytest

from helpers import load_json

pytestmark = pytest.mark.gpu


def sha(words):
    return hashlib.sha256(np.asarray(words, dtype=np.uint64).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def spk(spk_lib):
    return spk_lib


def test_two_tier_filter(spk):  # src/bloom.rs:139-156
    f = spk.TwoTierFilter(1024 * 1024)
    k1, k2 = 123456789, 987654321
    assert not f.is_solid(k1)
    f.insert(k1)
    assert not f.is_solid(k1)
    f.insert(k1)
    assert f.is_solid(k1)
    assert not f.is_solid(k2)


def test_two_tier_bloom_transitions(spk):  # tests/test_hammer_and_bloom.rs:39-70
    f = spk.TwoTierFilter(1024 * 1024)
    a, b, c = 0x123456789ABCDEF0, 0xFEDCBA9876543210, 0xA5A5A5A5A5A5A5A5
    assert not f.is_solid(a) and not f.is_solid(b) and not f.is_solid(c)
    assert not f.insert(a) and not f.is_solid(a)
    assert f.insert(a) and f.is_solid(a)
    assert f.insert(a) and f.is_solid(a)
    assert not f.is_solid(b) and not f.is_solid(c)


def test_sizes(spk):  # src/bloom.rs:26-43, 129-131
    for cap, words in ((0, 1), (1, 1), (64, 1), (65, 2), (1 << 20, 1 << 14)):
        f = spk.TwoTierFilter(cap)
        assert f.size_bits == words * 64
        assert f.memory_usage_bytes() == words * 16


def test_serial_trace_batched(spk):
    """A 2000-insert trace with repeats, submitted as one batch, returns the
    serial promotions and leaves the serial tiers (golden fixture)."""
    rec = load_json("bloom_vectors.json")["serial"]
    f = spk.TwoTierFilter(rec["capacity_bits"])
    keys = np.array([int(v) for v in rec["inserts"]], dtype=np.uint64)
    got = f.insert_batch(keys)
    assert got.tolist() == rec["promoted"]
    q = np.array([int(v) for v in rec["queries"]], dtype=np.uint64)
    assert f.is_solid_batch(q).tolist() == rec["solid"]
    seen, solid = f.download()
    assert sha(seen) == rec["seen_sha"] and sha(solid) == rec["solid_sha"]


@pytest.mark.parametrize("cap", [64, 100, 4096, 999_999_937])
def test_batched_k256_vs_serial_oracle(spk, ora, cap):
    """Random wide keys with many duplicates, in several batches, vs per-key oracle calls."""
    rng = np.random.default_rng(cap)
    pool = rng.integers(0, 2 ** 63, size=(500, 4), dtype=np.uint64)
    f = spk.TwoTierFilter(cap)
    o = ora.Bloom(cap)
    for _ in range(3):
        batch = pool[rng.integers(0, 500, size=3000)]
        got = f.insert_kmer256_batch(batch)
        exp = [o.insert_kmer256(ora.from_limbs(r)) for r in batch]
        assert got.tolist() == exp
        qs = pool[rng.integers(0, 500, size=700)]
        assert f.is_solid_kmer256_batch(qs).tolist() == [o.is_solid_kmer256(ora.from_limbs(r)) for r in qs]
    s1, t1 = f.download()
    s2, t2 = o.download()
    np.testing.assert_array_equal(s1, s2)
    np.testing.assert_array_equal(t1, t2)


def test_empty_batches(spk):
    f = spk.TwoTierFilter(1 << 16)
    assert f.insert_batch(np.zeros(0, np.uint64)).size == 0
    assert f.is_solid_batch(np.zeros(0, np.uint64)).size == 0
