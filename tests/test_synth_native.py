"""The native synthetic-read generator (spades-rs_b200/spk/synth_native.cpp)
that makes the batched and serving workloads: the same bytes whatever the
thread count, the PackedReads layout (src/packed_reads.rs:42-59, 547-578:
mates 1, then mates 2, each read on a byte boundary), genome GC share, and
reads that match the genome at the stated substitution rate."""
import numpy as np

from spk import synth


def decode(p, i):
    o, n = int(p.offsets[i]), int(p.lengths[i])
    by = p.data[o:o + (n + 3) // 4]
    return np.stack([(by >> 6) & 3, (by >> 4) & 3, (by >> 2) & 3, by & 3], 1).reshape(-1)[:n]


def test_threads_do_not_change_the_bytes(monkeypatch):
    a = synth.native_sample(200_000, 30, seed=3, stream=5, gc=0.4)
    monkeypatch.setattr(synth, "_threads", lambda: 3)
    b = synth.native_sample(200_000, 30, seed=3, stream=5, gc=0.4)
    np.testing.assert_array_equal(a.packed.data, b.packed.data)
    np.testing.assert_array_equal(a.packed.offsets, b.packed.offsets)
    c = synth.native_sample(200_000, 30, seed=3, stream=6, gc=0.4)
    assert not np.array_equal(a.packed.data, c.packed.data)


def test_layout_gc_and_error_rate():
    gc, err = 0.65, 0.01
    g = synth.native_genome(300_000, gc, 3, 10)
    assert abs(float(np.isin(g, (1, 2)).mean()) - gc) < 0.01
    p = synth.native_pairs([g], [5000], 3, 11, err=err)
    n = 10_000
    assert len(p) == n and p.pe_count == 5000
    np.testing.assert_array_equal(p.lengths, np.full(n, 150, np.uint32))
    np.testing.assert_array_equal(p.offsets, np.arange(n, dtype=np.uint64) * 38)
    assert p.data.size == n * 38
    gs = "".join("ACGT"[c] for c in g)
    rc = gs[::-1].translate(str.maketrans("ACGT", "TGCA"))
    mism, bases = 0, 0
    for i in range(0, 5000, 50):
        for r in (decode(p, i), decode(p, 5000 + i)):
            s = "".join("ACGT"[c] for c in r)
            best = 151
            for ref in (gs, rc):
                # the read's true place: the best of its 20-base seeds
                for o in range(0, 131, 10):
                    j = ref.find(s[o:o + 20])
                    while j >= 0 and best:
                        st = j - o
                        if 0 <= st and st + 150 <= len(ref):
                            best = min(best, sum(a != b for a, b in zip(s, ref[st:st + 150])))
                        j = ref.find(s[o:o + 20], j + 1)
            assert best < 151
            mism += best
            bases += 150
    assert abs(mism / bases - err) < 0.004
