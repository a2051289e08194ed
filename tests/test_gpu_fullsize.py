"""GPU parity at the full sizes of the benchmark configurations, and the
reference's own end-to-end fixture.

* The plain single-sample configuration in full: a 1 Mb genome read at 30x
  (100k pairs of 2x150, 0.5% substitutions, 0.01% N), canonical k = 21 (the
  one-limb key path), Bloom tiers of 512 Mi bits.  Every schedule's whole
  admitted table, both Bloom tiers, the cutoff and the edge list are compared
  bit for bit with the oracle's twice-tier count (src/assemble.rs:129-242,
  286-292, 692-735; src/graph.rs:78-102).  The oracle runs threaded here; its
  twice tier is order-free, so the threaded result is the serial one
  (pinned by tests/test_oracle_golden.py).
* The reference's integration test (tests/test_pipeline.rs:33-91): the
  E. coli 1K read pairs at k = 31 with a 16 Mi-bit Bloom and error
  correction assemble to data/reference_1K.fa.gz.  Counting, correction and
  unitig compaction run on the GPU here; the reference's tip clipping
  (src/simplify.rs) is outside the counting path, so the test asserts that
  the unitigs spell the reference contig as one path and that every other
  unitig is a short tip hanging off that path.
"""
import os

import numpy as np
import pytest

from helpers import ecoli_packed, revcomp, spelled_path

pytestmark = pytest.mark.gpu

EDGES, KEEP_BLOOM, GATED, DIRECT, CORRECT = 0x1, 0x4, 0x8, 0x10, 0x20


@pytest.fixture(scope="module")
def spk(spk_lib):
    return spk_lib


@pytest.fixture(scope="module")
def c1():
    from spk import synth
    return synth.c1(1.0).packed


def test_c1_full_size(spk, ora, c1):
    p = c1
    k, bits = 21, 512 << 20
    threads = os.cpu_count() or 1
    o = ora.count(p.data, p.offsets, p.lengths, k, bits, mode=ora.MODE_TWICE, threads=threads)
    tk, tc = o.table(1)
    oseen, otwice = o.bloom()
    assert o.stats()["occurrences"] == 25_944_828
    assert tk.shape[0] > 1_000_000
    solid_cut = ora.cutoff(tc, 5.0)
    want_edges = ora.edges(tk[tc >= solid_cut], k)
    for flags in (EDGES | KEEP_BLOOM, EDGES | KEEP_BLOOM | GATED, EDGES | KEEP_BLOOM | DIRECT):
        r = spk.count(p, [k], bloom_bits=bits, list_min_count=1, flags=flags)
        info = r.info(0)
        gk, gc = r.kmers(0, 1)
        np.testing.assert_array_equal(gk, tk)
        np.testing.assert_array_equal(gc, tc)
        seen, twice = r.bloom(0)
        np.testing.assert_array_equal(seen, oseen)
        np.testing.assert_array_equal(twice, otwice)
        assert info["occurrences"] == 25_944_828
        assert info["cutoff"] == solid_cut
        assert info["n_singletons"] == int((tc == 1).sum())
        assert info["admitted_occurrences"] == int(tc.astype(np.int64).sum())
        np.testing.assert_array_equal(r.edges(0), want_edges)
        r.close()


def test_ecoli_1k_pipeline_spells_reference(spk):
    data, offs, lens, d = ecoli_packed()
    ref = str(d["reference_1K"][0])
    k = 31
    r = spk.count((data, offs, lens), [k], bloom_bits=16 * 1024 * 1024, min_coverage=5.0,
                  flags=EDGES | CORRECT)
    seqs, cov, nk = r.unitigs(0)
    path = spelled_path(seqs, ref, k)
    assert path is not None, [len(s) for s in seqs]
    # every unitig off the path is a tip: shorter than 2k, one end on a
    # branch point of the path
    on_path = {ref[a:b] for a, b in path}
    for s in seqs:
        if s in on_path or revcomp(s) in on_path:
            continue
        assert len(s) < 2 * k, len(s)
        ends = {s[:k - 1], s[-(k - 1):], revcomp(s)[:k - 1], revcomp(s)[-(k - 1):]}
        assert any(e in ref for e in ends)
    # consecutive unitigs share k - 1 bases and no k-mer: the path holds each
    # of the reference's k-mers once
    assert sum(b - a - k + 1 for a, b in path) == len(ref) - k + 1
