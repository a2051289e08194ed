"""GPU unitigs (spk_result_unitigs, through the C ABI) against the oracle's
restatement of CompactedGraph::build (src/graph.rs:65-235), on the solid list
the GPU counted (that list is itself checked against the oracle elsewhere).
Sequences, k-mer counts and mean coverages compared exactly."""
import numpy as np
import pytest

from helpers import graph_sequences, reads_from, synth_small_packed
from oracle import pyref

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def spk(spk_lib):
    return spk_lib


def check(r, ora, k, ki=0, min_unitigs=1):
    keys, counts = r.solid(ki)
    want = ora.unitigs(keys, counts, k)
    got = r.unitigs(ki)
    assert got[0] == want[0]
    np.testing.assert_array_equal(got[2], want[2])
    np.testing.assert_array_equal(got[1], want[1])
    assert int(got[2].sum()) == keys.shape[0]
    assert len(got[0]) >= min_unitigs
    return got


@pytest.mark.parametrize("k", [21, 33, 55, 77, 127])
def test_graph_shapes(spk, ora, k):
    """Repeats, a tip, a bubble, an isolated circle, a hairpin and a short
    piece, read at 30x without errors."""
    rng = np.random.default_rng(k)
    seqs, circle = graph_sequences(rng, k)
    reads = reads_from(seqs, circle, rng)
    data, offs, lens = pyref.pack_reads(reads)
    p = (np.frombuffer(data, dtype=np.uint8), np.array(offs, dtype=np.uint64),
         np.array(lens, dtype=np.uint32))
    r = spk.count(p, [k], bloom_bits=1 << 22, min_count=2)
    check(r, ora, k, min_unitigs=6)


@pytest.mark.parametrize("k", [31, 55])
def test_small_sample(spk, ora, k):
    data, offs, lens = synth_small_packed()
    r = spk.count((data, offs, lens), [k], bloom_bits=1 << 22)
    check(r, ora, k)


def test_sample_with_errors_and_repeats(spk, ora):
    """200 kb genome at 40x with 0.5% substitutions and repeats: many tips and
    bubbles; two k values of one call."""
    from spk import synth
    p = synth.sample(200_000, 40, seed=11, repeats=10, err=(0.005, 0.005)).packed
    ks = [55, 77]
    r = spk.count(p, ks, bloom_bits=1 << 24)
    for ki, k in enumerate(ks):
        got = check(r, ora, k, ki, min_unitigs=50)
        again = r.unitigs(ki)  # cached
        assert again[0] == got[0]


def test_even_k_is_refused(spk):
    data, offs, lens = synth_small_packed()
    r = spk.count((data, offs, lens), [32], bloom_bits=1 << 22)
    with pytest.raises(spk.SpkError) as e:
        r.unitigs(0)
    assert e.value.code == 1


def test_no_solid_kmers(spk):
    reads = ["ACGT" * 10]  # shorter than k: no k-mer at all
    data, offs, lens = pyref.pack_reads(reads)
    p = (np.frombuffer(data, dtype=np.uint8), np.array(offs, dtype=np.uint64),
         np.array(lens, dtype=np.uint32))
    r = spk.count(p, [55], bloom_bits=1 << 20)
    seqs, cov, kmers = r.unitigs(0)
    assert seqs == [] and cov.size == 0 and kmers.size == 0
