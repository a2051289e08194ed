"""Unitigs of the solid k-mers (CompactedGraph::build, src/graph.rs:65-235):
the C++ oracle against known answers and against the independent Python
restatement (oracle/pyref.py), on graphs with repeats, tips, bubbles,
cycles and hairpins.  No GPU involved.

The reference ships no test of its own for this function, so the known
answers are the ones its definition fixes: a sequence with no repeated
(k-1)-mer is one unitig, and a circle is one unitig cut at its smallest
k-mer read forward (pass 2 walks the solid list in sorted order)."""
import numpy as np
import pytest

from helpers import graph_sequences, key_rows, rand_seq, revcomp, solid_from_sequences
from oracle import pyref


def canon(s):
    return min(s, revcomp(s))


@pytest.mark.parametrize("k", [21, 33, 77])
def test_linear_sequence_is_one_unitig(ora, k):
    rng = np.random.default_rng(k)
    g = rand_seq(rng, 1200)
    km1 = [canon(g[i:i + k - 1]) for i in range(len(g) - k + 2)]
    assert len(set(km1)) == len(km1)  # no repeated (k-1)-mer, no branch
    strs, counts = solid_from_sequences([g], k, rng)
    seqs, cov, kmers = ora.unitigs(key_rows(strs, k), counts, k)
    assert seqs == [canon(g)]
    assert kmers.tolist() == [len(g) - k + 1]
    assert cov[0] == float(counts.astype(np.float64).sum()) / (len(g) - k + 1)


@pytest.mark.parametrize("k", [21, 55])
def test_circle_is_cut_at_its_smallest_kmer(ora, k):
    rng = np.random.default_rng(100 + k)
    c = rand_seq(rng, 500)
    strs, counts = solid_from_sequences([c + c[:k - 1]], k, rng)
    assert len(strs) == len(c)
    m = strs[0]  # the smallest k-mer; the walk starts at it, forward
    for s in (c, revcomp(c)):
        p = (s + s).find(m)
        if 0 <= p < len(s):
            want = (s + s + s)[p:p + len(c) + k - 1]
            break
    seqs, cov, kmers = ora.unitigs(key_rows(strs, k), counts, k)
    assert seqs == [canon(want)]
    assert kmers.tolist() == [len(c)]


@pytest.mark.parametrize("k", [21, 31, 55, 77, 127])
@pytest.mark.parametrize("seed", [1, 2])
def test_oracle_matches_python_restatement(ora, k, seed):
    rng = np.random.default_rng(seed * 1000 + k)
    seqs_in, _ = graph_sequences(rng, k)
    strs, counts = solid_from_sequences(seqs_in, k, rng)
    a_seq, a_cov, a_km = ora.unitigs(key_rows(strs, k), counts, k)
    b_seq, b_cov, b_km = pyref.unitigs(strs, counts, k)
    assert a_seq == b_seq
    assert a_km.tolist() == b_km
    assert a_cov.tolist() == b_cov
    assert len(a_seq) > 5  # the graph really branches


@pytest.mark.parametrize("k", [21, 55])
def test_unitigs_partition_the_solid_kmers(ora, k):
    """Every solid k-mer lies in exactly one unitig, and consecutive k-mers of
    a unitig are solid (src/graph.rs:104-157 marks each k-mer visited once)."""
    rng = np.random.default_rng(7 + k)
    seqs_in, _ = graph_sequences(rng, k)
    strs, counts = solid_from_sequences(seqs_in, k, rng)
    seqs, _, kmers = ora.unitigs(key_rows(strs, k), counts, k)
    seen = []
    for s, n in zip(seqs, kmers):
        assert len(s) == n + k - 1
        seen += [canon(s[i:i + k]) for i in range(len(s) - k + 1)]
    assert sorted(seen) == strs


def test_empty_and_single(ora):
    k = 21
    seqs, cov, kmers = ora.unitigs(np.zeros((0, 1), dtype=np.uint64), np.zeros(0, dtype=np.uint32), k)
    assert seqs == [] and cov.size == 0 and kmers.size == 0
    s = canon("ACGTTGCAACGGTACCATGAA")
    seqs, cov, kmers = ora.unitigs(key_rows([s], k), np.array([9], dtype=np.uint32), k)
    assert seqs == [s] and cov.tolist() == [9.0] and kmers.tolist() == [1]
