"""Read error correction (ErrorCorrector::correct_read_in_place,
src/hammer.rs:34-121) in the oracle: the reference's own tests
(src/hammer.rs:160-193), and the C++ restatement against the independent
Python one (oracle/pyref.py) on reads with 0-4 substitutions against a dense
and a nearly saturated filter.  No GPU involved."""
import numpy as np
import pytest

from helpers import correction_case
from oracle import pyref


def oracle_filter(ora, bits, keys):
    b = ora.Bloom(bits)
    for row in keys:
        b.insert_kmer256((int(row[0]) | (int(row[1]) << 64), int(row[2]) | (int(row[3]) << 64)))
    return b


def test_reference_single_substitution(ora):
    """src/hammer.rs:160-185: k=5, a 1 Mi-bit filter holding ACGTACGTACGT's
    k-mers twice; ACGGACGTACGT is corrected back."""
    k = 5
    ref = "ACGTACGTACGT"
    b = ora.Bloom(1024 * 1024)
    for _ in range(2):
        for i in range(len(ref) - k + 1):
            b.insert_kmer256(pyref.k256_canonical(pyref.k256_from_str(ref[i:i + k], k), k)[0])
    assert b.correct_read(k, "ACGGACGTACGT") == (ref, True)


def test_reference_short_read_bypass(ora):
    """src/hammer.rs:187-193."""
    b = ora.Bloom(1024)
    assert b.correct_read(15, "ACGT") == ("ACGT", False)


@pytest.mark.parametrize("k,bits", [(11, 1 << 20), (21, 1 << 20), (21, 1 << 13), (33, 1 << 16)])
def test_oracle_matches_python_restatement(ora, k, bits):
    keys, reads = correction_case(k, seed=k + bits, genome_len=1500, n_reads=30)
    b = oracle_filter(ora, bits, keys)
    pf = pyref.TwoTierFilter(bits)
    for row in keys:
        pf.insert_kmer256((int(row[0]) | (int(row[1]) << 64), int(row[2]) | (int(row[3]) << 64)))
    n_changed = 0
    for r in reads:
        a = b.correct_read(k, r)
        p = pyref.correct_read(r, k, pf)
        assert a == p, r
        n_changed += a[1]
    assert n_changed > 5


def test_packed_form_equals_per_read(ora):
    """The Stage 3 form (every packed read decoded, corrected, written back)
    equals correcting each read on its own."""
    k = 21
    keys, reads = correction_case(k, seed=5, n_reads=40)
    b = oracle_filter(ora, 1 << 20, keys)
    data, offs, lens = pyref.pack_reads(reads)
    out, flags, nc = b.correct_packed(k, np.frombuffer(data, np.uint8), offs, lens)
    for i, r in enumerate(reads):
        want, m = b.correct_read(k, r) if len(r) >= k else (r, False)
        assert pyref.get_read(out, offs, lens, i) == want
        assert bool(flags[i]) == m
    assert nc == int(flags.sum()) > 5


def test_threaded_count_with_correction_equals_serial(ora):
    """The threaded restatement (the CPU baseline) corrects the same reads and,
    in the order-free twice mode, builds the same table as the serial one."""
    from spk import synth
    p = synth.sample(20_000, 20, seed=4, err=(0.003, 0.01)).packed
    k = 21
    a = ora.count(p.data, p.offsets, p.lengths, k, 1 << 20, mode=ora.MODE_TWICE, correct=True)
    b = ora.count(p.data, p.offsets, p.lengths, k, 1 << 20, mode=ora.MODE_TWICE, correct=True, threads=4)
    assert a.stats()["corrected_reads"] == b.stats()["corrected_reads"] > 100
    for x, y in zip(a.table(1), b.table(1)):
        np.testing.assert_array_equal(x, y)
