"""GPU read error correction (spk_bloom_correct_reads, through the C ABI)
against the oracle's restatement of ErrorCorrector::correct_read_in_place
(src/hammer.rs:34-121) on the same filter tiers.  Corrected packed bytes and
per-read flags compared bit for bit."""
import numpy as np
import pytest

from helpers import correction_case
from oracle import pyref

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def spk(spk_lib):
    return spk_lib


def both_filters(spk, ora, bits, keys):
    g = spk.TwoTierFilter(bits)
    g.insert_kmer256_batch(keys)
    o = ora.Bloom(bits)
    seen, solid = g.download()
    o.load(seen, solid)
    return g, o


def test_reference_single_substitution(spk):
    """src/hammer.rs:160-185 on the GPU."""
    k = 5
    ref = "ACGTACGTACGT"
    f = spk.TwoTierFilter(1024 * 1024)
    keys = [pyref.limbs(pyref.k256_canonical(pyref.k256_from_str(ref[i:i + k], k), k)[0])
            for i in range(len(ref) - k + 1)] * 2
    f.insert_kmer256_batch(np.array(keys, dtype=np.uint64))
    assert f.correct_read("ACGGACGTACGT", k) == (ref, True)


def test_reference_short_read_bypass(spk):
    """src/hammer.rs:187-193 on the GPU."""
    f = spk.TwoTierFilter(1024)
    assert f.correct_read("ACGT", 15) == ("ACGT", False)


@pytest.mark.parametrize("k,bits", [(11, 1 << 20), (21, 1 << 20), (21, 1 << 14), (33, 1 << 20),
                                    (55, 1 << 20), (64, 1 << 20), (77, 1 << 20), (127, 1 << 22),
                                    (55, 1 << 15)])
def test_matches_oracle(spk, ora, k, bits):
    keys, reads = correction_case(k, seed=3 * k + bits, genome_len=4000, n_reads=120)
    g, o = both_filters(spk, ora, bits, keys)
    data, offs, lens = pyref.pack_reads(reads)
    d = np.frombuffer(data, np.uint8)
    want, wflags, wn = o.correct_packed(k, d, offs, lens)
    got, gflags, gn = g.correct_reads((d, np.array(offs, np.uint64), np.array(lens, np.uint32)), k)
    np.testing.assert_array_equal(got.data, want)
    np.testing.assert_array_equal(gflags, wflags.astype(bool))
    assert gn == wn
    assert wn > 10


def test_sample_reads(spk, ora):
    """Reads of a 30 kb genome at 30x with 0.5-1% substitutions, the filter
    filled by inserting every read k-mer in read order (Stage 2)."""
    from spk import synth
    k = 33
    p = synth.sample(30_000, 30, seed=5, err=(0.005, 0.01)).packed
    n = 2000
    reads = [p.get_read(i) for i in range(n)]
    keys = []
    for r in reads:
        for i in range(len(r) - k + 1):
            keys.append(pyref.limbs(pyref.k256_canonical(pyref.k256_from_str(r[i:i + k], k), k)[0]))
    g, o = both_filters(spk, ora, 1 << 22, np.array(keys, dtype=np.uint64))
    data, offs, lens = p.data, p.offsets[:n], p.lengths[:n]
    want, wflags, wn = o.correct_packed(k, data, offs, lens)
    got, gflags, gn = g.correct_reads((data, offs, lens), k)
    np.testing.assert_array_equal(got.data, want)
    np.testing.assert_array_equal(gflags, wflags.astype(bool))
    assert gn == wn > 0


def test_bad_inputs(spk):
    f = spk.TwoTierFilter(1 << 16)
    d = np.zeros(8, np.uint8)
    with pytest.raises(spk.SpkError) as e:
        f.correct_reads((d, np.array([4], np.uint64), np.array([40], np.uint32)), 21)
    assert e.value.code == 1
    with pytest.raises(spk.SpkError) as e:
        f.correct_reads((d, np.array([0], np.uint64), np.array([20], np.uint32)), 128)
    assert e.value.code == 2
    out, flags, n = f.correct_reads((d, np.array([0], np.uint64), np.array([20], np.uint32)), 0)
    assert n == 0 and not flags.any()
    np.testing.assert_array_equal(out.data, d)


@pytest.mark.parametrize("k,genome", [(21, 40_000), (55, 40_000), (77, 12_000)])
def test_count_with_correction(spk, ora, k, genome):
    """SPK_F_CORRECT: Stage 3 corrects every read against the twice tier
    before counting (src/assemble.rs:183-191).  The admitted table, the
    cutoff and the number of corrected reads equal the oracle's serial count
    with the same correction."""
    from spk import synth
    p = synth.sample(genome, 25, seed=9, err=(0.003, 0.012)).packed
    bits = 1 << 22
    ref = ora.count(p.data, p.offsets, p.lengths, k, bits, mode=ora.MODE_TWICE, correct=True)
    tk, tc = ref.table(1)
    r = spk.count(p, [k], bloom_bits=bits, list_min_count=1, flags=0x1 | 0x4 | spk.SPK_F_CORRECT)
    info = r.info(0)
    assert info["schedule"] == 0  # gated
    assert info["n_corrected_reads"] == ref.stats()["corrected_reads"] > 100
    gk, gc = r.kmers(0, 1)
    np.testing.assert_array_equal(gk, tk)
    np.testing.assert_array_equal(gc, tc)
    assert info["cutoff"] == ora.cutoff(tc, 5.0)
    # fewer distinct k-mers than without correction
    plain = spk.count(p, [k], bloom_bits=bits, list_min_count=1, flags=0x1 | 0x4 | 0x8)
    assert info["n_table"] < plain.info(0)["n_table"]
    np.testing.assert_array_equal(r.bloom(0)[0], ref.bloom()[0])
