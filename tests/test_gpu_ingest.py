"""GPU ingest (spk_ingest, through the C ABI) of FASTQ / FASTA texts into
the three-block PackedReads store, against the oracle's restatement of
FastxReader and the ingest gates (src/packed_reads.rs:69-690).  Packed
bytes, offsets, lengths, pe_count and the ambiguous sidecar compared exactly."""
import numpy as np
import pytest

from helpers import fasta_text, fastq_text, messy_reads, rand_seq

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def spk(spk_lib):
    return spk_lib


def same(ora, spk, t1, t2=None):
    want = ora.Packed.from_texts(t1, t2)
    got = spk.ingest(t1, t2)
    pr, side = got.download()
    d, o, ln = want.arrays()
    np.testing.assert_array_equal(pr.data, d)
    np.testing.assert_array_equal(pr.offsets, o)
    np.testing.assert_array_equal(pr.lengths, ln)
    assert pr.pe_count == want.sizes()["pe_count"]
    assert side == want.sidecar()
    return got


@pytest.mark.parametrize("crlf,blank", [(False, False), (True, True)])
def test_paired_fastq(spk, ora, crlf, blank):
    rng = np.random.default_rng(11 + int(crlf))
    g = rand_seq(rng, 30000)
    r1 = messy_reads(rng, 700, g)
    r2 = messy_reads(rng, 640, g)
    t1 = b" \n\r\n" + fastq_text(r1, rng, crlf=crlf, blank_between=blank, plus_name=True)
    t2 = fastq_text(r2, rng, crlf=not crlf, blank_between=blank)
    got = same(ora, spk, t1, t2)
    i = got.info()
    assert i["pe_count"] > 50 and i["n_sidecar"] > 10


def test_single_fastq_and_fasta(spk, ora):
    rng = np.random.default_rng(2)
    reads = messy_reads(rng, 500)
    same(ora, spk, fastq_text(reads, rng))
    same(ora, spk, fasta_text(reads + [""]) + b">last_empty\n")
    same(ora, spk, fasta_text(reads, width=17))
    # a FASTQ R1 with a FASTA R2
    same(ora, spk, fastq_text(reads[:200], rng), fasta_text(reads[100:400]))


def test_many_lines(spk, ora):
    """Enough lines for several scan blocks of the record machine and many
    newline chunks; blank lines between records."""
    rng = np.random.default_rng(4)
    g = rand_seq(rng, 200000)
    reads = messy_reads(rng, 40000, g)
    same(ora, spk, fastq_text(reads, rng, blank_between=True))


@pytest.mark.parametrize("text", [b"", b"\n \n", b">a", b">a\n>b\nAC\n", b"@a\n\n+\n\n",
                                  b"@a\r\nACGTACGTACGTACGTACGTACGT\r\r\n+\r\nIIIIIIIIIIIIIIIIIIIIIIII\r\n"])
def test_edge_texts(spk, ora, text):
    same(ora, spk, text)


@pytest.mark.parametrize("text", [
    b"@r\nACGT\n+\nIII\n", b"@r\nACGT\n-\nIIII\n", b"@r\nACGT\n+\nIIII\nr2\nACGT\n+\nIIII\n",
    b"@r\nACGT\n", b"@r\nACGT\n+\n", b"@r\n", b"xyz\n"])
def test_malformed(spk, ora, text):
    with pytest.raises(ValueError):
        ora.Packed.from_texts(text)
    with pytest.raises(spk.SpkError) as e:
        spk.ingest(text)
    assert e.value.code == 1


def test_count_from_ingest(spk, ora):
    """Counting the device-resident store equals counting the oracle's store."""
    rng = np.random.default_rng(6)
    from spk import synth
    s = synth.sample(30000, 30, seed=3, n_rate=0.002)
    p = s.packed
    reads = [p.get_read(i) for i in range(len(p))]
    # put some Ns back so the gates split reads
    reads = [r[:50] + "N" + r[51:] if i % 7 == 0 and len(r) > 60 else r for i, r in enumerate(reads)]
    half = len(reads) // 2
    t1, t2 = fastq_text(reads[:half], rng), fastq_text(reads[half:], rng)
    dev = same(ora, spk, t1, t2)
    want = ora.Packed.from_texts(t1, t2)
    d, o, ln = want.arrays()
    a = dev.count([33], bloom_bits=1 << 22, list_min_count=1)
    b = spk.count((d, o, ln), [33], bloom_bits=1 << 22, list_min_count=1)
    ka, ca = a.kmers(0, 1)
    kb, cb = b.kmers(0, 1)
    np.testing.assert_array_equal(ka, kb)
    np.testing.assert_array_equal(ca, cb)
