"""FASTQ / FASTA text ingest in the oracle (FastxReader, src/packed_reads.rs:
69-234, into from_paired_files / append_from_file): the C++ restatement
against the independent Python one (oracle/pyref.py fastx_records) on
messy texts and malformed ones, and against the golden packed store of the
reference's own E. coli reads.  No GPU involved."""
import gzip
import os

import numpy as np
import pytest

from helpers import fasta_text, fastq_text, load_npz, messy_reads, rand_seq
from oracle import pyref

# The spades-rs checkout whose data/ holds the reference's own test reads, if
# the caller points at one (SPK_REFERENCE_ROOT); the test that reads them is
# skipped otherwise.
REF_DATA = os.path.join(os.environ.get("SPK_REFERENCE_ROOT", ""), "data")


def py_paired(t1, t2):
    a, b = pyref.fastx_records(t1), pyref.fastx_records(t2)
    return a, b


@pytest.mark.parametrize("crlf,blank", [(False, False), (True, False), (False, True), (True, True)])
def test_fastq_records_match_python(ora, crlf, blank):
    rng = np.random.default_rng(int(crlf) * 2 + int(blank))
    reads = messy_reads(rng, 300)
    t = b"\n \t\n" + fastq_text(reads, rng, crlf=crlf, blank_between=blank, plus_name=True)
    assert pyref.fastx_records(t) == [r.encode() for r in reads]
    p = ora.Packed.from_texts(t)
    q = ora.Packed()
    for r in reads:
        q.ingest_read(r)
    for x, y in zip(p.arrays(), q.arrays()):
        np.testing.assert_array_equal(x, y)
    assert p.sidecar() == q.sidecar()


def test_fasta_records(ora):
    rng = np.random.default_rng(3)
    seqs = messy_reads(rng, 50) + [""]
    t = fasta_text(seqs) + b">empty_at_end\n"
    recs = pyref.fastx_records(t)
    assert recs == [s.encode() for s in seqs]  # the empty last record is not a record
    p = ora.Packed.from_texts(t)
    q = ora.Packed()
    for r in seqs:
        q.ingest_read(r)
    for x, y in zip(p.arrays(), q.arrays()):
        np.testing.assert_array_equal(x, y)


def test_paired_unequal_counts(ora):
    rng = np.random.default_rng(5)
    r1 = messy_reads(rng, 120)
    r2 = messy_reads(rng, 90)
    t1, t2 = fastq_text(r1, rng), fastq_text(r2, rng, crlf=True)
    p = ora.Packed.from_texts(t1, t2)
    q = ora.Packed.from_paired(r1, r2)
    for x, y in zip(p.arrays(), q.arrays()):
        np.testing.assert_array_equal(x, y)
    assert p.sizes()["pe_count"] == q.sizes()["pe_count"] > 10
    assert p.sidecar() == q.sidecar()


@pytest.mark.parametrize("text", [
    b"@r\nACGT\n+\nIII\n",                 # quality length
    b"@r\nACGT\n-\nIIII\n",                # separator
    b"@r\nACGT\n+\nIIII\nr2\nACGT\n+\nIIII\n",  # header
    b"@r\nACGT\n",                         # EOF before '+'
    b"@r\nACGT\n+\n",                      # EOF before quality
    b"@r\n",                               # EOF before sequence
    b"xyz\n",                              # neither '@' nor '>'
])
def test_malformed_texts(ora, text):
    with pytest.raises(ValueError):
        pyref.fastx_records(text)
    with pytest.raises(ValueError):
        ora.Packed.from_texts(text)


def test_edge_texts(ora):
    for t, want in [(b"", []), (b"\n\n", []), (b">a", []), (b">a\n>b\nAC\n", [b"", b"AC"]),
                    (b"@a\n\n+\n\n", [b""]), (b"@a\r\nAC\r\r\n+\r\nII\r\n", [b"AC"]),
                    (b"@a\nACGT\n+x\nIIII", [b"ACGT"])]:
        assert pyref.fastx_records(t) == want, t
        p = ora.Packed.from_texts(t)
        assert p.sizes()["n_reads"] == 0


@pytest.mark.skipif(not os.environ.get("SPK_REFERENCE_ROOT")
                    or not os.path.exists(os.path.join(REF_DATA, "ecoli_1K_1.fq.gz")),
                    reason="SPK_REFERENCE_ROOT does not name a spades-rs checkout with its test data")
def test_reference_ecoli_reads_match_golden(ora):
    """The reference's data/ecoli_1K_{1,2}.fq.gz parsed by the oracle equal the
    golden packed store (made from the same files by the Python restatement)."""
    t1 = gzip.open(os.path.join(REF_DATA, "ecoli_1K_1.fq.gz")).read()
    t2 = gzip.open(os.path.join(REF_DATA, "ecoli_1K_2.fq.gz")).read()
    p = ora.Packed.from_texts(t1, t2)
    g = load_npz("ecoli_1K_packed.npz")
    d, o, ln = p.arrays()
    np.testing.assert_array_equal(d, g["data"])
    np.testing.assert_array_equal(o, g["offsets"])
    np.testing.assert_array_equal(ln, g["lengths"])


def test_fuzzed_texts_agree(ora):
    """Random texts built from FASTQ/FASTA line fragments (headers, bases with
    N and lowercase, '+' lines, qualities of matching or wrong length, blank,
    whitespace and CR-terminated lines): the C++ and Python restatements of
    the reader accept the same texts, refuse the same ones, and ingest the
    same store."""
    rng = np.random.default_rng(2024)
    nl_choices = [b"\n", b"\r\n", b"\r\r\n"]

    def seq():
        n = int(rng.integers(0, 60))
        return bytes(rng.choice(list(b"ACGTacgtN"), n).tolist())

    def fastq_record():
        s = seq()
        q = b"I" * (len(s) if rng.random() < 0.9 else len(s) + 1)
        nl = nl_choices[int(rng.integers(0, 3))]
        plus = b"+" if rng.random() < 0.95 else b"-"
        head = b"@r" if rng.random() < 0.97 else b"r"
        rec = head + nl + s + nl + plus + nl + q
        if rng.random() < 0.95:
            rec += nl
        return rec

    def fasta_record():
        out = b">h\n"
        for _ in range(int(rng.integers(0, 4))):
            out += seq() + nl_choices[int(rng.integers(0, 3))]
        return out

    agree = refused = 0
    for case in range(300):
        lead = b"".join([b"\n", b" \t\n", b"\r\n"][int(rng.integers(0, 3))] for _ in range(int(rng.integers(0, 3))))
        if case % 2:
            body = b"".join(fastq_record() + (b"\n" if rng.random() < 0.2 else b"") for _ in range(int(rng.integers(0, 6))))
        else:
            body = b"".join(fasta_record() for _ in range(int(rng.integers(0, 6))))
        text = lead + body
        try:
            want = pyref.fastx_records(text)
        except ValueError:
            with pytest.raises(ValueError):
                ora.Packed.from_texts(text)
            refused += 1
            continue
        p = ora.Packed.from_texts(text)
        q = ora.Packed()
        for r in want:
            q.ingest_read(r)
        for x, y in zip(p.arrays(), q.arrays()):
            np.testing.assert_array_equal(x, y)
        assert p.sidecar() == q.sidecar()
        agree += 1
    assert agree > 100 and refused > 20
