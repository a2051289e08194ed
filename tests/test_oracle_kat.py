"""The reference's own known-answer tests for the counting path, run on the
C++ oracle and the independent Python restatement.

Each test restates a spades-rs test (file:line given) so that the oracle is
pinned to the reference's expectations before it is used to check the GPU.
"""
import random

import numpy as np
import pytest

from oracle import pyref

TEMPLATE = ("ATGCGATCGATCGATAGCTAGCTAGCTAGCTAAGCTAGCTAGCTAGCTAATGCGATCGATCGATAGCTAGCTAGCTAGCTAAGCT"
            "AGCTAGCTAGCTAATGCGATCGATCGATAGCTAGCTAGCTAGCTAAGCTAGCTAGCTAGCTAATGCGATCGATCGATAGCTAGCT"
            "AGCTAGCTAAGCTAGCTAGCTAGCTA")


# ---- src/dna.rs tests ---------------------------------------------------------
def test_revcomp_kmer(ora):  # src/dna.rs:329-342
    k = ora.lib()
    import ctypes as C
    v = C.c_uint64()
    assert k.ora_string_to_kmer(b"ACGT", 4, 4, C.byref(v))
    acgt = v.value
    assert ora.lib().ora_revcomp_u64(acgt, 4) == acgt
    k.ora_string_to_kmer(b"AAAA", 4, 4, C.byref(v)); a4 = v.value
    k.ora_string_to_kmer(b"TTTT", 4, 4, C.byref(v)); t4 = v.value
    assert k.ora_revcomp_u64(a4, 4) == t4 and k.ora_revcomp_u64(t4, 4) == a4


def test_encode_decode_roundtrip():  # src/dna.rs:345-351
    s = "ATGCGATCGATCGAT"
    assert pyref.kmer_to_string(pyref.string_to_kmer(s.encode(), len(s)), len(s)) == s


@pytest.mark.parametrize("k", [21, 33, 55, 64, 77, 99, 127])
def test_kmer256_roundtrip_and_revcomp(ora, k):  # src/dna.rs:354-367
    seq = TEMPLATE[:k]
    km = ora.k256_from_bytes(seq.encode(), k)
    assert ora.k256_to_string(km, k) == seq
    assert ora.k256_revcomp(ora.k256_revcomp(km, k), k) == km
    assert pyref.k256_to_str(pyref.k256_from_str(seq, k), k) == seq


def test_kmer256_revcomp_known_answer(ora):  # src/dna.rs:370-414
    base = "ACGT" * 16 + "A"
    km = ora.k256_from_bytes(base.encode(), 65)
    rc = ora.k256_revcomp(km, 65)
    assert ora.k256_to_string(rc, 65) == "T" + "ACGT" * 16
    assert ora.k256_revcomp(rc, 65) == km
    b96 = "ACGT" * 24
    assert ora.k256_to_string(ora.k256_revcomp(ora.k256_from_bytes(b96.encode(), 96), 96), 96) == b96
    s127 = "ATCG" * 31 + "ATG"
    rc127 = ora.k256_revcomp(ora.k256_from_bytes(s127.encode(), 127), 127)
    assert ora.k256_to_string(rc127, 127) == pyref.revcomp_str(s127)


@pytest.mark.parametrize("k", [21, 33, 55, 64, 77, 99, 127])
def test_kmer256_extend_and_prepend(ora, k):  # src/dna.rs:416-432
    seq = TEMPLATE[:k]
    km = ora.k256_from_bytes(seq.encode(), k)
    assert ora.k256_to_string(ora.k256_extend_right(km, 1, k), k) == seq[1:] + "C"
    assert ora.k256_to_string(ora.k256_prepend_left(km, 2, k), k) == "G" + seq[:-1]


# ---- tests/test_dna_kmer.rs -------------------------------------------------------
def test_base_encoding_and_invalid_chars(ora):  # tests/test_dna_kmer.rs:9-33
    L = ora.lib()
    for ch, v in zip(b"AaCcGgTt", (0, 0, 1, 1, 2, 2, 3, 3)):
        assert L.ora_base_to_2bit(ch) == v
    for bad in (b"ACGTN", b"ACGT1", b"AC GT", b"AC-GT"):
        assert pyref.string_to_kmer(bad, 5) is None
        assert ora.k256_from_bytes(bad, 5) is None
    assert pyref.string_to_kmer(b"ACGT", 5) is None


def test_revcomp_bytes_properties():  # tests/test_dna_kmer.rs:35-45
    assert pyref.revcomp_str("AAAA") == "TTTT"
    assert pyref.revcomp_str("CCCC") == "GGGG"
    assert pyref.revcomp_str("ACGT") == "ACGT"
    assert pyref.revcomp_str("CGCG") == "CGCG"


def test_revcomp_u64_invariance(ora):  # tests/test_dna_kmer.rs:48-74
    L = ora.lib()
    for k in range(1, 33):
        seq = "".join("ACGT"[i % 4] for i in range(k))
        v = pyref.string_to_kmer(seq.encode(), k)
        rc = L.ora_revcomp_u64(v, k)
        assert L.ora_revcomp_u64(rc, k) == v
        assert pyref.kmer_to_string(v, k) == seq


@pytest.mark.parametrize("k", [1, 7, 15, 21, 31, 32])
def test_canonical_kmer_u64_idempotence(ora, k):  # tests/test_dna_kmer.rs:76-107
    import ctypes as C
    L = ora.lib()
    seq = "".join("ACGT"[(i * 7) % 4] for i in range(k))
    v = pyref.string_to_kmer(seq.encode(), k)
    r1, r2 = C.c_int(), C.c_int()
    c1 = L.ora_canonical_u64(v, k, C.byref(r1))
    assert L.ora_canonical_u64(c1, k, None) == c1
    rc = L.ora_revcomp_u64(v, k)
    assert L.ora_canonical_u64(rc, k, C.byref(r2)) == c1
    if v != rc:
        assert r1.value != r2.value


@pytest.mark.parametrize("k", [33, 55, 64, 65, 77, 99, 111, 127, 128])
def test_kmer256_large_k_invariance(ora, k):  # tests/test_dna_kmer.rs:109-147
    seq = "".join("ACGT"[(i * 13 + 5) % 4] for i in range(k))
    km = ora.k256_from_bytes(seq.encode(), k)
    rc = ora.k256_revcomp(km, k)
    assert ora.k256_revcomp(rc, k) == km
    assert ora.k256_canonical(km, k)[0] == ora.k256_canonical(rc, k)[0]
    assert ora.k256_to_string(km, k) == seq


def test_kmer256_extend_and_prepend_exactness(ora):  # tests/test_dna_kmer.rs:149-175
    k = 63
    seq = "".join("ACGT"[i % 4] for i in range(k))
    km = ora.k256_from_bytes(seq.encode(), k)
    assert ora.k256_to_string(ora.k256_extend_right(km, 3, k), k) == seq[1:] + "T"
    assert ora.k256_to_string(ora.k256_prepend_left(km, 2, k), k) == "G" + seq[:-1]


# ---- src/bloom.rs and tests/test_hammer_and_bloom.rs ------------------------------
@pytest.mark.parametrize("impl", ["cpp", "py"])
def test_two_tier_filter(ora, impl):  # src/bloom.rs:139-156
    f = ora.Bloom(1024 * 1024) if impl == "cpp" else pyref.TwoTierFilter(1024 * 1024)
    k1, k2 = 123456789, 987654321
    assert not f.is_solid(k1)
    f.insert(k1)
    assert not f.is_solid(k1)
    f.insert(k1)
    assert f.is_solid(k1)
    assert not f.is_solid(k2)


@pytest.mark.parametrize("impl", ["cpp", "py"])
def test_two_tier_bloom_transitions(ora, impl):  # tests/test_hammer_and_bloom.rs:39-70
    f = ora.Bloom(1024 * 1024) if impl == "cpp" else pyref.TwoTierFilter(1024 * 1024)
    a, b, c = 0x123456789ABCDEF0, 0xFEDCBA9876543210, 0xA5A5A5A5A5A5A5A5
    assert not f.is_solid(a) and not f.is_solid(b) and not f.is_solid(c)
    assert not f.insert(a) and not f.is_solid(a)
    assert f.insert(a) and f.is_solid(a)
    assert f.insert(a) and f.is_solid(a)
    assert not f.is_solid(b) and not f.is_solid(c)


def test_filter_sizes(ora):  # src/bloom.rs:26-43, 129-131
    for cap, words in ((0, 1), (1, 1), (64, 1), (65, 2), (1024 * 1024, 16384)):
        f = ora.Bloom(cap)
        assert f.num_words == words and f.size_bits == words * 64
        assert f.memory_usage_bytes() == words * 16


# ---- tests/test_packed_reads.rs and src/packed_reads.rs tests ---------------------
def test_packed_reads_all_modulo4_lengths(ora):  # tests/test_packed_reads.rs:6-38
    p = ora.Packed()
    seqs = ["".join("ACGT"[i % 4] for i in range(n)) for n in range(65)]
    for s in seqs:
        p.pack_clean(s)
    assert p.sizes()["n_reads"] == 65
    for i, s in enumerate(seqs):
        assert p.get_read(i) == s


def test_packed_reads_synthetic_workload(ora):  # tests/test_packed_reads.rs:41-79
    p = ora.Packed()
    st = 0x12345678
    M = (1 << 64) - 1
    exp = []
    for _ in range(2000):
        st = (st * 6364136223846793005 + 1) & M
        n = 50 + st % 200
        s = []
        for j in range(n):
            st = (st * 6364136223846793005 + 1) & M
            s.append("ACGT"[(st ^ j) % 4])
        s = "".join(s)
        p.pack_clean(s)
        exp.append(s)
    assert p.sizes()["n_reads"] == 2000
    for i in range(0, 2000, 37):
        assert p.get_read(i) == exp[i]
    data, offs, lens = p.arrays()
    d2, o2, l2 = pyref.pack_reads(exp)
    assert bytes(data) == d2 and list(offs) == o2 and list(lens) == l2


def test_packed_reads_boundary_cases(ora):  # tests/test_packed_reads.rs:82-116
    p = ora.Packed()
    for s in ("", "G", "TA", "CGC", "ACGT", "ACGTA"):
        p.pack_clean(s)
    for i, s in enumerate(("", "G", "TA", "CGC", "ACGT", "ACGTA")):
        assert p.get_read(i) == s


@pytest.mark.parametrize("read,n_primary,n_side,first", [
    ("NNNACGTACGTACGTACGTACGTA", 1, 0, "ACGTACGTACGTACGTACGTA"),   # test_packed_reads.rs:122-136
    ("ACGTACGTACGTACGTACGTANNN", 1, 0, "ACGTACGTACGTACGTACGTA"),   # :138-151
    ("ACGTACGTACGTACGTACGTANNNACGTACGTACGTACGTACGTA", 2, 0, None),  # :153-162
    ("ACGTN" + "ACGTACGTACGTACGTACGTA", 1, 0, "ACGTACGTACGTACGTACGTA"),  # :164-176
    ("ACGTNNCGTA", 0, 1, None),                                      # :178-186
    ("NNNNNNNNNNN", 0, 0, None),                                     # :188-198
    ("ACGTNACGT", 0, 1, None),                                       # :200-217
    ("ACGTACGTACGTACGTACGTACGT", 1, 0, "ACGTACGTACGTACGTACGTACGT"),  # :233-246
    ("NNACGTNN", 0, 1, None),
    ("NNNNNN", 0, 0, None),                                          # src/packed_reads.rs:795-800
])
def test_ingest_n_handling(ora, read, n_primary, n_side, first):
    p = ora.Packed()
    p.ingest_read(read)
    s = p.sizes()
    assert s["n_reads"] == n_primary and s["n_sidecar"] == n_side
    if first is not None:
        assert p.get_read(0) == first
    r, pe, side = pyref.from_paired_slices([read], [])
    assert len(r) == n_primary and side == n_side


def test_three_block_paired_synchronization_and_trimming(ora):  # tests/test_packed_reads.rs:259-320
    r1 = ["ACGTACGTACGTACGTACGTACGT", "NNAAACCCGGGTTTAAACCCGGGTTTNN",
          "ACGTACGTACGTACGTACGTACNNNGTGCATGCATGCATGCATGCAT", "GGGGGGGGGGGGGGGGGGGGGGGG"]
    r2 = ["TGCATGCATGCATGCATGCATGCA", "TTTGGGCCCAAATTTGGGCCCAAA", "CCCCCCCCCCCCCCCCCCCCCCCC",
          "AAAAAAAAAAAAAAAAAAAAAAAA"]
    p = ora.Packed.from_paired(r1, r2)
    s = p.sizes()
    assert s["pe_count"] == 3 and s["n_reads"] == 9
    pe = 3
    assert p.get_read(0) == r1[0] and p.get_read(0 + pe) == r2[0]
    assert p.get_read(1) == "AAACCCGGGTTTAAACCCGGGTTT" and p.get_read(1 + pe) == r2[1]
    assert p.get_read(2) == r1[3] and p.get_read(2 + pe) == r2[3]
    reads, pe2, side = pyref.from_paired_slices(r1, r2)
    assert pe2 == 3 and len(reads) == 9
    assert [p.get_read(i) for i in range(9)] == reads


def test_three_block_paired_synchronization(ora):  # src/packed_reads.rs:846-891
    r1 = ["AAAAACCCCCGGGGGTTTTTAAAA", "ACGTACGTACGTACGTACGTACNNACGTACGTACGTACGTACGTAC",
          "NNNCCCCCGGGGTTTTTAAAAACCCCCNN"]
    r2 = ["TTTTTAAAAAGGGGGCCCCCTTTT", "GGGGGGGGGGGGCCCCCCCCCCCC", "NNNGGGGGCCCCTTTTTAAAAAGGGGGNN"]
    p = ora.Packed.from_paired(r1, r2)
    s = p.sizes()
    assert s["pe_count"] == 2 and s["n_reads"] == 7
    assert p.get_read(1) == "CCCCCGGGGTTTTTAAAAACCCCC"
    assert p.get_read(3) == "GGGGGCCCCTTTTTAAAAAGGGGG"
    assert p.get_read(4) == "ACGTACGTACGTACGTACGTAC"
    assert p.get_read(5) == "ACGTACGTACGTACGTACGTAC"
    assert p.get_read(6) == r2[1]
