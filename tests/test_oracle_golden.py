"""Pins the C++ oracle against the golden fixtures made by the independent
Python restatement (tests/golden/make_golden.py), and cross-checks the two
restatements on many random keys.  No GPU involved."""
import hashlib
import os

import numpy as np
import pytest

from helpers import ecoli_packed, load_json, load_npz, nlimbs, rows, synth_small_packed
from oracle import pyref

HASH_KS = [21, 31, 32, 33, 55, 63, 64, 65, 77, 127]


def sha(words):
    return hashlib.sha256(np.asarray(words, dtype=np.uint64).tobytes()).hexdigest()


def random_kmer_limbs(rng, n, k):
    """n random k-mers as 4-limb Kmer256 arrays (src/dna.rs:134-138 layout)."""
    w = rng.integers(0, 2 ** 63, size=(n, 4), dtype=np.uint64) * np.uint64(2) + \
        rng.integers(0, 2, size=(n, 4), dtype=np.uint64)
    if k <= 64:
        bits = 2 * k
        if bits < 64:
            w[:, 0] &= np.uint64((1 << bits) - 1)
            w[:, 1] = 0
        elif bits < 128:
            w[:, 1] &= np.uint64((1 << (bits - 64)) - 1)
        w[:, 2:] = 0
    else:
        hb = 2 * (k - 64)
        if hb < 64:
            w[:, 2] &= np.uint64((1 << hb) - 1)
            w[:, 3] = 0
        else:
            w[:, 3] &= np.uint64((1 << (hb - 64)) - 1)
    return w


@pytest.mark.parametrize("k", HASH_KS)
def test_hash_cpp_vs_numpy_1e6(ora, k):
    """hash_kmer256 (src/bloom.rs:61-78): C++ oracle == vectorised Python on 10^6 keys per k."""
    rng = np.random.default_rng(k)
    w = random_kmer_limbs(rng, 1_000_000, k)
    for seed in pyref.SEEDS:
        np.testing.assert_array_equal(ora.hash_batch(w, seed), pyref.hash_batch_np(w, seed))


def test_hash_golden_vectors(ora):
    d = load_npz("hash_vectors.npz")
    for s, seed in enumerate(pyref.SEEDS):
        np.testing.assert_array_equal(ora.hash_batch(d["keys"], seed), d["hashes"][:, s])


def test_dna_golden_vectors(ora):
    """from_bytes / revcomp / canonical / extend_right / prepend_left / hash against the fixtures."""
    for rec in load_json("dna_vectors.json"):
        k = rec["k"]
        fb = lambda v: tuple(int(x) for x in v)
        km = ora.k256_from_bytes(rec["seq"].encode(), k)
        assert fb(ora.to4(km)) == fb(rec["kmer"])
        assert fb(ora.to4(ora.k256_revcomp(km, k))) == fb(rec["revcomp"])
        can, is_rc = ora.k256_canonical(km, k)
        assert fb(ora.to4(can)) == fb(rec["canonical"]) and is_rc == rec["is_rc"]
        for b in range(4):
            assert fb(ora.to4(ora.k256_extend_right(km, b, k))) == fb(rec["extend_right"][b])
            assert fb(ora.to4(ora.k256_prepend_left(km, b, k))) == fb(rec["prepend_left"][b])
        for s, seed in enumerate(pyref.SEEDS):
            assert ora.hash_kmer256(can, seed) == int(rec["hashes"][s])


def test_bloom_positions_non_power_of_two(ora):
    """hash % size_bits for filter sizes that are not powers of two (src/bloom.rs:84-86)."""
    for rec in load_json("bloom_vectors.json")["positions"]:
        f = ora.Bloom(rec["capacity_bits"])
        assert f.size_bits == rec["size_bits"]
        for key, pos in zip(rec["keys"], rec["positions"]):
            for s, seed in enumerate(pyref.SEEDS):
                assert ora.hash_kmer256((int(key), 0), seed) % f.size_bits == int(pos[s])


def test_bloom_serial_trace(ora):
    """insert/is_solid return values and final tiers of a serial trace with repeats."""
    rec = load_json("bloom_vectors.json")["serial"]
    f = ora.Bloom(rec["capacity_bits"])
    got = [f.insert(int(v)) for v in rec["inserts"]]
    assert got == rec["promoted"]
    assert [f.is_solid(int(v)) for v in rec["queries"]] == rec["solid"]
    seen, solid = f.download()
    assert sha(seen) == rec["seen_sha"] and sha(solid) == rec["solid_sha"]


def test_cutoff_golden(ora):
    """determine_solid_kmer_cutoff (src/assemble.rs:692-735)."""
    d = load_npz("cutoff_vectors.npz")
    for i in range(d["cutoff"].size):
        assert ora.cutoff(d[f"counts_{i}"], float(d["min_coverage"][i])) == int(d["cutoff"][i])


COUNT_FIXTURES = ["counts_ecoli_1K_k21.npz", "counts_ecoli_1K_k31.npz", "counts_ecoli_1K_k55.npz",
                  "counts_synth_k55.npz", "counts_synth_k77.npz", "counts_synth_k32.npz",
                  "counts_synth_k64.npz"]


def _inputs(name):
    if "ecoli" in name:
        data, offs, lens, _ = ecoli_packed()
    else:
        data, offs, lens = synth_small_packed()
    return data, offs, lens


@pytest.mark.parametrize("name", COUNT_FIXTURES)
@pytest.mark.parametrize("threads", [0, 3])
def test_count_tables_golden(ora, name, threads):
    """Stages 2-3 (src/assemble.rs:129-242): serial and threaded oracle vs the fixtures."""
    g = load_npz(name)
    k, bits = int(g["k"]), int(g["bloom_bits"])
    data, offs, lens = _inputs(name)
    ref = ora.count(data, offs, lens, k, bits, mode=ora.MODE_REF, threads=threads)
    keys, counts = ref.table(2)
    # the count >= 2 list is order-free even in reference semantics
    np.testing.assert_array_equal(keys, g["ge2_keys"])
    np.testing.assert_array_equal(counts, g["ge2_counts"])
    seen, solid = ref.bloom()
    assert sha(seen) == str(g["seen_sha"][0])
    if threads == 0:
        assert sha(solid) == str(g["ref_solid_sha"][0])
        assert ref.table(1)[0].shape[0] == int(g["ref_table_size"][0])
        allc = ref.table(1)[1]
        assert ora.cutoff(allc, 5.0) == int(g["cutoff"][0])
    tw = ora.count(data, offs, lens, k, bits, mode=ora.MODE_TWICE, threads=threads)
    tk, tc = tw.table(1)
    np.testing.assert_array_equal(tk, g["twice_keys"])
    np.testing.assert_array_equal(tc, g["twice_counts"])
    s2, t2 = tw.bloom()
    assert sha(s2) == str(g["seen_sha"][0]) and sha(t2) == str(g["twice_sha"][0])


@pytest.mark.parametrize("name", ["counts_ecoli_1K_k31.npz", "counts_synth_k55.npz",
                                  "counts_synth_k77.npz"])
def test_edges_golden(ora, name):
    """(k+1)-mer edges implied by get_successors (src/graph.rs:78-102)."""
    g = load_npz(name)
    k = int(g["k"])
    e = ora.edges(g["ge2_keys"], k)
    np.testing.assert_array_equal(e, g["edges"])


def test_edges_successor_predecessor_symmetry(ora):
    """Every edge seen from the successor side is seen from the predecessor side (src/graph.rs:91-102)."""
    g = load_npz("counts_synth_k55.npz")
    k = 55
    solid = set(rows(g["ge2_keys"]))
    keys = [ora.from_limbs(r) for r in g["ge2_keys"][:400]]
    for s in keys:
        for o in range(2):
            ex = ora.k256_revcomp(s, k) if o else s
            for b in range(4):
                nx = ora.k256_extend_right(ex, b, k)
                can, _ = ora.k256_canonical(nx, k)
                if tuple(int(v) for v in ora.to4(can)[: nlimbs(k)]) not in solid:
                    continue
                # prepending the dropped first base to the successor gives s back
                back = ora.k256_prepend_left(nx, "ACGT".index(pyref.k256_to_str(ex, k)[0]), k)
                assert back == ex


def test_ecoli_reference_kmers_are_solid(ora):
    """Every k-mer of data/reference_1K.fa.gz has count >= 2 in the ecoli_1K reads at
    k = 21 and the reference test's k = 31 (tests/test_pipeline.rs:33-91).  At k = 55
    the trimmed reads (30-100 bp) leave a 16-position gap, so k = 55 is not asserted."""
    data, offs, lens, d = ecoli_packed()
    ref_seq = str(d["reference_1K"][0])
    for k in (21, 31):
        res = ora.count(data, offs, lens, k, 16 << 20, mode=ora.MODE_REF)
        solid = set(rows(res.table(2)[0]))
        for i in range(len(ref_seq) - k + 1):
            x = pyref.k256_from_str(ref_seq[i:i + k], k)
            can, _ = pyref.k256_canonical(x, k)
            assert tuple(pyref.limbs(can)[: nlimbs(k)]) in solid


def test_ecoli_pipeline_spells_reference(ora):
    """The reference's integration test (tests/test_pipeline.rs:33-91) on the
    oracle: k = 31, a 16 Mi-bit Bloom, error correction, the adaptive cutoff
    at min_coverage 5, then CompactedGraph::build.  The unitigs spell
    data/reference_1K.fa.gz as one path; the only others are error tips,
    which the reference's simplifier (outside the counting path) clips."""
    from helpers import revcomp, spelled_path
    data, offs, lens, d = ecoli_packed()
    ref = str(d["reference_1K"][0])
    k = 31
    res = ora.count(data, offs, lens, k, 16 * 1024 * 1024, mode=ora.MODE_TWICE, correct=True)
    tk, tc = res.table(1)
    keep = tc >= ora.cutoff(tc, 5.0)
    seqs, _, _ = ora.unitigs(tk[keep], tc[keep], k)
    path = spelled_path(seqs, ref, k)
    assert path is not None
    assert len(path) < len(seqs)  # the tips split the contig at their branch points
    off = [s for s in seqs if s not in {ref[a:b] for a, b in path} and revcomp(s) not in {ref[a:b] for a, b in path}]
    assert all(len(s) < 2 * k for s in off)


def test_threaded_twice_count_equals_serial(ora):
    """The twice tier is order-free, so the threaded oracle (the checker of the
    full-size GPU tests and of the benchmark's parity check) gives the serial
    table and tiers exactly, whatever its thread count."""
    from spk import synth
    p = synth.c2(0.004).packed
    for k in (21, 55, 77):
        s = ora.count(p.data, p.offsets, p.lengths, k, 1 << 22, mode=ora.MODE_TWICE)
        sk, sc = s.table(1)
        ss, st = s.bloom()
        for threads in (2, 7):
            t = ora.count(p.data, p.offsets, p.lengths, k, 1 << 22, mode=ora.MODE_TWICE, threads=threads)
            tk, tc = t.table(1)
            ts, tt = t.bloom()
            np.testing.assert_array_equal(tk, sk)
            np.testing.assert_array_equal(tc, sc)
            np.testing.assert_array_equal(ts, ss)
            np.testing.assert_array_equal(tt, st)


def test_ecoli_packing_matches_oracle_ingest(ora):
    """The committed ecoli_1K packing equals the C++ oracle's ingest of the same reads."""
    data, offs, lens, d = ecoli_packed()
    assert int(d["pe_count"][0]) > 0 and lens.size == offs.size
    assert int(d["n_raw"][0]) == 2054 and int(d["n_raw"][1]) == 2054


def test_prior_injection_matches_python_restatement(ora):
    """src/assemble.rs:267-283 on the C++ oracle against the Python
    restatement: windows with a non-ACGT byte are skipped, either case is
    accepted, contigs shorter than k add nothing, and absent k-mers are
    inserted with the boost."""
    data, offs, lens = synth_small_packed()
    k, boost = 21, 50
    r = ora.count(data, offs, lens, k, 1 << 20, mode=ora.MODE_TWICE)
    before_k, before_c = r.table(1)
    reads = [pyref.get_read(data, offs, lens, i) for i in (0, 5, 9)]
    priors = [reads[0][10:90].encode(), reads[1][:40].lower().encode(),
              (reads[2][:30] + "N" + reads[2][30:70]).encode(), b"ACGTACGT",
              b"GATTACAGATTACATTTTGGGGCCCCAAAATTTT"]
    r.inject_priors(priors, boost)
    got_k, got_c = r.table(1)
    want = {tuple(int(x) for x in row): int(c) for row, c in zip(before_k, before_c)}
    for p in priors:
        s = p.decode()
        for i in range(len(s) - k + 1):
            x = pyref.k256_from_str(s[i:i + k], k)
            if x is None:
                continue
            key = tuple(int(v) for v in pyref.limbs(pyref.k256_canonical(x, k)[0]))[: nlimbs(k)]
            want[key] = want.get(key, 0) + boost
    keys = sorted(want)
    np.testing.assert_array_equal(got_k, np.array(keys, dtype=np.uint64))
    np.testing.assert_array_equal(got_c, np.array([want[t] for t in keys], dtype=np.uint32))
