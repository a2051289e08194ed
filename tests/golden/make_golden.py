"""Generates the golden fixtures in tests/golden/ from the Python restatement.

Run once with a spades-rs checkout at hand, named on the command line or by
the SPK_REFERENCE_ROOT environment variable:

    python tests/golden/make_golden.py /path/to/spades-rs

The fixtures are produced by ``oracle/pyref.py`` (pure Python, unbounded
integers, string-level reverse complements), i.e. independently of the C++
oracle they pin.  The only inputs read from the spades-rs tree are its own
test data: ``data/ecoli_1K_{1,2}.fq.gz`` and ``data/reference_1K.fa.gz``
(used by tests/test_pipeline.rs:33-91).  Synthetic inputs come from the
seeded generator in spades-rs_b200/spk/synth.py.
"""
from __future__ import annotations

import gzip
import hashlib
import json
import os
import random
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "spades-rs_b200"))

from oracle import pyref  # noqa: E402
from spk import synth  # noqa: E402

DNA_KS = [1, 7, 11, 15, 21, 31, 32, 33, 55, 63, 64, 65, 77, 96, 99, 111, 127, 128]


def limbs4(x):
    return [int(v) for v in pyref.limbs(x)]


def nlimbs(k):
    return (k + 31) // 32


def sha(words) -> str:
    return hashlib.sha256(np.asarray(words, dtype=np.uint64).tobytes()).hexdigest()


def dna_vectors():
    rng = random.Random(20240601)
    out = []
    for k in DNA_KS:
        for _ in range(24):
            s = "".join(rng.choice("ACGT") for _ in range(k))
            x = pyref.k256_from_str(s, k)
            can, is_rc = pyref.k256_canonical(x, k)
            rec = dict(k=k, seq=s, kmer=limbs4(x), revcomp=limbs4(pyref.k256_revcomp(x, k)),
                       canonical=limbs4(can), is_rc=bool(is_rc),
                       extend_right=[limbs4(pyref.k256_extend_right(x, b, k)) for b in range(4)],
                       prepend_left=[limbs4(pyref.k256_prepend_left(x, b, k)) for b in range(4)],
                       hashes=[str(pyref.hash_kmer256(can, sd)) for sd in pyref.SEEDS])
            out.append(rec)
    return out


def hash_vectors(n=3000):
    rng = random.Random(7)
    keys, hs = [], []
    for i in range(n):
        nl = 1 + i % 4
        w = [rng.getrandbits(64) if j < nl else 0 for j in range(4)]
        x = (w[0] | (w[1] << 64), w[2] | (w[3] << 64))
        keys.append(w)
        hs.append([pyref.hash_kmer256(x, sd) for sd in pyref.SEEDS])
    return np.array(keys, dtype=np.uint64), np.array(hs, dtype=np.uint64)


def bloom_bits_vectors():
    """Positions (hash % size_bits) for non-power-of-two filter sizes."""
    rng = random.Random(11)
    out = []
    for cap in (64, 100, 1000, 12345, 1 << 20, (1 << 20) + 1, 999_999_937):
        f = pyref.TwoTierFilter(cap)
        keys = []
        for _ in range(64):
            w = rng.getrandbits(64)
            keys.append(w)
        pos = [[pyref.hash_kmer256((w, 0), sd) % f.size_bits for sd in pyref.SEEDS] for w in keys]
        out.append(dict(capacity_bits=cap, size_bits=f.size_bits, keys=[str(w) for w in keys],
                        positions=[[str(p) for p in q] for q in pos]))
    return out


def serial_bloom_sequence():
    """A serial insert/is_solid trace with repeats (reference semantics)."""
    rng = random.Random(5)
    f = pyref.TwoTierFilter(4096)
    keys = [rng.getrandbits(62) for _ in range(300)]
    seq = [keys[rng.randrange(len(keys))] for _ in range(2000)]
    promoted = [f.insert(v) for v in seq]
    solid = [f.is_solid(v) for v in keys]
    return dict(capacity_bits=4096, inserts=[str(v) for v in seq], promoted=promoted,
                queries=[str(v) for v in keys], solid=solid, seen_sha=sha(f.seen),
                solid_sha=sha(f.solid))


def counts_record(reads, k, bloom_bits, name, with_edges=False):
    ref_counts, ref_f = pyref.count_serial(reads, k, bloom_bits, "ref")
    tw_counts, tw_f = pyref.count_serial(reads, k, bloom_bits, "twice")
    L = nlimbs(k)
    ge2 = sorted((kk, c) for kk, c in ref_counts.items() if c >= 2)
    tw = sorted(tw_counts.items())
    rec = dict(
        name=name, k=k, bloom_bits=bloom_bits,
        ge2_keys=np.array([limbs4(kk)[:L] for kk, _ in ge2], dtype=np.uint64).reshape(-1, L),
        ge2_counts=np.array([c for _, c in ge2], dtype=np.uint32),
        twice_keys=np.array([limbs4(kk)[:L] for kk, _ in tw], dtype=np.uint64).reshape(-1, L),
        twice_counts=np.array([c for _, c in tw], dtype=np.uint32),
        ref_table_size=np.array([len(ref_counts)], dtype=np.uint64),
        seen_sha=np.array([sha(ref_f.seen)]), ref_solid_sha=np.array([sha(ref_f.solid)]),
        twice_sha=np.array([sha(tw_f.solid)]),
        seen_popcount=np.array([sum(bin(w).count("1") for w in ref_f.seen)], dtype=np.uint64),
        cutoff=np.array([pyref.determine_solid_kmer_cutoff(list(ref_counts.values()), 5.0)],
                        dtype=np.uint32),
    )
    assert sha(ref_f.seen) == sha(tw_f.seen)  # the seen tier does not depend on the mode
    if with_edges:
        solid = [kk for kk, c in ge2]
        e = pyref.edges(solid, k)
        rec["edges"] = np.array([limbs4(x)[:nlimbs(k + 1)] for x in e], dtype=np.uint64).reshape(-1, nlimbs(k + 1))
    return rec


def cutoff_vectors():
    rng = np.random.default_rng(3)
    cases = []
    # branch min_coverage > 5
    cases.append(dict(counts=[2, 3, 4], min_coverage=10.0))
    cases.append(dict(counts=[2, 3, 4], min_coverage=5.5))
    # <= 100 entries
    cases.append(dict(counts=list(range(1, 90)), min_coverage=5.0))
    # low coverage (top < 30)
    cases.append(dict(counts=rng.integers(1, 20, 5000).tolist(), min_coverage=5.0))
    # error peak + coverage peak with a valley
    for mu in (40, 64, 90, 150, 400):
        err = np.clip(rng.geometric(0.5, 20000), 1, None)
        cov = np.clip(rng.normal(mu, mu * 0.15, 30000).astype(int), 1, None)
        cases.append(dict(counts=np.concatenate([err, cov]).tolist(), min_coverage=5.0))
    # flat histogram (no valley found)
    cases.append(dict(counts=np.repeat(np.arange(1, 200), 50).tolist(), min_coverage=5.0))
    for c in cases:
        c["cutoff"] = pyref.determine_solid_kmer_cutoff(c["counts"], c["min_coverage"])
    return cases


def main(ref_root: str):
    os.makedirs(HERE, exist_ok=True)
    with open(os.path.join(HERE, "dna_vectors.json"), "w") as f:
        json.dump(dna_vectors(), f)
    keys, hs = hash_vectors()
    np.savez_compressed(os.path.join(HERE, "hash_vectors.npz"), keys=keys, hashes=hs)
    with open(os.path.join(HERE, "bloom_vectors.json"), "w") as f:
        json.dump(dict(positions=bloom_bits_vectors(), serial=serial_bloom_sequence()), f)
    cv = cutoff_vectors()
    np.savez_compressed(os.path.join(HERE, "cutoff_vectors.npz"),
                        **{f"counts_{i}": np.array(c["counts"], dtype=np.uint32) for i, c in enumerate(cv)},
                        min_coverage=np.array([c["min_coverage"] for c in cv]),
                        cutoff=np.array([c["cutoff"] for c in cv], dtype=np.uint32))

    # ---- real reads: the reference's own ecoli_1K test data -------------------
    r1 = pyref.read_fastq_gz(os.path.join(ref_root, "data", "ecoli_1K_1.fq.gz"))
    r2 = pyref.read_fastq_gz(os.path.join(ref_root, "data", "ecoli_1K_2.fq.gz"))
    with gzip.open(os.path.join(ref_root, "data", "reference_1K.fa.gz"), "rt") as f:
        ref_seq = "".join(l.strip() for l in f if not l.startswith(">"))
    reads, pe, side = pyref.from_paired_slices(r1, r2)
    data, offs, lens = pyref.pack_reads(reads)
    np.savez_compressed(os.path.join(HERE, "ecoli_1K_packed.npz"),
                        data=np.frombuffer(data, dtype=np.uint8), offsets=np.array(offs, np.uint64),
                        lengths=np.array(lens, np.uint32), pe_count=np.array([pe], np.uint64),
                        sidecar=np.array([side], np.uint64), n_raw=np.array([len(r1), len(r2)]),
                        reference_1K=np.array([ref_seq]))
    for k in (21, 31, 55):
        rec = counts_record(reads, k, 16 * 1024 * 1024, f"ecoli_1K_k{k}", with_edges=(k == 31))
        np.savez_compressed(os.path.join(HERE, f"counts_ecoli_1K_k{k}.npz"), **rec)
        print("ecoli", k, len(rec["ge2_counts"]), len(rec["twice_counts"]))

    # ---- synthetic reads ---------------------------------------------------------
    s = synth.c2(scale=0.0006)  # 3 kb genome at 100x
    sreads = [s.packed.get_read(i) for i in range(len(s.packed))]
    np.savez_compressed(os.path.join(HERE, "synth_c2_small_packed.npz"), data=s.packed.data,
                        offsets=s.packed.offsets, lengths=s.packed.lengths)
    for k, bits in ((55, 1 << 20), (77, 1 << 20), (32, 1 << 16), (64, 100_003)):
        rec = counts_record(sreads, k, bits, f"synth_k{k}", with_edges=(k in (55, 77)))
        np.savez_compressed(os.path.join(HERE, f"counts_synth_k{k}.npz"), **rec)
        print("synth", k, len(rec["ge2_counts"]), len(rec["twice_counts"]))


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SPK_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: make_golden.py /path/to/spades-rs (or set SPK_REFERENCE_ROOT)")
    main(root)
