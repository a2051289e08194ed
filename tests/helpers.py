"""Helpers shared by the tests (fixtures loading, key conversions)."""
import json
import os

import numpy as np

from conftest import GOLDEN

M64 = (1 << 64) - 1


def load_npz(name):
    return dict(np.load(os.path.join(GOLDEN, name), allow_pickle=False))


def load_json(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def nlimbs(k):
    return (k + 31) // 32


def rows(a):
    """Set-comparable tuples of a (n, L) key array."""
    a = np.asarray(a, dtype=np.uint64)
    return [tuple(int(v) for v in r) for r in a]


def ecoli_packed():
    d = load_npz("ecoli_1K_packed.npz")
    return d["data"], d["offsets"], d["lengths"], d


def synth_small_packed():
    d = load_npz("synth_c2_small_packed.npz")
    return d["data"], d["offsets"], d["lengths"]


def kmer_strings(data, offsets, lengths, k):
    """All k-mer strings of packed reads (small inputs only)."""
    out = []
    for o, n in zip(offsets, lengths):
        o, n = int(o), int(n)
        by = data[o:o + (n + 3) // 4]
        codes = np.stack([(by >> 6) & 3, (by >> 4) & 3, (by >> 2) & 3, by & 3], 1).reshape(-1)[:n]
        s = "".join("ACGT"[c] for c in codes)
        out.extend(s[i:i + k] for i in range(n - k + 1))
    return out


# ---- unitig cases -------------------------------------------------------------
_COMP = str.maketrans("ACGT", "TGCA")


def revcomp(s):
    return s.translate(_COMP)[::-1]


def spelled_path(unitigs, ref, k):
    """The unitigs that lie inside ref (either strand), ordered along it,
    when consecutive ones overlap by k - 1 bases and together cover ref from
    its first base to its last; else None."""
    placed = []
    for s in unitigs:
        for t in (s, revcomp(s)):
            i = ref.find(t)
            if i >= 0:
                placed.append((i, i + len(t)))
                break
    placed.sort()
    if not placed or placed[0][0] != 0 or placed[-1][1] != len(ref):
        return None
    for (a0, a1), (b0, b1) in zip(placed, placed[1:]):
        if b0 != a1 - (k - 1):
            return None
    return placed


def rand_seq(rng, n):
    return "".join("ACGT"[c] for c in rng.integers(0, 4, n))


def key_rows(strs, k):
    """Canonical k-mer strings -> (n, nlimbs(k)) u64 keys in Kmer256 limb order."""
    from oracle import pyref
    L = nlimbs(k)
    out = np.zeros((len(strs), L), dtype=np.uint64)
    for i, s in enumerate(strs):
        out[i] = pyref.limbs(pyref.k256_from_str(s, k))[:L]
    return out


def graph_sequences(rng, k):
    """Sequences whose k-mers make a graph with every shape the unitig walk
    meets: a genome with a repeat (two branch points each side), a tip (an
    error-like side branch), a bubble, a circle (an isolated cycle), a
    hairpin (a sequence followed by its own reverse complement) and a short
    isolated piece."""
    rep = rand_seq(rng, 2 * k)
    g = rand_seq(rng, 700) + rep + rand_seq(rng, 500) + rep + rand_seq(rng, 600)
    tip = g[300:300 + k + 5] + rand_seq(rng, 12)
    bub = g[900:900 + 3 * k]
    bub = bub[:k + 10] + ("A" if bub[k + 10] != "A" else "C") + bub[k + 11:]
    circle = rand_seq(rng, 400)
    circ_seq = circle + circle[:k - 1]
    h = rand_seq(rng, 90)
    hairpin = h + revcomp(h)
    piece = rand_seq(rng, k + 3)
    return [g, tip, bub, circ_seq, hairpin, piece], circle


def solid_from_sequences(seqs, k, rng):
    """Sorted canonical k-mer strings of the sequences with counts 2..60."""
    ks = set()
    for s in seqs:
        for i in range(len(s) - k + 1):
            w = s[i:i + k]
            ks.add(min(w, revcomp(w)))
    strs = sorted(ks)
    counts = rng.integers(2, 61, len(strs)).astype(np.uint32)
    return strs, counts


def reads_from(seqs, circle, rng, cov=30, rl=(90, 150)):
    """Error-free reads tiling every sequence, and the circle with reads that
    wrap around its end, at about cov-fold coverage; half of them reverse
    complemented."""
    out = []

    def take(s, n_start):
        for _ in range(max(1, cov * n_start // 120)):
            L = min(int(rng.integers(rl[0], rl[1] + 1)), len(s))
            st = int(rng.integers(0, min(n_start, len(s) - L + 1)))
            r = s[st:st + L]
            out.append(revcomp(r) if rng.integers(0, 2) else r)

    for s in seqs:
        take(s, len(s))
    take(circle + circle[:rl[1]], len(circle))
    return out


# ---- error-correction cases -------------------------------------------------
def correction_case(k, seed, genome_len=3000, n_reads=60, filter_bits=1 << 20):
    """A genome whose canonical k-mers are inserted twice (solid), plus reads
    drawn from it (either strand) with 0-4 substitutions, some of them
    adjacent or at the read ends; a few reads shorter than k and a few longer
    than 256 bases.  Returns (key list in insertion order as 4-limb rows,
    reads as strings)."""
    from oracle import pyref
    rng = np.random.default_rng(seed)
    g = rand_seq(rng, genome_len)
    keys = []
    for _ in range(2):
        for i in range(len(g) - k + 1):
            x = pyref.k256_canonical(pyref.k256_from_str(g[i:i + k], k), k)[0]
            keys.append(pyref.limbs(x))
    reads = []
    for j in range(n_reads):
        if j % 20 == 7:
            L = int(rng.integers(max(1, k - 10), k))          # shorter than k
        elif j % 20 == 11:
            L = int(rng.integers(300, 900))                   # several words
        else:
            L = int(rng.integers(k + 5, 200))
        L = min(L, len(g))
        st = int(rng.integers(0, len(g) - L + 1))
        r = list(g[st:st + L])
        ne = int(rng.integers(0, 5))
        for e in range(ne):
            if e == 1 and rng.integers(0, 3) == 0:
                p = min(L - 1, int(rng.integers(0, L)) + 1)  # may sit next to another error
            elif rng.integers(0, 6) == 0:
                p = int(rng.choice([0, L - 1]))               # read ends
            else:
                p = int(rng.integers(0, L))
            r[p] = "ACGT"[("ACGT".index(r[p]) + int(rng.integers(1, 4))) % 4]
        s = "".join(r)
        reads.append(revcomp(s) if rng.integers(0, 2) else s)
    return np.array(keys, dtype=np.uint64), reads


# ---- FASTQ / FASTA texts ---------------------------------------------------------
def fastq_text(seqs, rng, crlf=False, blank_between=False, plus_name=False):
    """A FASTQ text of the given sequences (bytes or str) with random qualities."""
    nl = b"\r\n" if crlf else b"\n"
    out = []
    for i, s in enumerate(seqs):
        s = s.encode() if isinstance(s, str) else bytes(s)
        q = bytes(rng.integers(35, 75, len(s)).astype(np.uint8).tolist())
        out.append(b"@read_%d/1" % i + nl + s + nl + (b"+read_%d" % i if plus_name else b"+") + nl + q + nl)
        if blank_between and i % 3 == 0:
            out.append(nl)
    return b"".join(out)


def fasta_text(seqs, width=60):
    out = []
    for i, s in enumerate(seqs):
        s = s.encode() if isinstance(s, str) else bytes(s)
        out.append(b">contig_%d some description\n" % i)
        for j in range(0, len(s), width):
            out.append(s[j:j + width] + b"\n")
    return b"".join(out)


def messy_reads(rng, n, genome=None):
    """Reads with every case the ingest gates meet: leading/trailing N runs,
    internal N (one or several, sub-reads short and long), all-N, lowercase,
    other IUPAC letters, lengths 0..400 (and a few of 2000)."""
    g = genome if genome is not None else rand_seq(rng, 20000)
    out = []
    for i in range(n):
        kind = i % 10
        L = int(rng.integers(0, 400)) if kind != 9 else 2000
        st = int(rng.integers(0, max(1, len(g) - L)))
        r = list(g[st:st + L])
        if kind == 1 and L:
            r[: int(rng.integers(1, 6))] = "N" * min(L, int(rng.integers(1, 6)))
        if kind == 2 and L:
            r[-int(rng.integers(1, 6)):] = "n" * min(L, int(rng.integers(1, 6)))
        if kind in (3, 4) and L > 2:
            for _ in range(1 if kind == 3 else int(rng.integers(2, 6))):
                r[int(rng.integers(0, L))] = "N"
        if kind == 5:
            r = ["N"] * L
        if kind == 6:
            r = [c.lower() if rng.integers(0, 2) else c for c in r]
        if kind == 7 and L:
            r[int(rng.integers(0, L))] = "RYKMSWBDHV"[int(rng.integers(0, 10))]
        out.append("".join(r))
    return out
