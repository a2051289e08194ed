"""Independent Python restatement of the spades-rs k-mer path (test infrastructure).

This module is the second, independent restatement that cross-checks the C++
oracle (``oracle/spk_oracle.cpp``).  It is deliberately written a different way:
reverse complements are computed on strings rather than with bit permutations,
and all arithmetic uses unbounded Python integers with explicit masking.  It is
used only by ``tests/`` and by ``tests/golden/make_golden.py``; nothing in the
product library imports it.

Citations are to the spades-rs sources (path:line).
"""
from __future__ import annotations

import numpy as np

M64 = (1 << 64) - 1
M128 = (1 << 128) - 1

# src/dna.rs:11-22
ASCII_TO_2BIT = {ord(c): v for c, v in zip("AaCcGgTt", (0, 0, 1, 1, 2, 2, 3, 3))}
BASES = "ACGT"
_COMP = {"A": "T", "C": "G", "G": "C", "T": "A"}

# src/bloom.rs:84-86
SEEDS = (0x517CC1B727220A95, 0x9E3779B97F4A7C15, 0x6C62272E07BB0142)


def base_to_2bit(b: int):
    """src/dna.rs:30-37 (None for non-ACGT)."""
    return ASCII_TO_2BIT.get(b)


def revcomp_str(s: str) -> str:
    """src/dna.rs:46-60 restricted to ACGT."""
    return "".join(_COMP[c] for c in reversed(s))


def string_to_kmer(s: bytes, k: int):
    """src/dna.rs:104-114."""
    if k == 0 or k > 32 or len(s) < k:
        return None
    v = 0
    for b in s[:k]:
        c = base_to_2bit(b)
        if c is None:
            return None
        v = (v << 2) | c
    return v


def kmer_to_string(v: int, k: int) -> str:
    """src/dna.rs:92-100."""
    k = min(k, 32)
    return "".join(BASES[(v >> (2 * (k - 1 - i))) & 3] for i in range(k))


def k256_from_str(s: str, k: int):
    """src/dna.rs:299-321: returns (lo, hi) or None."""
    if k == 0 or len(s) < k or k > 128:
        return None
    lo = hi = 0
    for i, ch in enumerate(s[:k]):
        c = ASCII_TO_2BIT.get(ord(ch))
        if c is None:
            return None
        if i < 64:
            lo = (lo << 2) | c
        else:
            hi = (hi << 2) | c
    return (lo, hi)


def k256_to_str(x, k: int) -> str:
    """src/dna.rs:274-295."""
    lo, hi = x
    if k <= 64:
        return "".join(BASES[(lo >> (2 * (k - 1 - i))) & 3] for i in range(k))
    a = "".join(BASES[(lo >> (2 * (63 - i))) & 3] for i in range(64))
    b = "".join(BASES[(hi >> (2 * (k - 1 - i))) & 3] for i in range(64, k))
    return a + b


def k256_revcomp(x, k: int):
    """src/dna.rs:152-180, computed on the string form."""
    return k256_from_str(revcomp_str(k256_to_str(x, k)), k)


def k256_canonical(x, k: int):
    """src/dna.rs:185-192: (canonical, is_rc); ties keep the forward strand."""
    rc = k256_revcomp(x, k)
    return (x, False) if x <= rc else (rc, True)


def k256_extend_right(x, b: int, k: int):
    """src/dna.rs:196-221."""
    return k256_from_str(k256_to_str(x, k)[1:] + BASES[b & 3], k)


def k256_prepend_left(x, a: int, k: int):
    """src/dna.rs:225-245."""
    return k256_from_str(BASES[a & 3] + k256_to_str(x, k)[:-1], k)


def limbs(x):
    """Kmer256 (lo, hi) -> the four u64 limbs hashed by bloom.rs:62-65."""
    lo, hi = x
    return (lo & M64, (lo >> 64) & M64, hi & M64, (hi >> 64) & M64)


def _rotl(v: int, r: int) -> int:
    return ((v << r) | (v >> (64 - r))) & M64


def hash_kmer256(x, seed: int) -> int:
    """src/bloom.rs:61-78 with unbounded ints masked to 64 bits."""
    w0, w1, w2, w3 = limbs(x)
    h = w0 ^ seed
    h = ((h ^ ((_rotl(w1, 21) * 0x9E3779B97F4A7C15) & M64)) * 0xFF51AFD7ED558CCD) & M64
    h ^= h >> 33
    h = ((h ^ ((_rotl(w2, 43) * 0xBF58476D1CE4E5B9) & M64)) * 0xC4CEB9FE1A85EC53) & M64
    h ^= h >> 33
    h = ((h ^ ((_rotl(w3, 11) * 0x94D049BB133111EB) & M64)) * 0xFF51AFD7ED558CCD) & M64
    h ^= h >> 33
    return h


def hash_batch_np(w: np.ndarray, seed: int) -> np.ndarray:
    """Vectorised bloom.rs:61-78 over an (n, 4) uint64 limb array (numpy wraps mod 2^64)."""
    w = np.asarray(w, dtype=np.uint64)
    with np.errstate(over="ignore"):
        def rotl(v, r):
            return (v << np.uint64(r)) | (v >> np.uint64(64 - r))
        s33 = np.uint64(33)
        x = w[:, 0] ^ np.uint64(seed)
        x = (x ^ (rotl(w[:, 1], 21) * np.uint64(0x9E3779B97F4A7C15))) * np.uint64(0xFF51AFD7ED558CCD)
        x ^= x >> s33
        x = (x ^ (rotl(w[:, 2], 43) * np.uint64(0xBF58476D1CE4E5B9))) * np.uint64(0xC4CEB9FE1A85EC53)
        x ^= x >> s33
        x = (x ^ (rotl(w[:, 3], 11) * np.uint64(0x94D049BB133111EB))) * np.uint64(0xFF51AFD7ED558CCD)
        x ^= x >> s33
    return x


class TwoTierFilter:
    """src/bloom.rs:13-131 (serial; Python ints as words)."""

    def __init__(self, capacity_bits: int):
        self.num_words = max((capacity_bits + 63) // 64, 1)   # bloom.rs:27
        self.size_bits = self.num_words * 64                   # bloom.rs:28
        self.seen = [0] * self.num_words
        self.solid = [0] * self.num_words

    def _pos(self, x):
        return [hash_kmer256(x, s) % self.size_bits for s in SEEDS]

    def insert_kmer256(self, x) -> bool:                       # bloom.rs:83-107
        prev = []
        pos = self._pos(x)
        for h in pos:
            w, b = divmod(h, 64)
            prev.append((self.seen[w] >> b) & 1)
            self.seen[w] |= 1 << b
        if all(prev):
            for h in pos:
                w, b = divmod(h, 64)
                self.solid[w] |= 1 << b
            return True
        return False

    def insert_twice(self, x) -> bool:
        """Order-free twice tier: a seen fetch_or that finds its bit set also sets it here."""
        allp = True
        for h in self._pos(x):
            w, b = divmod(h, 64)
            if (self.seen[w] >> b) & 1:
                self.solid[w] |= 1 << b
            else:
                allp = False
            self.seen[w] |= 1 << b
        return allp

    def is_solid_kmer256(self, x) -> bool:                     # bloom.rs:111-126
        return all((self.solid[h // 64] >> (h % 64)) & 1 for h in self._pos(x))

    def insert(self, v: int) -> bool:                          # bloom.rs:48-50
        return self.insert_kmer256((v & M128, 0))

    def is_solid(self, v: int) -> bool:                        # bloom.rs:54-56
        return self.is_solid_kmer256((v & M128, 0))

    def memory_usage_bytes(self) -> int:                       # bloom.rs:129-131
        return self.num_words * 8 * 2


def correct_read(seq: str, k: int, filt: TwoTierFilter):
    """src/hammer.rs:34-121 on a string read against filt's solid tier:
    (corrected read, changed).  Written over strings with a memo of window
    solidity (the filter does not change during a correction)."""
    if k == 0 or k > 128 or len(seq) < k:
        return seq, False
    memo = {}

    def solid(w: str) -> bool:
        if w not in memo:
            x = k256_from_str(w, k)
            memo[w] = x is not None and filt.is_solid_kmer256(k256_canonical(x, k)[0])
        return memo[w]

    cur = list(seq)
    changed = False
    n = len(cur)
    for i in range(n - k + 1):
        win = "".join(cur[i:i + k])
        if k256_from_str(win, k) is None or solid(win):
            continue
        best, best_gain = None, 0
        for off in range(k):
            pos = i + off
            lo, hi = max(pos - (k - 1), 0), min(pos, n - k)
            others = [s for s in range(lo, hi + 1) if s != i]
            base = sum(solid("".join(cur[s:s + k])) for s in others)
            orig = cur[pos]
            for c in "ACGT":
                if c == orig.upper():
                    continue
                cur[pos] = c
                if solid("".join(cur[i:i + k])):
                    cnt = 1 + sum(solid("".join(cur[s:s + k])) for s in others)
                    gain = max(cnt - base, 0)
                    if gain > best_gain:
                        best, best_gain = (pos, c), gain
                cur[pos] = orig
        if best is not None:
            cur[best[0]] = best[1]
            changed = True
    return "".join(cur), changed


def pack_reads(reads):
    """src/packed_reads.rs:547-578 for a list of clean ACGT strings -> (data, offsets, lengths)."""
    data = bytearray()
    offsets, lengths = [], []
    for r in reads:
        offsets.append(len(data))
        byte, shift, n = 0, 6, 0
        for ch in r:
            c = ASCII_TO_2BIT.get(ord(ch))
            if c is None:
                continue
            n += 1
            byte |= c << shift
            if shift == 0:
                data.append(byte)
                byte, shift = 0, 6
            else:
                shift -= 2
        if shift != 6:
            data.append(byte)
        lengths.append(n)
    return bytes(data), offsets, lengths


def get_read(data, offsets, lengths, idx) -> str:
    """src/packed_reads.rs:592-613."""
    n = lengths[idx]
    o = offsets[idx]
    return "".join(BASES[(data[o + i // 4] >> (6 - 2 * (i % 4))) & 3] for i in range(n))


def count_serial(reads, k: int, bloom_bits: int, mode: str = "ref"):
    """src/assemble.rs:129-242 on decoded reads, serial order.

    Returns (counts dict canonical->count, filter).  mode 'ref' uses the
    reference TwoTierFilter; mode 'twice' uses the order-free twice tier.
    """
    f = TwoTierFilter(bloom_bits)
    ins = f.insert_kmer256 if mode == "ref" else f.insert_twice
    cans = []
    for r in reads:
        if len(r) < k:
            continue
        rc_r = revcomp_str(r)
        L = len(r)
        for i in range(L - k + 1):
            fw = r[i:i + k]
            rv = rc_r[L - i - k:L - i]
            a, b = k256_from_str(fw, k), k256_from_str(rv, k)
            cans.append(a if a <= b else b)
    for c in cans:
        ins(c)
    counts = {}
    for c in cans:
        if f.is_solid_kmer256(c):
            counts[c] = counts.get(c, 0) + 1
    return counts, f


def determine_solid_kmer_cutoff(counts, min_coverage: float) -> int:
    """src/assemble.rs:692-735."""
    if min_coverage > 5.0:
        return int(max(min_coverage * 0.35, 2.0))
    s = sorted(counts)
    if len(s) <= 100:
        return 2
    top = s[len(s) * 95 // 100]
    if top < 30:
        return 2
    mvs = min(max(top // 4, 10), 35)
    hist = [0] * (mvs + 1)
    for c in s:
        if c <= mvs:
            hist[c] += 1
    valley, min_val, found = 2, None, False
    for c in range(2, mvs + 1):
        h = hist[c]
        if min_val is None or h <= min_val:
            min_val, valley = h, c
        elif h > min_val * 2 and c > valley + 2:
            found = True
            break
    return valley if found else 2


def edges(solid, k: int):
    """src/graph.rs:78-102: canonical (k+1)-mers s+b over both orientations of every solid s."""
    sset = set(solid)
    out = set()
    for s in solid:
        st = k256_to_str(s, k)
        for ex in (st, revcomp_str(st)):
            for b in BASES:
                nx = k256_from_str(ex[1:] + b, k)
                nc, _ = k256_canonical(nx, k)
                if nc in sset:
                    e = ex + b
                    re = revcomp_str(e)
                    out.add(k256_from_str(min(e, re, key=lambda z: k256_from_str(z, k + 1)), k + 1))
    return sorted(out)


def unitigs(solid_strs, counts, k: int):
    """CompactedGraph::build (src/graph.rs:65-235) on string k-mers.

    solid_strs: the canonical solid k-mers as strings, sorted (string order is
    the 2-bit value order); counts: their counts.  The walk follows the
    reference step by step on oriented k-mers (kmer, is_rc): pass 1 starts at
    k-mers with an orientation that has no unique unvisited predecessor of
    out-degree one (:183-216), pass 2 takes what is left, i.e. isolated cycles
    (:219-231).  Returns (sequences, mean coverages, k-mer counts), each
    sequence in the orientation not greater than its reverse complement, sorted
    by sequence (the reference's own order follows its hash-set iteration)."""
    idx = {s: i for i, s in enumerate(solid_strs)}

    def explicit(o):  # :24-30
        return revcomp_str(o[0]) if o[1] else o[0]

    def canon(x):  # src/dna.rs:185-192
        r = revcomp_str(x)
        return (x, False) if x <= r else (r, True)

    def succs(o):  # :78-90
        e = explicit(o)
        return [c for c in (canon(e[1:] + b) for b in BASES) if c[0] in idx]

    def preds(o):  # :91-102
        e = explicit(o)
        return [c for c in (canon(a + e[:-1]) for a in BASES) if c[0] in idx]

    visited = set()

    def extract(start):  # :104-157
        path, curr = [], start
        while curr[0] not in visited:
            visited.add(curr[0])
            path.append(curr)
            sc = succs(curr)
            if len(sc) != 1:
                break
            nx = sc[0]
            if nx[0] in visited or len(preds(nx)) != 1:
                break
            curr = nx
        if not path:
            return path
        back, bc = [], path[0]
        while True:
            pr = preds(bc)
            if len(pr) != 1:
                break
            pv = pr[0]
            if pv[0] in visited or len(succs(pv)) != 1:
                break
            visited.add(pv[0])
            back.append(pv)
            bc = pv
        return back[::-1] + path

    out = []

    def build(path):  # :159-177
        seq = explicit(path[0]) + "".join(explicit(o)[-1] for o in path[1:])
        cov = sum(int(counts[idx[o[0]]]) for o in path)
        out.append((seq, cov / len(path), len(path)))

    for km in solid_strs:  # pass 1
        if km in visited:
            continue
        start = (km, False)
        pf, pr = preds((km, False)), preds((km, True))
        if len(pf) == 1 and len(succs(pf[0])) == 1 and pf[0][0] not in visited:
            if len(pr) == 1 and len(succs(pr[0])) == 1 and pr[0][0] not in visited:
                continue
            start = (km, True)
        p = extract(start)
        if p:
            build(p)
    for km in solid_strs:  # pass 2
        if km not in visited:
            p = extract((km, False))
            if p:
                build(p)
    norm = [(min(s, revcomp_str(s)), c, n) for s, c, n in out]
    norm.sort(key=lambda t: t[0])
    return [t[0] for t in norm], [t[1] for t in norm], [t[2] for t in norm]


MIN_K = 21  # src/packed_reads.rs:38


def trim_n_ends(r: str) -> str:
    """src/packed_reads.rs:635-648."""
    ok = [i for i, c in enumerate(r) if ord(c) in ASCII_TO_2BIT]
    return r[ok[0]:ok[-1] + 1] if ok else ""


def split_on_n(r: str):
    """src/packed_reads.rs:659-662: maximal ACGT runs."""
    out, cur = [], []
    for c in r:
        if ord(c) in ASCII_TO_2BIT:
            cur.append(c)
        elif cur:
            out.append("".join(cur))
            cur = []
    if cur:
        out.append("".join(cur))
    return out


def from_paired_slices(r1, r2):
    """src/packed_reads.rs:438-461, 481-489, 668-690, 521-540.

    Returns (reads in store order, pe_count, sidecar count).
    """
    b1, b2, b3, side = [], [], [], 0

    def unpaired(t):
        nonlocal side
        if not t:
            return
        segs = [s for s in split_on_n(t) if len(s) >= MIN_K]
        b3.extend(segs)
        if not segs:
            side += 1

    common = min(len(r1), len(r2))
    for a, b in zip(r1[:common], r2[:common]):
        t1, t2 = trim_n_ends(a), trim_n_ends(b)
        n1 = any(ord(c) not in ASCII_TO_2BIT for c in t1)
        n2 = any(ord(c) not in ASCII_TO_2BIT for c in t2)
        if not n1 and not n2 and len(t1) >= MIN_K and len(t2) >= MIN_K:
            b1.append(t1)
            b2.append(t2)
        else:
            unpaired(t1)
            unpaired(t2)
    for r in list(r1[common:]) + list(r2[common:]):
        unpaired(trim_n_ends(r))
    return b1 + b2 + b3, len(b1), side


def fastx_records(text: bytes):
    """FastxReader::open + next_seq (src/packed_reads.rs:69-234) on a
    decompressed text: the record sequences as bytes.  Raises ValueError on a
    malformed text.  Written over a list of lines (the Rust reader streams)."""
    raw = text.split(b"\n")
    if raw and raw[-1] == b"":
        raw.pop()  # a final '\n' ends the last line; it does not start another
    lines = [(r, r.rstrip(b"\r\n")) for r in raw]
    i = 0
    ws = b" \t\r\x0c"
    while i < len(lines) and all(c in ws for c in lines[i][0]):
        i += 1  # open(): blank or whitespace-only leading lines
    if i == len(lines):
        return []
    first = lines[i][0][:1]
    out = []
    if first == b"@":
        while i < len(lines):
            if lines[i][1] == b"":
                i += 1
                continue
            if not lines[i][1].startswith(b"@"):
                raise ValueError("expected '@' header")
            if i + 1 >= len(lines):
                raise ValueError("unexpected EOF waiting for sequence line")
            seq = lines[i + 1][1]
            if i + 2 >= len(lines):
                raise ValueError("unexpected EOF waiting for '+' separator")
            if not lines[i + 2][0].startswith(b"+"):
                raise ValueError("expected '+' separator line")
            if i + 3 >= len(lines):
                raise ValueError("unexpected EOF waiting for quality scores")
            if len(lines[i + 3][1]) != len(seq):
                raise ValueError("sequence length != quality length")
            out.append(seq)
            i += 4
        return out
    if first != b">":
        raise ValueError("expected '@' or '>' header")
    i += 1
    cur = b""
    while i < len(lines):
        c = lines[i][1]
        if c.startswith(b">"):
            out.append(cur)
            cur = b""
        else:
            cur += c
        i += 1
    if cur:
        out.append(cur)
    return out


def read_fastq_gz(path):
    """Sequence lines of a (gzipped) FASTQ file (src/packed_reads.rs:141-216, no validation)."""
    import gzip
    out = []
    with gzip.open(path, "rt") as f:
        lines = [l.rstrip("\r\n") for l in f]
    i = 0
    while i + 3 < len(lines) + 1 and i < len(lines):
        if not lines[i]:
            i += 1
            continue
        out.append(lines[i + 1])
        i += 4
    return out
