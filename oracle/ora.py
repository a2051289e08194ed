"""ctypes wrapper of the C++ CPU oracle (``oracle/liboracle.so``).

TEST INFRASTRUCTURE ONLY: used by ``tests/``, the smoke check and the
CPU-baseline leg of ``bench.py`` as the checker / reported baseline.  The
product library never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

u64p = C.POINTER(C.c_uint64)
u32p = C.POINTER(C.c_uint32)
u8p = C.POINTER(C.c_uint8)

MODE_REF = 0
MODE_TWICE = 1


def build() -> str:
    """Compile liboracle.so with the committed Makefile (gcc only)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return os.path.join(_HERE, "liboracle.so")


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.ora_hash_kmer256.restype = C.c_uint64
        L.ora_hash_kmer256.argtypes = [u64p, C.c_uint64]
        L.ora_hash_batch.argtypes = [u64p, C.c_size_t, C.c_uint64, u64p]
        L.ora_revcomp_u64.restype = C.c_uint64
        L.ora_revcomp_u64.argtypes = [C.c_uint64, C.c_uint]
        L.ora_canonical_u64.restype = C.c_uint64
        L.ora_canonical_u64.argtypes = [C.c_uint64, C.c_uint, C.POINTER(C.c_int)]
        L.ora_string_to_kmer.argtypes = [C.c_char_p, C.c_size_t, C.c_uint, u64p]
        L.ora_k256_from_bytes.argtypes = [C.c_char_p, C.c_size_t, C.c_uint, u64p]
        L.ora_k256_to_string.argtypes = [u64p, C.c_uint, C.c_char_p]
        L.ora_k256_revcomp.argtypes = [u64p, C.c_uint, u64p]
        L.ora_k256_canonical.argtypes = [u64p, C.c_uint, u64p]
        L.ora_k256_extend_right.argtypes = [u64p, C.c_uint8, C.c_uint, u64p]
        L.ora_k256_prepend_left.argtypes = [u64p, C.c_uint8, C.c_uint, u64p]
        L.ora_bloom_new.restype = C.c_void_p
        L.ora_bloom_new.argtypes = [C.c_uint64]
        L.ora_bloom_free.argtypes = [C.c_void_p]
        for n in ("ora_bloom_size_bits", "ora_bloom_num_words", "ora_bloom_memory_usage_bytes"):
            getattr(L, n).restype = C.c_uint64
            getattr(L, n).argtypes = [C.c_void_p]
        L.ora_bloom_insert_k256.argtypes = [C.c_void_p, u64p]
        L.ora_bloom_is_solid_k256.argtypes = [C.c_void_p, u64p]
        L.ora_bloom_insert_u64.argtypes = [C.c_void_p, C.c_uint64]
        L.ora_bloom_is_solid_u64.argtypes = [C.c_void_p, C.c_uint64]
        L.ora_bloom_download.argtypes = [C.c_void_p, u64p, u64p]
        L.ora_packed_new.restype = C.c_void_p
        L.ora_packed_free.argtypes = [C.c_void_p]
        L.ora_packed_pack_clean.argtypes = [C.c_void_p, C.c_char_p, C.c_size_t]
        L.ora_packed_ingest_read.argtypes = [C.c_void_p, C.c_char_p, C.c_size_t]
        L.ora_packed_from_paired.restype = C.c_void_p
        L.ora_packed_from_paired.argtypes = [C.c_char_p, u64p, C.c_size_t, C.c_char_p, u64p, C.c_size_t]
        L.ora_packed_sizes.argtypes = [C.c_void_p, u64p, u64p, u64p, u64p]
        L.ora_packed_copy.argtypes = [C.c_void_p, u8p, u64p, u32p]
        L.ora_packed_get_read.restype = C.c_size_t
        L.ora_packed_get_read.argtypes = [C.c_void_p, C.c_size_t, C.c_char_p]
        L.ora_count.restype = C.c_void_p
        L.ora_count.argtypes = [u8p, C.c_size_t, u64p, u32p, C.c_size_t, C.c_uint, C.c_uint64,
                                C.c_int, C.c_int, C.c_int]
        L.ora_count_free.argtypes = [C.c_void_p]
        L.ora_unitigs.restype = C.c_void_p
        L.ora_unitigs.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_uint]
        L.ora_unitigs_count.restype = C.c_size_t
        L.ora_unitigs_count.argtypes = [C.c_void_p]
        L.ora_unitigs_bases.restype = C.c_size_t
        L.ora_unitigs_bases.argtypes = [C.c_void_p]
        L.ora_unitigs_get.restype = None
        L.ora_unitigs_get.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ora_unitigs_free.restype = None
        L.ora_unitigs_free.argtypes = [C.c_void_p]
        L.ora_packed_from_texts.restype = C.c_void_p
        L.ora_packed_from_texts.argtypes = [C.c_char_p, C.c_size_t, C.c_char_p, C.c_size_t, C.c_char_p]
        L.ora_packed_sidecar_get.restype = C.c_size_t
        L.ora_packed_sidecar_get.argtypes = [C.c_void_p, C.c_size_t, C.c_char_p]
        L.ora_count_sample3.restype = C.c_void_p
        L.ora_count_sample3.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p, C.c_size_t, C.c_uint,
                                        C.c_uint64, C.c_int, C.c_int, C.c_size_t]
        L.ora_bloom_load.restype = None
        L.ora_bloom_load.argtypes = [C.c_void_p, u64p, u64p]
        L.ora_correct_ascii.restype = C.c_int
        L.ora_correct_ascii.argtypes = [C.c_void_p, C.c_uint, C.c_char_p, C.c_size_t]
        L.ora_correct_packed.restype = C.c_size_t
        L.ora_correct_packed.argtypes = [C.c_void_p, C.c_uint, C.c_void_p, C.c_size_t, C.c_void_p,
                                         C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p]
        L.ora_count_inject_priors.restype = None
        L.ora_count_inject_priors.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                              C.c_size_t, C.c_uint, C.c_uint32]
        L.ora_count_size.restype = C.c_size_t
        L.ora_count_size.argtypes = [C.c_void_p, C.c_uint32]
        L.ora_count_table.restype = C.c_size_t
        L.ora_count_table.argtypes = [C.c_void_p, C.c_uint, C.c_uint32, u64p, u32p]
        L.ora_count_bloom_words.restype = C.c_size_t
        L.ora_count_bloom_words.argtypes = [C.c_void_p]
        L.ora_count_bloom.argtypes = [C.c_void_p, u64p, u64p]
        L.ora_count_stats.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        L.ora_cutoff.restype = C.c_uint32
        L.ora_cutoff.argtypes = [u32p, C.c_size_t, C.c_double]
        L.ora_edges.restype = C.c_size_t
        L.ora_edges.argtypes = [u64p, C.c_size_t, C.c_uint, C.POINTER(u64p)]
        L.ora_free.argtypes = [C.c_void_p]
        L.ora_shard_bloom.restype = None
        L.ora_shard_bloom.argtypes = [u8p, C.c_size_t, u64p, u32p, C.c_size_t, C.c_uint, C.c_uint64,
                                      C.c_uint64, C.c_uint64, u64p, u64p]
        L.ora_shard_count.restype = C.c_void_p
        L.ora_shard_count.argtypes = [u8p, C.c_size_t, u64p, u32p, C.c_size_t, C.c_uint, C.c_uint64, u64p,
                                      C.c_uint, C.c_uint]
        _LIB = L
    return _LIB


def _p(a, t):
    return a.ctypes.data_as(t)


def nlimbs(k: int) -> int:
    return (k + 31) // 32


def to4(x):
    """Kmer256 (lo, hi) python ints -> 4-limb uint64 array."""
    lo, hi = x
    M = (1 << 64) - 1
    return np.array([lo & M, lo >> 64 & M, hi & M, hi >> 64 & M], dtype=np.uint64)


def from_limbs(row) -> tuple:
    w = [int(v) for v in row] + [0] * (4 - len(row))
    return (w[0] | (w[1] << 64), w[2] | (w[3] << 64))


def hash_kmer256(x, seed: int) -> int:
    a = to4(x)
    return int(lib().ora_hash_kmer256(_p(a, u64p), C.c_uint64(seed)))


def hash_batch(w4: np.ndarray, seed: int) -> np.ndarray:
    w4 = np.ascontiguousarray(w4, dtype=np.uint64)
    out = np.empty(w4.shape[0], dtype=np.uint64)
    lib().ora_hash_batch(_p(w4, u64p), w4.shape[0], C.c_uint64(seed), _p(out, u64p))
    return out


def _k256_call(fn, x, k, *extra):
    a = to4(x)
    o = np.zeros(4, dtype=np.uint64)
    r = fn(_p(a, u64p), *extra, C.c_uint(k), _p(o, u64p)) if extra else fn(_p(a, u64p), C.c_uint(k), _p(o, u64p))
    return from_limbs(o), r


def k256_from_bytes(s: bytes, k: int):
    o = np.zeros(4, dtype=np.uint64)
    ok = lib().ora_k256_from_bytes(s, len(s), k, _p(o, u64p))
    return from_limbs(o) if ok else None


def k256_to_string(x, k: int) -> str:
    a = to4(x)
    buf = C.create_string_buffer(k)
    lib().ora_k256_to_string(_p(a, u64p), k, buf)
    return buf.raw[:k].decode()


def k256_revcomp(x, k):
    return _k256_call(lib().ora_k256_revcomp, x, k)[0]


def k256_canonical(x, k):
    v, r = _k256_call(lib().ora_k256_canonical, x, k)
    return v, bool(r)


def k256_extend_right(x, b, k):
    a = to4(x)
    o = np.zeros(4, dtype=np.uint64)
    lib().ora_k256_extend_right(_p(a, u64p), b, k, _p(o, u64p))
    return from_limbs(o)


def k256_prepend_left(x, b, k):
    a = to4(x)
    o = np.zeros(4, dtype=np.uint64)
    lib().ora_k256_prepend_left(_p(a, u64p), b, k, _p(o, u64p))
    return from_limbs(o)


class Bloom:
    """TwoTierFilter (bloom.rs:13-131) in the C++ oracle."""

    def __init__(self, capacity_bits: int):
        self.h = lib().ora_bloom_new(capacity_bits)

    def __del__(self):
        if getattr(self, "h", None):
            lib().ora_bloom_free(self.h)
            self.h = None

    @property
    def size_bits(self):
        return lib().ora_bloom_size_bits(self.h)

    @property
    def num_words(self):
        return lib().ora_bloom_num_words(self.h)

    def memory_usage_bytes(self):
        return lib().ora_bloom_memory_usage_bytes(self.h)

    def insert(self, v: int) -> bool:
        return bool(lib().ora_bloom_insert_u64(self.h, v))

    def is_solid(self, v: int) -> bool:
        return bool(lib().ora_bloom_is_solid_u64(self.h, v))

    def insert_kmer256(self, x) -> bool:
        a = to4(x)
        return bool(lib().ora_bloom_insert_k256(self.h, _p(a, u64p)))

    def is_solid_kmer256(self, x) -> bool:
        a = to4(x)
        return bool(lib().ora_bloom_is_solid_k256(self.h, _p(a, u64p)))

    def download(self):
        n = self.num_words
        seen = np.zeros(n, dtype=np.uint64)
        solid = np.zeros(n, dtype=np.uint64)
        lib().ora_bloom_download(self.h, _p(seen, u64p), _p(solid, u64p))
        return seen, solid

    def load(self, seen=None, solid=None):
        """Overwrite the tiers with word arrays of num_words u64 each."""
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.uint64) for a in (seen, solid)]
        for a in arrs:
            assert a is None or a.size == self.num_words
        lib().ora_bloom_load(self.h, *[None if a is None else _p(a, u64p) for a in arrs])

    def correct_read(self, k: int, seq: str):
        """ErrorCorrector::correct_read_in_place (hammer.rs:34-121): (read, changed)."""
        b = C.create_string_buffer(seq.encode(), len(seq))
        m = lib().ora_correct_ascii(self.h, k, b, len(seq))
        return b.raw[: len(seq)].decode(), bool(m)

    def correct_packed(self, k: int, data, offsets, lengths):
        """Every packed read corrected as Stage 3 does (assemble.rs:183-191):
        (corrected packed data, per-read flags uint8, number corrected)."""
        d = np.ascontiguousarray(data, dtype=np.uint8)
        o = np.ascontiguousarray(offsets, dtype=np.uint64)
        ln = np.ascontiguousarray(lengths, dtype=np.uint32)
        out = np.zeros(max(d.size, 1), dtype=np.uint8)
        fl = np.zeros(max(ln.size, 1), dtype=np.uint8)
        nc = lib().ora_correct_packed(self.h, k, d.ctypes.data, d.size, o.ctypes.data, ln.ctypes.data,
                                      ln.size, out.ctypes.data, fl.ctypes.data)
        return out[: d.size], fl[: ln.size], int(nc)


class Packed:
    """PackedReads (packed_reads.rs:42-59) built by the oracle's ingest restatement."""

    def __init__(self, h=None):
        self.h = h if h is not None else lib().ora_packed_new()

    def __del__(self):
        if getattr(self, "h", None):
            lib().ora_packed_free(self.h)
            self.h = None

    @staticmethod
    def from_paired(r1, r2):
        def cat(rs):
            bs = [r.encode() if isinstance(r, str) else bytes(r) for r in rs]
            lens = np.array([len(b) for b in bs], dtype=np.uint64)
            return b"".join(bs), lens
        a, la = cat(r1)
        b, lb = cat(r2)
        la = la if la.size else np.zeros(1, np.uint64)
        lb = lb if lb.size else np.zeros(1, np.uint64)
        return Packed(lib().ora_packed_from_paired(a, _p(la, u64p), len(r1), b, _p(lb, u64p), len(r2)))

    @staticmethod
    def from_texts(t1: bytes, t2: bytes = None):
        """FASTQ/FASTA texts (decompressed) as from_paired_files (two texts) or
        append_from_file on an empty store (one text), packed_reads.rs:300-504.
        Raises ValueError for a malformed text."""
        err = C.create_string_buffer(256)
        h = lib().ora_packed_from_texts(t1, len(t1), t2, len(t2) if t2 is not None else 0, err)
        if not h:
            raise ValueError(err.value.decode())
        return Packed(h)

    def sidecar(self):
        out = []
        for i in range(self.sizes()["n_sidecar"]):
            n = lib().ora_packed_sidecar_get(self.h, i, None)
            buf = C.create_string_buffer(max(n, 1))
            lib().ora_packed_sidecar_get(self.h, i, buf)
            out.append(buf.raw[:n])
        return out

    def pack_clean(self, s):
        s = s.encode() if isinstance(s, str) else bytes(s)
        lib().ora_packed_pack_clean(self.h, s, len(s))

    def ingest_read(self, s):
        s = s.encode() if isinstance(s, str) else bytes(s)
        lib().ora_packed_ingest_read(self.h, s, len(s))

    def sizes(self):
        v = [C.c_uint64() for _ in range(4)]
        lib().ora_packed_sizes(self.h, *[C.byref(x) for x in v])
        return dict(n_reads=v[0].value, data_len=v[1].value, pe_count=v[2].value, n_sidecar=v[3].value)

    def arrays(self):
        s = self.sizes()
        data = np.zeros(max(s["data_len"], 1), dtype=np.uint8)
        offs = np.zeros(max(s["n_reads"], 1), dtype=np.uint64)
        lens = np.zeros(max(s["n_reads"], 1), dtype=np.uint32)
        lib().ora_packed_copy(self.h, _p(data, u8p), _p(offs, u64p), _p(lens, u32p))
        return data[: s["data_len"]], offs[: s["n_reads"]], lens[: s["n_reads"]]

    def get_read(self, idx: int) -> str:
        n = self.arrays()[2][idx]
        buf = C.create_string_buffer(int(n) + 1)
        m = lib().ora_packed_get_read(self.h, idx, buf)
        return buf.raw[:m].decode()


class CountResult:
    """Output of assemble.rs:129-242 restated: the admitted table, Bloom tiers and stats."""

    def __init__(self, h, k):
        self.h, self.k = h, k

    def __del__(self):
        if getattr(self, "h", None):
            lib().ora_count_free(self.h)
            self.h = None

    def inject_priors(self, priors, boost: int):
        """src/assemble.rs:267-283 on this table: every accepted k-window of every
        prior contig (ASCII bytes) adds `boost` to its canonical k-mer."""
        seqs = [bytes(p) for p in priors]
        if not seqs:
            return
        buf = np.frombuffer(b"".join(seqs) or b"\0", dtype=np.uint8).copy()
        lens = np.array([len(p) for p in seqs], dtype=np.uint32)
        offs = np.concatenate([[0], np.cumsum(lens.astype(np.uint64))[:-1]]).astype(np.uint64)
        lib().ora_count_inject_priors(self.h, buf.ctypes.data, offs.ctypes.data, lens.ctypes.data,
                                      len(seqs), self.k, boost)

    def table(self, min_count: int = 1):
        n = lib().ora_count_size(self.h, min_count)
        L = nlimbs(self.k)
        keys = np.zeros((max(n, 1), L), dtype=np.uint64)
        counts = np.zeros(max(n, 1), dtype=np.uint32)
        lib().ora_count_table(self.h, self.k, min_count, _p(keys, u64p), _p(counts, u32p))
        return keys[:n], counts[:n]

    def bloom(self):
        n = lib().ora_count_bloom_words(self.h)
        seen = np.zeros(max(n, 1), dtype=np.uint64)
        solid = np.zeros(max(n, 1), dtype=np.uint64)
        lib().ora_count_bloom(self.h, _p(seen, u64p), _p(solid, u64p))
        return seen[:n], solid[:n]

    def stats(self):
        o = (C.c_double * 6)()
        lib().ora_count_stats(self.h, o)
        return dict(occurrences=int(o[0]), admitted_occurrences=int(o[1]),
                    seconds_stage2=o[2], seconds_stage3=o[3], seconds_total=o[4],
                    corrected_reads=int(o[5]))


def count(data, offsets, lengths, k: int, bloom_bits: int, mode: int = MODE_TWICE,
          threads: int = 0, keep_bloom: bool = True, correct: bool = False) -> CountResult:
    """assemble.rs:129-242.  correct: the error-correcting Stage 3
    (config.error_correct, :183-191)."""
    if correct:
        mode |= 0x100
    data = np.ascontiguousarray(data, dtype=np.uint8)
    offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
    lengths = np.ascontiguousarray(lengths, dtype=np.uint32)
    d = data if data.size else np.zeros(1, np.uint8)
    o = offsets if offsets.size else np.zeros(1, np.uint64)
    ln = lengths if lengths.size else np.zeros(1, np.uint32)
    h = lib().ora_count(_p(d, u8p), data.size, _p(o, u64p), _p(ln, u32p), lengths.size, k,
                        C.c_uint64(bloom_bits), mode, threads, 1 if keep_bloom else 0)
    return CountResult(h, k)


def count_sample3(data, offsets, lengths, k: int, bloom_bits: int, threads: int, stage3_reads: int,
                  mode: int = MODE_REF, correct: bool = True) -> CountResult:
    """The threaded count (Stage 2 over every read) with Stage 3 over the first
    stage3_reads reads only; stats() times both stages."""
    d = np.ascontiguousarray(data, dtype=np.uint8)
    o = np.ascontiguousarray(offsets, dtype=np.uint64)
    ln = np.ascontiguousarray(lengths, dtype=np.uint32)
    h = lib().ora_count_sample3(d.ctypes.data, d.size, o.ctypes.data, ln.ctypes.data, ln.size, k,
                                bloom_bits, mode | (0x100 if correct else 0), threads, stage3_reads)
    return CountResult(h, k)


def cutoff(counts, min_coverage: float) -> int:
    c = np.ascontiguousarray(counts, dtype=np.uint32)
    cc = c if c.size else np.zeros(1, np.uint32)
    return int(lib().ora_cutoff(_p(cc, u32p), c.size, C.c_double(min_coverage)))


def unitigs(solid_keys: np.ndarray, counts: np.ndarray, k: int):
    """CompactedGraph::build (src/graph.rs:65-235) on a sorted solid list:
    (sequences as a list of str, mean coverage float64[n], k-mer counts
    uint64[n]), each unitig in the orientation not greater than its reverse
    complement, sorted by sequence."""
    keys = np.ascontiguousarray(solid_keys, dtype=np.uint64)
    cnt = np.ascontiguousarray(counts, dtype=np.uint32)
    h = lib().ora_unitigs(keys.ctypes.data, cnt.ctypes.data, cnt.size, k)
    try:
        n = lib().ora_unitigs_count(h)
        nb = lib().ora_unitigs_bases(h)
        buf = np.zeros(max(nb, 1), dtype=np.uint8)
        lens = np.zeros(max(n, 1), dtype=np.uint64)
        cov = np.zeros(max(n, 1), dtype=np.float64)
        km = np.zeros(max(n, 1), dtype=np.uint64)
        lib().ora_unitigs_get(h, buf.ctypes.data, lens.ctypes.data, cov.ctypes.data, km.ctypes.data)
    finally:
        lib().ora_unitigs_free(h)
    seqs, o = [], 0
    for ln in lens[:n]:
        seqs.append(buf[o:o + int(ln)].tobytes().decode())
        o += int(ln)
    return seqs, cov[:n], km[:n]


def edges(solid_keys: np.ndarray, k: int) -> np.ndarray:
    s = np.ascontiguousarray(solid_keys, dtype=np.uint64)
    if s.size == 0:
        return np.zeros((0, nlimbs(k + 1)), dtype=np.uint64)
    out = u64p()
    n = lib().ora_edges(_p(s, u64p), s.shape[0], k, C.byref(out))
    Le = nlimbs(k + 1)
    arr = np.ctypeslib.as_array(out, shape=(max(n, 1) * Le,)).copy()[: n * Le].reshape(n, Le)
    lib().ora_free(out)
    return arr


def shard_words(num_words: int, rank: int, world: int):
    """Bloom words [lo, hi) of one rank in the sharded design."""
    return num_words * rank // world, num_words * (rank + 1) // world


def shard_bloom(data, offsets, lengths, k: int, bloom_bits: int, rank: int, world: int):
    """Phase 1 of one rank: the seen and twice words of its word range."""
    num_words = max((bloom_bits + 63) // 64, 1)
    lo, hi = shard_words(num_words, rank, world)
    d = np.ascontiguousarray(data, dtype=np.uint8)
    o = np.ascontiguousarray(offsets, dtype=np.uint64)
    ln = np.ascontiguousarray(lengths, dtype=np.uint32)
    seen = np.zeros(max(hi - lo, 1), dtype=np.uint64)
    twice = np.zeros(max(hi - lo, 1), dtype=np.uint64)
    lib().ora_shard_bloom(_p(d, u8p), d.size, _p(o, u64p), _p(ln, u32p), ln.size, k, C.c_uint64(bloom_bits),
                          lo, hi, _p(seen, u64p), _p(twice, u64p))
    return seen[: hi - lo], twice[: hi - lo]


def shard_count(data, offsets, lengths, k: int, bloom_bits: int, twice, rank: int, world: int):
    """Phase 2 of one rank: its own k-mers counted and admitted against the
    gathered twice tier; (keys, counts) sorted."""
    d = np.ascontiguousarray(data, dtype=np.uint8)
    o = np.ascontiguousarray(offsets, dtype=np.uint64)
    ln = np.ascontiguousarray(lengths, dtype=np.uint32)
    tw = np.ascontiguousarray(twice, dtype=np.uint64)
    h = lib().ora_shard_count(_p(d, u8p), d.size, _p(o, u64p), _p(ln, u32p), ln.size, k, C.c_uint64(bloom_bits),
                              _p(tw, u64p), rank, world)
    return CountResult(h, k).table(1)
