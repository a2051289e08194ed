"""Reference-shaped Python API over libspk (see package docstring)."""
from __future__ import annotations

import ctypes as C
import threading
from dataclasses import dataclass, field
from typing import Dict, Iterable, List, Optional, Sequence, Tuple

import numpy as np

from ._lib import (SPK_F_EDGES, SPK_F_KEEP_BLOOM, CountOpts, JobC, ResultInfo, SpkError,
                   TableView, check, lib, u8p, u32p, u64p, vp)

Kmer256 = Tuple[int, int]  # (lo, hi) as in src/dna.rs:138

_M64 = (1 << 64) - 1


def nlimbs(k: int) -> int:
    """u64 limbs per k-mer key in lists: ceil(k/32)."""
    return (k + 31) // 32


def limbs_from_kmer256(x: Kmer256, n: int = 4) -> List[int]:
    lo, hi = x
    w = [lo & _M64, (lo >> 64) & _M64, hi & _M64, (hi >> 64) & _M64]
    return w[:n]


def kmer256_from_limbs(row) -> Kmer256:
    w = [int(v) for v in row] + [0] * (4 - len(row))
    return (w[0] | (w[1] << 64), w[2] | (w[3] << 64))


def _ptr(a: np.ndarray, t):
    return a.ctypes.data_as(t)


# ---------------------------------------------------------------------------
# Context
# ---------------------------------------------------------------------------
class Context:
    """An spk_ctx: one device, one stream, a cached device memory pool."""

    def __init__(self, device: int = 0):
        h = vp()
        check(lib().spk_ctx_create(device, C.byref(h)))
        self.h = h.value
        self.device = device

    def close(self):
        if getattr(self, "h", None):
            lib().spk_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, cuda_stream: Optional[int]) -> None:
        """Run this context's work on a caller-owned cudaStream_t (None: its own)."""
        check(lib().spk_ctx_set_stream(self.h, cuda_stream))

    def memory(self) -> Tuple[int, int]:
        r, f = C.c_uint64(), C.c_uint64()
        check(lib().spk_ctx_memory(self.h, C.byref(r), C.byref(f)))
        return r.value, f.value


_DEFAULT: Dict[int, Context] = {}
_DEFAULT_LOCK = threading.Lock()


def default_context(device: int = 0) -> Context:
    with _DEFAULT_LOCK:
        if device not in _DEFAULT:
            _DEFAULT[device] = Context(device)
        return _DEFAULT[device]


# ---------------------------------------------------------------------------
# TwoTierFilter (src/bloom.rs:13-131)
# ---------------------------------------------------------------------------
class TwoTierFilter:
    """Device-resident ``TwoTierFilter``; single-key methods match the reference's.

    Batched methods take numpy arrays and return what per-key calls in array
    order would return.
    """

    def __init__(self, capacity_bits: int, ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        h = vp()
        check(lib().spk_bloom_create(self.ctx.h, capacity_bits, C.byref(h)))
        self.h = h.value

    def close(self):
        if getattr(self, "h", None):
            lib().spk_bloom_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def size_bits(self) -> int:
        return int(lib().spk_bloom_size_bits(self.h))

    def memory_usage_bytes(self) -> int:          # bloom.rs:129-131
        return int(lib().spk_bloom_memory_usage_bytes(self.h))

    # batched
    def insert_batch(self, keys) -> np.ndarray:   # bloom.rs:48-50 per key
        k = np.ascontiguousarray(keys, dtype=np.uint64).reshape(-1)
        out = np.zeros(max(k.size, 1), dtype=np.uint8)
        check(lib().spk_bloom_insert_u64(self.h, _ptr(k, u64p), k.size, _ptr(out, u8p)))
        return out[: k.size].astype(bool)

    def insert_kmer256_batch(self, keys4) -> np.ndarray:  # bloom.rs:83-107 per key
        k = np.ascontiguousarray(keys4, dtype=np.uint64).reshape(-1, 4)
        out = np.zeros(max(k.shape[0], 1), dtype=np.uint8)
        check(lib().spk_bloom_insert_k256(self.h, _ptr(k, u64p), k.shape[0], _ptr(out, u8p)))
        return out[: k.shape[0]].astype(bool)

    def is_solid_batch(self, keys) -> np.ndarray:  # bloom.rs:54-56 per key
        k = np.ascontiguousarray(keys, dtype=np.uint64).reshape(-1)
        out = np.zeros(max(k.size, 1), dtype=np.uint8)
        check(lib().spk_bloom_is_solid_u64(self.h, _ptr(k, u64p), k.size, _ptr(out, u8p)))
        return out[: k.size].astype(bool)

    def is_solid_kmer256_batch(self, keys4) -> np.ndarray:  # bloom.rs:111-126 per key
        k = np.ascontiguousarray(keys4, dtype=np.uint64).reshape(-1, 4)
        out = np.zeros(max(k.shape[0], 1), dtype=np.uint8)
        check(lib().spk_bloom_is_solid_k256(self.h, _ptr(k, u64p), k.shape[0], _ptr(out, u8p)))
        return out[: k.shape[0]].astype(bool)

    # single key, reference names
    def insert(self, kmer: int) -> bool:
        return bool(self.insert_batch(np.array([kmer], dtype=np.uint64))[0])

    def is_solid(self, kmer: int) -> bool:
        return bool(self.is_solid_batch(np.array([kmer], dtype=np.uint64))[0])

    def insert_kmer256(self, kmer: Kmer256) -> bool:
        return bool(self.insert_kmer256_batch(np.array([limbs_from_kmer256(kmer)], dtype=np.uint64))[0])

    def is_solid_kmer256(self, kmer: Kmer256) -> bool:
        return bool(self.is_solid_kmer256_batch(np.array([limbs_from_kmer256(kmer)], dtype=np.uint64))[0])

    def correct_reads(self, packed, k: int):
        """ErrorCorrector::correct_read_in_place (src/hammer.rs:34-121) on every
        read, against this filter's solid tier, as Stage 3 does before counting
        (src/assemble.rs:183-191).  Returns (PackedReads with the corrected
        bases, per-read bool flags, number of corrected reads)."""
        data, offsets, lengths = _as_arrays(packed)
        d = np.ascontiguousarray(data, dtype=np.uint8)
        o = np.ascontiguousarray(offsets, dtype=np.uint64)
        ln = np.ascontiguousarray(lengths, dtype=np.uint32)
        out = np.empty(max(d.size, 1), dtype=np.uint8)
        flags = np.zeros(max(ln.size, 1), dtype=np.uint8)
        nc = C.c_uint64(0)
        check(lib().spk_bloom_correct_reads(self.h, k, d.ctypes.data, d.size, o.ctypes.data, ln.ctypes.data,
                                            ln.size, out.ctypes.data, flags.ctypes.data, C.byref(nc)))
        pe = getattr(packed, "pe_count", 0)
        return (PackedReads(out[: d.size], o.copy(), ln.copy(), pe), flags[: ln.size].astype(bool),
                int(nc.value))

    def correct_read(self, seq: str, k: int) -> Tuple[str, bool]:
        """One ACGT read, as correct_read_in_place on it: (read, changed)."""
        pr = PackedReads.from_clean_reads([seq])
        if len(pr.lengths) != 1 or int(pr.lengths[0]) != len(seq):
            raise SpkError(1, "correct_read takes a read of A, C, G and T only")
        out, flags, _ = self.correct_reads(pr, k)
        return out.get_read(0), bool(flags[0])

    def download(self) -> Tuple[np.ndarray, np.ndarray]:
        """(seen_bits, solid_bits) word arrays of src/bloom.rs:19-21."""
        n = self.size_bits // 64
        seen = np.zeros(n, dtype=np.uint64)
        solid = np.zeros(n, dtype=np.uint64)
        check(lib().spk_bloom_download(self.h, _ptr(seen, u64p), _ptr(solid, u64p)))
        return seen, solid


# ---------------------------------------------------------------------------
# Packed reads (src/packed_reads.rs:42-59)
# ---------------------------------------------------------------------------
_CODE = np.full(256, 255, dtype=np.uint8)
for _c, _v in zip(b"AaCcGgTt", (0, 0, 1, 1, 2, 2, 3, 3)):
    _CODE[_c] = _v


@dataclass
class PackedReads:
    """The reference PackedReads layout: 2-bit MSB-first bytes, byte-aligned reads."""

    data: np.ndarray
    offsets: np.ndarray
    lengths: np.ndarray
    pe_count: int = 0

    def __len__(self) -> int:
        return int(self.lengths.size)

    @staticmethod
    def from_clean_reads(reads: Iterable) -> "PackedReads":
        """pack_clean (src/packed_reads.rs:547-578) of each read, in order; non-ACGT bytes are skipped."""
        codes, offsets, lengths, data_parts = [], [], [], []
        off = 0
        for r in reads:
            b = np.frombuffer(r.encode() if isinstance(r, str) else bytes(r), dtype=np.uint8)
            c = _CODE[b]
            c = c[c != 255]
            n = c.size
            nb = (n + 3) // 4
            pad = np.zeros(nb * 4, dtype=np.uint8)
            pad[:n] = c
            q = pad.reshape(-1, 4) if nb else pad.reshape(0, 4)
            packed = (q[:, 0] << 6) | (q[:, 1] << 4) | (q[:, 2] << 2) | q[:, 3]
            data_parts.append(packed.astype(np.uint8))
            offsets.append(off)
            lengths.append(n)
            off += nb
        data = np.concatenate(data_parts) if data_parts else np.zeros(0, np.uint8)
        return PackedReads(data, np.array(offsets, dtype=np.uint64), np.array(lengths, dtype=np.uint32))

    def get_read(self, idx: int) -> str:
        """get_read (src/packed_reads.rs:592-613)."""
        n = int(self.lengths[idx])
        o = int(self.offsets[idx])
        by = self.data[o:o + (n + 3) // 4]
        codes = np.stack([(by >> 6) & 3, (by >> 4) & 3, (by >> 2) & 3, by & 3], axis=1).reshape(-1)[:n]
        return bytes(np.frombuffer(b"ACGT", dtype=np.uint8)[codes]).decode()


# ---------------------------------------------------------------------------
# Counting
# ---------------------------------------------------------------------------
def make_opts(bloom_bits: int = 512 << 20, min_count: int = 0, list_min_count: int = 2,
              min_coverage: float = 5.0, flags: Optional[int] = None,
              table_log2: int = 0, priors: Optional[Sequence[bytes]] = None,
              span_groups_log2: int = 0, solid_out=None) -> CountOpts:
    """spk_count_opts.  priors: prior/trusted contigs as ASCII byte strings
    (src/assemble.rs:244-284); the returned options keep them alive.
    solid_out: (keys, counts) arrays (u64 (capacity, ceil(k/32)) and u32
    (capacity,), C-contiguous; pinned host memory copies fastest) that the
    count fills with the first k's solid list while it builds the edges
    (CountResult.info()["solid_copied"], ["n_solid"])."""
    o = CountOpts()
    lib().spk_count_opts_default(C.byref(o))
    o.bloom_bits = bloom_bits
    o.min_count = min_count
    o.list_min_count = list_min_count
    o.min_coverage = min_coverage
    o.table_log2 = table_log2
    o.span_groups_log2 = span_groups_log2
    if flags is not None:
        o.flags = flags
    if priors:
        seqs = [bytes(p) for p in priors]
        buf = np.frombuffer(b"".join(seqs) + b"\0", dtype=np.uint8).copy()
        lens = np.array([len(p) for p in seqs], dtype=np.uint32)
        offs = np.concatenate([[0], np.cumsum(lens.astype(np.uint64))[:-1]]).astype(np.uint64)
        o._prior_arrays = (buf, offs, lens)
        o.prior_seqs = buf.ctypes.data
        o.prior_offsets = offs.ctypes.data
        o.prior_lengths = lens.ctypes.data
        o.n_prior = len(seqs)
    if solid_out is not None:
        keys, counts = solid_out
        if (keys.dtype != np.uint64 or counts.dtype != np.uint32 or keys.ndim != 2 or counts.ndim != 1
                or keys.shape[0] != counts.shape[0] or not keys.flags.c_contiguous
                or not counts.flags.c_contiguous):
            raise SpkError(1, "solid_out must be C-contiguous u64 keys (n, limbs) and u32 counts (n,)")
        o._solid_arrays = (keys, counts)
        o.solid_keys_out = keys.ctypes.data
        o.solid_counts_out = counts.ctypes.data
        o.solid_capacity = counts.shape[0]
    return o


class CountResult:
    """Owner of an spk_result: per-k solid lists, edges, Bloom tiers and stats."""

    def __init__(self, h, ctx: Context):
        self.h = h
        self.ctx = ctx

    def close(self):
        if getattr(self, "h", None):
            lib().spk_result_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self) -> int:
        n = C.c_int()
        check(lib().spk_result_count(self.h, C.byref(n)))
        return n.value

    def info(self, ki: int = 0) -> dict:
        i = ResultInfo()
        check(lib().spk_result_info_get(self.h, ki, C.byref(i)))
        return i.as_dict()

    def _list(self, fn, ki, *extra, out=None):
        """keys (n, ceil(k/32)) u64 and counts (n,) u32.  out = (keys, counts)
        arrays to fill (C-contiguous, enough rows; pinned host memory makes
        the copy faster); views of their first n rows are returned."""
        k = self.info(ki)["k"]
        L = nlimbs(k)
        n = C.c_size_t(0)
        check(fn(self.h, ki, *extra, None, None, C.byref(n)))
        m = n.value
        if out is None:
            keys = np.empty((max(m, 1), L), dtype=np.uint64)
            counts = np.empty(max(m, 1), dtype=np.uint32)
        else:
            keys, counts = out
            if (keys.dtype != np.uint64 or counts.dtype != np.uint32 or keys.ndim != 2
                    or keys.shape[1] != L or keys.shape[0] < m or counts.shape[0] < m
                    or not keys.flags.c_contiguous or not counts.flags.c_contiguous):
                raise SpkError(1, f"output arrays must hold {m} keys of {L} u64 limbs and {m} u32 counts")
        n = C.c_size_t(max(m, keys.shape[0]) if out is not None else m)
        check(fn(self.h, ki, *extra, _ptr(keys, u64p), _ptr(counts, u32p), C.byref(n)))
        return keys[: n.value], counts[: n.value]

    def solid(self, ki: int = 0, out=None) -> Tuple[np.ndarray, np.ndarray]:
        """Sorted (keys, counts) of the solid k-mers (count >= cutoff, src/assemble.rs:288-292)."""
        return self._list(lib().spk_result_solid, ki, out=out)

    def kmers(self, ki: int = 0, min_count: int = 0, out=None) -> Tuple[np.ndarray, np.ndarray]:
        """Sorted (keys, counts) of every listed k-mer with count >= min_count."""
        return self._list(lib().spk_result_kmers, ki, C.c_uint32(min_count), out=out)

    def edges(self, ki: int = 0) -> np.ndarray:
        """Sorted canonical (k+1)-mer edges, ceil((k+1)/32) limbs each."""
        k = self.info(ki)["k"]
        L = nlimbs(k + 1)
        n = C.c_size_t(0)
        check(lib().spk_result_edges(self.h, ki, None, C.byref(n)))
        m = n.value
        e = np.empty((max(m, 1), L), dtype=np.uint64)
        n = C.c_size_t(m)
        check(lib().spk_result_edges(self.h, ki, _ptr(e, u64p), C.byref(n)))
        return e[: n.value]

    def unitigs(self, ki: int = 0):
        """Unitigs of the solid k-mers (CompactedGraph::build, src/graph.rs:65-235):
        (sequences, mean_coverage float64[n], kmers_count uint64[n]), each
        sequence in the orientation not greater than its reverse complement,
        sorted by sequence.  k must be odd."""
        n = C.c_uint64(0)
        nb = C.c_uint64(0)
        check(lib().spk_result_unitigs(self.h, ki, None, C.byref(nb), None, None, None, C.byref(n)))
        m, b = n.value, nb.value
        buf = C.create_string_buffer(max(b, 1))
        lengths = np.zeros(max(m, 1), dtype=np.uint64)
        cov = np.zeros(max(m, 1), dtype=np.float64)
        kmers = np.zeros(max(m, 1), dtype=np.uint64)
        check(lib().spk_result_unitigs(self.h, ki, buf, C.byref(nb), _ptr(lengths, u64p),
                                       cov.ctypes.data_as(C.POINTER(C.c_double)), _ptr(kmers, u64p),
                                       C.byref(n)))
        raw = buf.raw[: nb.value].decode("ascii")
        seqs, o = [], 0
        for L in lengths[: n.value].tolist():
            seqs.append(raw[o : o + L])
            o += L
        return seqs, cov[: n.value], kmers[: n.value]

    def bloom(self, ki: int = 0, ref_solid: bool = False):
        """(seen, twice[, ref_solid]) Bloom word arrays of this k."""
        n = self.info(ki)["bloom_size_bits"] // 64
        seen = np.zeros(n, dtype=np.uint64)
        twice = np.zeros(n, dtype=np.uint64)
        rs = np.zeros(n, dtype=np.uint64) if ref_solid else None
        check(lib().spk_result_bloom(self.h, ki, _ptr(seen, u64p), _ptr(twice, u64p),
                                     _ptr(rs, u64p) if ref_solid else None))
        return (seen, twice, rs) if ref_solid else (seen, twice)

    def table_view(self, ki: int = 0) -> dict:
        v = TableView()
        check(lib().spk_result_table_view(self.h, ki, C.byref(v)))
        return {name: getattr(v, name) for name, _ in v._fields_}


def _as_arrays(packed):
    if isinstance(packed, PackedReads):
        return packed.data, packed.offsets, packed.lengths
    data, offsets, lengths = packed
    return data, offsets, lengths


def _check_solid_out(opt_kw, ks_arr) -> None:
    so = opt_kw.get("solid_out")
    if so is not None and ks_arr.size and so[0].ndim == 2 and so[0].shape[1] != nlimbs(int(ks_arr[0])):
        raise SpkError(1, f"solid_out keys need {nlimbs(int(ks_arr[0]))} u64 limbs per k-mer")


def count(packed, ks: Sequence[int] | int, ctx: Optional[Context] = None, **opt_kw) -> CountResult:
    """spk_count on host-resident packed reads (copied to the device inside the call)."""
    ctx = ctx or default_context()
    data, offsets, lengths = _as_arrays(packed)
    data = np.ascontiguousarray(data, dtype=np.uint8)
    offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
    lengths = np.ascontiguousarray(lengths, dtype=np.uint32)
    if offsets.size != lengths.size:
        raise SpkError(1, "offsets and lengths differ in size")
    ks_arr = np.ascontiguousarray(np.atleast_1d(ks), dtype=np.uint32)
    _check_solid_out(opt_kw, ks_arr)
    o = make_opts(**opt_kw)
    h = vp()
    check(lib().spk_count(ctx.h, data.ctypes.data if data.size else None, data.size,
                          offsets.ctypes.data if offsets.size else None,
                          lengths.ctypes.data if lengths.size else None, lengths.size,
                          _ptr(ks_arr, u32p), ks_arr.size, C.byref(o), C.byref(h)))
    return CountResult(h.value, ctx)


def count_device(d_data: int, data_len: int, d_offsets: int, d_lengths: int, n_reads: int,
                 ks, ctx: Optional[Context] = None, **opt_kw) -> CountResult:
    """spk_count_device: packed reads already resident on the device (raw pointers)."""
    ctx = ctx or default_context()
    ks_arr = np.ascontiguousarray(np.atleast_1d(ks), dtype=np.uint32)
    _check_solid_out(opt_kw, ks_arr)
    o = make_opts(**opt_kw)
    h = vp()
    check(lib().spk_count_device(ctx.h, d_data, data_len, d_offsets, d_lengths, n_reads,
                                 _ptr(ks_arr, u32p), ks_arr.size, C.byref(o), C.byref(h)))
    return CountResult(h.value, ctx)


class DevicePackedReads:
    """A PackedReads store built on the device by spk_ingest from FASTQ/FASTA
    texts (PackedReads::from_paired_files / append_from_file,
    src/packed_reads.rs:300-504)."""

    def __init__(self, text1: bytes, text2: Optional[bytes] = None, ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        h = vp()
        t1 = bytes(text1)
        t2 = None if text2 is None else bytes(text2)
        check(lib().spk_ingest(self.ctx.h, t1, len(t1), t2, 0 if t2 is None else len(t2), C.byref(h)))
        self.h = h.value

    def close(self):
        if getattr(self, "h", None):
            lib().spk_packed_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> dict:
        v = [C.c_uint64() for _ in range(5)]
        check(lib().spk_packed_info(self.h, *[C.byref(x) for x in v]))
        ms, nl = C.c_float(), C.c_uint32()
        check(lib().spk_packed_stats(self.h, C.byref(ms), C.byref(nl)))
        return dict(n_reads=v[0].value, data_len=v[1].value, pe_count=v[2].value, n_sidecar=v[3].value,
                    sidecar_bytes=v[4].value, ms_device=ms.value, kernel_launches=nl.value)

    def download(self) -> Tuple[PackedReads, list]:
        """(PackedReads on the host, sidecar reads as bytes)."""
        i = self.info()
        data = np.zeros(max(i["data_len"], 1), np.uint8)
        offs = np.zeros(max(i["n_reads"], 1), np.uint64)
        lens = np.zeros(max(i["n_reads"], 1), np.uint32)
        sc = np.zeros(max(i["sidecar_bytes"], 1), np.uint8)
        scl = np.zeros(max(i["n_sidecar"], 1), np.uint64)
        check(lib().spk_packed_download(self.h, data.ctypes.data, offs.ctypes.data, lens.ctypes.data,
                                        sc.ctypes.data, scl.ctypes.data))
        side, o = [], 0
        for n in scl[: i["n_sidecar"]].tolist():
            side.append(sc[o:o + n].tobytes())
            o += n
        pr = PackedReads(data[: i["data_len"]], offs[: i["n_reads"]], lens[: i["n_reads"]], i["pe_count"])
        return pr, side

    def device(self) -> Tuple[int, int, int]:
        d, o, ln = vp(), vp(), vp()
        check(lib().spk_packed_device(self.h, C.byref(d), C.byref(o), C.byref(ln)))
        return d.value or 0, o.value or 0, ln.value or 0

    def count(self, ks, **opt_kw) -> "CountResult":
        """spk_count_device on the resident store."""
        i = self.info()
        d, o, ln = self.device()
        return count_device(d, i["data_len"], o, ln, i["n_reads"], ks, ctx=self.ctx, **opt_kw)


def ingest(text1: bytes, text2: Optional[bytes] = None, ctx: Optional[Context] = None) -> DevicePackedReads:
    """spk_ingest: FASTQ/FASTA text(s) to a device-resident PackedReads store."""
    return DevicePackedReads(text1, text2, ctx)


def count_solid_kmers(packed, k: int, bloom_bits: int = 512 << 20,
                      ctx: Optional[Context] = None) -> Dict[Kmer256, int]:
    """The Stage 2-3 seam: HashMap<Kmer256, u32> of the admitted k-mers with count >= 2.

    Replaces src/assemble.rs:129-242 (without error correction) for one k.
    """
    r = count(packed, [k], ctx=ctx, bloom_bits=bloom_bits, flags=0)
    try:
        keys, counts = r.kmers(0)
        return {kmer256_from_limbs(row): int(c) for row, c in zip(keys, counts)}
    finally:
        r.close()


# ---------------------------------------------------------------------------
# Batched and serving
# ---------------------------------------------------------------------------
@dataclass
class Job:
    """One counting job (spk_job); arrays are kept alive for the job's lifetime."""

    packed: object
    ks: Sequence[int]
    opts: dict = field(default_factory=dict)

    def to_c(self) -> JobC:
        data, offsets, lengths = _as_arrays(self.packed)
        self._data = np.ascontiguousarray(data, dtype=np.uint8)
        self._off = np.ascontiguousarray(offsets, dtype=np.uint64)
        self._len = np.ascontiguousarray(lengths, dtype=np.uint32)
        self._ks = np.ascontiguousarray(np.atleast_1d(self.ks), dtype=np.uint32)
        j = JobC()
        j.data = self._data.ctypes.data if self._data.size else None
        j.data_len = self._data.size
        j.offsets = self._off.ctypes.data if self._off.size else None
        j.lengths = self._len.ctypes.data if self._len.size else None
        j.n_reads = self._len.size
        j.ks = self._ks.ctypes.data
        j.n_k = self._ks.size
        self._opts = make_opts(**self.opts)  # keeps any prior contig arrays alive
        j.opts = self._opts
        return j


def count_batch(jobs: List[Job], ctx: Optional[Context] = None) -> List[CountResult]:
    """spk_count_batch: every job's result, each identical to count() on that job alone."""
    ctx = ctx or default_context()
    cj = (JobC * len(jobs))(*[j.to_c() for j in jobs])
    outs = (vp * len(jobs))()
    check(lib().spk_count_batch(ctx.h, cj, len(jobs), outs))
    return [CountResult(outs[i], ctx) for i in range(len(jobs))]


def count_batch_iter(jobs: List[Job], ctx: Optional[Context] = None):
    """spk_batch_start / spk_batch_next / spk_batch_end: yields (index,
    result) in job order as each job finishes, while the jobs after it are
    still uploading and counting.  A failed job raises SpkError (the batch is
    ended, and the results not yet yielded are freed)."""
    ctx = ctx or default_context()
    cj = (JobC * len(jobs))(*[j.to_c() for j in jobs])
    b = vp()
    check(lib().spk_batch_start(ctx.h, cj, len(jobs), C.byref(b)))
    try:
        for _ in range(len(jobs)):
            i, r = C.c_int(-1), vp()
            check(lib().spk_batch_next(b, C.byref(i), C.byref(r)))
            yield i.value, CountResult(r.value, ctx)
    finally:
        lib().spk_batch_end(b)


class Server:
    """The serving loop: jobs admitted by HBM budget, run concurrently, results resident."""

    def __init__(self, ctx: Optional[Context] = None, hbm_budget_bytes: int = 0, max_inflight: int = 4):
        self.ctx = ctx or default_context()
        check(lib().spk_serve_start(self.ctx.h, hbm_budget_bytes, max_inflight))
        self._jobs: Dict[int, Job] = {}
        self._cjobs: Dict[int, JobC] = {}

    def stop(self):
        if self.ctx is not None and getattr(self.ctx, "h", None):
            lib().spk_serve_stop(self.ctx.h)

    @staticmethod
    def estimate(job: Job) -> int:
        cj = job.to_c()
        b = C.c_uint64()
        check(lib().spk_job_hbm_estimate(C.byref(cj), C.byref(b)))
        return b.value

    def submit(self, job: Job) -> int:
        cj = job.to_c()
        t = C.c_uint64()
        check(lib().spk_submit(self.ctx.h, C.byref(cj), C.byref(t)))
        self._jobs[t.value] = job
        self._cjobs[t.value] = cj
        return t.value

    def poll(self, ticket: int) -> bool:
        d = C.c_int()
        check(lib().spk_poll(self.ctx.h, ticket, C.byref(d)))
        return bool(d.value)

    def wait(self, ticket: int, timeout_ms: int = -1) -> Tuple[CountResult, float]:
        h = vp()
        lat = C.c_double()
        rc = lib().spk_wait(self.ctx.h, ticket, timeout_ms, C.byref(h), C.byref(lat))
        if rc != 9:  # SPK_E_NOT_READY keeps the job (and its host buffers) alive
            self._jobs.pop(ticket, None)
            self._cjobs.pop(ticket, None)
        check(rc)
        return CountResult(h.value, self.ctx), lat.value
