"""Seeded synthetic read sets in the reference PackedReads layout.

The counting path is measured on synthetic paired-end reads of the shapes
the benchmark configurations name (no public dataset is involved):

* ``c1`` -- 1 Mb uniform genome, 100k pairs of 2x150, fragment ~N(300,30),
  0.5% uniform substitutions, 0.01% N bases; k = 21.
* ``c2`` -- 5 Mb genome at 50% GC with 20 inserted repeat copies of 1-5 kb at
  99% identity, 1.667M pairs (100x), substitution rate ramping from 0.1% at
  the read start to 1.0% at the read end; k = 55.
* ``c3`` -- the ``c2`` reads with k in {21, 33, 55, 77}.
* ``c4`` -- 64 samples, genome log-uniform in 0.5-12 Mb, GC U[30%,70%],
  coverage U[20,200]x, 0.5% errors; k = 33.
* ``c5`` -- the serving mix: isolates of 1-8 Mb at 30-100x and metagenome-like
  sets of 20 genomes (1-5 Mb, log-normal abundance sigma=1.5); k = 55.

Every configuration is seeded with its index (c1 -> 0, c2 -> 1, ...) and
generated with numpy's counter-based Philox generator, so a given
(config, scale) always produces the same bytes.  ``scale`` shrinks genome
size (and read count with it) for tests.

Packing follows src/packed_reads.rs: clean pairs (no N after terminal
trimming, both mates >= 21 bp) go to blocks 1 and 2; other pairs are split on
N and their sub-reads >= 21 bp go to block 3 (src/packed_reads.rs:668-690,
521-540); every read starts on a byte boundary (src/packed_reads.rs:547-578).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np

from .api import PackedReads

N_CODE = 4
MIN_K = 21  # src/packed_reads.rs:38


def rng_for(seed: int, stream: int = 0) -> np.random.Generator:
    return np.random.Generator(np.random.Philox(key=[seed, stream]))


def make_genome(rng: np.random.Generator, length: int, gc: float = 0.5) -> np.ndarray:
    """i.i.d. bases with P(C) = P(G) = gc/2, P(A) = P(T) = (1-gc)/2 (codes A0 C1 G2 T3)."""
    p = np.array([(1 - gc) / 2, gc / 2, gc / 2, (1 - gc) / 2])
    u = rng.random(length, dtype=np.float32)
    return np.searchsorted(np.cumsum(p)[:-1], u, side="right").astype(np.uint8)


def insert_repeats(rng: np.random.Generator, g: np.ndarray, n: int, lo: int, hi: int,
                   identity: float) -> None:
    """Copies n random segments of lo..hi bp to random places at the given identity."""
    G = g.size
    for _ in range(n):
        L = int(rng.integers(lo, hi + 1))
        if L >= G:
            continue
        src = int(rng.integers(0, G - L))
        dst = int(rng.integers(0, G - L))
        seg = g[src:src + L].copy()
        m = rng.random(L) >= identity
        seg[m] = (seg[m] + rng.integers(1, 4, size=int(m.sum()), dtype=np.uint8)) % 4
        g[dst:dst + L] = seg


def simulate_pairs(rng: np.random.Generator, g: np.ndarray, n_pairs: int, read_len: int = 150,
                   frag_mean: float = 300.0, frag_sd: float = 30.0,
                   err: Tuple[float, float] = (0.005, 0.005), n_rate: float = 0.0,
                   chunk: int = 50000):
    """Yields (r1, r2) code arrays (pairs x read_len, code 4 = N) in chunks."""
    G = g.size
    pos_err = np.linspace(err[0], err[1], read_len, dtype=np.float32)[None, :]
    ar = np.arange(read_len, dtype=np.int64)[None, :]
    done = 0
    while done < n_pairs:
        n = min(chunk, n_pairs - done)
        frag = np.rint(rng.normal(frag_mean, frag_sd, n)).astype(np.int64)
        frag = np.clip(frag, read_len, G)
        start = (rng.random(n) * (G - frag + 1)).astype(np.int64)
        fwd = g[start[:, None] + ar]
        end = g[(start + frag - read_len)[:, None] + ar]
        end_rc = (3 - end)[:, ::-1]
        minus = rng.random(n) < 0.5
        r1 = np.where(minus[:, None], end_rc, fwd)
        r2 = np.where(minus[:, None], fwd, end_rc)
        out = []
        for r in (r1, r2):
            r = np.ascontiguousarray(r)
            m = rng.random(r.shape, dtype=np.float32) < pos_err
            sub = rng.integers(1, 4, size=r.shape, dtype=np.uint8)
            r = np.where(m, (r + sub) % 4, r).astype(np.uint8)
            if n_rate > 0:
                r[rng.random(r.shape, dtype=np.float32) < n_rate] = N_CODE
            out.append(r)
        yield out[0], out[1]
        done += n


def _pack_fixed(codes: np.ndarray) -> np.ndarray:
    """(n, L) codes 0..3 -> (n, ceil(L/4)) packed bytes, first base in the high bits."""
    n, L = codes.shape
    nb = (L + 3) // 4
    pad = np.zeros((n, nb * 4), dtype=np.uint8)
    pad[:, :L] = codes
    q = pad.reshape(n, nb, 4)
    return ((q[:, :, 0] << 6) | (q[:, :, 1] << 4) | (q[:, :, 2] << 2) | q[:, :, 3]).astype(np.uint8)


def _pack_one(c: np.ndarray) -> np.ndarray:
    return _pack_fixed(c[None, :])[0] if c.size else np.zeros(0, np.uint8)


def _trim(c: np.ndarray) -> np.ndarray:
    ok = np.nonzero(c != N_CODE)[0]
    if ok.size == 0:
        return c[:0]
    return c[ok[0]:ok[-1] + 1]


class _Builder:
    """Accumulates the three blocks of src/packed_reads.rs:9-27."""

    def __init__(self):
        self.b1: List[np.ndarray] = []  # fixed-length packed chunks (n, nb) or variable reads
        self.b2: List[np.ndarray] = []
        self.len1: List[np.ndarray] = []
        self.len2: List[np.ndarray] = []
        self.b3: List[np.ndarray] = []
        self.len3: List[int] = []

    def add(self, r1: np.ndarray, r2: np.ndarray):
        has_n = (r1 == N_CODE).any(axis=1) | (r2 == N_CODE).any(axis=1)
        clean = ~has_n
        if clean.any():
            p1 = _pack_fixed(r1[clean])
            p2 = _pack_fixed(r2[clean])
            self.b1.append(p1)
            self.b2.append(p2)
            self.len1.append(np.full(p1.shape[0], r1.shape[1], np.uint32))
            self.len2.append(np.full(p2.shape[0], r2.shape[1], np.uint32))
        for i in np.nonzero(has_n)[0]:
            t1, t2 = _trim(r1[i]), _trim(r2[i])
            n1, n2 = (t1 == N_CODE).any(), (t2 == N_CODE).any()
            if not n1 and not n2 and t1.size >= MIN_K and t2.size >= MIN_K:
                # terminal Ns only: the trimmed pair stays paired (src/packed_reads.rs:683-685)
                self.b1.append(_pack_one(t1)[None, :] if t1.size else np.zeros((1, 0), np.uint8))
                self.b2.append(_pack_one(t2)[None, :] if t2.size else np.zeros((1, 0), np.uint8))
                self.len1.append(np.array([t1.size], np.uint32))
                self.len2.append(np.array([t2.size], np.uint32))
            else:
                for t in (t1, t2):  # src/packed_reads.rs:521-540
                    if t.size == 0:
                        continue
                    cuts = np.nonzero(t == N_CODE)[0]
                    bounds = np.concatenate([[-1], cuts, [t.size]])
                    for a, b in zip(bounds[:-1], bounds[1:]):
                        seg = t[a + 1:b]
                        if seg.size >= MIN_K:
                            self.b3.append(_pack_one(seg))
                            self.len3.append(seg.size)

    def finish(self) -> PackedReads:
        parts, lens, offs = [], [], []
        off = 0
        for blocks, lengths in ((self.b1, self.len1), (self.b2, self.len2)):
            for p, ln in zip(blocks, lengths):
                nb = p.shape[1]
                parts.append(p.reshape(-1))
                offs.append(off + np.arange(p.shape[0], dtype=np.uint64) * nb)
                lens.append(ln)
                off += p.size
        pe = int(sum(x.size for x in self.len1))
        for p, ln in zip(self.b3, self.len3):
            parts.append(p)
            offs.append(np.array([off], np.uint64))
            lens.append(np.array([ln], np.uint32))
            off += p.size
        data = np.concatenate(parts) if parts else np.zeros(0, np.uint8)
        offsets = np.concatenate(offs) if offs else np.zeros(0, np.uint64)
        lengths = np.concatenate(lens) if lens else np.zeros(0, np.uint32)
        return PackedReads(data, offsets.astype(np.uint64), lengths.astype(np.uint32), pe)


@dataclass
class Sample:
    name: str
    packed: PackedReads
    genome_len: int
    coverage: float
    ks: Tuple[int, ...]


def sample(genome_len: int, coverage: float, seed: int, stream: int = 0, gc: float = 0.5,
           err=(0.005, 0.005), n_rate: float = 0.0, repeats: int = 0, read_len: int = 150,
           ks=(31,), name: str = "sample", genome: Optional[np.ndarray] = None) -> Sample:
    rng = rng_for(seed, stream)
    g = genome if genome is not None else make_genome(rng, genome_len, gc)
    if repeats and genome is None:
        insert_repeats(rng, g, repeats, 1000, 5000, 0.99)
    n_pairs = max(1, int(round(genome_len * coverage / (2 * read_len))))
    b = _Builder()
    for r1, r2 in simulate_pairs(rng, g, n_pairs, read_len, err=err, n_rate=n_rate):
        b.add(r1, r2)
    return Sample(name, b.finish(), genome_len, coverage, tuple(ks))


def c1(scale: float = 1.0) -> Sample:
    G = max(2000, int(1_000_000 * scale))
    return sample(G, 30.0, seed=0, err=(0.005, 0.005), n_rate=0.0001, ks=(21,), name="c1")


def c2(scale: float = 1.0, ks=(55,)) -> Sample:
    G = max(2000, int(5_000_000 * scale))
    return sample(G, 100.0, seed=1, gc=0.5, err=(0.001, 0.01), repeats=20, ks=ks, name="c2")


def c3(scale: float = 1.0) -> Sample:
    s = c2(scale, ks=(21, 33, 55, 77))
    s.name = "c3"
    return s


def c4_plan(n_samples: int = 64, scale: float = 1.0) -> List[dict]:
    """Genome size, GC and coverage of each c4 sample (seed 3)."""
    rng = rng_for(3, 0)
    out = []
    for i in range(n_samples):
        G = math.exp(rng.uniform(math.log(0.5e6), math.log(12e6)))
        out.append(dict(index=i, genome_len=max(2000, int(G * scale)), gc=float(rng.uniform(0.3, 0.7)),
                        coverage=float(rng.uniform(20, 200))))
    return out


def c4(n_samples: int = 64, scale: float = 1.0) -> List[Sample]:
    out = []
    for p in c4_plan(n_samples, scale):
        out.append(sample(p["genome_len"], p["coverage"], seed=3, stream=1 + p["index"], gc=p["gc"],
                          err=(0.005, 0.005), ks=(33,), name=f"c4_{p['index']}"))
    return out


def c5_job(i: int, scale: float = 1.0) -> Sample:
    """The i-th serving request (seed 4): 1 in 4 is metagenome-like, the rest isolates."""
    rng = rng_for(4, 10_000 + i)
    if rng.random() < 0.25:
        # 20 genomes of 1-5 Mb with log-normal abundances (sigma 1.5), one pooled read set.
        sizes = (rng.uniform(1e6, 5e6, 20) * scale).astype(np.int64).clip(2000)
        ab = rng.lognormal(0.0, 1.5, 20)
        total_cov = rng.uniform(20, 100)
        genomes = [make_genome(rng, int(s), float(rng.uniform(0.3, 0.7))) for s in sizes]
        g = np.concatenate(genomes)
        # coverage of each genome proportional to its abundance
        cov = total_cov * ab / ab.mean()
        b = _Builder()
        for gi, (gg, c) in enumerate(zip(genomes, cov)):
            n_pairs = max(1, int(gg.size * c / 300))
            for r1, r2 in simulate_pairs(rng, gg, n_pairs, err=(0.005, 0.005)):
                b.add(r1, r2)
        return Sample(f"c5_meta_{i}", b.finish(), int(g.size), float(total_cov), (55,))
    G = int(rng.uniform(1e6, 8e6) * scale)
    return sample(max(G, 2000), float(rng.uniform(30, 100)), seed=4, stream=20_000 + i,
                  gc=float(rng.uniform(0.3, 0.7)), ks=(55,), name=f"c5_iso_{i}")


# ---------------------------------------------------------------------------
# Native generator (spk/libspksynth.so, synth_native.cpp): the batched and
# serving workloads at their full sizes (tens of Gbp), seeded per sample and
# independent of the thread count.  Reads are 2x150 N-free pairs, so every
# pair is clean (blocks 1 and 2 of src/packed_reads.rs:9-27).
# ---------------------------------------------------------------------------
_NATIVE = None


def _native():
    global _NATIVE
    if _NATIVE is None:
        import ctypes as C
        import os
        here = os.path.dirname(os.path.abspath(__file__))
        path = os.path.join(here, "libspksynth.so")
        if not os.path.exists(path):
            import subprocess
            subprocess.run(["make", "-s", "-C", os.path.dirname(here), "spk/libspksynth.so"], check=True)
        L = C.CDLL(path)
        L.spk_synth_genome.restype = None
        L.spk_synth_genome.argtypes = [C.c_void_p, C.c_uint64, C.c_double, C.c_uint64, C.c_uint64, C.c_int]
        L.spk_synth_pairs.restype = None
        L.spk_synth_pairs.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint32, C.c_double, C.c_double,
                                      C.c_double, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_int]
        _NATIVE = L
    return _NATIVE


def _threads() -> int:
    import os
    return os.cpu_count() or 1


def native_genome(length: int, gc: float, seed: int, stream: int) -> np.ndarray:
    g = np.empty(max(length, 1), dtype=np.uint8)
    _native().spk_synth_genome(g.ctypes.data, length, gc, seed, stream, _threads())
    return g[:length]


def native_pairs(genomes: Sequence[np.ndarray], pairs: Sequence[int], seed: int, stream: int,
                 err: float = 0.005, read_len: int = 150, frag_mean: float = 300.0,
                 frag_sd: float = 30.0) -> PackedReads:
    """pairs[g] read pairs from genomes[g] (stream stream + g), as one store:
    every mate 1 in genome and pair order, then every mate 2."""
    total = int(sum(pairs))
    nb = (read_len + 3) // 4
    data = np.empty(max(2 * total * nb, 1), dtype=np.uint8)
    offsets = np.empty(max(2 * total, 1), dtype=np.uint64)
    lengths = np.empty(max(2 * total, 1), dtype=np.uint32)
    first = 0
    for gi, (g, n) in enumerate(zip(genomes, pairs)):
        if n:
            _native().spk_synth_pairs(g.ctypes.data, g.size, int(n), read_len, frag_mean, frag_sd, err, seed,
                                      stream + gi, first, total + first, data.ctypes.data,
                                      offsets.ctypes.data, lengths.ctypes.data, _threads())
        first += int(n)
    return PackedReads(data[: 2 * total * nb], offsets[: 2 * total], lengths[: 2 * total], total)


def native_sample(genome_len: int, coverage: float, seed: int, stream: int, gc: float = 0.5,
                  err: float = 0.005, ks=(33,), name: str = "sample") -> Sample:
    g = native_genome(genome_len, gc, seed, 2 * stream)
    n_pairs = max(1, int(round(genome_len * coverage / 300)))
    return Sample(name, native_pairs([g], [n_pairs], seed, 2 * stream + 1, err), genome_len, coverage,
                  tuple(ks))


def c4_native(n_samples: int = 64, scale: float = 1.0) -> List[Sample]:
    """The 64-sample batch with the plan of c4_plan, made by the native generator."""
    return [native_sample(p["genome_len"], p["coverage"], seed=3, stream=1 + p["index"], gc=p["gc"],
                          err=0.005, ks=(33,), name=f"c4_{p['index']}")
            for p in c4_plan(n_samples, scale)]


def c5_plan(i: int, scale: float = 1.0, iso_scale: float = 1.0) -> dict:
    """The i-th serving request (seed 4): 1 in 4 is metagenome-like (20
    genomes of 1-5 Mb, log-normal abundances with sigma 1.5, 20-100x in
    total), the rest isolates (1-8 Mb, 30-100x).  scale multiplies the
    metagenomes' genome sizes, iso_scale the isolates'."""
    rng = rng_for(4, 10_000 + i)
    if rng.random() < 0.25:
        sizes = (rng.uniform(1e6, 5e6, 20) * scale).astype(np.int64).clip(2000)
        ab = rng.lognormal(0.0, 1.5, 20)
        total_cov = float(rng.uniform(20, 100))
        gcs = rng.uniform(0.3, 0.7, 20)
        cov = total_cov * ab / ab.mean()
        return dict(kind="meta", sizes=[int(x) for x in sizes], gcs=[float(x) for x in gcs],
                    covs=[float(x) for x in cov], coverage=total_cov)
    G = max(int(rng.uniform(1e6, 8e6) * iso_scale), 2000)
    return dict(kind="iso", sizes=[G], gcs=[float(rng.uniform(0.3, 0.7))], covs=[float(rng.uniform(30, 100))],
                coverage=None)


def c5_native(i: int, scale: float = 1.0, iso_scale: float = 1.0) -> Sample:
    """The i-th serving request of c5_plan, made by the native generator."""
    p = c5_plan(i, scale, iso_scale)
    genomes = [native_genome(sz, gc, 4, 40_000 + 64 * i + j) for j, (sz, gc) in enumerate(zip(p["sizes"], p["gcs"]))]
    pairs = [max(1, int(sz * c / 300)) for sz, c in zip(p["sizes"], p["covs"])]
    packed = native_pairs(genomes, pairs, 4, 80_000 + 64 * i)
    cov = p["coverage"] if p["coverage"] is not None else p["covs"][0]
    return Sample(f"c5_{p['kind']}_{i}", packed, int(sum(p["sizes"])), float(cov), (55,))


def occurrences(p: PackedReads, k: int) -> int:
    L = p.lengths.astype(np.int64)
    return int(np.clip(L - k + 1, 0, None).sum())
