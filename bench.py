#!/usr/bin/env python
"""Headline benchmark: canonical k-mer counting of the 5 Mb x 100x read set at
k = 55 on B200 (Gk-mers/s), with the reference algorithm's CPU restatement
timed beside it.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

One step = one complete counting job on one read set: Bloom population,
twice-tier admission and count table, adaptive cutoff, sorted solid list and
(k+1)-mer edge list (src/assemble.rs:129-292, src/graph.rs:78-102).  With N
GPUs (torchrun) every rank counts its own copy of the read set (replicas, no
data-path collective); value = all ranks' k-mer occurrences / max time.

Output: one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [ROOT, os.path.join(ROOT, "spades-rs_b200")]

METRIC = "Gk-mers/s at k=55 (5Mb,100x) batched vs plain on 1 B200; p50/p99 job latency"
K = 55
L2_FLUSH_BYTES = 512 << 20  # > the 126 MB L2, written between timed steps
# Algorithmic bytes per k-mer occurrence, counted at the 32-byte sector
# granularity of random DRAM/L2 accesses.
#   fused pass:     the packed-read stream, 3 random Bloom word-pair sectors
#                   and the one-sector count-table slot.
#   Stage 2 insert: 3 random Bloom word-pair sectors + the packed-read stream.
#   Stage 3 count:  3 random twice-tier sectors + the stream, and for each
#                   admitted occurrence one table slot sector.
SECTOR = 32


def stream_bytes_per_occ(read_len=150, k=K):
    return ((read_len + 3) // 4 + 12) / (read_len - k + 1)


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.p.terminate()
        self.p.wait()
        self.f.seek(0)
        sm, smax, reasons = [], None, set()
        for line in self.f.read().splitlines():
            c = [x.strip() for x in line.split(",")]
            if len(c) < 9:
                continue
            try:
                sm.append(float(c[1]))
                smax = float(c[2])
            except ValueError:
                continue
            for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                                "sw_power_cap"), c[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# N GPUs: replicas (every rank counts its own copy of the read set, no
# data-path collective); the step time is the slowest rank's
# ---------------------------------------------------------------------------
def max_over_ranks(ms, world, device):
    """The largest per-step time of all ranks (every rank calls this)."""
    if world <= 1:
        return ms
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(occ_per_rank, world, ms):
    """Gk-mers/s of the whole job: all ranks' occurrences over the slowest step."""
    return occ_per_rank * world / (ms / 1e3) / 1e9


# ---------------------------------------------------------------------------
# reference CPU arm
def run_unitigs(args, ctx, log_rank0):
    """Unitig compaction (CompactedGraph::build, src/graph.rs:65-235) of the
    solid k-mers of the 5 Mb x 100x reads (scaled by --scale) at k=55.  Each
    step counts the reads on the device (untimed) and then builds the unitigs
    (timed): the device time of the build from its events, the host's
    orientation and sort, and the host clock around spk_result_unitigs with
    the unitigs copied into host buffers.  CPU baseline: the oracle's
    restatement of the reference walk on the same solid list, one thread."""
    import numpy as np
    import torch
    import spk
    from spk import synth
    from oracle import ora
    p = synth.c2(args.scale).packed
    dev = torch.device("cuda", 0)
    d_data = torch.zeros(p.data.size + 64, dtype=torch.uint8, device=dev)
    d_data[: p.data.size] = torch.from_numpy(p.data).to(dev)
    d_off = torch.from_numpy(p.offsets.view(np.int64)).to(dev)
    d_len = torch.from_numpy(p.lengths.view(np.int32)).to(dev)
    torch.cuda.synchronize()
    opts = dict(bloom_bits=args.bloom_bits, flags=spk.SPK_F_EDGES)

    def count():
        return spk.count_device(d_data.data_ptr(), p.data.size, d_off.data_ptr(), d_len.data_ptr(),
                                p.lengths.size, [K], ctx=ctx, **opts)

    dev_ms, host_ms, wall_ms = [], [], []
    n_solid = n_unitigs = launches = 0
    out_bytes = 0
    for i in range(args.warmup + args.steps):
        r = count()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        seqs, cov, kmers = r.unitigs(0)
        t1 = time.perf_counter()
        info = r.info(0)
        if i >= args.warmup:
            dev_ms.append(info["ms_unitigs"])
            host_ms.append(info["ms_unitigs_host"])
            wall_ms.append((t1 - t0) * 1e3)
        n_solid, n_unitigs, launches = info["n_solid"], info["n_unitigs"], info["unitig_launches"]
        out_bytes = sum(len(x) for x in seqs) + 16 * len(seqs)
        if i == args.warmup + args.steps - 1:
            keys, counts = r.solid(0)
        r.close()
    med = lambda a: float(np.median(a))
    t_build = med(dev_ms) + med(host_ms)
    line = {"metric": "unitig compaction throughput (solid k-mers per second)",
            "value": n_solid / (t_build / 1e3) / 1e6, "unit": "M solid k-mers/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_build,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic (seeded; no public dataset)",
            "config": {"workload": f"unitigs of the k=55 solid k-mers of the 5 Mb x 100x reads at "
                                   f"scale {args.scale}", "n_solid": n_solid, "n_unitigs": n_unitigs,
                       "timing": "CUDA events around the device build (through the copy of the "
                                 "unitigs to the host) plus the host's orientation and sort; "
                                 "median over steps"},
            "device_ms": med(dev_ms), "host_ms": med(host_ms), "gpu_launches": launches,
            "e2e": {"value": n_solid / (med(wall_ms) / 1e3) / 1e6, "unit": "M solid k-mers/s",
                    "h2d_bytes_per_step": 0, "d2h_bytes_per_step": out_bytes,
                    "what": "host clock around spk_result_unitigs through the Python binding, "
                            "results in host buffers"}}
    if not args.no_cpu_baseline:
        t0 = time.perf_counter()
        ref = ora.unitigs(keys, counts, K)
        sec = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": n_solid / sec / 1e6, "unit": "M solid k-mers/s", "cores": 1,
                                "kind": "port", "seconds": sec,
                                "sample": "the whole solid list of the workload; the oracle's C++ "
                                          "restatement of the reference walk, one thread"}
        line["parity"] = bool(ref[0] == seqs and np.array_equal(ref[2], kmers)
                              and np.array_equal(ref[1], cov))
    return line


def run_correct(args, ctx, log_rank0):
    """Stage 3 with error correction (config.error_correct,
    src/assemble.rs:183-191; ErrorCorrector, src/hammer.rs:34-121) on the
    5 Mb x 100x reads (scaled by --scale) at k=55: each step is one counting
    job with SPK_F_CORRECT (Bloom pass, correction of every read into a
    device copy, gated count of the corrected reads, cutoff, sort, edges),
    reads resident in HBM; host clock around the synchronised call.  Also:
    the correction kernel alone (its device time), the same job without
    correction, and the job end to end from host reads.  CPU baseline: the
    threaded restatement of the same Stage 2 + corrected Stage 3 on a sample
    of the reads, all host threads."""
    import numpy as np
    import torch
    import spk
    from spk import synth
    from oracle import ora
    p = synth.c2(args.scale).packed
    occ = synth.occurrences(p, K)
    dev = torch.device("cuda", 0)
    d_data = torch.zeros(p.data.size + 64, dtype=torch.uint8, device=dev)
    d_data[: p.data.size] = torch.from_numpy(p.data).to(dev)
    d_off = torch.from_numpy(p.offsets.view(np.int64)).to(dev)
    d_len = torch.from_numpy(p.lengths.view(np.int32)).to(dev)
    torch.cuda.synchronize()
    corr = dict(bloom_bits=args.bloom_bits, flags=spk.SPK_F_EDGES | spk.SPK_F_CORRECT)
    gated = dict(bloom_bits=args.bloom_bits, flags=spk.SPK_F_EDGES | spk.SPK_F_GATED)

    def run(opts):
        return spk.count_device(d_data.data_ptr(), p.data.size, d_off.data_ptr(), d_len.data_ptr(),
                                p.lengths.size, [K], ctx=ctx, **opts)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        ms, infos = [], []
        for _ in range(args.steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            info = fn()
            torch.cuda.synchronize()
            ms.append((time.perf_counter() - t0) * 1e3)
            infos.append(info)
        return float(np.median(ms)), infos

    def job(opts):
        r = run(opts)
        info = r.info(0)
        r.close()
        return info

    t_corr, infos = timed(lambda: job(corr))
    t_plain, _ = timed(lambda: job(gated))
    ms_kernel = float(np.median([i["ms_correct"] for i in infos]))
    n_corr = infos[-1]["n_corrected_reads"]
    e2e_ms, _ = timed(lambda: spk.count(p, [K], ctx=ctx, **corr).close())
    line = {"metric": "k-mer counting with error correction (k-mer occurrences per second)",
            "value": occ / (t_corr / 1e3) / 1e9, "unit": "Gk-mers/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_corr,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic (seeded; no public dataset)",
            "config": {"workload": f"c2 reads at scale {args.scale}, k={K}, SPK_F_CORRECT (Stage 3 "
                                   "corrects every read against the twice tier, then counts)",
                       "occurrences": occ, "reads": int(p.lengths.size), "bloom_bits": args.bloom_bits,
                       "timing": "host clock around synchronised calls, median"},
            "correct_kernel": {"ms": ms_kernel, "reads_per_s": p.lengths.size / (ms_kernel / 1e3),
                               "corrected_reads": n_corr},
            "without_correction": {"ms_per_step": t_plain,
                                   "value": occ / (t_plain / 1e3) / 1e9, "schedule": "gated"},
            "gpu_launches": infos[-1]["kernel_launches"],
            "e2e": {"value": occ / (e2e_ms / 1e3) / 1e9, "unit": "Gk-mers/s",
                    "h2d_bytes_per_step": int(p.data.size + p.offsets.nbytes + p.lengths.nbytes),
                    "d2h_bytes_per_step": 0,
                    "what": "spk.count on host reads (H2D of the reads inside the call); the solid "
                            "list stays on the device"}}
    if not args.no_cpu_baseline:
        # Stage 2 over every read (the filter must be the full job's), then the
        # correcting Stage 3 over a sample of the reads, scaled to all of them.
        threads = os.cpu_count() or 1
        n3 = min(p.lengths.size, 20000)
        for _ in range(3):
            r = ora.count_sample3(p.data, p.offsets, p.lengths, K, args.bloom_bits, threads, n3)
            st = r.stats()
            if st["seconds_stage3"] > 5 or n3 == p.lengths.size:
                break
            n3 = min(p.lengths.size, int(n3 * min(20.0, 10.0 / max(st["seconds_stage3"], 1e-3))))
        t_full = st["seconds_stage2"] + st["seconds_stage3"] * p.lengths.size / n3
        line["cpu_baseline"] = {"value": occ / t_full / 1e9, "unit": "Gk-mers/s", "cores": threads,
                                "kind": "port", "seconds_stage2": st["seconds_stage2"],
                                "seconds_stage3_sample": st["seconds_stage3"],
                                "sample": f"Stage 2 over all {p.lengths.size} reads, the correcting Stage 3 "
                                          f"over the first {n3} reads, scaled to all reads; threaded C++ "
                                          f"restatement, {threads} threads, full-size Bloom (reference "
                                          f"solid tier)",
                                "corrected_reads_in_sample": st["corrected_reads"]}
    return line


def c2_fastq_texts(p, n_rate=0.001, seed=7):
    """The c2 read pairs as two FASTQ texts (R1 = reads [0, pe), R2 = [pe, 2pe)),
    fixed-width headers, Phred+33 qualities, about n_rate of the bases N."""
    import numpy as np
    n, L = p.lengths.size, int(p.lengths[0])
    assert np.all(p.lengths == L) and p.pe_count * 2 == n
    nb = (L + 3) // 4
    by = p.data[(p.offsets[:, None] + np.arange(nb)[None, :]).astype(np.int64)]
    codes = np.stack([(by >> 6) & 3, (by >> 4) & 3, (by >> 2) & 3, by & 3], axis=2).reshape(n, -1)[:, :L]
    seq = np.frombuffer(b"ACGT", np.uint8)[codes]
    rng = np.random.default_rng(seed)
    seq[rng.random(seq.shape, dtype=np.float32) < n_rate] = ord("N")
    qual = rng.integers(35, 75, seq.shape, dtype=np.uint8)

    def text(lo, hi):
        m = hi - lo
        hdr = np.frombuffer(b"".join(b"@c2_%09d\n" % i for i in range(lo, hi)), np.uint8).reshape(m, -1)
        nl = np.full((m, 1), ord("\n"), np.uint8)
        plus = np.tile(np.frombuffer(b"+\n", np.uint8), (m, 1))
        return np.concatenate([hdr, seq[lo:hi], nl, plus, qual[lo:hi], nl], axis=1).tobytes()

    pe = int(p.pe_count)
    return text(0, pe), text(pe, n)


def run_ingest(args, ctx, log_rank0):
    """FASTQ ingest (FastxReader and the three-gate, three-block
    PackedReads::from_paired_files, src/packed_reads.rs:69-690) of the c2
    read pairs (scaled by --scale) as two decompressed FASTQ texts in host
    memory: each step uploads both texts, parses and packs them on the device
    (spk_ingest); then, as a second figure, the same plus the k=55 count of
    the resident store.  Host clock around synchronised calls.  CPU baseline:
    the oracle's restatement of the reference's single-threaded streaming
    reader and packer on a sample of the pairs."""
    import ctypes as C
    import numpy as np
    import torch
    import spk
    from spk import synth
    from oracle import ora
    p = synth.c2(args.scale).packed
    t0 = time.time()
    t1, t2 = c2_fastq_texts(p)
    log_rank0(f"ingest: {len(t1) + len(t2)} FASTQ bytes built in {time.time() - t0:.1f}s")
    h1 = torch.frombuffer(bytearray(t1), dtype=torch.uint8).pin_memory()
    h2 = torch.frombuffer(bytearray(t2), dtype=torch.uint8).pin_memory()
    nbytes = len(t1) + len(t2)

    def ingest_only():
        """spk_ingest straight from the pinned texts (the binding would copy bytes)."""
        d = spk.DevicePackedReads.__new__(spk.DevicePackedReads)
        d.ctx = ctx
        h = C.c_void_p()
        spk.api.check(spk.lib().spk_ingest(ctx.h, C.cast(h1.data_ptr(), C.c_char_p), len(t1),
                                           C.cast(h2.data_ptr(), C.c_char_p), len(t2), C.byref(h)))
        d.h = h.value
        return d

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        ms = []
        for _ in range(args.steps):
            torch.cuda.synchronize()
            a = time.perf_counter()
            fn()
            torch.cuda.synchronize()
            ms.append((time.perf_counter() - a) * 1e3)
        return float(np.median(ms))

    infos = []

    def step():
        d = ingest_only()
        infos.append(d.info())
        d.close()

    t_ing = timed(step)
    info = infos[-1]
    occ = synth.occurrences(p, K)

    def with_count():
        d = ingest_only()
        r = d.count([K], bloom_bits=args.bloom_bits, flags=spk.SPK_F_EDGES)
        r.close()
        d.close()

    t_all = timed(with_count)
    line = {"metric": "FASTQ ingest throughput (FASTQ bytes per second)",
            "value": nbytes / (t_ing / 1e3) / 1e9, "unit": "GB/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_ing, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded; no public dataset)",
            "config": {"workload": f"c2 read pairs at scale {args.scale} as two FASTQ texts "
                                   f"({nbytes} bytes, {p.lengths.size} records, 0.1% N)",
                       "timing": "host clock around synchronised calls, median; the upload of both "
                                 "texts from pinned host memory is inside every step"},
            "device_ms": info["ms_device"], "gpu_launches": info["kernel_launches"],
            "store": {k: info[k] for k in ("n_reads", "pe_count", "n_sidecar", "data_len")},
            "e2e": {"value": nbytes / (t_ing / 1e3) / 1e9, "unit": "GB/s", "h2d_bytes_per_step": nbytes,
                    "d2h_bytes_per_step": 0,
                    "what": "spk_ingest from pinned host texts; the store stays on the device"},
            "ingest_and_count": {"ms_per_step": t_all, "Gk_mers_per_s": occ / (t_all / 1e3) / 1e9,
                                 "what": f"FASTQ texts to the k={K} solid list and edges, one step"}}
    if not args.no_cpu_baseline:
        n = min(len(p) // 2, 20000)
        for _ in range(4):
            rec = 318 * n  # fixed-width records
            a = time.perf_counter()
            q = ora.Packed.from_texts(t1[:rec], t2[:rec])
            sec = time.perf_counter() - a
            if sec > 5 or n == len(p) // 2:
                break
            n = min(len(p) // 2, int(n * min(20.0, 10.0 / max(sec, 1e-3))))
        line["cpu_baseline"] = {"value": 2 * rec / sec / 1e9, "unit": "GB/s", "cores": 1, "kind": "port",
                                "seconds": sec,
                                "sample": f"the first {n} pairs ({2 * rec} bytes); the oracle's C++ "
                                          "restatement of the reference's streaming reader and "
                                          "three-block packer (single-threaded, as the reference)"}
        ref = ora.Packed.from_texts(t1[:rec], t2[:rec])
        got = spk.ingest(t1[:rec], t2[:rec], ctx=ctx).download()[0]
        line["parity"] = bool(np.array_equal(got.data, ref.arrays()[0])
                              and np.array_equal(got.lengths, ref.arrays()[2]))
    return line


def cpu_sample(packed, target_occ):
    """The first reads of the workload holding about target_occ k-mer
    occurrences (target_occ <= 0: the whole workload)."""
    import numpy as np
    per = np.clip(packed.lengths.astype(np.int64) - K + 1, 0, None)
    if target_occ <= 0:
        return packed.data, packed.offsets, packed.lengths, int(per.sum())
    n = int(np.searchsorted(np.cumsum(per), target_occ)) + 1
    n = min(n, packed.lengths.size)
    end = int(packed.offsets[n - 1]) + (int(packed.lengths[n - 1]) + 3) // 4
    return packed.data[:end], packed.offsets[:n], packed.lengths[:n], int(per[:n].sum())


def run_cpu_baseline(packed, steps, warmup, target_occ, bloom_bits):
    """The reference algorithm (C++ restatement of src/assemble.rs:129-242 with
    the rayon chunking and sharded maps) on all host cores."""
    import numpy as np
    from oracle import ora
    data, offs, lens, occ = cpu_sample(packed, target_occ)
    total = int(np.clip(packed.lengths.astype(np.int64) - K + 1, 0, None).sum())
    threads = os.cpu_count() or 1
    times = []
    for i in range(warmup + steps):
        r = ora.count(data, offs, lens, K, bloom_bits, mode=ora.MODE_REF, threads=threads,
                      keep_bloom=False)
        st = r.stats()
        if i >= warmup:
            times.append(st["seconds_total"])
        r.table(2)
    sec = sum(times) / len(times)
    what = ("the whole workload" if occ == total else
            f"the first {lens.size} reads of the workload ({occ / total:.1%} of its occurrences)")
    return {"value": occ / sec / 1e9, "unit": "Gk-mers/s", "cores": threads, "kind": "port",
            "seconds_per_step": sec,
            "sample": f"{what}: {lens.size} reads, {occ} k-mer occurrences, Bloom {bloom_bits} "
                      f"bits/tier; C++ restatement of spades-rs Stages 2-3, {threads} threads, timed "
                      f"from packed reads in RAM to the sorted count>=2 list"}


def c2_config(p, occ, args, world):
    """config of the k=55 line (both arms print the same one)."""
    return {"workload": "c2: 5 Mb genome (50% GC, 20 repeats of 1-5 kb at 99% identity), "
                        "2x150 bp pairs at 100x, substitution errors 0.1%->1.0% along the "
                        "read; canonical k=55; Bloom 512 Mi bits/tier; adaptive cutoff; "
                        "sorted solid list + (k+1)-mer edges",
            "k": K, "reads": int(len(p)), "occurrences_per_gpu": occ,
            "bloom_bits": args.bloom_bits, "scale": args.scale,
            "l2": "flushed between steps (512 MiB write)",
            "parallelism": f"replicas x{world} (one read set per GPU, no collective)"}


def run_parity(p, run_job, bloom_bits, timed_info, k=K):
    """The full result of one more (untimed) job against the oracle's
    twice-tier count of the same reads (threaded; order-free, so equal to the
    serial restatement): the whole admitted table with its counts, both Bloom
    tiers, the cutoff and the edge list, bit for bit; and the timed steps'
    result sizes against this job's."""
    import hashlib
    import numpy as np
    import spk
    from oracle import ora
    t0 = time.time()
    r = run_job(flags=spk.SPK_F_EDGES | spk.SPK_F_KEEP_BLOOM, list_min_count=1)
    info = r.info(0)
    gk, gc = r.kmers(0, 1)
    seen, twice = r.bloom(0)
    ge = r.edges(0)
    r.close()
    t1 = time.time()
    threads = os.cpu_count() or 1
    o = ora.count(p.data, p.offsets, p.lengths, k, bloom_bits, mode=ora.MODE_TWICE, threads=threads)
    tk, tc = o.table(1)
    oseen, otwice = o.bloom()
    cut = ora.cutoff(tc, 5.0)
    solid = tc >= cut
    oe = ora.edges(tk[solid], k)
    checks = {
        "table": bool(np.array_equal(gk, tk) and np.array_equal(gc, tc)),
        "count_ge2_list": bool(np.array_equal(gk[gc >= 2], tk[tc >= 2]) and np.array_equal(gc[gc >= 2], tc[tc >= 2])),
        "seen_tier": bool(np.array_equal(seen, oseen)),
        "twice_tier": bool(np.array_equal(twice, otwice)),
        "cutoff": int(info["cutoff"]) == cut,
        "edges": bool(np.array_equal(ge, oe)),
        "singletons": int(info["n_singletons"]) == int((tc == 1).sum()),
        "timed_steps_same_sizes": all(
            ti[key] == info[key] for ti in timed_info
            for key in ("n_solid", "n_edges", "cutoff", "n_table", "admitted_occurrences")),
    }
    sha = hashlib.sha256(tk[solid].tobytes() + tc[solid].tobytes()).hexdigest()[:16]
    return bool(all(checks.values())), {
        "checks": checks, "oracle": f"C++ restatement, twice-tier mode, {threads} threads",
        "n_table": int(tk.shape[0]), "n_count_ge2": int((tc >= 2).sum()), "n_solid": int(solid.sum()),
        "n_edges": int(oe.shape[0]), "cutoff": cut, "solid_sha256_16": sha,
        "gpu_seconds": round(t1 - t0, 2), "oracle_seconds": round(time.time() - t1, 2)}


# ---------------------------------------------------------------------------
# the other workloads (one JSON line each; the default run is the k=55 one)
# ---------------------------------------------------------------------------
def _gk(occ, sec):
    return occ / sec / 1e9


def run_c1(args, ctx, log_rank0):
    """Plain single-sample counting: the 1 Mb x 30x read set (2 x 150 bp
    pairs, 0.5% substitution errors, 0.01% N) at k=21 with one-limb keys and
    the 512 Mi-bit Bloom.  Device-resident steps timed with CUDA events (L2
    flushed between steps); end to end through spk_count from pinned host
    buffers, the solid list copied to pinned buffers during the count; and
    the whole result of one more job against the oracle."""
    import numpy as np
    import torch
    import spk
    from spk import synth
    k = 21
    p = synth.c1(args.scale).packed
    occ = synth.occurrences(p, k)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    d_data = torch.zeros(p.data.size + 64, dtype=torch.uint8, device=dev)
    d_data[: p.data.size] = torch.from_numpy(p.data).to(dev)
    d_off = torch.from_numpy(p.offsets.view(np.int64)).to(dev)
    d_len = torch.from_numpy(p.lengths.view(np.int32)).to(dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    torch.cuda.synchronize()
    opts = dict(bloom_bits=args.bloom_bits, flags=spk.SPK_F_EDGES)

    def job(**kw):
        return spk.count_device(d_data.data_ptr(), p.data.size, d_off.data_ptr(), d_len.data_ptr(),
                                p.lengths.size, [k], ctx=ctx, **{**opts, **kw})

    def timed(fn):
        out, infos = [], []
        for i in range(args.warmup + args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(1)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            r = fn()
            e1.record(stream)
            e1.synchronize()
            if i >= args.warmup:
                out.append(e0.elapsed_time(e1))
                infos.append(r.info(0))
            r.close()
        return out, infos

    step_ms, infos = timed(job)
    ms = sum(step_ms) / len(step_ms)
    h_data = torch.from_numpy(p.data).pin_memory()
    h_off = torch.from_numpy(p.offsets.view(np.int64)).pin_memory()
    h_len = torch.from_numpy(p.lengths.view(np.int32)).pin_memory()
    packed_pinned = (h_data.numpy(), h_off.numpy().view(np.uint64), h_len.numpy().view(np.uint32))
    n_out = int(infos[0]["n_solid"]) + 1024
    o_keys = torch.empty((n_out, 1), dtype=torch.int64).pin_memory().numpy().view(np.uint64)
    o_counts = torch.empty(n_out, dtype=torch.int32).pin_memory().numpy().view(np.uint32)
    e2e_ms, _ = timed(lambda: spk.count(packed_pinned, [k], ctx=ctx, solid_out=(o_keys, o_counts), **opts))
    em = sum(e2e_ms) / len(e2e_ms)
    parity, detail = run_parity(p, job, args.bloom_bits, infos, k=k)
    info = infos[0]
    return {"metric": METRIC, "value": _gk(occ, ms / 1e3), "unit": "Gk-mers/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "step_ms": [round(x, 3) for x in step_ms],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic (seeded; no public dataset)",
            "config": {"workload": f"c1: 1 Mb genome, 2x150 bp pairs at 30x, 0.5% substitution errors, "
                                   f"0.01% N, scale {args.scale}; canonical k=21 (u64 keys); Bloom "
                                   f"{args.bloom_bits} bits/tier; adaptive cutoff; sorted solid list + edges",
                       "k": k, "reads": int(len(p)), "occurrences": occ,
                       "l2": "flushed between steps (512 MiB write)"},
            "e2e": {"value": _gk(occ, em / 1e3), "unit": "Gk-mers/s", "ms_per_step": em,
                    "h2d_bytes_per_step": int(p.data.nbytes + p.offsets.nbytes + p.lengths.nbytes),
                    "d2h_bytes_per_step": int(info["n_solid"]) * 12},
            "parity": parity, "parity_detail": detail,
            "result": {key: int(info[key]) for key in ("n_solid", "n_edges", "cutoff", "n_table")}}


def run_c3(args, ctx, log_rank0):
    """Multi-k: the 5 Mb x 100x reads (scaled by --scale) at k in {21,33,55,77},
    one call counting the four k values against four one-k calls in a row.
    Both are device-resident; time = host clock around synchronised calls."""
    import numpy as np
    import torch
    import spk
    from spk import synth
    ks = [21, 33, 55, 77]
    p = synth.c2(args.scale).packed
    occ = sum(synth.occurrences(p, k) for k in ks)
    dev = torch.device("cuda", 0)
    d_data = torch.zeros(p.data.size + 64, dtype=torch.uint8, device=dev)
    d_data[: p.data.size] = torch.from_numpy(p.data).to(dev)
    d_off = torch.from_numpy(p.offsets.view(np.int64)).to(dev)
    d_len = torch.from_numpy(p.lengths.view(np.int32)).to(dev)
    torch.cuda.synchronize()
    opts = dict(bloom_bits=args.bloom_bits, flags=spk.SPK_F_EDGES)

    def run(kset):
        return spk.count_device(d_data.data_ptr(), p.data.size, d_off.data_ptr(), d_len.data_ptr(),
                                p.lengths.size, kset, ctx=ctx, **opts)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        out = []
        for _ in range(args.steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            fn()
            torch.cuda.synchronize()
            out.append(time.perf_counter() - t0)
        return sum(out) / len(out)

    def plain():
        for k in ks:
            run([k]).close()

    def multi():
        run(ks).close()

    t_plain = timed(plain)
    t_multi = timed(multi)
    return {"metric": METRIC, "value": _gk(occ, t_multi), "unit": "Gk-mers/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_multi * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic (seeded; no public dataset)",
            "config": {"workload": f"c3: the 5 Mb x 100x reads at scale {args.scale}, k in {ks} in "
                                   "one call",
                       "occurrences": occ, "bloom_bits": args.bloom_bits,
                       "timing": "host clock around synchronised calls"},
            "plain": {"what": "one call per k, in a row", "value": _gk(occ, t_plain),
                      "ms_per_step": t_plain * 1e3},
            "speedup_vs_plain": t_plain / t_multi}


def batched_vs_plain(ctx, scale, steps, warmup, bloom_bits, log_rank0):
    """64 uneven samples (genome log-uniform 0.5-12 Mb x scale, GC 30-70%,
    20-200x, 0.5% errors, k=33) from the native generator, host buffers in
    and solid lists out: the batch pipeline (spk_batch_start / spk_batch_next) against spk_count on one sample
    after another.  Returns the measurement as a dict."""
    import torch
    import spk
    from spk import synth
    t0 = time.time()
    ss = synth.c4_native(64, scale)
    packs = [s.packed for s in ss]
    occ = sum(synth.occurrences(p, 33) for p in packs)
    log_rank0(f"c4: {len(packs)} samples, {occ} occurrences, generated in {time.time() - t0:.1f}s")
    opts = dict(bloom_bits=bloom_bits, flags=spk.SPK_F_EDGES)

    # job latency: from the start of the step's work on that job (plain) or
    # of the batch (batched) to the job's solid list on the host
    lat_plain, lat_batch = [], []
    same = []

    def plain(lat=None, keep=None):
        for p in packs:
            a = time.perf_counter()
            r = spk.count(p, [33], ctx=ctx, **opts)
            sk = r.solid(0)
            r.close()
            if lat is not None:
                lat.append((time.perf_counter() - a) * 1e3)
            if keep is not None:
                keep.append(sk)

    def batched(lat=None, keep=None):
        # results handed out in job order as they finish (spk_batch_next), each
        # downloaded while the samples after it still upload and count
        a = time.perf_counter()
        for _, r in spk.count_batch_iter([spk.Job(p, [33], dict(opts)) for p in packs], ctx=ctx):
            sk = r.solid(0)
            r.close()
            if lat is not None:
                lat.append((time.perf_counter() - a) * 1e3)
            if keep is not None:
                keep.append(sk)

    def timed(fn, lat):
        for _ in range(warmup):
            fn()
        out = []
        for _ in range(steps):
            torch.cuda.synchronize()
            a = time.perf_counter()
            fn(lat)
            torch.cuda.synchronize()
            out.append(time.perf_counter() - a)
        return out

    steps_plain = timed(plain, lat_plain)
    steps_batch = timed(batched, lat_batch)
    t_plain = sum(steps_plain) / len(steps_plain)
    t_batch = sum(steps_batch) / len(steps_batch)
    # identical exact output: every sample's solid list, batched and alone
    kp, kb = [], []
    plain(keep=kp)
    batched(keep=kb)
    import numpy as np
    identical = all(np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) for a, b in zip(kp, kb))

    def pct(v):
        v = sorted(v)
        return {"p50": v[len(v) // 2], "p99": v[min(len(v) - 1, int(0.99 * len(v)))]} if v else None
    return {"workload": f"64 samples, genome 0.5-12 Mb x {scale}, 20-200x, k=33, host buffers in, "
                        "solid lists out", "occurrences": occ,
            "value": _gk(occ, t_batch), "ms_per_step": t_batch * 1e3,
            "step_ms": [round(x * 1e3, 1) for x in steps_batch],
            "plain": {"what": "spk_count on one sample after another", "value": _gk(occ, t_plain),
                      "ms_per_step": t_plain * 1e3, "step_ms": [round(x * 1e3, 1) for x in steps_plain],
                      "job_latency_ms": pct(lat_plain)},
            "job_latency_ms": pct(lat_batch), "speedup_vs_plain": t_plain / t_batch,
            "identical_output": identical, "timing": "host clock around synchronised calls"}


def run_c4(args, ctx, log_rank0):
    """Batched uneven samples at --scale (1.0: the workload as specified)."""
    b = batched_vs_plain(ctx, args.scale, args.steps, args.warmup, args.bloom_bits, log_rank0)
    return {"metric": METRIC, "value": b["value"], "unit": "Gk-mers/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": b["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic (seeded; no public dataset)",
            "config": {"workload": "c4: " + b["workload"] + "; spk_batch_start / spk_batch_next", "occurrences": b["occurrences"],
                       "bloom_bits": args.bloom_bits, "timing": b["timing"]},
            "plain": b["plain"], "job_latency_ms": b["job_latency_ms"],
            "speedup_vs_plain": b["speedup_vs_plain"], "identical_output": b["identical_output"]}


def run_c5(args, ctx, log_rank0):
    """Serving: counting jobs (isolates of 1-8 Mb at 30-100x; 1 in 4
    metagenome-like, 20 genomes of 1-5 Mb x --scale with log-normal
    abundances, 20-100x in total), k=55, arriving as a Poisson process (mean
    4 jobs/s), admitted by HBM budget with up to 4 in flight; p50/p99 latency
    from submit to result and throughput.  The read sets come from the native
    seeded generator."""
    import numpy as np
    import spk
    from spk import synth
    n_jobs = max(8, args.steps * 4)
    t0 = time.time()
    jobs = [synth.c5_native(i, args.scale).packed for i in range(n_jobs)]
    occ = sum(synth.occurrences(p, 55) for p in jobs)
    log_rank0(f"c5: {n_jobs} jobs, {occ} occurrences, generated in {time.time() - t0:.1f}s")
    opts = dict(bloom_bits=args.bloom_bits, flags=spk.SPK_F_EDGES)
    rng = np.random.default_rng(4)
    gaps = rng.exponential(1.0 / 4.0, n_jobs)
    srv = spk.Server(ctx, hbm_budget_bytes=0, max_inflight=4)
    try:
        # warm-up: the first eight jobs submitted together, as a running service
        # has seen before (the memory pool holds the buffers of jobs in flight)
        for t in [srv.submit(spk.Job(p, [55], dict(opts))) for p in jobs[:8]]:
            r, _ = srv.wait(t)
            r.close()
        start = time.perf_counter()
        tickets = []
        for i, p in enumerate(jobs):
            due = start + gaps[: i + 1].sum()
            while time.perf_counter() < due:
                time.sleep(min(0.002, max(0.0, due - time.perf_counter())))
            tickets.append(srv.submit(spk.Job(p, [55], dict(opts))))
        lat, per_job = [], []
        for i, t in enumerate(tickets):
            r, ms = srv.wait(t)
            r.solid(0)
            inf = r.info(0)
            r.close()
            lat.append(ms)
            per_job.append({"kind": synth.c5_plan(i, args.scale)["kind"],
                            "occurrences": int(inf["occurrences"]), "latency_ms": round(ms, 1),
                            "job_ms": round(inf["ms_total"], 1), "schedule": int(inf["schedule"]),
                            "relayouts": int(inf["part_rescatters"])})
        wall = time.perf_counter() - start
    finally:
        srv.stop()
    lat = np.array(lat)
    return {"metric": METRIC, "value": _gk(occ, wall), "unit": "Gk-mers/s", "n_gpus": 1,
            "steps": n_jobs, "warmup": 1, "ms_per_step": wall * 1e3 / n_jobs,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic (seeded; no public dataset)",
            "config": {"workload": f"c5: {n_jobs} serving jobs, isolates at full size, metagenome genomes "
                                   f"at scale {args.scale}, k=55, Poisson arrivals at 4/s, up to 4 in flight",
                       "occurrences": occ, "bloom_bits": args.bloom_bits,
                       "timing": "host clock; throughput over the arrival span"},
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                           "max": float(lat.max())},
            # each job: its kind, size, latency (submit to result), device time of the
            # count, schedule and layout repeats
            "jobs": per_job}


# ---------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="spk", choices=["spk", "reference"])
    ap.add_argument("--scale", type=float, default=None,
                    help="genome scale (default 1.0; c5: 0.1 for the metagenome-like jobs)")
    ap.add_argument("--bloom-bits", type=int, default=512 << 20)
    ap.add_argument("--cpu-occ", type=int, default=0,
                    help="k-mer occurrences in the CPU baseline sample (0: the whole workload)")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched-vs-plain measurement of the default run")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the full-size check of one job's result against the oracle")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--workload", default="c2",
                    choices=["c1", "c2", "c3", "c4", "c5", "unitigs", "correct", "ingest"],
                    help="c2 (default): k=55 on the 5 Mb x 100x reads; c1: k=21 on the 1 Mb x 30x "
                         "reads; c3: multi-k; "
                         "c4: 64 batched samples; c5: serving; unitigs: unitig compaction "
                         "of the c2 solid k-mers; correct: c2 with error correction; ingest: c2 "
                         "as FASTQ texts")
    args = ap.parse_args()
    assert args.warmup >= 1
    if args.scale is None:
        args.scale = {"c1": 1.0, "c2": 1.0, "c3": 1.0, "c4": 1.0, "c5": 0.1, "unitigs": 1.0,
                      "correct": 1.0, "ingest": 1.0}[args.workload]

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    import numpy as np
    from spk import synth

    if args.impl == "reference":
        if rank != 0:
            return
        s = synth.c2(args.scale)
        occ = synth.occurrences(s.packed, K)
        cb = run_cpu_baseline(s.packed, args.steps, args.warmup, args.cpu_occ, args.bloom_bits)
        line = {"metric": METRIC, "value": cb["value"], "unit": "Gk-mers/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": cb["seconds_per_step"] * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "u64",
                "data": "synthetic (seeded; no public dataset)", "impl": "reference",
                "config": c2_config(s.packed, occ, args, world),
                "cpu_baseline": cb,
                "e2e": {"value": cb["value"], "unit": "Gk-mers/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch
    import spk

    if args.workload != "c2":
        if rank != 0:
            return
        torch.cuda.set_device(local_rank)
        ctx = spk.Context(local_rank)
        fn = {"c1": run_c1, "c3": run_c3, "c4": run_c4, "c5": run_c5, "unitigs": run_unitigs,
              "correct": run_correct, "ingest": run_ingest}[args.workload]
        print(json.dumps(fn(args, ctx, log)), flush=True)
        ctx.close()
        return

    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local_rank)

    t0 = time.time()
    s = synth.c2(args.scale)
    p = s.packed
    occ = synth.occurrences(p, K)
    log(f"[rank {rank}] generated {len(p)} reads, {occ} occurrences in {time.time() - t0:.1f}s")

    ctx = spk.Context(local_rank)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    dev = torch.device("cuda", local_rank)
    d_data = torch.zeros(p.data.size + 64, dtype=torch.uint8, device=dev)
    d_data[: p.data.size] = torch.from_numpy(p.data).to(dev)
    d_off = torch.from_numpy(p.offsets.view(np.int64)).to(dev)
    d_len = torch.from_numpy(p.lengths.view(np.int32)).to(dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    torch.cuda.synchronize()
    opts = dict(bloom_bits=args.bloom_bits, flags=spk.SPK_F_EDGES)

    def device_step():
        return spk.count_device(d_data.data_ptr(), p.data.size, d_off.data_ptr(), d_len.data_ptr(),
                                p.lengths.size, [K], ctx=ctx, **opts)

    # The clock sampler starts before the warm-up (its start-up queries the
    # driver) and runs until after the timed steps.
    clk = Clocks(local_rank)
    for _ in range(args.warmup):
        device_step().close()

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    barrier()
    step_ms, infos = [], []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(1)  # evict the previous step's tables from L2 (outside the timing)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = device_step()
        e1.record(stream)
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        infos.append(r.info(0))
        r.close()
    barrier()
    clocks = clk.stop()

    ms = sum(step_ms) / len(step_ms)
    # phase times of the median step
    info = infos[sorted(range(len(step_ms)), key=lambda i: step_ms[i])[len(step_ms) // 2]]
    bloom_ms = sum(i["ms_bloom_kernel"] for i in infos) / len(infos)
    count_ms = sum(i["ms_count_kernel"] for i in infos) / len(infos)
    launches = sum(i["kernel_launches"] for i in infos) // len(infos)
    ms = max_over_ranks(ms, world, dev)
    value = replica_throughput(occ, world, ms)

    # e2e: host buffers (pinned) through spk_count, H2D and the D2H of the
    # solid list inside the timing; the solid list goes to the caller's
    # buffers during the count (spk_count_opts.solid_*_out, copied while the
    # edges are built)
    e2e = None
    if not args.no_e2e:
        h_data = torch.from_numpy(p.data).pin_memory()
        h_off = torch.from_numpy(p.offsets.view(np.int64)).pin_memory()
        h_len = torch.from_numpy(p.lengths.view(np.int32)).pin_memory()
        packed_pinned = (h_data.numpy(), h_off.numpy().view(np.uint64), h_len.numpy().view(np.uint32))
        e2e_ms, d2h = [], 0
        # pinned result buffers, sized from the solid list and reused by every step
        n_out = info["n_solid"] + 1024
        o_keys = torch.empty((n_out, (K + 31) // 32), dtype=torch.int64).pin_memory().numpy().view(np.uint64)
        o_counts = torch.empty(n_out, dtype=torch.int32).pin_memory().numpy().view(np.uint32)
        for i in range(args.warmup + args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(1)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            r = spk.count(packed_pinned, [K], ctx=ctx, solid_out=(o_keys, o_counts), **opts)
            ri = r.info(0)
            if not ri["solid_copied"]:  # (the buffers are sized from the first job)
                r.solid(0, out=(o_keys, o_counts))
            e1.record(stream)
            e1.synchronize()
            if i >= args.warmup:
                e2e_ms.append(e0.elapsed_time(e1))
            d2h = int(ri["n_solid"]) * (o_keys.shape[1] * 8 + 4)
            r.close()
        em = sum(e2e_ms) / len(e2e_ms)
        em = max_over_ranks(em, world, dev)
        e2e = {"value": replica_throughput(occ, world, em), "unit": "Gk-mers/s", "ms_per_step": em,
               "h2d_bytes_per_step": int(p.data.nbytes + p.offsets.nbytes + p.lengths.nbytes),
               "d2h_bytes_per_step": int(d2h)}

    # roofline of the dominant kernel (largest share of the step)
    f_adm = info["admitted_occurrences"] / max(info["occurrences"], 1)
    sb = stream_bytes_per_occ()
    kernel_rates = None
    if info["schedule"] == 3:
        # Partitioned: the dominant of its kernels, each with its own
        # algorithmic bytes (what the kernel must read and write).
        scatter_ms = sum(i["ms_scatter_kernel"] for i in infos) / len(infos)
        ops = 3 * info["n_distinct"]
        n_ge2 = info["n_table"] - info["n_singletons"]  # k-mers counted at least twice
        # the read pass that leaves every key in its span's region: one kernel,
        # or two (coarse buckets, then spans) timed together
        sname = "k_part_coarse+k_part_fine" if info.get("part_passes") == 2 else "k_part_scatter"
        coarse_ms = sum(i.get("ms_coarse_kernel", 0.0) for i in infos) / len(infos)
        cands = []
        if coarse_ms > 0 and info.get("part_passes") == 2:
            # the two partition passes on their own: the coarse pass reads the
            # read stream and writes one key per occurrence; the fine pass
            # reads every key back and writes it to its span
            cands += [("k_part_coarse", coarse_ms, occ * (sb + 16)),
                      ("k_part_fine", scatter_ms - coarse_ms, occ * 32)]
        else:
            # read stream and one streamed key write per occurrence (the
            # algorithm's need; the two-level form moves the keys twice more)
            cands += [(sname, scatter_ms, occ * (sb + 16))]
        cands += [
            # keys read back; out: the k-mers counted twice or more as list
            # entries (key + count), the singleton keys, and three 4-byte Bloom
            # operations per distinct k-mer (the table itself is not written)
            ("k_part_count", count_ms,
             occ * 16 + n_ge2 * 20 + (info["n_distinct"] - n_ge2) * 16 + ops * 4),
            # Bloom ops read, both tiers written
            ("k_bloom_apply", bloom_ms, ops * 4 + 2 * info["bloom_size_bits"] / 8),
        ]
        kname, kms, kbytes = max(cands, key=lambda c: c[1])
        # every partitioned kernel's algorithmic rate, beside the dominant one
        kernel_rates = {n: {"ms": round(t, 3), "algorithmic_bytes": int(b),
                            "achieved_gbs": round(b / (t / 1e3) / 1e9, 1) if t > 0 else None}
                        for n, t, b in cands}
    elif info["schedule"] == 2 and count_ms >= bloom_ms:
        # Count-first: the read stream and a read-modify-write of the table
        # slot's sector (read + write back) per occurrence.
        kname, kms = "k_count_all", count_ms
        kbytes = occ * (sb + 2 * SECTOR)
    elif info["schedule"] == 2:
        # Bloom tiers from the table: a table scan plus three word-pair
        # sector read-modify-writes per distinct k-mer.
        kname, kms = "k_bloom_from_table", bloom_ms
        kbytes = info["table_capacity"] * 32 + info["n_distinct"] * 3 * 2 * SECTOR
    elif info["schedule"] == 1:
        # One pass: the read stream, three Bloom word-pair sectors and the
        # one-sector table slot of every occurrence.
        kname, kms = "k_fused_pass", bloom_ms
        kbytes = occ * (sb + 3 * SECTOR + SECTOR)
    elif count_ms >= bloom_ms:
        kname, kms = "k_count_pass", count_ms
        kbytes = occ * (3 * SECTOR + sb + f_adm * SECTOR)
    else:
        kname, kms = "k_bloom_pass", bloom_ms
        kbytes = occ * (3 * SECTOR + sb)
    # Whole job against the design-independent 217 B per occurrence of the
    # reference's two-pass algorithm (stream x2, Bloom insert + query, table,
    # output).
    job_bytes_per_occ = 2 * sb + 6 * SECTOR + f_adm * SECTOR + 0.3
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        with open(peaks_path) as f:
            pk = json.load(f)
        peak, peak_src = float(pk["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    else:
        peak, peak_src = 6650.0, "fallback"
    achieved = kbytes / (kms / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "dram_traffic_c2_k55.json")
    if os.path.exists(tpath) and args.scale == 1.0 and K == 55:
        # captured on the full-size k=55 job only
        with open(tpath) as f:
            traffic = json.load(f).get(kname)
    roofline = {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                # the captured DRAM bytes of the kernel over its live time: what
                # it really moves (the two-level partition moves every key three
                # times against the algorithm's once)
                "traffic_achieved": (traffic / (kms / 1e3) / 1e9) if traffic else None,
                "traffic_frac": (traffic / (kms / 1e3) / 1e9 / peak) if traffic else None,
                "peak_source": peak_src, "algorithmic_bytes_per_launch": kbytes,
                "kernel_ms": kms, "kernel_share": kms / ms, "kernels": kernel_rates,
                "job": {"bytes_per_occurrence": job_bytes_per_occ,
                        "achieved": value * job_bytes_per_occ / world,
                        "frac": value * job_bytes_per_occ / world / peak},
                "phases_ms": {"bloom_kernel": bloom_ms, "count_kernel": count_ms,
                              "bloom_phase": info["ms_bloom"], "count_phase": info["ms_count"],
                              "cutoff_compact": info["ms_finish"], "sort": info["ms_sort"],
                              "edges": info["ms_edges"]}}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = run_cpu_baseline(p, 1, 0, args.cpu_occ, args.bloom_bits)

    # the metric's batched-vs-plain part: a 64-sample batch at a tenth of the
    # specified genome sizes (the full batch: --workload c4)
    batched = None
    if rank == 0 and not args.no_batched:
        batched = batched_vs_plain(ctx, 0.1, 5, 4, args.bloom_bits, log)

    # full-size parity of one more job against the oracle (rank 0 alone; every
    # rank counts the same reads)
    parity, parity_detail = None, None
    if rank == 0 and not args.no_parity:
        parity, parity_detail = run_parity(p, lambda **kw: spk.count_device(
            d_data.data_ptr(), p.data.size, d_off.data_ptr(), d_len.data_ptr(), p.lengths.size, [K],
            ctx=ctx, bloom_bits=args.bloom_bits, **kw), args.bloom_bits, infos)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "Gk-mers/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "step_ms": [round(x, 3) for x in step_ms],
            # the library's own device time of each step's job (first to last event)
            "job_ms": [round(i["ms_total"], 3) for i in infos],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic (seeded; no public dataset)",
            "config": c2_config(p, occ, args, world),
            "parity": parity, "parity_detail": parity_detail,
            "batched": batched,
            "speedup_vs_plain": batched["speedup_vs_plain"] if batched else None,
            "job_latency_ms": batched["job_latency_ms"] if batched else None,
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
            "clocks": clocks,
            "result": {"n_solid": info["n_solid"], "n_list": info["n_list"],
                       "n_table": info["n_table"], "n_edges": info["n_edges"],
                       "cutoff": info["cutoff"], "admitted_fraction": f_adm,
                       "table_capacity": info["table_capacity"]},
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
