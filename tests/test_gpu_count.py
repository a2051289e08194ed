"""GPU parity of the counting path (spk_count, through the C ABI) against the
oracle and the golden fixtures.  Integer work: every comparison is bit-exact.

What is compared (per k):
  * the seen tier, bit for bit (src/bloom.rs:95-97 is order-free);
  * the full count table (every admitted k-mer and its count) against the
    order-free twice-tier oracle, and the sorted (k-mer, count) list for
    count >= 2 against the reference-semantics oracle (src/assemble.rs:129-242);
  * the (k+1)-mer edge list (src/graph.rs:78-102);
  * the reference-semantics solid tier as a counted difference.
"""
import hashlib

import numpy as np
import pytest

from helpers import ecoli_packed, load_npz, nlimbs, rows, synth_small_packed

pytestmark = pytest.mark.gpu

BASE = 0x1 | 0x4        # SPK_F_EDGES | SPK_F_KEEP_BLOOM
ALL = BASE | 0x2        # ... | SPK_F_REF_SOLID
GATED = 0x8             # SPK_F_GATED: the two-pass schedule
DIRECT = 0x10           # SPK_F_DIRECT: count-first with global-table atomics
KEEP_TABLE = 0x40       # SPK_F_KEEP_TABLE: the partitioned schedule also writes the table


def sha(words):
    return hashlib.sha256(np.asarray(words, dtype=np.uint64).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def spk(spk_lib):
    return spk_lib


def occ(lengths, k):
    L = np.asarray(lengths, dtype=np.int64)
    return int(np.clip(L - k + 1, 0, None).sum())


def check_against_oracle(spk, ora, data, offs, lens, k, bits, edges=True, **kw):
    """Full GPU result vs the C++ oracle (twice semantics for the table, reference
    semantics for the count >= 2 list), for every schedule: the default one
    (d: partitioned count-first for k <= 64), count-first with global atomics
    (x), the fused pass that builds the reference solid tier (r) and the gated
    one (p)."""
    tw = ora.count(data, offs, lens, k, bits, mode=ora.MODE_TWICE)
    tk, tc = tw.table(1)
    oseen, otwice = tw.bloom()
    p = spk.count((data, offs, lens), [k], bloom_bits=bits, list_min_count=1, flags=BASE | GATED, **kw)
    pk, pc = p.kmers(0, 1)
    np.testing.assert_array_equal(pk, tk)
    np.testing.assert_array_equal(pc, tc)
    ps, pt = p.bloom(0)
    np.testing.assert_array_equal(ps, oseen)
    np.testing.assert_array_equal(pt, otwice)
    pinfo = p.info(0)
    d = spk.count((data, offs, lens), [k], bloom_bits=bits, list_min_count=1, flags=BASE, **kw)
    dk, dc = d.kmers(0, 1)
    np.testing.assert_array_equal(dk, tk)
    np.testing.assert_array_equal(dc, tc)
    # the default schedule with the table kept (its admission scans the table)
    t = spk.count((data, offs, lens), [k], bloom_bits=bits, list_min_count=1, flags=BASE | KEEP_TABLE, **kw)
    tkk, tcc = t.kmers(0, 1)
    np.testing.assert_array_equal(tkk, tk)
    np.testing.assert_array_equal(tcc, tc)
    assert t.info(0)["cutoff"] == d.info(0)["cutoff"]
    np.testing.assert_array_equal(t.edges(0), d.edges(0))
    t.close()
    ds, dt = d.bloom(0)
    np.testing.assert_array_equal(ds, oseen)
    np.testing.assert_array_equal(dt, otwice)
    dinfo = d.info(0)
    x = spk.count((data, offs, lens), [k], bloom_bits=bits, list_min_count=1, flags=BASE | DIRECT, **kw)
    xk, xc = x.kmers(0, 1)
    np.testing.assert_array_equal(xk, tk)
    np.testing.assert_array_equal(xc, tc)
    xs, xt = x.bloom(0)
    np.testing.assert_array_equal(xs, oseen)
    np.testing.assert_array_equal(xt, otwice)
    xinfo = x.info(0)
    r = spk.count((data, offs, lens), [k], bloom_bits=bits, list_min_count=1, flags=ALL, **kw)
    info = r.info(0)
    for key in ("occurrences", "admitted_occurrences", "n_table", "n_list", "n_solid", "n_edges",
                "seen_popcount", "twice_popcount", "cutoff"):
        assert pinfo[key] == info[key], key
        assert dinfo[key] == info[key], key
        assert xinfo[key] == info[key], key
    assert dinfo["n_distinct"] == xinfo["n_distinct"] >= info["n_table"]
    assert pinfo["n_distinct"] == pinfo["n_table"]  # the gated table holds admitted k-mers only
    ref = ora.count(data, offs, lens, k, bits, mode=ora.MODE_REF)
    gk, gc = r.kmers(0, 1)
    np.testing.assert_array_equal(gk, tk)
    np.testing.assert_array_equal(gc, tc)
    rk, rc = ref.table(2)
    g2k, g2c = r.kmers(0, 2)
    np.testing.assert_array_equal(g2k, rk)
    np.testing.assert_array_equal(g2c, rc)
    seen, twice, ref_solid = r.bloom(0, ref_solid=True)
    np.testing.assert_array_equal(seen, oseen)
    np.testing.assert_array_equal(twice, otwice)
    # reference-semantics solid tier: a subset of the twice tier; its difference
    # against the serial reference is reported and bounded
    _, oref_solid = ref.bloom()
    assert not np.any(ref_solid & ~twice)
    diff = int(np.unpackbits((ref_solid ^ oref_solid).view(np.uint8)).sum())
    pop = int(np.unpackbits(oref_solid.view(np.uint8)).sum())
    assert diff <= max(64, pop // 50), (diff, pop)
    assert info["occurrences"] == occ(lens, k)
    assert info["admitted_occurrences"] == int(tc.astype(np.int64).sum())
    assert info["n_table"] == tk.shape[0]
    assert info["n_singletons"] == int((tc == 1).sum())
    assert info["cutoff"] == ora.cutoff(tc, 5.0)
    if edges:
        sk, sc = r.solid(0)
        e = r.edges(0)
        np.testing.assert_array_equal(e, ora.edges(sk, k))
        np.testing.assert_array_equal(p.edges(0), e)
        np.testing.assert_array_equal(d.edges(0), e)
        np.testing.assert_array_equal(x.edges(0), e)
    r.close()
    p.close()
    d.close()
    x.close()
    return info


GOLDEN = ["counts_ecoli_1K_k21.npz", "counts_ecoli_1K_k31.npz", "counts_ecoli_1K_k55.npz",
          "counts_synth_k55.npz", "counts_synth_k77.npz", "counts_synth_k32.npz",
          "counts_synth_k64.npz"]


@pytest.mark.parametrize("flags", [BASE, BASE | GATED, ALL, ALL | GATED],
                         ids=["count-first", "gated", "fused-ref", "gated-ref"])
@pytest.mark.parametrize("name", GOLDEN)
def test_count_matches_golden(spk, name, flags):
    g = load_npz(name)
    k, bits = int(g["k"]), int(g["bloom_bits"])
    if "ecoli" in name:
        data, offs, lens, _ = ecoli_packed()
    else:
        data, offs, lens = synth_small_packed()
    r = spk.count((data, offs, lens), [k], bloom_bits=bits, list_min_count=1, flags=flags)
    gk, gc = r.kmers(0, 1)
    np.testing.assert_array_equal(gk, g["twice_keys"])
    np.testing.assert_array_equal(gc, g["twice_counts"])
    g2k, g2c = r.kmers(0, 2)
    np.testing.assert_array_equal(g2k, g["ge2_keys"])
    np.testing.assert_array_equal(g2c, g["ge2_counts"])
    seen, twice = r.bloom(0)
    assert sha(seen) == str(g["seen_sha"][0])
    assert sha(twice) == str(g["twice_sha"][0])
    if "edges" in g:
        # edges over the count >= 2 set
        r2 = spk.count((data, offs, lens), [k], bloom_bits=bits, min_count=2)
        np.testing.assert_array_equal(r2.edges(0), g["edges"])


@pytest.mark.parametrize("k", [1, 11, 15, 21, 31, 32, 33, 47, 55, 63, 64, 65, 77, 89, 90, 95, 96, 97, 99, 121,
                               122, 127])
def test_count_all_key_widths(spk, ora, k):
    data, offs, lens = synth_small_packed()
    check_against_oracle(spk, ora, data, offs, lens, k, 1 << 20)


@pytest.mark.parametrize("bits", [64, 100, 100_003, 12345 * 64 + 17, (1 << 22) + 64])
def test_count_bloom_sizes(spk, ora, bits):
    """Non-power-of-two sizes use the invariant-divisor path; 64 bits admits everything."""
    data, offs, lens, _ = ecoli_packed()
    check_against_oracle(spk, ora, data, offs, lens, 31, bits)


def packed_from(reads):
    import spk as _spk
    p = _spk.PackedReads.from_clean_reads(reads)
    return p.data, p.offsets, p.lengths


def test_homopolymer_and_tandem_repeats(spk, ora):
    """Hot keys: identical k-mers inside a warp go through the aggregated add."""
    reads = ["A" * 150] * 40 + ["AC" * 75] * 40 + ["ACGT" * 40] * 40 + ["T" * 97] * 7
    data, offs, lens = packed_from(reads)
    for k in (21, 33, 55, 77):
        check_against_oracle(spk, ora, data, offs, lens, k, 1 << 16)


def test_all_read_lengths_and_offsets(spk, ora):
    """Read lengths 0..200 (every byte-boundary case) at several k."""
    rng = np.random.default_rng(9)
    reads = ["".join(rng.choice(list("ACGT"), n)) for n in range(201)] * 2
    data, offs, lens = packed_from(reads)
    for k in (1, 17, 32, 33, 64, 65, 127):
        check_against_oracle(spk, ora, data, offs, lens, k, 1 << 18)


def test_empty_and_short_inputs(spk):
    r = spk.count((np.zeros(0, np.uint8), np.zeros(0, np.uint64), np.zeros(0, np.uint32)), [31])
    i = r.info(0)
    assert i["occurrences"] == 0 and i["n_list"] == 0 and i["n_edges"] == 0
    assert r.kmers(0)[0].shape[0] == 0 and r.edges(0).shape[0] == 0
    data, offs, lens = packed_from(["ACGT" * 5, "A" * 30, "ACGTACGTAC"])
    r = spk.count((data, offs, lens), [31])
    assert r.info(0)["occurrences"] == 0
    data, offs, lens = packed_from(["ACGTTGCAAC" * 3 + "A"])
    r = spk.count((data, offs, lens), [31], list_min_count=1)
    i = r.info(0)
    assert i["occurrences"] == 1 and i["n_list"] <= 1


def test_table_regrow(spk, ora):
    """A deliberately undersized table overflows its probe limit; the host
    regrows it and recounts, with the same result."""
    data, offs, lens = synth_small_packed()
    want = spk.count((data, offs, lens), [55], bloom_bits=1 << 20, list_min_count=1)
    r = spk.count((data, offs, lens), [55], bloom_bits=1 << 20, list_min_count=1, table_log2=4)
    assert r.info(0)["table_regrows"] > 0
    a, b = want.kmers(0, 1), r.kmers(0, 1)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])


def test_invalid_inputs(spk):
    data, offs, lens = packed_from(["ACGT" * 20])
    with pytest.raises(spk.SpkError) as e:
        spk.count((data, offs + np.uint64(100), lens), [21])
    assert e.value.code == 1
    for bad_k in (0, 128, 500):
        with pytest.raises(spk.SpkError) as e:
            spk.count((data, offs, lens), [bad_k])
        assert e.value.code == 2
    with pytest.raises(spk.SpkError):
        spk.count((data, offs, lens), [])


def test_multik_equals_single_k(spk):
    """One call over several k (the per-k loop of src/multik.rs:109-178) gives,
    per k, exactly the single-k result."""
    data, offs, lens = synth_small_packed()
    ks = [21, 33, 55, 77]
    multi = spk.count((data, offs, lens), ks, bloom_bits=1 << 22)
    for i, k in enumerate(ks):
        one = spk.count((data, offs, lens), [k], bloom_bits=1 << 22)
        for a, b in zip(multi.kmers(i), one.kmers(0)):
            np.testing.assert_array_equal(a, b)
        np.testing.assert_array_equal(multi.edges(i), one.edges(0))


@pytest.mark.parametrize("k,flags", [(21, BASE), (55, BASE), (77, BASE), (55, BASE | GATED), (55, BASE | DIRECT)])
def test_solid_out_buffers(spk, k, flags):
    """spk_count_opts.solid_*_out: the count fills the caller's host buffers
    with the first k's solid list (the default job while it builds the edges,
    the other schedules after the job), exactly what spk_result_solid gives;
    a list longer than the buffers is not copied and leaves them untouched."""
    data, offs, lens = synth_small_packed()
    want_k, want_c = spk.count((data, offs, lens), [k], bloom_bits=1 << 22, flags=flags).solid(0)
    n = len(want_c)
    assert n > 0
    L = nlimbs(k)
    keys = np.full((n + 5, L), 0xAB, dtype=np.uint64)
    counts = np.full(n + 5, 7, dtype=np.uint32)
    r = spk.count((data, offs, lens), [k], bloom_bits=1 << 22, flags=flags, solid_out=(keys, counts))
    info = r.info(0)
    assert info["solid_copied"] == 1 and info["n_solid"] == n
    np.testing.assert_array_equal(keys[:n], want_k)
    np.testing.assert_array_equal(counts[:n], want_c)
    assert (keys[n:] == 0xAB).all() and (counts[n:] == 7).all()
    gk, gc = r.solid(0)  # the download after it gives the same list
    np.testing.assert_array_equal(gk, want_k)
    np.testing.assert_array_equal(gc, want_c)
    small_k = np.full((n - 1, L), 0xAB, dtype=np.uint64)
    small_c = np.full(n - 1, 7, dtype=np.uint32)
    r2 = spk.count((data, offs, lens), [k], bloom_bits=1 << 22, flags=flags, solid_out=(small_k, small_c))
    assert r2.info(0)["solid_copied"] == 0
    assert (small_k == 0xAB).all() and (small_c == 7).all()
    np.testing.assert_array_equal(r2.solid(0)[0], want_k)


def test_solid_out_first_k_of_several(spk):
    """With several k, the buffers receive the first k's solid list only."""
    data, offs, lens = synth_small_packed()
    want_k, want_c = spk.count((data, offs, lens), [33], bloom_bits=1 << 22).solid(0)
    n = len(want_c)
    keys = np.zeros((n, nlimbs(33)), dtype=np.uint64)
    counts = np.zeros(n, dtype=np.uint32)
    r = spk.count((data, offs, lens), [33, 55], bloom_bits=1 << 22, solid_out=(keys, counts))
    assert r.info(0)["solid_copied"] == 1 and r.info(1)["solid_copied"] == 0
    np.testing.assert_array_equal(keys, want_k)
    np.testing.assert_array_equal(counts, want_c)


def test_count_device_pointers(spk):
    """spk_count_device on device-resident reads, including an unaligned base pointer."""
    import torch
    data, offs, lens = synth_small_packed()
    host = spk.count((data, offs, lens), [55], bloom_bits=1 << 22)
    for shift in (0, 3):
        buf = torch.zeros(data.size + 64 + shift, dtype=torch.uint8, device="cuda")
        buf[shift:shift + data.size] = torch.from_numpy(data).cuda()
        d_off = torch.from_numpy(offs.astype(np.int64)).cuda()
        d_len = torch.from_numpy(lens.astype(np.int32)).cuda()
        torch.cuda.synchronize()
        r = spk.count_device(buf.data_ptr() + shift, data.size, d_off.data_ptr(), d_len.data_ptr(),
                             lens.size, [55], bloom_bits=1 << 22)
        for a, b in zip(r.kmers(0), host.kmers(0)):
            np.testing.assert_array_equal(a, b)


def test_solid_cutoff_and_seam(spk, ora):
    """count_solid_kmers (the Stage 2-3 seam) returns the HashMap of count >= 2
    k-mers; the solid list applies the adaptive cutoff (src/assemble.rs:286-292)."""
    data, offs, lens, _ = ecoli_packed()
    m = spk.count_solid_kmers((data, offs, lens), 31, bloom_bits=16 << 20)
    ref = ora.count(data, offs, lens, 31, 16 << 20, mode=ora.MODE_REF)
    rk, rc = ref.table(2)
    assert m == {spk.kmer256_from_limbs(k): int(c) for k, c in zip(rk, rc)}
    r = spk.count((data, offs, lens), [31], bloom_bits=16 << 20)
    sk, sc = r.solid(0)
    cut = r.info(0)["cutoff"]
    assert np.all(sc >= cut)
    assert sk.shape[0] == int((rc >= cut).sum())


def test_schedules(spk):
    """Partitioned count-first by default: with a one-level partition for k
    <= 64 on small read sets, two levels otherwise, and for k > 64 once the
    read set has enough spans for two levels (else, and for k = 96, whose keys
    fill three limbs, count-first with global atomics); the reference solid
    tier selects the fused pass and SPK_F_GATED the two-pass schedule."""
    from spk import synth
    data, offs, lens = synth_small_packed()
    assert spk.count((data, offs, lens), [55]).info(0)["schedule"] == 3
    assert spk.count((data, offs, lens), [21]).info(0)["schedule"] == 3
    assert spk.count((data, offs, lens), [77]).info(0)["schedule"] == 2
    p = synth.c2(0.05).packed
    for k, sched in ((77, 3), (127, 3), (96, 2)):
        i = spk.count(p, [k], bloom_bits=1 << 26).info(0)
        assert i["schedule"] == sched, k
        assert i["part_passes"] == (2 if sched == 3 else 0), k
    assert spk.count((data, offs, lens), [55], flags=DIRECT).info(0)["schedule"] == 2
    assert spk.count((data, offs, lens), [55], flags=ALL).info(0)["schedule"] == 1
    assert spk.count((data, offs, lens), [55], flags=GATED).info(0)["schedule"] == 0
    assert spk.count((data, offs, lens), [55], flags=ALL | GATED).info(0)["schedule"] == 0


def test_fused_table_regrow(spk, ora):
    """The one-pass table (every distinct k-mer) starting far too small regrows and recounts."""
    data, offs, lens = synth_small_packed()
    check_against_oracle(spk, ora, data, offs, lens, 31, 1 << 20, table_log2=6)


def test_list_threshold_above_two(spk, ora):
    """list_min_count above 2 with the adaptive cutoff: the list and its length
    hold exactly the k-mers with count >= min(list_min_count, cutoff)."""
    data, offs, lens = synth_small_packed()
    ref = ora.count(data, offs, lens, 55, 1 << 20, mode=ora.MODE_TWICE)
    tk, tc = ref.table(1)
    r = spk.count((data, offs, lens), [55], bloom_bits=1 << 20, list_min_count=5)
    i = r.info(0)
    thr = min(5, i["cutoff"])
    keys, counts = r.kmers(0)
    np.testing.assert_array_equal(keys, tk[tc >= thr])
    np.testing.assert_array_equal(counts, tc[tc >= thr])
    assert i["n_list"] == int((tc >= thr).sum())
    assert i["n_solid"] == int((tc >= i["cutoff"]).sum())


@pytest.mark.parametrize("table_log2", [16, 21])
def test_partition_rescatter_on_skew(spk, ora, table_log2):
    """A k-mer that makes up most occurrences overflows its span's region:
    the read pass is repeated with exact region sizes and the result is
    unchanged."""
    data, offs, lens = synth_small_packed()
    # 400 poly-A reads of 150 bases: 48,000 occurrences of one k-mer, more
    # than its span's region holds next to that span's share of the rest.
    extra = np.zeros(38 * 400, dtype=np.uint8)
    d2 = np.concatenate([data[: int(offs[-1]) + (int(lens[-1]) + 3) // 4], extra])
    o2 = np.concatenate([offs, int(offs[-1]) + (int(lens[-1]) + 3) // 4 + 38 * np.arange(400, dtype=np.uint64)])
    l2 = np.concatenate([lens, np.full(400, 150, dtype=np.uint32)])
    info = check_against_oracle(spk, ora, d2, o2.astype(np.uint64), l2.astype(np.uint32), 31,
                                1 << 20, table_log2=table_log2)
    r = spk.count((d2, o2.astype(np.uint64), l2.astype(np.uint32)), [31], bloom_bits=1 << 20,
                  table_log2=table_log2, flags=BASE | KEEP_TABLE)
    ri = r.info(0)
    assert ri["schedule"] == 3 and ri["part_rescatters"] >= 1
    assert ri["part_passes"] == (2 if table_log2 == 21 else 1)  # 256 spans: two-level partition
    assert ri["n_table"] == info["n_table"]
    v = r.table_view(0)
    assert v["log2span"] == 13 and v["capacity"] == 1 << table_log2  # 8192-slot spans for k <= 32


def test_two_level_rescatter_on_skew_k55(spk, ora):
    """The two-level read partition (16-byte keys) with one k-mer making up
    most occurrences: its coarse bucket and its span both overflow, both
    passes are repeated with exact sizes, and the result equals the oracle's."""
    data, offs, lens = synth_small_packed()
    extra = np.zeros(38 * 400, dtype=np.uint8)  # 400 poly-A reads of 150 bases
    d2 = np.concatenate([data[: int(offs[-1]) + (int(lens[-1]) + 3) // 4], extra])
    o2 = np.concatenate([offs, int(offs[-1]) + (int(lens[-1]) + 3) // 4 + 38 * np.arange(400, dtype=np.uint64)])
    l2 = np.concatenate([lens, np.full(400, 150, dtype=np.uint32)])
    o2, l2 = o2.astype(np.uint64), l2.astype(np.uint32)
    info = check_against_oracle(spk, ora, d2, o2, l2, 55, 1 << 20, table_log2=21)
    r = spk.count((d2, o2, l2), [55], bloom_bits=1 << 20, table_log2=21)
    ri = r.info(0)
    assert ri["schedule"] == 3 and ri["part_passes"] == 2 and ri["part_rescatters"] >= 1
    assert ri["n_table"] == info["n_table"]


def test_one_bloom_range_direct_emission(spk, ora):
    """A 2^19-bit Bloom is a single range, so a span's Bloom operations all
    fall into it; with 64 spans of ~790 distinct k-mers each they exceed half
    a span (2,048), and the span pass emits them directly instead of sorting
    them.  The tiers and the table equal the oracle's.  (The order-dependent
    reference solid tier is left out: a Bloom this small is saturated.)"""
    data, offs, lens = synth_small_packed()
    bits = 1 << 19
    tw = ora.count(data, offs, lens, 55, bits, mode=ora.MODE_TWICE)
    tk, tc = tw.table(1)
    oseen, otwice = tw.bloom()
    r = spk.count((data, offs, lens), [55], bloom_bits=bits, list_min_count=1, flags=BASE, table_log2=18)
    assert r.info(0)["schedule"] == 3
    gk, gc = r.kmers(0, 1)
    np.testing.assert_array_equal(gk, tk)
    np.testing.assert_array_equal(gc, tc)
    seen, twice = r.bloom(0)
    np.testing.assert_array_equal(seen, oseen)
    np.testing.assert_array_equal(twice, otwice)
    sk, _ = r.solid(0)
    np.testing.assert_array_equal(r.edges(0), ora.edges(sk, 55))


@pytest.mark.parametrize("k,table_log2", [(21, 22), (55, 22), (55, 20), (64, 23)])
def test_many_spans(spk, ora, k, table_log2):
    """Tables of hundreds of spans: the result equals the oracle's."""
    data, offs, lens = synth_small_packed()
    check_against_oracle(spk, ora, data, offs, lens, k, 1 << 20, table_log2=table_log2)
    r = spk.count((data, offs, lens), [k], bloom_bits=1 << 20, table_log2=table_log2,
                  flags=BASE | KEEP_TABLE)
    v = r.table_view(0)
    assert r.info(0)["schedule"] == 3 and v["capacity"] == 1 << table_log2
    assert (table_log2 - v["log2span"]) >= 8


def _pack_codes(rows):
    """Packed reads (src/packed_reads.rs:547-578) from rows of 2-bit codes."""
    data, offs, lens = [], [], []
    o = 0
    for c in rows:
        c = np.asarray(c, dtype=np.uint8)
        pad = np.zeros((len(c) + 3) // 4 * 4, dtype=np.uint8)
        pad[: len(c)] = c
        q = pad.reshape(-1, 4)
        data.append((q[:, 0] << 6) | (q[:, 1] << 4) | (q[:, 2] << 2) | q[:, 3])
        offs.append(o)
        lens.append(len(c))
        o += q.shape[0]
    return np.concatenate(data).astype(np.uint8), np.array(offs, np.uint64), np.array(lens, np.uint32)


def test_large_lists_bucket_sort(spk, ora):
    """Lists long enough for the bucketed sort (2^18 entries and more), with
    one top-bits bucket far over its shared-memory size (k-mers that start
    with eight A): the sorted list and edges equal the oracle's."""
    from spk import synth
    p = synth.c2(0.05).packed
    rng = np.random.default_rng(5)
    rows = []
    for _ in range(1500):
        blocks = [np.concatenate([np.zeros(8, np.uint8), rng.integers(0, 4, 8, dtype=np.uint8)])
                  for _ in range(10)]
        r = np.concatenate(blocks)[:150]
        rows += [r, r]  # twice, so that its k-mers are listed (count >= 2)
    d2, o2, l2 = _pack_codes(rows)
    data = np.concatenate([p.data, d2])
    offs = np.concatenate([p.offsets, o2 + np.uint64(p.data.size)])
    lens = np.concatenate([p.lengths, l2])
    k, bits = 55, 1 << 26
    ref = ora.count(data, offs, lens, k, bits, mode=ora.MODE_TWICE, keep_bloom=False)
    tk, tc = ref.table(2)
    assert tk.shape[0] > (1 << 18)
    assert int((tk[:, 1] >> np.uint64(2 * k - 64 - 16) == 0).sum()) > 2048  # the big bucket
    r = spk.count((data, offs, lens), [k], bloom_bits=bits)
    gk, gc = r.kmers(0)
    np.testing.assert_array_equal(gk, tk)
    np.testing.assert_array_equal(gc, tc)
    sk, _ = r.solid(0)
    np.testing.assert_array_equal(r.edges(0), ora.edges(sk, k))


@pytest.mark.parametrize("k,table_log2", [(55, 21), (77, 22)])
def test_span_count_grows_full_spans(spk, ora, k, table_log2):
    """Too few slots for the distinct k-mers (forced with table_log2): spans
    run out of slots, the job stops early and runs again with twice the
    slots; the admitted table, tiers, cutoff and edges equal the oracle's."""
    import os
    from spk import synth
    p = synth.c2(0.05).packed
    bits = 1 << 26
    tw = ora.count(p.data, p.offsets, p.lengths, k, bits, mode=ora.MODE_TWICE, threads=os.cpu_count() or 1)
    tk, tc = tw.table(1)
    oseen, otwice = tw.bloom()
    r = spk.count(p, [k], bloom_bits=bits, list_min_count=1, table_log2=table_log2, flags=BASE)
    info = r.info(0)
    assert info["n_distinct"] > 3 << (table_log2 - 2)  # most spans over their slots at first
    assert info["schedule"] == 3 and info["table_regrows"] >= 1
    assert info["table_capacity"] == 1 << (table_log2 + info["table_regrows"])
    gk, gc = r.kmers(0, 1)
    np.testing.assert_array_equal(gk, tk)
    np.testing.assert_array_equal(gc, tc)
    seen, twice = r.bloom(0)
    np.testing.assert_array_equal(seen, oseen)
    np.testing.assert_array_equal(twice, otwice)
    assert info["cutoff"] == ora.cutoff(tc, 5.0)
    sk, _ = r.solid(0)
    np.testing.assert_array_equal(r.edges(0), ora.edges(sk, k))


@pytest.mark.parametrize("k", [55, 77])
def test_many_large_buckets_sort(spk, ora, k):
    """Lists with many top-bits buckets over their shared-memory size (40
    eight-base prefixes with 3000 listed k-mers each): those buckets are
    sorted together as one array, and the list and edges equal the oracle's."""
    import os
    from spk import synth
    p = synth.c2(0.05).packed
    rng = np.random.default_rng(11)
    prefixes = rng.integers(0, 4, (40, 8), dtype=np.uint8)
    prefixes[:, 0] = 0  # a leading A: mostly the canonical strand
    rows = []
    for pre in prefixes:
        for _ in range(3000):
            r = np.concatenate([pre, rng.integers(0, 4, k - 8, dtype=np.uint8)])
            rows += [r, r]  # twice, so that the k-mer is listed (count >= 2)
    d2, o2, l2 = _pack_codes(rows)
    data = np.concatenate([p.data, d2])
    offs = np.concatenate([p.offsets, o2 + np.uint64(p.data.size)])
    lens = np.concatenate([p.lengths, l2])
    bits = 1 << 26
    ref = ora.count(data, offs, lens, k, bits, mode=ora.MODE_TWICE, keep_bloom=False,
                    threads=os.cpu_count() or 1)
    tk, tc = ref.table(2)
    # the first eight bases: the top 16 bits of the key (Kmer256 keeps the
    # first 64 bases of a k > 64 in its low half, limb 1 on top)
    nl = nlimbs(k)
    top = tk[:, 1] >> np.uint64(48) if k > 64 else tk[:, nl - 1] >> np.uint64(2 * k - 64 * (nl - 1) - 16)
    _, sizes = np.unique(top, return_counts=True)
    assert tk.shape[0] > (1 << 18) and int((sizes > 2048).sum()) >= 20
    r = spk.count((data, offs, lens), [k], bloom_bits=bits)
    assert r.info(0)["schedule"] == 3
    gk, gc = r.kmers(0)
    np.testing.assert_array_equal(gk, tk)
    np.testing.assert_array_equal(gc, tc)
    sk, _ = r.solid(0)
    np.testing.assert_array_equal(r.edges(0), ora.edges(sk, k))


@pytest.mark.parametrize("k", [31, 55, 77])
def test_prior_contigs(spk, ora, k):
    """Prior and trusted contigs (src/assemble.rs:244-284) add their boost to
    every accepted k-window after singleton admission and before the cutoff:
    the table, the cutoff and the edges equal the oracle's count followed by
    its prior injection."""
    from oracle import pyref
    data, offs, lens = synth_small_packed()
    reads = [pyref.get_read(data, offs, lens, i) for i in range(0, 200, 7)]
    rng = np.random.default_rng(k)
    priors = [r[5:120].encode() for r in reads[:20]]                       # known k-mers, singletons
    priors += ["".join("ACGT"[b] for b in rng.integers(0, 4, 300)).encode()]  # new k-mers
    priors += [(reads[20][:60].lower() + "NN" + reads[20][60:]).encode()]   # case, ambiguous bases
    priors += [b"ACGT" * 5]                                                  # shorter than k
    bits = 1 << 20
    ref = ora.count(data, offs, lens, k, bits, mode=ora.MODE_TWICE)
    ref.inject_priors(priors, 50)  # max(4 * 5, 50) with the default min_coverage 5.0
    tk, tc = ref.table(1)
    for flags in (BASE, BASE | GATED):
        r = spk.count((data, offs, lens), [k], bloom_bits=bits, list_min_count=1, flags=flags,
                      priors=priors)
        gk, gc = r.kmers(0, 1)
        np.testing.assert_array_equal(gk, tk)
        np.testing.assert_array_equal(gc, tc)
        info = r.info(0)
        assert info["cutoff"] == ora.cutoff(tc, 5.0)
        assert info["n_table"] == tk.shape[0]
        sk, _ = r.solid(0)
        np.testing.assert_array_equal(r.edges(0), ora.edges(sk, k))


@pytest.mark.parametrize("k", [77, 127])
def test_claim_wait_times_out(spk, ora, k):
    """A wide-key table slot left claimed and never published (a writer gone
    mid-claim): the reader's bounded wait gives up after a fraction of a
    second, the call returns SPK_E_TIMEOUT (5), and the context still counts."""
    import time
    from spk._lib import lib
    ctx = spk.Context(0)
    t0 = time.time()
    rc = lib().spk_diag_stuck_claim(ctx.h, k)
    assert rc == 5, spk._lib.last_error()
    assert "claim wait timed out" in spk._lib.last_error()
    assert time.time() - t0 < 30
    data, offs, lens = synth_small_packed()
    r = spk.count((data, offs, lens), [k], ctx=ctx, bloom_bits=1 << 20, list_min_count=1)
    tw = ora.count(data, offs, lens, k, 1 << 20, mode=ora.MODE_TWICE)
    gk, gc = r.kmers(0, 1)
    tk, tc = tw.table(1)
    np.testing.assert_array_equal(gk, tk)
    np.testing.assert_array_equal(gc, tc)
    r.close()
    with pytest.raises(spk.SpkError):
        spk._lib.check(lib().spk_diag_stuck_claim(ctx.h, 55))


def test_table_view_needs_keep_table(spk):
    """Without SPK_F_KEEP_TABLE the partitioned schedule writes the list from
    its spans and keeps no table: the view is refused; with it, the view
    describes the table; the lists are the same either way."""
    data, offs, lens = synth_small_packed()
    a = spk.count((data, offs, lens), [55], bloom_bits=1 << 20)
    assert a.info(0)["schedule"] == 3
    with pytest.raises(spk.SpkError) as e:
        a.table_view(0)
    assert e.value.code == 1 and "SPK_F_KEEP_TABLE" in str(e.value)
    b = spk.count((data, offs, lens), [55], bloom_bits=1 << 20, flags=BASE | KEEP_TABLE)
    v = b.table_view(0)
    assert v["slots"] and v["capacity"] == b.info(0)["table_capacity"]
    for x, y in zip(a.kmers(0), b.kmers(0)):
        np.testing.assert_array_equal(x, y)
    np.testing.assert_array_equal(a.edges(0), b.edges(0))


@pytest.mark.parametrize("k", [21, 55, 77])
def test_span_groups_equal_one_pass(spk, ora, k):
    """Read sets too large for one partition pass are counted in groups of
    spans, one pass over the reads each (forced here with span_groups_log2):
    the whole admitted table, both tiers, cutoff and edges equal the oracle's
    and the one-pass result."""
    import os
    from spk import synth
    p = synth.c2(0.05).packed
    bits = 1 << 26
    tw = ora.count(p.data, p.offsets, p.lengths, k, bits, mode=ora.MODE_TWICE, threads=os.cpu_count() or 1)
    tk, tc = tw.table(1)
    oseen, otwice = tw.bloom()
    one = spk.count(p, [k], bloom_bits=bits, list_min_count=1, table_log2=24)
    for lg in (1, 2):
        r = spk.count(p, [k], bloom_bits=bits, list_min_count=1, table_log2=24, span_groups_log2=lg)
        info = r.info(0)
        assert info["span_groups"] == 1 << lg and info["schedule"] == 3
        gk, gc = r.kmers(0, 1)
        np.testing.assert_array_equal(gk, tk)
        np.testing.assert_array_equal(gc, tc)
        seen, twice = r.bloom(0)
        np.testing.assert_array_equal(seen, oseen)
        np.testing.assert_array_equal(twice, otwice)
        assert info["occurrences"] == one.info(0)["occurrences"]
        assert info["cutoff"] == ora.cutoff(tc, 5.0) == one.info(0)["cutoff"]
        np.testing.assert_array_equal(r.edges(0), one.edges(0))
        # the default listing (count >= 2) through the same groups
        d = spk.count(p, [k], bloom_bits=bits, table_log2=24, span_groups_log2=lg)
        dk, dc = d.kmers(0)
        np.testing.assert_array_equal(dk, tk[tc >= 2])
        np.testing.assert_array_equal(dc, tc[tc >= 2])
        r.close()
        d.close()
