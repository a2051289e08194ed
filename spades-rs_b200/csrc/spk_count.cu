// spk_count.cu -- the k-mer counting pipeline on one B200.
//
// Replaces Stages 2-3 of run_assembly_with_packed_reads (src/assemble.rs:
// 129-292) and the implicit edge probes of CompactedGraph::build
// (src/graph.rs:78-102).
//
// Admission.  The reference promotes a k-mer to its solid tier only when an
// insert finds all three seen bits already set, which depends on the order of
// the rayon chunks (src/bloom.rs:95-106), and counts (Stage 3) every
// occurrence of a k-mer whose three solid bits are set.  The GPU keeps an
// order-free twice tier instead: a seen-tier fetch_or that finds its bit set
// also sets that bit in the twice tier.  The admitted set is every k-mer whose
// three twice bits are set; it contains every k-mer that occurs at least twice,
// so the count >= 2 list is exact and equals the reference's.  The
// reference-semantics solid tier is still produced on request
// (SPK_F_REF_SOLID).
//
// Three schedules compute that same admitted table:
//   count-first  (default) one pass over the reads counts every canonical
//                k-mer occurrence in a table that holds every distinct
//                k-mer, with one hash and one table update per occurrence.
//                The Bloom tiers are then derived from the table (a k-mer
//                counted c times makes c insert operations on each of its
//                three bits; the tiers do not depend on their order), and
//                each k-mer seen once is kept only if its three twice bits
//                are set (a k-mer seen twice always has them).
//   fused        (SPK_F_REF_SOLID without SPK_F_GATED) the same single read
//                pass with the three Bloom insert operations of every
//                occurrence in it, which the reference-semantics solid tier
//                needs because it depends on the order of the inserts.
//   gated        (SPK_F_GATED) the reference's two passes: Stage 2 fills the
//                Bloom, Stage 3 counts only occurrences whose three twice
//                bits are set.  The table then holds only admitted k-mers,
//                which bounds memory on very large read sets.
// All are followed by the cutoff (src/assemble.rs:692-735), a compaction of
// the table into the k-mer list, a radix sort and the edge list.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "spk_internal.h"

namespace spk {

constexpr unsigned FULL = 0xffffffffu;
constexpr int kBlock = 256;
constexpr uint64_t kEmpty = ~0ULL;
constexpr uint32_t kMaxProbe = 4096;
constexpr int kSpinLimit = 1 << 22;
constexpr uint32_t kRejected = 0x80000000u;  // count flag: a singleton the twice tier does not admit

struct alignas(16) U128 {
  unsigned long long x, y;
};

// ---------------------------------------------------------------------------
// Count table slots: one slot per 16/32/64 bytes, key limbs first, the count
// right after them, so a lookup and its increment touch one DRAM sector.
//   NL = 1 (k <= 32):  16 B  key[1] count pad
//   NL = 2 (k <= 64):  32 B  key[2] count pad pad
//   NL = 3 (k <= 96):  32 B  key[3] count state
//   NL = 4 (k <= 127): 64 B  key[4] count state pad...
// ---------------------------------------------------------------------------
template <int NL>
struct Slot {
  static constexpr uint32_t bytes = NL == 1 ? 16 : (NL <= 3 ? 32 : 64);
  static constexpr uint32_t count_off = NL * 8;
  static constexpr uint32_t state_off = NL * 8 + 4;
};
__host__ __device__ constexpr uint32_t slot_bytes(int nl) { return nl == 1 ? 16 : (nl <= 3 ? 32 : 64); }

template <int NL>
__device__ __forceinline__ uint64_t* slot_key(const TableView& t, uint64_t s) {
  return (uint64_t*)(t.slots + s * Slot<NL>::bytes);
}
template <int NL>
__device__ __forceinline__ uint32_t* slot_count(const TableView& t, uint64_t s) {
  return (uint32_t*)(t.slots + s * Slot<NL>::bytes + Slot<NL>::count_off);
}
template <int NL>
__device__ __forceinline__ uint32_t* slot_state(const TableView& t, uint64_t s) {
  return (uint32_t*)(t.slots + s * Slot<NL>::bytes + Slot<NL>::state_off);
}

// Empty slots: keys of <= 128 bits hold the all-ones sentinel (no canonical
// k-mer equals it: for k < 32 / k < 64 the top bits are unused, for k = 32 /
// 64 all-ones is poly-T whose reverse complement poly-A is smaller); wider
// keys are empty while their state word is 0.  Counts start at 0.
template <int NL>
__global__ void __launch_bounds__(kBlock) k_table_init(uint8_t* __restrict__ slots, uint64_t cap) {
  const uint64_t words = cap * Slot<NL>::bytes / 16;
  ulonglong2* p = (ulonglong2*)slots;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < words;
       i += (uint64_t)gridDim.x * blockDim.x) {
    ulonglong2 v = make_ulonglong2(0ULL, 0ULL);
    if (NL == 1) v = make_ulonglong2(~0ULL, 0ULL);                        // key | count, pad
    if (NL == 2 && (i & 1) == 0) v = make_ulonglong2(~0ULL, ~0ULL);       // key limbs
    p[i] = v;
  }
}

// ---------------------------------------------------------------------------
// Position iteration.  A warp takes 32 consecutive reads, scans their k-mer
// counts and then walks the concatenated positions 32 at a time, so lanes
// stay busy regardless of read length.  f(active, bitpos) is called by all 32
// lanes (it may use warp collectives); inactive lanes must not touch memory.
// ---------------------------------------------------------------------------
template <class F>
__device__ __forceinline__ void foreach_position(const ReadsView& R, unsigned k, F& f) {
  const unsigned lane = threadIdx.x & 31;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t b = warp * 32; b < R.n_reads; b += nwarps * 32) {
    const uint64_t r = b + lane;
    uint32_t len = 0;
    uint64_t off = 0;
    if (r < R.n_reads) {
      len = __ldg(R.lengths + r);
      off = __ldg(R.offsets + r);
      // get_read slices data[off .. off + ceil(len/4)] (src/packed_reads.rs:600-602)
      if (off + ((uint64_t)len + 3) / 4 > R.data_len) {
        atomicOr(R.err, 4);
        len = 0;
      }
    }
    const uint32_t np = len >= k ? len - k + 1 : 0;
    uint32_t incl = np;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      uint32_t t = __shfl_up_sync(FULL, incl, d);
      if ((int)lane >= d) incl += t;
    }
    const uint32_t excl = incl - np;
    const uint32_t total = __shfl_sync(FULL, incl, 31);
    for (uint32_t base = 0; base < total; base += 32) {
      const uint32_t p = base + lane;
      unsigned j = 0;
#pragma unroll
      for (unsigned step = 16; step >= 1; step >>= 1) {
        uint32_t c = __shfl_sync(FULL, incl, j + step - 1);
        if (p >= c) j += step;
      }
      const uint64_t o = __shfl_sync(FULL, off, j);
      const uint32_t e = __shfl_sync(FULL, excl, j);
      const bool active = p < total;
      const uint64_t bitpos = 8ull * (R.byte_base + o) + 2ull * (uint64_t)(p - e);
      f(active, bitpos);
    }
  }
}

template <int NL>
__device__ __forceinline__ void bloom_positions(const Seq<NL>& C, unsigned k, const FastMod& fm,
                                                uint64_t raw[3], uint64_t pos[3]) {
  uint64_t w4[4];
  kmer256_limbs<NL>(C, k, w4);
  HashPre hp = hash_pre(w4);
  raw[0] = hash_seed(hp, kSeed1);
  raw[1] = hash_seed(hp, kSeed2);
  raw[2] = hash_seed(hp, kSeed3);
#pragma unroll
  for (int i = 0; i < 3; i++) pos[i] = fastmod(fm, raw[i]);
}

__device__ __forceinline__ void warp_add_u64(unsigned long long* dst, uint64_t v) {
#pragma unroll
  for (int d = 16; d >= 1; d >>= 1) v += __shfl_xor_sync(FULL, v, d);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(dst, (unsigned long long)v);
}

// The three seen fetch_or of src/bloom.rs:95-97 on interleaved (seen, twice)
// word pairs; a fetch_or that finds its bit already set also sets the twice
// bit.  Returns whether all three bits were already seen (src/bloom.rs:99).
__device__ __forceinline__ bool bloom_insert3(U128* __restrict__ tiers, const uint64_t pos[3]) {
  U128 t[3];
#pragma unroll
  for (int i = 0; i < 3; i++) t[i] = tiers[pos[i] >> 6];
  bool allprev = true;
#pragma unroll
  for (int i = 0; i < 3; i++) {
    const uint64_t w = pos[i] >> 6;
    const unsigned long long bit = 1ULL << (pos[i] & 63);
    bool prev;
    if (t[i].x & bit) {
      // Seen bits are only ever set, so a set bit read here (even from a
      // stale cached line) was set by an earlier insert.
      prev = true;
      if (!(t[i].y & bit)) atomicOr(&tiers[w].y, bit);
    } else {
      const unsigned long long p = atomicOr(&tiers[w].x, bit);
      prev = (p & bit) != 0;
      if (prev) atomicOr(&tiers[w].y, bit);
    }
    allprev &= prev;
  }
  return allprev;
}

__device__ __forceinline__ void ref_promote(unsigned long long* __restrict__ ref_solid,
                                            const uint64_t pos[3]) {  // src/bloom.rs:99-103
#pragma unroll
  for (int i = 0; i < 3; i++) {
    const unsigned long long bit = 1ULL << (pos[i] & 63);
    unsigned long long* a = ref_solid + (pos[i] >> 6);
    if (!(*a & bit)) atomicOr(a, bit);
  }
}

// ---------------------------------------------------------------------------
// Count table operations
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t table_home(const TableView& t, uint64_t raw0) {
  return raw0 >> (64 - t.log2cap);
}

// Adds n to key C.  Keys of <= 128 bits claim a slot with one 64- or 128-bit
// CAS against the sentinel; wider keys claim the state word, publish the key
// and mark the slot ready.
// The first key words of the home slot, loaded early so the table probe
// overlaps the Bloom accesses of the same occurrence.
struct SlotPeek {
  unsigned long long x, y;
};
template <int NL>
__device__ __forceinline__ SlotPeek table_peek(const TableView& t, uint64_t home) {
  SlotPeek p{kEmpty, kEmpty};
  if (NL == 1) p.x = __ldcg((const unsigned long long*)slot_key<NL>(t, home));
  if (NL == 2) {
    const ulonglong2 v = __ldcg((const ulonglong2*)slot_key<NL>(t, home));
    p.x = v.x;
    p.y = v.y;
  }
  return p;
}

template <int NL>
__device__ __forceinline__ void table_add(const TableView& t, const Seq<NL>& C, uint64_t home,
                                          uint32_t n, const SlotPeek* peek = nullptr) {
  const uint64_t mask = t.capacity - 1;
  for (uint32_t i = 0; i < t.max_probe; i++) {
    const uint64_t s = (home + i) & mask;
    uint64_t* kp = slot_key<NL>(t, s);
    if (NL == 1) {
      unsigned long long cur = (i == 0 && peek) ? peek->x : __ldcg((const unsigned long long*)kp);
      if (cur == C.v[0]) { atomicAdd(slot_count<NL>(t, s), n); return; }
      if (cur == kEmpty) {
        unsigned long long old = atomicCAS((unsigned long long*)kp, kEmpty, (unsigned long long)C.v[0]);
        if (old == kEmpty || old == C.v[0]) { atomicAdd(slot_count<NL>(t, s), n); return; }
      }
    } else if (NL == 2) {
      ulonglong2 cur;
      if (i == 0 && peek) cur = make_ulonglong2(peek->x, peek->y);
      else cur = __ldcg((const ulonglong2*)kp);
      if (cur.x != kEmpty && cur.y != kEmpty) {
        // A settled key (a 16-byte load may tear only while a slot is being
        // claimed, and a claimed slot never changes afterwards).
        if (cur.x == C.v[0] && cur.y == C.v[NL - 1]) { atomicAdd(slot_count<NL>(t, s), n); return; }
        continue;
      }
      U128 e{kEmpty, kEmpty}, mine{C.v[0], C.v[NL - 1]};
      U128 old = atomicCAS((U128*)kp, e, mine);
      if ((old.x == kEmpty && old.y == kEmpty) || (old.x == mine.x && old.y == mine.y)) {
        atomicAdd(slot_count<NL>(t, s), n);
        return;
      }
    } else {
      uint32_t* sp = slot_state<NL>(t, s);
      uint32_t st = __ldcg(sp);
      if (st == 0) {
        uint32_t old = atomicCAS(sp, 0u, 1u);
        if (old == 0) {
#pragma unroll
          for (int j = 0; j < NL; j++) __stcg(kp + j, C.v[j]);
          atomicAdd(slot_count<NL>(t, s), n);
          __threadfence();
          atomicExch(sp, 2u);
          return;
        }
        st = old;
      }
      if (st == 1) {
        int spins = 0;
        while ((st = *(volatile uint32_t*)sp) != 2u) {
          if (++spins > kSpinLimit) { atomicOr(t.err, 2); return; }
          __nanosleep(64);
        }
        __threadfence();
      }
      bool eq = true;
#pragma unroll
      for (int j = 0; j < NL; j++) eq &= __ldcg(kp + j) == C.v[j];
      if (eq) { atomicAdd(slot_count<NL>(t, s), n); return; }
    }
  }
  atomicOr(t.err, 1);  // probe limit: the host regrows the table and recounts
}

// Read-only lookup after counting: the count (with the kRejected flag) or 0.
template <int NL>
__device__ __forceinline__ uint32_t table_find(const TableView& t, const Seq<NL>& C, uint64_t home) {
  const uint64_t mask = t.capacity - 1;
  for (uint32_t i = 0; i < t.max_probe; i++) {
    const uint64_t s = (home + i) & mask;
    const uint32_t c = __ldg(slot_count<NL>(t, s));
    if (c == 0) return 0;  // empty slot ends the probe sequence
    const uint64_t* kp = slot_key<NL>(t, s);
    bool eq = true;
#pragma unroll
    for (int j = 0; j < NL; j++) eq &= __ldg(kp + j) == C.v[j];
    if (eq) return c;
  }
  return 0;
}

template <int NL>
__device__ __forceinline__ void warp_table_add(const TableView& t, bool take, const Seq<NL>& C,
                                               uint64_t raw0, const SlotPeek* peek = nullptr) {
  const unsigned am = __ballot_sync(FULL, take);
  if (take) {
    // Equal keys in the warp (repeats, hot k-mers) become one atomic add.
    unsigned peers = am;
#pragma unroll
    for (int j = 0; j < NL; j++) peers &= __match_any_sync(am, (unsigned long long)C.v[j]);
    if ((threadIdx.x & 31) == (unsigned)(__ffs(peers) - 1))
      table_add<NL>(t, C, table_home(t, raw0), __popc(peers), peek);
  }
}

// ---------------------------------------------------------------------------
// Fused pass: Stage 2 Bloom population (src/assemble.rs:141-157) and the
// count of every k-mer (src/assemble.rs:193-207 without the gate) in one walk
// over the reads.
// ---------------------------------------------------------------------------
template <int NL, bool REF>
__global__ void __launch_bounds__(kBlock) k_fused_pass(ReadsView R, unsigned k, FastMod fm,
                                                        U128* __restrict__ tiers,
                                                        unsigned long long* __restrict__ ref_solid,
                                                        TableView t,
                                                        unsigned long long* __restrict__ occ_out) {
  uint64_t occ = 0;
  auto fn = [&](bool active, uint64_t bitpos) {
    Seq<NL> C;
    uint64_t raw[3] = {0, 0, 0};
    SlotPeek peek{kEmpty, kEmpty};
    if (active) {
      occ++;
      const Seq<NL> V = extract<NL>(R.words, bitpos, k);
      C = canonical<NL>(V, k);
      uint64_t pos[3];
      bloom_positions<NL>(C, k, fm, raw, pos);
      peek = table_peek<NL>(t, table_home(t, raw[0]));
      const bool allprev = bloom_insert3(tiers, pos);
      if (REF && allprev) ref_promote(ref_solid, pos);
    }
    warp_table_add<NL>(t, active, C, raw[0], NL <= 2 ? &peek : nullptr);
  };
  foreach_position(R, k, fn);
  warp_add_u64(occ_out, occ);
}

// ---------------------------------------------------------------------------
// Count-first schedule, pass 1: the count of every canonical k-mer occurrence
// (src/assemble.rs:193-207 without the gate), with one hash (the table's home
// slot) and one table update per occurrence and no Bloom work.  Both Bloom
// tiers depend only on the distinct k-mers and their counts, so
// k_bloom_from_table derives them from the finished table.
// ---------------------------------------------------------------------------
template <int NL>
__global__ void __launch_bounds__(kBlock) k_count_all(ReadsView R, unsigned k, TableView t,
                                                       unsigned long long* __restrict__ occ_out) {
  uint64_t occ = 0;
  auto fn = [&](bool active, uint64_t bitpos) {
    Seq<NL> C;
    uint64_t raw0 = 0;
    SlotPeek peek{kEmpty, kEmpty};
    if (active) {
      occ++;
      const Seq<NL> V = extract<NL>(R.words, bitpos, k);
      C = canonical<NL>(V, k);
      uint64_t w4[4];
      kmer256_limbs<NL>(C, k, w4);
      raw0 = hash_seed(hash_pre(w4), kSeed1);
      if (NL <= 2) peek = table_peek<NL>(t, table_home(t, raw0));
    }
    warp_table_add<NL>(t, active, C, raw0, NL <= 2 ? &peek : nullptr);
  };
  foreach_position(R, k, fn);
  warp_add_u64(occ_out, occ);
}

// Count-first schedule, pass 2: the Bloom tiers from the table.  An insert
// operation sets its seen bit, and its twice bit when the seen bit was
// already set (src/bloom.rs:95-97 plus the twice tier), so once every
// occurrence is inserted seen[p] = "some operation hit p" and twice[p] = "at
// least two operations hit p", whatever the order.  A k-mer counted c times
// makes c operations on each of its three positions: for c >= 2 all three
// twice bits are set outright, and a k-mer seen once makes its three
// operations one after another (so a position it hits twice still gets its
// twice bit).  The tiers equal those of inserting every occurrence.
template <int NL>
__global__ void __launch_bounds__(kBlock) k_bloom_from_table(TableView t, unsigned k, FastMod fm,
                                                              U128* __restrict__ tiers) {
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < t.capacity;
       s += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t c = *slot_count<NL>(t, s);
    if (c == 0) continue;  // empty slot
    Seq<NL> C;
    const uint64_t* kp = slot_key<NL>(t, s);
#pragma unroll
    for (int j = 0; j < NL; j++) C.v[j] = kp[j];
    uint64_t raw[3], pos[3];
    bloom_positions<NL>(C, k, fm, raw, pos);
    if (c == 1) {
      bloom_insert3(tiers, pos);
    } else {
#pragma unroll
      for (int i = 0; i < 3; i++) {
        const uint64_t w = pos[i] >> 6;
        const unsigned long long bit = 1ULL << (pos[i] & 63);
        const U128 cur = tiers[w];
        if (!(cur.x & bit)) atomicOr(&tiers[w].x, bit);
        if (!(cur.y & bit)) atomicOr(&tiers[w].y, bit);
      }
    }
  }
}

// Gated schedule, Stage 2 alone.
template <int NL, bool REF>
__global__ void __launch_bounds__(kBlock) k_bloom_pass(ReadsView R, unsigned k, FastMod fm,
                                                        U128* __restrict__ tiers,
                                                        unsigned long long* __restrict__ ref_solid,
                                                        unsigned long long* __restrict__ occ_out) {
  uint64_t occ = 0;
  auto fn = [&](bool active, uint64_t bitpos) {
    if (!active) return;
    occ++;
    const Seq<NL> V = extract<NL>(R.words, bitpos, k);
    const Seq<NL> C = canonical<NL>(V, k);
    uint64_t raw[3], pos[3];
    bloom_positions<NL>(C, k, fm, raw, pos);
    const bool allprev = bloom_insert3(tiers, pos);
    if (REF && allprev) ref_promote(ref_solid, pos);
  };
  foreach_position(R, k, fn);
  warp_add_u64(occ_out, occ);
}

// Gated schedule, Stage 3: count occurrences whose three twice bits are set
// (src/assemble.rs:193-207).
template <int NL>
__global__ void __launch_bounds__(kBlock) k_count_pass(ReadsView R, unsigned k, FastMod fm,
                                                        const uint64_t* __restrict__ twice,
                                                        TableView t) {
  auto fn = [&](bool active, uint64_t bitpos) {
    bool admitted = false;
    Seq<NL> C;
    uint64_t raw0 = 0;
    if (active) {
      const Seq<NL> V = extract<NL>(R.words, bitpos, k);
      C = canonical<NL>(V, k);
      uint64_t raw[3], pos[3];
      bloom_positions<NL>(C, k, fm, raw, pos);
      raw0 = raw[0];
      const uint64_t a = __ldg(twice + (pos[0] >> 6));
      const uint64_t b = __ldg(twice + (pos[1] >> 6));
      const uint64_t c = __ldg(twice + (pos[2] >> 6));
      admitted = ((a >> (pos[0] & 63)) & (b >> (pos[1] & 63)) & (c >> (pos[2] & 63)) & 1) != 0;
    }
    warp_table_add<NL>(t, admitted, C, raw0);
  };
  foreach_position(R, k, fn);
}

// Interleaved word pairs -> compact seen and twice tiers, with popcounts.
__global__ void __launch_bounds__(kBlock) k_tier_finish(const U128* __restrict__ tiers, uint64_t n,
                                                         uint64_t* __restrict__ seen,
                                                         uint64_t* __restrict__ twice,
                                                         unsigned long long* __restrict__ pops) {
  uint64_t cs = 0, ct = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    U128 t = tiers[i];
    seen[i] = t.x;
    twice[i] = t.y;
    cs += __popcll(t.x);
    ct += __popcll(t.y);
  }
  warp_add_u64(pops + 0, cs);
  warp_add_u64(pops + 1, ct);
}

// ---------------------------------------------------------------------------
// One scan of the table: admission of k-mers seen once (their three twice
// bits), the count histogram of the admitted table (the input of
// src/assemble.rs:692-735), and the stream compaction of admitted k-mers with
// count >= lmin into the SoA list.  lmin is known before the cutoff: the
// adaptive cutoff is never below 2 (src/assemble.rs:692-735).
// sums: [0] admitted k-mers, [1] admitted count-1 k-mers, [2] admitted
// occurrences (sum of counts), [3] list length.
// ---------------------------------------------------------------------------
constexpr int kHistBins = 256;  // counts >= 255 share the last bin

template <int NL>
__global__ void __launch_bounds__(kBlock) k_admit_compact(TableView t, unsigned k, FastMod fm,
                                                          const uint64_t* __restrict__ twice,
                                                          int check_singletons, uint32_t lmin,
                                                          uint64_t* o0, uint64_t* o1, uint64_t* o2,
                                                          uint64_t* o3, uint32_t* __restrict__ ocnt,
                                                          uint64_t out_cap,
                                                          unsigned long long* __restrict__ hist,
                                                          unsigned long long* __restrict__ sums) {
  __shared__ unsigned sh[kHistBins];
  for (int i = threadIdx.x; i < kHistBins; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  const unsigned lane = threadIdx.x & 31;
  uint64_t n_adm = 0, n_one = 0, occ = 0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t start = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  // Uniform trip count per warp so the ballot below sees every lane.
  for (uint64_t base = start - lane; base < t.capacity; base += stride) {
    const uint64_t s = base + lane;
    uint32_t c = s < t.capacity ? *slot_count<NL>(t, s) : 0u;
    if (c & kRejected) c = 0;
    Seq<NL> C;
    if (c) {
      const uint64_t* kp = slot_key<NL>(t, s);
#pragma unroll
      for (int j = 0; j < NL; j++) C.v[j] = kp[j];
    }
    if (c == 1 && check_singletons) {
      uint64_t raw[3], pos[3];
      bloom_positions<NL>(C, k, fm, raw, pos);
      const uint64_t a = __ldg(twice + (pos[0] >> 6));
      const uint64_t b = __ldg(twice + (pos[1] >> 6));
      const uint64_t d = __ldg(twice + (pos[2] >> 6));
      if (!((a >> (pos[0] & 63)) & (b >> (pos[1] & 63)) & (d >> (pos[2] & 63)) & 1)) {
        *slot_count<NL>(t, s) = 1u | kRejected;
        c = 0;
      }
    }
    if (c) {
      n_adm++;
      n_one += c == 1;
      occ += c;
      atomicAdd(&sh[c < kHistBins - 1 ? c : kHistBins - 1], 1u);
    }
    const bool keep = c != 0 && c >= lmin;
    const unsigned m = __ballot_sync(FULL, keep);
    if (!m) continue;
    unsigned long long pos0 = 0;
    if (lane == (unsigned)(__ffs(m) - 1)) pos0 = atomicAdd(sums + 3, (unsigned long long)__popc(m));
    pos0 = __shfl_sync(FULL, pos0, __ffs(m) - 1);
    const uint64_t p = pos0 + __popc(m & lanemask_lt());
    if (keep && p < out_cap) {
      o0[p] = C.v[0];
      if (NL > 1) o1[p] = C.v[NL > 1 ? 1 : 0];
      if (NL > 2) o2[p] = C.v[NL > 2 ? 2 : 0];
      if (NL > 3) o3[p] = C.v[NL > 3 ? 3 : 0];
      ocnt[p] = c;
    }
  }
  warp_add_u64(sums + 0, n_adm);
  warp_add_u64(sums + 1, n_one);
  warp_add_u64(sums + 2, occ);
  __syncthreads();
  for (int i = threadIdx.x; i < kHistBins; i += blockDim.x)
    if (sh[i]) atomicAdd(hist + i, (unsigned long long)sh[i]);
}

// Solid k-mers of the list (count >= cutoff), for cutoffs the histogram cannot resolve.
__global__ void __launch_bounds__(256) k_count_solid(const uint32_t* __restrict__ cnt, uint64_t n,
                                                     const uint32_t* __restrict__ thr,
                                                     unsigned long long* __restrict__ out) {
  uint64_t s = 0;
  const uint32_t cutoff = thr[0];
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    s += cnt[i] >= cutoff;
  warp_add_u64(out, s);
}

// out: [0] cutoff, [1] list threshold
__global__ void k_cutoff(const unsigned long long* __restrict__ hist, uint32_t fixed,
                         uint32_t list_min, uint32_t* __restrict__ out) {
  if (threadIdx.x | blockIdx.x) return;
  uint32_t cutoff = 2;
  if (fixed) {
    cutoff = fixed;
  } else {
    unsigned long long n = 0;
    for (int c = 0; c < kHistBins; c++) n += hist[c];
    if (n > 100) {
      const unsigned long long rank = n * 95 / 100;
      unsigned long long cum = 0;
      uint32_t top = kHistBins - 1;  // bin 255 means >= 255
      for (int c = 0; c < kHistBins; c++) {
        cum += hist[c];
        if (cum > rank) { top = c; break; }
      }
      if (top >= 30) {
        uint32_t mvs = min(max(top / 4, 10u), 35u);
        uint32_t valley = 2;
        unsigned long long min_val = ~0ULL;
        bool found = false;
        for (uint32_t c = 2; c <= mvs; c++) {
          unsigned long long h = hist[c];
          if (h <= min_val) { min_val = h; valley = c; }
          else if (h > min_val * 2 && c > valley + 2) { found = true; break; }
        }
        cutoff = found ? valley : 2;
      }
    }
  }
  out[0] = cutoff;
  out[1] = max(1u, min(cutoff, list_min));
}

// ---------------------------------------------------------------------------
// (k+1)-mer edges (src/graph.rs:78-102 with OrientedKmer::explicit_seq
// src/graph.rs:24-30).  For a solid k-mer s in orientation o and base b the
// successor is canonical(explicit(s,o).extend_right(b)) (src/dna.rs:196-221);
// when it is solid too, the (k+1)-mer explicit(s,o)+b is an edge.  The same
// edge is generated once more from the other end as its reverse complement,
// so only the copy that is its own canonical form is emitted: every
// canonical (k+1)-mer comes out exactly once without a dedup pass.
// ---------------------------------------------------------------------------
template <int NL>
__device__ __forceinline__ Seq<NL> shl_append(const Seq<NL>& X, unsigned b, unsigned k) {
  Seq<NL> R;
#pragma unroll
  for (int i = NL - 1; i >= 1; i--) R.v[i] = shl2(X.v[i], X.v[i - 1], 2);
  R.v[0] = (X.v[0] << 2) | b;
  const unsigned topbits = 2u * k - 64u * (NL - 1);  // bits used in the top limb (1..64)
  if (topbits < 64) R.v[NL - 1] &= (1ULL << topbits) - 1;
  return R;
}
template <int NL, int NLE>
__device__ __forceinline__ Seq<NLE> widen_append(const Seq<NL>& X, unsigned b) {
  Seq<NLE> R;
#pragma unroll
  for (int i = NLE - 1; i >= 1; i--) {
    const uint64_t hi = i < NL ? X.v[i] : 0;
    R.v[i] = shl2(hi, X.v[i - 1], 2);
  }
  R.v[0] = (X.v[0] << 2) | b;
  return R;
}

template <int NL, int NLE>
__global__ void __launch_bounds__(kBlock) k_edges(const uint64_t* l0, const uint64_t* l1,
                                                   const uint64_t* l2, const uint64_t* l3,
                                                   const uint32_t* __restrict__ cnt, uint64_t n,
                                                   const uint32_t* __restrict__ thr, TableView t,
                                                   unsigned k, uint64_t* e0, uint64_t* e1,
                                                   uint64_t* e2, uint64_t* e3, uint64_t out_cap,
                                                   unsigned long long* __restrict__ counter) {
  const uint32_t cutoff = thr[0];
  const unsigned lane = threadIdx.x & 31;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t start = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  for (uint64_t base = start - lane; base < n; base += stride) {
    const uint64_t i = base + lane;
    Seq<NL> S;
    bool solid = false;
    if (i < n) {
      S.v[0] = l0[i];
      if (NL > 1) S.v[NL > 1 ? 1 : 0] = l1[i];
      if (NL > 2) S.v[NL > 2 ? 2 : 0] = l2[i];
      if (NL > 3) S.v[NL > 3 ? 3 : 0] = l3[i];
      solid = cnt[i] >= cutoff;
    }
    for (int o = 0; o < 2; o++) {
      Seq<NL> EX = S;
      bool ok = solid;
      if (o == 1 && ok) {
        EX = revcomp<NL>(S, k);
        ok = !seq_eq<NL>(EX, S);  // a palindromic k-mer (even k) has one orientation
      }
      for (unsigned b = 0; b < 4; b++) {
        bool emit = false;
        Seq<NLE> E;
        if (ok) {
          const Seq<NL> NB = shl_append<NL>(EX, b, k);
          const Seq<NL> CN = canonical<NL>(NB, k);
          uint64_t w4[4];
          kmer256_limbs<NL>(CN, k, w4);
          const HashPre hp = hash_pre(w4);
          const uint32_t c = table_find<NL>(t, CN, table_home(t, hash_seed(hp, kSeed1)));
          if (c && !(c & kRejected) && c >= cutoff) {
            E = widen_append<NL, NLE>(EX, b);
            emit = seq_le<NLE>(E, revcomp<NLE>(E, k + 1));
          }
        }
        const unsigned m = __ballot_sync(FULL, emit);
        if (!m) continue;
        unsigned long long p0 = 0;
        if (lane == (unsigned)(__ffs(m) - 1)) p0 = atomicAdd(counter, (unsigned long long)__popc(m));
        p0 = __shfl_sync(FULL, p0, __ffs(m) - 1);
        const uint64_t p = p0 + __popc(m & lanemask_lt());
        if (emit && p < out_cap) {
          e0[p] = E.v[0];
          if (NLE > 1) e1[p] = E.v[NLE > 1 ? 1 : 0];
          if (NLE > 2) e2[p] = E.v[NLE > 2 ? 2 : 0];
          if (NLE > 3) e3[p] = E.v[NLE > 3 ? 3 : 0];
        }
      }
    }
  }
}

// Occurrences of a read set (sum of max(len - k + 1, 0)).
__global__ void __launch_bounds__(kBlock) k_occ(const uint32_t* __restrict__ lengths, uint64_t n,
                                               unsigned k, unsigned long long* __restrict__ out) {
  uint64_t s = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t len = lengths[i];
    s += len >= k ? len - k + 1 : 0;
  }
  warp_add_u64(out, s);
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
static int grid_for(spk_ctx* ctx, int blocks_per_sm) { return ctx->sm_count * blocks_per_sm; }

#define SPK_DISPATCH_NL(nl, F, ...)                 \
  switch (nl) {                                     \
    case 1: F<1>(__VA_ARGS__); break;               \
    case 2: F<2>(__VA_ARGS__); break;               \
    case 3: F<3>(__VA_ARGS__); break;               \
    default: F<4>(__VA_ARGS__); break;              \
  }

template <int NL>
static void launch_fused(spk_ctx* ctx, cudaStream_t st, const ReadsView& rv, unsigned k,
                         const FastMod& fm, U128* tiers, unsigned long long* ref,
                         const TableView& t, unsigned long long* occ) {
  const int g = grid_for(ctx, 8);
  if (ref) k_fused_pass<NL, true><<<g, kBlock, 0, st>>>(rv, k, fm, tiers, ref, t, occ);
  else k_fused_pass<NL, false><<<g, kBlock, 0, st>>>(rv, k, fm, tiers, nullptr, t, occ);
}
template <int NL>
static void launch_count_all(spk_ctx* ctx, cudaStream_t st, const ReadsView& rv, unsigned k,
                             const TableView& t, unsigned long long* occ) {
  k_count_all<NL><<<grid_for(ctx, 8), kBlock, 0, st>>>(rv, k, t, occ);
}
template <int NL>
static void launch_bloom_from_table(spk_ctx* ctx, cudaStream_t st, const TableView& t, unsigned k,
                                    const FastMod& fm, U128* tiers) {
  k_bloom_from_table<NL><<<grid_for(ctx, 8), kBlock, 0, st>>>(t, k, fm, tiers);
}
template <int NL>
static void launch_bloom(spk_ctx* ctx, cudaStream_t st, const ReadsView& rv, unsigned k,
                         const FastMod& fm, U128* tiers, unsigned long long* ref,
                         unsigned long long* occ) {
  const int g = grid_for(ctx, 8);
  if (ref) k_bloom_pass<NL, true><<<g, kBlock, 0, st>>>(rv, k, fm, tiers, ref, occ);
  else k_bloom_pass<NL, false><<<g, kBlock, 0, st>>>(rv, k, fm, tiers, nullptr, occ);
}
template <int NL>
static void launch_count(spk_ctx* ctx, cudaStream_t st, const ReadsView& rv, unsigned k,
                         const FastMod& fm, const uint64_t* twice, const TableView& t) {
  k_count_pass<NL><<<grid_for(ctx, 8), kBlock, 0, st>>>(rv, k, fm, twice, t);
}
template <int NL>
static void launch_init(spk_ctx* ctx, cudaStream_t st, uint8_t* slots, uint64_t cap) {
  k_table_init<NL><<<grid_for(ctx, 4), kBlock, 0, st>>>(slots, cap);
}
template <int NL>
static void launch_admit(spk_ctx* ctx, cudaStream_t st, const TableView& t, unsigned k,
                         const FastMod& fm, const uint64_t* twice, int check, uint32_t lmin,
                         uint64_t** o, uint32_t* oc, uint64_t out_cap, unsigned long long* hist,
                         unsigned long long* sums) {
  k_admit_compact<NL><<<grid_for(ctx, 8), kBlock, 0, st>>>(t, k, fm, twice, check, lmin, o[0], o[1],
                                                          o[2], o[3], oc, out_cap, hist, sums);
}
template <int NL, int NLE>
static void launch_edges_t(spk_ctx* ctx, cudaStream_t st, uint64_t* l[4], const uint32_t* cnt,
                           uint64_t n, const uint32_t* thr, const TableView& t, unsigned k,
                           uint64_t* e[4], uint64_t out_cap, unsigned long long* counter) {
  k_edges<NL, NLE><<<grid_for(ctx, 8), kBlock, 0, st>>>(l[0], l[1], l[2], l[3], cnt, n, thr, t, k,
                                                       e[0], e[1], e[2], e[3], out_cap, counter);
}
static void launch_edges(spk_ctx* ctx, cudaStream_t st, int nl, int nle, uint64_t* l[4],
                         const uint32_t* cnt, uint64_t n, const uint32_t* thr, const TableView& t,
                         unsigned k, uint64_t* e[4], uint64_t out_cap, unsigned long long* counter) {
  if (nl == 1 && nle == 1) launch_edges_t<1, 1>(ctx, st, l, cnt, n, thr, t, k, e, out_cap, counter);
  else if (nl == 1) launch_edges_t<1, 2>(ctx, st, l, cnt, n, thr, t, k, e, out_cap, counter);
  else if (nl == 2 && nle == 2) launch_edges_t<2, 2>(ctx, st, l, cnt, n, thr, t, k, e, out_cap, counter);
  else if (nl == 2) launch_edges_t<2, 3>(ctx, st, l, cnt, n, thr, t, k, e, out_cap, counter);
  else if (nl == 3 && nle == 3) launch_edges_t<3, 3>(ctx, st, l, cnt, n, thr, t, k, e, out_cap, counter);
  else if (nl == 3) launch_edges_t<3, 4>(ctx, st, l, cnt, n, thr, t, k, e, out_cap, counter);
  else launch_edges_t<4, 4>(ctx, st, l, cnt, n, thr, t, k, e, out_cap, counter);
}

static uint64_t next_pow2(uint64_t x) {
  uint64_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

// Gated table capacity from the Bloom fill.  With m bits and 3 hashes a
// filter holding n items has fill 1 - exp(-3n/m), so n = -(m/3) ln(1 - fill).
// The twice tier estimates the k-mers seen at least twice (plus collisions,
// an overestimate); singletons admitted by chance add (twice fill)^3 of the
// rest.  Sized for a load factor of at most 1/2.
static uint64_t gated_capacity(uint64_t m, uint64_t pop_seen, uint64_t pop_twice) {
  const double md = (double)m;
  const double fs = std::min((double)pop_seen / md, 0.999999);
  const double ft = std::min((double)pop_twice / md, 0.999999);
  const double n_all = -(md / 3.0) * std::log1p(-fs);
  const double n2 = -(md / 3.0) * std::log1p(-ft);
  const double est = n2 + std::max(n_all - n2, 0.0) * ft * ft * ft;
  return std::max<uint64_t>(next_pow2((uint64_t)(est * 2.0) + 1024), 1024);
}

// Fused table capacity: every distinct k-mer, unknown before the pass.  At
// 20-200x coverage and 0.1-1% substitution errors distinct k-mers are 5-35%
// of the occurrences; the table starts at 30% (load <= ~0.6 after rounding
// up) and doubles, with a recount, if a probe sequence overflows.
static uint64_t fused_capacity(uint64_t occ) {
  return std::max<uint64_t>(next_pow2(occ * 3 / 10 + 1), 1024);
}

struct Ev {
  cudaEvent_t e = nullptr;
  Ev() { cudaEventCreate(&e); }
  ~Ev() { if (e) cudaEventDestroy(e); }
  Ev(const Ev&) = delete;
  Ev& operator=(const Ev&) = delete;
};
static float ms_between(const Ev& a, const Ev& b) {
  float ms = 0;
  if (cudaEventElapsedTime(&ms, a.e, b.e) != cudaSuccess) {
    cudaGetLastError();
    ms = 0;
  }
  return ms;
}

static int alloc_table(spk_ctx* ctx, KResult& kr, cudaStream_t st, uint64_t cap) {
  const uint32_t sb = slot_bytes(kr.nl);
  int rc;
  if ((rc = kr.tslots.alloc(cap * sb, st))) return rc;
  SPK_DISPATCH_NL(kr.nl, launch_init, ctx, st, kr.tslots.as<uint8_t>(), cap);
  SPK_CUDA(cudaGetLastError());
  TableView& t = kr.table;
  t.slots = kr.tslots.as<uint8_t>();
  t.capacity = cap;
  t.log2cap = 0;
  while ((1ULL << t.log2cap) < cap) t.log2cap++;
  t.slot_bytes = sb;
  t.max_probe = (uint32_t)std::min<uint64_t>(kMaxProbe, cap);
  return SPK_OK;
}

// Scratch layout (u64 words) in the per-k scratch buffer.
enum {
  S_OCC = 0, S_POPS = 1, /* 2 words */
  S_ERR = 3,             /* int */
  S_THR = 4,             /* 2 x u32 */
  S_SUMS = 5,            /* 4 words: admitted, admitted singletons, admitted occurrences, list */
  S_CNT = 9,             /* solid */
  S_EDGES = 10,
  S_OCC0 = 11,           /* occurrences before the pass */
  S_HIST = 16,           /* 256 words */
  S_WORDS = 16 + kHistBins
};

int count_one_k(spk_ctx* ctx, cudaStream_t st, uint64_t* host, const ReadsView& rv_in, unsigned k,
                const spk_count_opts& o, KResult& kr) {
  kr.k = k;
  kr.nl = (int)((k + 31) / 32);
  const int nl = kr.nl;
  const uint64_t bloom_bits = o.bloom_bits ? o.bloom_bits : (512ULL << 20);
  kr.num_words = std::max<uint64_t>((bloom_bits + 63) / 64, 1);  // src/bloom.rs:27
  const uint64_t size_bits = kr.num_words * 64;                   // src/bloom.rs:28
  kr.fm = make_fastmod(size_bits);
  spk_result_info& info = kr.info;
  memset(&info, 0, sizeof info);
  info.k = k;
  info.bloom_size_bits = size_bits;
  int rc;

  DevBuf scratch;
  if ((rc = scratch.alloc(S_WORDS * 8, st))) return rc;
  uint64_t* sw = scratch.as<uint64_t>();
  SPK_CUDA(cudaMemsetAsync(sw, 0, S_WORDS * 8, st));
  unsigned long long* su = (unsigned long long*)sw;
  int* errp = (int*)(sw + S_ERR);
  ReadsView rv = rv_in;
  rv.err = errp;
  const bool ref = (o.flags & SPK_F_REF_SOLID) != 0;
  const bool gated = (o.flags & SPK_F_GATED) != 0;
  // The reference-semantics solid tier depends on the order of the inserts,
  // so it needs the per-occurrence Bloom of the fused pass.
  const bool count_first = !gated && !ref;

  Ev e0, e1, e2, e3, e4, e5, e6, kb0, kb1, kc0, kc1;
  uint32_t launches = 0;
  SPK_CUDA(cudaEventRecord(e0.e, st));

  // Bloom tiers as interleaved (seen, twice) word pairs.
  if ((rc = kr.tiers.alloc(kr.num_words * 16, st))) return rc;
  if (ref && (rc = kr.ref_solid.alloc(kr.num_words * 8, st))) return rc;
  U128* tiers = kr.tiers.as<U128>();
  unsigned long long* refp = ref ? kr.ref_solid.as<unsigned long long>() : nullptr;
  auto reset_tiers = [&]() -> int {
    SPK_CUDA(cudaMemsetAsync(kr.tiers.p, 0, kr.num_words * 16, st));
    if (ref) SPK_CUDA(cudaMemsetAsync(kr.ref_solid.p, 0, kr.num_words * 8, st));
    return SPK_OK;
  };
  auto fetch = [&](int words) -> int {
    SPK_CUDA(cudaMemcpyAsync(host, sw, words * 8, cudaMemcpyDeviceToHost, st));
    SPK_CUDA(cudaStreamSynchronize(st));
    if ((int)host[S_ERR] & 4)
      return fail(SPK_E_INVALID_ARG, "a read extends past the end of the packed data");
    if ((int)host[S_ERR] & 2) return fail(SPK_E_TIMEOUT, "count table: claim wait timed out");
    return SPK_OK;
  };

  uint64_t cap = 0;
  if (!gated) {
    // ---- fused: Bloom and the count of every k-mer in one pass ----
    k_occ<<<grid_for(ctx, 2), kBlock, 0, st>>>(rv.lengths, rv.n_reads, k, su + S_OCC0);
    SPK_CUDA(cudaGetLastError());
    launches++;
    if ((rc = fetch(S_OCC0 + 1))) return rc;
    cap = o.table_log2 ? (1ULL << std::min<uint32_t>(o.table_log2, 40)) : fused_capacity(host[S_OCC0]);
    for (int attempt = 0;; attempt++) {
      if ((rc = reset_tiers())) return rc;
      if ((rc = alloc_table(ctx, kr, st, cap))) return rc;
      kr.table.err = errp;
      SPK_CUDA(cudaMemsetAsync(sw, 0, (S_ERR + 1) * 8, st));
      if (count_first) {
        SPK_CUDA(cudaEventRecord(kc0.e, st));
        SPK_DISPATCH_NL(nl, launch_count_all, ctx, st, rv, k, kr.table, su + S_OCC);
        SPK_CUDA(cudaGetLastError());
        SPK_CUDA(cudaEventRecord(kc1.e, st));
      } else {
        SPK_CUDA(cudaEventRecord(kb0.e, st));
        SPK_DISPATCH_NL(nl, launch_fused, ctx, st, rv, k, kr.fm, tiers, refp, kr.table, su + S_OCC);
        SPK_CUDA(cudaGetLastError());
        SPK_CUDA(cudaEventRecord(kb1.e, st));
      }
      launches += 2;
      if ((rc = fetch(S_ERR + 1))) return rc;
      if (!((int)host[S_ERR] & 1)) break;
      if (attempt >= 24) return fail(SPK_E_TABLE_FULL, "count table overflow after regrow attempts");
      cap *= 2;
      info.table_regrows++;
    }
    if (count_first) {
      SPK_CUDA(cudaEventRecord(kb0.e, st));
      SPK_DISPATCH_NL(nl, launch_bloom_from_table, ctx, st, kr.table, k, kr.fm, tiers);
      SPK_CUDA(cudaGetLastError());
      SPK_CUDA(cudaEventRecord(kb1.e, st));
      launches++;
    }
  } else {
    // ---- gated: Stage 2 first ----
    if ((rc = reset_tiers())) return rc;
    SPK_CUDA(cudaEventRecord(kb0.e, st));
    SPK_DISPATCH_NL(nl, launch_bloom, ctx, st, rv, k, kr.fm, tiers, refp, su + S_OCC);
    SPK_CUDA(cudaGetLastError());
    SPK_CUDA(cudaEventRecord(kb1.e, st));
    launches++;
  }
  // compact tiers (both schedules)
  if ((rc = kr.seen.alloc(kr.num_words * 8, st))) return rc;
  if ((rc = kr.twice.alloc(kr.num_words * 8, st))) return rc;
  k_tier_finish<<<grid_for(ctx, 4), kBlock, 0, st>>>(tiers, kr.num_words, kr.seen.as<uint64_t>(),
                                                    kr.twice.as<uint64_t>(), su + S_POPS);
  SPK_CUDA(cudaGetLastError());
  launches++;
  kr.tiers.release();
  SPK_CUDA(cudaEventRecord(e1.e, st));
  if ((rc = fetch(S_POPS + 2))) return rc;
  info.occurrences = host[S_OCC];
  info.seen_popcount = host[S_POPS];
  info.twice_popcount = host[S_POPS + 1];

  if (gated) {
    // ---- gated: Stage 3 over admitted occurrences ----
    cap = o.table_log2 ? (1ULL << std::min<uint32_t>(o.table_log2, 40))
                       : gated_capacity(size_bits, info.seen_popcount, info.twice_popcount);
    for (int attempt = 0;; attempt++) {
      if ((rc = alloc_table(ctx, kr, st, cap))) return rc;
      kr.table.err = errp;
      SPK_CUDA(cudaMemsetAsync(errp, 0, 8, st));
      SPK_CUDA(cudaEventRecord(kc0.e, st));
      SPK_DISPATCH_NL(nl, launch_count, ctx, st, rv, k, kr.fm, kr.twice.as<uint64_t>(), kr.table);
      SPK_CUDA(cudaGetLastError());
      SPK_CUDA(cudaEventRecord(kc1.e, st));
      launches += 2;
      if ((rc = fetch(S_ERR + 1))) return rc;
      if (!((int)host[S_ERR] & 1)) break;
      if (attempt >= 24) return fail(SPK_E_TABLE_FULL, "count table overflow after regrow attempts");
      cap *= 2;
      info.table_regrows++;
    }
  }
  info.table_capacity = cap;
  SPK_CUDA(cudaEventRecord(e2.e, st));

  // ---- admission of singletons, histogram, compaction, cutoff ----
  uint32_t fixed = o.min_count;
  if (!fixed && o.min_coverage > 5.0) {  // src/assemble.rs:693-694
    double v = std::max(o.min_coverage * 0.35, 2.0);
    fixed = v >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)v;
  }
  const uint32_t list_min = o.list_min_count ? o.list_min_count : 2;
  // The list keeps counts >= min(cutoff, list_min).  The adaptive cutoff is
  // never below 2, so compacting counts >= min(2 or the fixed cutoff,
  // list_min) keeps a superset; the exact threshold filters downloads.
  const uint32_t lmin_pre = std::max(1u, std::min(fixed ? fixed : 2u, list_min));
  kr.list_min = lmin_pre;
  // List capacity from the Bloom: k-mers seen at least twice (twice-tier
  // estimate, an overestimate), plus admitted singletons if they are listed.
  uint64_t lcap;
  {
    const double md = (double)size_bits;
    const double fs = std::min((double)info.seen_popcount / md, 0.999999);
    const double ft = std::min((double)info.twice_popcount / md, 0.999999);
    const double n_all = -(md / 3.0) * std::log1p(-fs);
    const double n2 = -(md / 3.0) * std::log1p(-ft);
    double est = n2 * 1.25 + 65536;
    if (kr.list_min <= 1) est += std::max(n_all - n2, 0.0) * ft * ft * ft * 1.5 + 65536;
    lcap = std::min<uint64_t>((uint64_t)est, cap);
  }
  uint64_t* lp[4] = {nullptr, nullptr, nullptr, nullptr};
  for (int pass = 0;; pass++) {
    for (int j = 0; j < nl; j++) {
      if ((rc = kr.list[j].alloc(std::max<uint64_t>(lcap, 1) * 8, st))) return rc;
      lp[j] = kr.list[j].as<uint64_t>();
    }
    if ((rc = kr.list[4].alloc(std::max<uint64_t>(lcap, 1) * 4, st))) return rc;
    SPK_CUDA(cudaMemsetAsync(sw + S_SUMS, 0, 4 * 8, st));
    SPK_CUDA(cudaMemsetAsync(sw + S_HIST, 0, kHistBins * 8, st));
    SPK_DISPATCH_NL(nl, launch_admit, ctx, st, kr.table, k, kr.fm, kr.twice.as<uint64_t>(),
                    gated ? 0 : 1, lmin_pre, lp, kr.list[4].as<uint32_t>(), lcap, su + S_HIST,
                    su + S_SUMS);
    SPK_CUDA(cudaGetLastError());
    launches++;
    if ((rc = fetch(S_SUMS + 4))) return rc;
    if (host[S_SUMS + 3] <= lcap) break;
    // Underestimated: size exactly and scan again (rejections are already
    // marked, so the second scan admits the same k-mers).
    lcap = host[S_SUMS + 3];
    if (pass >= 1) return fail(SPK_E_CUDA, "k-mer list size changed between scans");
  }
  uint32_t* thr = (uint32_t*)(sw + S_THR);
  k_cutoff<<<1, 32, 0, st>>>(su + S_HIST, fixed, list_min, thr);
  SPK_CUDA(cudaGetLastError());
  launches++;
  if ((rc = fetch(S_WORDS))) return rc;
  const uint32_t* hthr = (const uint32_t*)(host + S_THR);
  info.cutoff = hthr[0];
  kr.list_min = hthr[1];
  info.n_table = host[S_SUMS + 0];
  info.n_singletons = host[S_SUMS + 1];
  info.admitted_occurrences = host[S_SUMS + 2];
  kr.list_len = host[S_SUMS + 3];
  auto hist_from = [&](uint32_t c0) {
    uint64_t ns = 0;
    for (int c = (int)c0; c < kHistBins; c++) ns += host[S_HIST + c];
    return ns;
  };
  info.n_list = kr.list_min == lmin_pre ? kr.list_len : hist_from(kr.list_min);
  if (kr.list_min != lmin_pre && kr.list_min >= (uint32_t)(kHistBins - 1))
    return fail(SPK_E_INVALID_ARG, "list_min_count above 254 needs a fixed min_count");
  if (info.cutoff < (uint32_t)(kHistBins - 1)) {
    info.n_solid = hist_from(info.cutoff);
  } else {
    SPK_CUDA(cudaMemsetAsync(sw + S_CNT, 0, 8, st));
    k_count_solid<<<grid_for(ctx, 2), 256, 0, st>>>(kr.list[4].as<uint32_t>(), kr.list_len, thr,
                                                   su + S_CNT);
    SPK_CUDA(cudaGetLastError());
    launches++;
    if ((rc = fetch(S_CNT + 1))) return rc;
    info.n_solid = host[S_CNT];
  }
  SPK_CUDA(cudaEventRecord(e3.e, st));

  // ---- sort ----
  if ((rc = radix_sort_bufs(st, nl, kr.list_len, 2 * k, kr.list, &kr.list[4], &launches))) return rc;
  for (int j = 0; j < nl; j++) lp[j] = kr.list[j].as<uint64_t>();
  SPK_CUDA(cudaEventRecord(e4.e, st));

  // ---- edges ----
  kr.nle = (int)((k + 1 + 31) / 32);
  if ((o.flags & SPK_F_EDGES) && info.n_solid > 0) {
    uint64_t* ep[4] = {nullptr, nullptr, nullptr, nullptr};
    const uint64_t ecap = info.n_solid * 8;  // at most 8 canonical edges per solid k-mer
    for (int j = 0; j < kr.nle; j++) {
      if ((rc = kr.edges[j].alloc(ecap * 8, st))) return rc;
      ep[j] = kr.edges[j].as<uint64_t>();
    }
    launch_edges(ctx, st, nl, kr.nle, lp, kr.list[4].as<uint32_t>(), kr.list_len, thr, kr.table, k,
                 ep, ecap, su + S_EDGES);
    SPK_CUDA(cudaGetLastError());
    launches++;
    if ((rc = fetch(S_EDGES + 1))) return rc;
    info.n_edges = host[S_EDGES];
    if (info.n_edges > ecap) return fail(SPK_E_CUDA, "edge list larger than its bound");
    if ((rc = radix_sort_bufs(st, kr.nle, info.n_edges, 2 * (k + 1), kr.edges, nullptr, &launches)))
      return rc;
  }
  SPK_CUDA(cudaEventRecord(e5.e, st));
  if (!(o.flags & SPK_F_KEEP_BLOOM)) {
    kr.seen.release();
    kr.twice.release();
  }
  SPK_CUDA(cudaEventRecord(e6.e, st));
  SPK_CUDA(cudaStreamSynchronize(st));
  info.ms_bloom = ms_between(e0, e1);
  info.ms_count = ms_between(e1, e2);
  info.ms_finish = ms_between(e2, e3);
  info.ms_sort = ms_between(e3, e4);
  info.ms_edges = ms_between(e4, e5);
  info.ms_total = ms_between(e0, e6);
  info.ms_bloom_kernel = ms_between(kb0, kb1);
  info.ms_count_kernel = (gated || count_first) ? ms_between(kc0, kc1) : 0.f;
  info.kernel_launches = launches;
  info.schedule = gated ? SPK_SCHEDULE_GATED : count_first ? SPK_SCHEDULE_COUNT_FIRST : SPK_SCHEDULE_FUSED;
  return SPK_OK;
}

int count_pipeline(spk_ctx* ctx, cudaStream_t st, const ReadsView& rv, uint32_t max_len,
                   const uint32_t* ks, int n_k, const spk_count_opts& o, spk_result* res) {
  (void)max_len;
  for (int i = 0; i < n_k; i++) {
    auto kr = std::make_unique<KResult>();
    int rc = count_one_k(ctx, st, res->h_staging, rv, ks[i], o, *kr);
    if (rc) return rc;
    res->ks.push_back(std::move(kr));
  }
  return SPK_OK;
}

// ---------------------------------------------------------------------------
// Downloads
// ---------------------------------------------------------------------------
static int copy_out(spk_result* res, int nl, DevBuf* limbs, const uint32_t* cin, uint64_t n,
                    unsigned k, uint32_t minc, uint64_t* keys, uint32_t* counts, size_t* n_inout) {
  cudaStream_t st = res->stream;
  DevBuf okeys, ocnt;
  uint64_t m = 0;
  int rc = ordered_convert(st, nl, n, k, limbs, cin, minc, &okeys, cin ? &ocnt : nullptr,
                           res->h_staging, &m);
  if (rc) return rc;
  if (!keys && !counts) {
    SPK_CUDA(cudaStreamSynchronize(st));
    *n_inout = m;
    return SPK_OK;
  }
  if (*n_inout < m) {
    SPK_CUDA(cudaStreamSynchronize(st));
    *n_inout = m;
    return fail(SPK_E_INVALID_ARG, "output buffer too small");
  }
  if (m) {
    if (keys) SPK_CUDA(cudaMemcpyAsync(keys, okeys.p, m * nl * 8, cudaMemcpyDeviceToHost, st));
    if (counts && cin) SPK_CUDA(cudaMemcpyAsync(counts, ocnt.p, m * 4, cudaMemcpyDeviceToHost, st));
  }
  SPK_CUDA(cudaStreamSynchronize(st));
  *n_inout = m;
  return SPK_OK;
}

int download_list(spk_result* res, int ki, uint32_t min_count, bool solid_only, uint64_t* keys,
                  uint32_t* counts, size_t* n_inout) {
  KResult& kr = *res->ks[ki];
  const uint32_t minc = solid_only ? kr.info.cutoff : std::max(min_count, kr.list_min);
  return copy_out(res, kr.nl, kr.list, kr.list[4].as<uint32_t>(), kr.list_len, kr.k, minc,
                  keys, counts, n_inout);
}

int download_edges(spk_result* res, int ki, uint64_t* out, size_t* n_inout) {
  KResult& kr = *res->ks[ki];
  return copy_out(res, kr.nle, kr.edges, nullptr, kr.info.n_edges, kr.k + 1, 0, out, nullptr,
                  n_inout);
}

int download_bloom(spk_result* res, int ki, uint64_t* seen, uint64_t* twice, uint64_t* ref_solid) {
  KResult& kr = *res->ks[ki];
  cudaStream_t st = res->stream;
  if (!kr.seen.p) return fail(SPK_E_INVALID_ARG, "Bloom tiers were not kept (SPK_F_KEEP_BLOOM)");
  const uint64_t n = kr.num_words;
  if (seen) SPK_CUDA(cudaMemcpyAsync(seen, kr.seen.p, n * 8, cudaMemcpyDeviceToHost, st));
  if (twice) SPK_CUDA(cudaMemcpyAsync(twice, kr.twice.p, n * 8, cudaMemcpyDeviceToHost, st));
  if (ref_solid) {
    if (!kr.ref_solid.p) return fail(SPK_E_INVALID_ARG, "reference solid tier not built (SPK_F_REF_SOLID)");
    SPK_CUDA(cudaMemcpyAsync(ref_solid, kr.ref_solid.p, n * 8, cudaMemcpyDeviceToHost, st));
  }
  SPK_CUDA(cudaStreamSynchronize(st));
  return SPK_OK;
}

}  // namespace spk
