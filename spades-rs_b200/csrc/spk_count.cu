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
#include <string>
#include <thread>
#include <vector>

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

// The same walk handing every lane U positions per call, f(active[U],
// bitpos[U]), so that a lane can keep U independent memory operations in
// flight.  Position u of a call is base + 32u + lane.
template <int U, class F>
__device__ __forceinline__ void foreach_position_n(const ReadsView& R, unsigned k, F& f) {
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
    for (uint32_t base = 0; base < total; base += 32 * U) {
      bool active[U];
      uint64_t bitpos[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const uint32_t p = base + 32 * u + lane;
        unsigned j = 0;
#pragma unroll
        for (unsigned step = 16; step >= 1; step >>= 1) {
          uint32_t c = __shfl_sync(FULL, incl, j + step - 1);
          if (p >= c) j += step;
        }
        const uint64_t o = __shfl_sync(FULL, off, j);
        const uint32_t e = __shfl_sync(FULL, excl, j);
        active[u] = p < total;
        bitpos[u] = 8ull * (R.byte_base + o) + 2ull * (uint64_t)(p - e);
      }
      f(active, bitpos);
    }
  }
}

// Rolling walk (k <= 64): one read per thread.  The first window of a read
// is extracted, later windows roll in one base each (extend_right,
// src/dna.rs:196-221) with the reverse complement rolled alongside, so a
// position costs a few shifts instead of a full extract and reverse
// complement.  f(active[U], canonical[U]) gets U consecutive windows of the
// thread's read per call (all 32 lanes call f; inactive entries are junk).
template <int NL, int U, class F>
__device__ __forceinline__ void foreach_read_roll(const ReadsView& R, unsigned k, F& f) {
  static_assert(NL <= 2, "rolling walk holds keys of up to 128 bits");
  const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t first = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const unsigned topsh = 2 * k - 2 - 64 * (NL - 1);  // bit of the first base in the top limb
  const uint64_t topmask = (2 * k - 64 * (NL - 1)) >= 64 ? ~0ULL : ((1ULL << (2 * k - 64 * (NL - 1))) - 1);
  // Warps walk 32 consecutive reads per round; a warp keeps going while any
  // of its lanes has windows left, so f sees all 32 lanes.
  for (uint64_t r0 = first - (threadIdx.x & 31); r0 < R.n_reads; r0 += nthreads) {
    const uint64_t r = r0 + (threadIdx.x & 31);
    uint32_t np = 0;
    uint64_t bit0 = 0;
    if (r < R.n_reads) {
      const uint32_t len = __ldg(R.lengths + r);
      const uint64_t off = __ldg(R.offsets + r);
      if (off + ((uint64_t)len + 3) / 4 > R.data_len) {  // src/packed_reads.rs:600-602
        atomicOr(R.err, 4);
      } else if (len >= k) {
        np = len - k + 1;
        bit0 = 8ull * (R.byte_base + off);
      }
    }
    Seq<NL> V, Rc;
    if (np) {
      V = extract<NL>(R.words, bit0, k);
      Rc = revcomp<NL>(V, k);
    }
    uint64_t buf = 0, nextbit = bit0 + 2ull * k;
    unsigned bleft = 0;
    uint32_t i = 0;
    for (;;) {
      if (!__any_sync(FULL, i < np)) break;
      bool act[U];
      Seq<NL> C[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        act[u] = i < np;
        if (act[u]) {
          if (i > 0) {
            if (bleft == 0) {
              buf = extract<1>(R.words, nextbit, 32).v[0];
              bleft = 32;
            }
            const uint64_t b = buf >> 62;
            buf <<= 2;
            bleft--;
            nextbit += 2;
            if (NL == 1) {
              V.v[0] = ((V.v[0] << 2) | b) & topmask;
              Rc.v[0] = (Rc.v[0] >> 2) | ((3 - b) << topsh);
            } else {
              V.v[NL - 1] = ((V.v[NL - 1] << 2) | (V.v[0] >> 62)) & topmask;
              V.v[0] = (V.v[0] << 2) | b;
              Rc.v[0] = (Rc.v[0] >> 2) | (Rc.v[NL - 1] << 62);
              Rc.v[NL - 1] = (Rc.v[NL - 1] >> 2) | ((3 - b) << topsh);
            }
          }
          C[u] = seq_le<NL>(V, Rc) ? V : Rc;  // canonical, src/dna.rs:185-192
          i++;
        }
      }
      f(act, C);
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

// The Bloom insert operations of U distinct k-mers with counts c[u] (0 =
// none): a k-mer counted c >= 2 times sets its three seen and twice bits; a
// k-mer seen once makes its three operations in order (as bloom_insert3).
// All word pairs are loaded first and all fetch_or issued before their
// results are used, so a thread keeps up to 3U operations in flight.
template <int U>
__device__ __forceinline__ void bloom_ops_distinct(U128* __restrict__ tiers, const uint64_t (&pos)[U][3],
                                                   const uint32_t (&c)[U]) {
  U128 t[U][3];
#pragma unroll
  for (int u = 0; u < U; u++)
#pragma unroll
    for (int i = 0; i < 3; i++) t[u][i] = c[u] ? tiers[pos[u][i] >> 6] : U128{0, 0};
  unsigned long long prev[U][3];
#pragma unroll
  for (int u = 0; u < U; u++)
#pragma unroll
    for (int i = 0; i < 3; i++) {
      const uint64_t w = pos[u][i] >> 6;
      const unsigned long long bit = 1ULL << (pos[u][i] & 63);
      prev[u][i] = 0;
      if (c[u] >= 2) {
        if (!(t[u][i].x & bit)) atomicOr(&tiers[w].x, bit);
        if (!(t[u][i].y & bit)) atomicOr(&tiers[w].y, bit);
      } else if (c[u] == 1) {
        // A set seen bit (even from a stale read) was set by an earlier operation.
        prev[u][i] = (t[u][i].x & bit) ? bit : atomicOr(&tiers[w].x, bit);
      }
    }
#pragma unroll
  for (int u = 0; u < U; u++)
#pragma unroll
    for (int i = 0; i < 3; i++) {
      const unsigned long long bit = 1ULL << (pos[u][i] & 63);
      if (c[u] == 1 && (prev[u][i] & bit) && !(t[u][i].y & bit))
        atomicOr(&tiers[pos[u][i] >> 6].y, bit);
    }
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
// Slot i of the probe sequence from `home`: linear, wrapping inside the span.
__device__ __forceinline__ uint64_t probe_slot(const TableView& t, uint64_t home, uint32_t i) {
  const uint64_t m = (1ULL << t.log2span) - 1;
  return (home & ~m) | ((home + i) & m);
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
  for (uint32_t i = 0; i < t.max_probe; i++) {
    // A table too full for its k-mers is regrown and the pass repeated: once
    // another thread has found that out, long probe sequences stop.
    if ((i & 63) == 63 && (*(volatile int*)t.err & 1)) return;
    const uint64_t s = probe_slot(t, home, i);
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
  for (uint32_t i = 0; i < t.max_probe; i++) {
    const uint64_t s = probe_slot(t, home, i);
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

// ---------------------------------------------------------------------------
// Partitioned count-first schedule (k <= 64).  The table's spans double as
// partitions: a k-mer belongs to the span of its home slot (the top bits of
// hash_kmer256(key, seed 1)).
//   k_part_scatter  one read pass appends every canonical occurrence to the
//                   region of its span (one relaxed counter per span; the
//                   regions' write frontiers stay in L2, so DRAM sees whole
//                   lines).
//   k_part_count    one CTA per span counts the span's region in a shared-
//                   memory copy of the span and writes the span to the table
//                   (every slot, so the table needs no initialisation).  The
//                   Bloom insert operations of its distinct k-mers (see
//                   k_bloom_from_table) are binned by Bloom range: ranges of
//                   2^19 bits, one u32 operation (bit offset in the range,
//                   and whether the k-mer was seen twice) appended to the
//                   range's region with one reservation per (span, range).
//   k_bloom_apply   one CTA per Bloom range applies its operations to a
//                   shared-memory copy of the range's seen and twice words
//                   and writes both tiers out once.
// The random read-modify-write of a table slot per occurrence becomes a
// streamed write and read of the key, the table is written once, and every
// random Bloom update happens in shared memory.
// ---------------------------------------------------------------------------
struct PartView {
  uint64_t* keys;            // region entries, NL u64 limbs each
  const uint64_t* base;      // region of span p = entries [base[p], base[p + 1])
  unsigned int* fill;        // entries appended to span p: fill[p * kFillStride]
  uint64_t uniform;          // > 0: every region holds `uniform` entries and base[p] =
                             // p * uniform (no lookup); 0: use base[]
  uint32_t log2parts;        // spans = 2^log2parts
  uint32_t packed_home;      // 1: entries carry their home slot in the span in the top
                             // kHomeBits bits of their top limb (keys leave them zero)
  int* err;                  // bit 3: some region overflowed
  uint32_t log2groups;       // > 0: the spans come in 2^log2groups groups counted one after
                             // another; a pass keeps the keys of group `group` only, and its
                             // regions, buckets and span indices are the group's
  uint32_t group;
};
constexpr uint32_t kHomeBits = 13;  // >= log2 of the largest span
// Whether keys of k (NL limbs) leave the top kHomeBits bits of their top limb free.
__host__ __device__ constexpr bool home_fits(unsigned k, int nl) {
  return 2u * k - 64u * (nl - 1) <= 64u - kHomeBits;
}
// One fill counter per 32-byte sector, so that claims on different spans
// never queue behind each other on one L2 line.
constexpr uint32_t kFillStride = 8;

// Launch shapes of the partitioned passes (build-time tunables).
#ifndef SPK_PART_BLOCK
#define SPK_PART_BLOCK 512
#endif
#ifndef SPK_PART_CTAS_PER_SM
#define SPK_PART_CTAS_PER_SM 2
#endif
#ifndef SPK_SCATTER_BATCH
#define SPK_SCATTER_BATCH 4
#endif
constexpr int kPartBlock = SPK_PART_BLOCK;
constexpr int kPartCtasPerSm = SPK_PART_CTAS_PER_SM;
constexpr int kScatterBatch = SPK_SCATTER_BATCH;  // positions per lane in flight in k_part_scatter
constexpr int kSpanBatch = 2;      // slots per thread in flight in k_part_count's write-out
#ifndef SPK_COUNT_PREFETCH
#define SPK_COUNT_PREFETCH 1
#endif
constexpr uint32_t kErrRegion = 8;

// Region, bucket and tile entries: the key's NL limbs side by side (one
// 16-byte access for k <= 64, two for k > 96, three 8-byte ones for 65-96).
template <int NL>
__device__ __forceinline__ void key_put(uint64_t* p, uint64_t i, const Seq<NL>& C) {
  if constexpr (NL == 1) {
    p[i] = C.v[0];
  } else if constexpr (NL == 2) {
    *(ulonglong2*)(p + 2 * i) = make_ulonglong2(C.v[0], C.v[1]);
  } else if constexpr (NL == 4) {
    ((ulonglong2*)(p + 4 * i))[0] = make_ulonglong2(C.v[0], C.v[1]);
    ((ulonglong2*)(p + 4 * i))[1] = make_ulonglong2(C.v[2], C.v[3]);
  } else {
#pragma unroll
    for (int j = 0; j < NL; j++) p[(uint64_t)NL * i + j] = C.v[j];
  }
}
template <int NL>
__device__ __forceinline__ Seq<NL> key_get(const uint64_t* p, uint64_t i) {
  Seq<NL> C;
  if constexpr (NL == 1) {
    C.v[0] = p[i];
  } else if constexpr (NL == 2) {
    const ulonglong2 v = *(const ulonglong2*)(p + 2 * i);
    C.v[0] = v.x;
    C.v[1] = v.y;
  } else if constexpr (NL == 4) {
    const ulonglong2 a = ((const ulonglong2*)(p + 4 * i))[0], b = ((const ulonglong2*)(p + 4 * i))[1];
    C.v[0] = a.x;
    C.v[1] = a.y;
    C.v[2] = b.x;
    C.v[3] = b.y;
  } else {
#pragma unroll
    for (int j = 0; j < NL; j++) C.v[j] = p[(uint64_t)NL * i + j];
  }
  return C;
}
// The same load from global memory, streaming (each entry is read once).
template <int NL>
__device__ __forceinline__ Seq<NL> key_get_cs(const uint64_t* p, uint64_t i) {
  Seq<NL> C;
  if constexpr (NL == 1) {
    C.v[0] = __ldcs(p + i);
  } else if constexpr (NL == 2) {
    const ulonglong2 v = __ldcs((const ulonglong2*)(p + 2 * i));
    C.v[0] = v.x;
    C.v[1] = v.y;
  } else if constexpr (NL == 4) {
    const ulonglong2 a = __ldcs((const ulonglong2*)(p + 4 * i)), b = __ldcs((const ulonglong2*)(p + 4 * i) + 1);
    C.v[0] = a.x;
    C.v[1] = a.y;
    C.v[2] = b.x;
    C.v[3] = b.y;
  } else {
#pragma unroll
    for (int j = 0; j < NL; j++) C.v[j] = __ldcs(p + (uint64_t)NL * i + j);
  }
  return C;
}
template <int NL>
__device__ __forceinline__ void key_copy(uint64_t* d, uint64_t di, const uint64_t* s, uint64_t si) {
  key_put<NL>(d, di, key_get<NL>(s, si));
}

template <int NL>
__global__ void __launch_bounds__(kBlock) k_part_scatter(ReadsView R, unsigned k, PartView pv,
                                                          unsigned long long* __restrict__ occ_out) {
  constexpr int U = kScatterBatch;
  uint64_t occ = 0;
  auto fn = [&](const bool (&active)[U], const Seq<NL> (&Cin)[U]) {
    Seq<NL> C[U];
#pragma unroll
    for (int u = 0; u < U; u++) C[u] = Cin[u];
    uint32_t p[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      p[u] = 0;
      if (!active[u]) continue;
      occ++;
      uint64_t w4[4];
      kmer256_limbs<NL>(C[u], k, w4);
      const uint64_t raw0 = hash_seed(hash_pre(w4), kSeed1);
      p[u] = pv.log2parts ? (uint32_t)(raw0 >> (64 - pv.log2parts)) : 0u;
      if (pv.packed_home)  // the slot within the span, for k_part_count
        C[u].v[NL - 1] |= (raw0 << pv.log2parts) >> (64 - kHomeBits) << (64 - kHomeBits);
    }
    // U independent claims in flight before any is used.
    uint64_t i[U], e[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      i[u] = 0;
      e[u] = 0;
      if (!active[u]) continue;
      const uint32_t got = atomicAdd(pv.fill + (uint64_t)p[u] * kFillStride, 1u);
      if (pv.uniform) {
        i[u] = (uint64_t)p[u] * pv.uniform + got;
        e[u] = (uint64_t)(p[u] + 1) * pv.uniform;
      } else {
        i[u] = __ldg(pv.base + p[u]) + got;
        e[u] = __ldg(pv.base + p[u] + 1);
      }
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      if (!active[u]) continue;
      if (i[u] < e[u]) {
        if (NL == 1) pv.keys[i[u]] = C[u].v[0];
        else *(ulonglong2*)(pv.keys + 2 * i[u]) = make_ulonglong2(C[u].v[0], C[u].v[NL - 1]);
      } else {
        atomicOr(pv.err, (int)kErrRegion);
      }
    }
  };
  foreach_read_roll<NL, U>(R, k, fn);
  warp_add_u64(occ_out, occ);
}

// Two-level form of the read pass (k <= 64).  k_part_scatter appends every
// key to its span's region with a 16-byte store of its own, and those
// scattered stores, not the claims, bound it.  Here the keys are partitioned
// twice, each time through shared memory, so every global store is part of a
// contiguous run:
//   k_part_coarse  one read per thread; per round each thread rolls
//                  coarse_w windows into a shared-memory tile, the tile is
//                  counting-sorted by coarse bucket (the top kCoarseBits bits
//                  of the span index), each bucket's run is reserved with one
//                  atomic and written out contiguously.
//   k_part_fine    chunks of a coarse bucket's keys are sorted the same way
//                  by span and written to the span regions k_part_count reads.
// The keys, and the home bits packed into them, are those k_part_scatter
// writes; only the order inside a region differs, and k_part_count is
// order-free.
constexpr uint32_t kCoarseBits = 6;
constexpr uint32_t kCoarse = 1u << kCoarseBits;
constexpr int kCoarseBlock = 512;
// windows per thread per round: the tile (its keys, and a bucket, rank and
// sorted slot per key) stays within half an SM's shared memory, so two CTAs
// share an SM
// (4,096 keys for k <= 64: 2.90 -> 2.57 ms at k = 55 against 2,048, and
// 3.19 -> 2.75 at k = 21; 24-byte keys keep 2,048, which leaves two CTAs)
template <int NL>
constexpr int coarse_w() { return NL <= 2 ? 8 : 4; }
template <int NL>
constexpr uint32_t coarse_slots() { return kCoarseBlock * coarse_w<NL>(); }
constexpr int kFineBlock = 512;
// keys per chunk of k_part_fine
template <int NL>
constexpr uint32_t fine_chunk() { return NL <= 2 ? 2048 : 1024; }
constexpr uint32_t kFineMaxBits = 12;                    // spans per coarse bucket <= 2^12
static_assert(fine_chunk<1>() % kFineBlock == 0 && fine_chunk<4>() % kFineBlock == 0,
              "k_part_fine loads whole rounds of keys");

struct CoarseView {
  uint64_t* keys;        // NL u64 per entry
  const uint64_t* base;  // bucket b = entries [base[b], base[b + 1]) when uniform == 0
  unsigned int* fill;    // entries appended to bucket b: fill[b * kFillStride]
  uint64_t uniform;      // > 0: base[b] = b * uniform
  int* err;              // bit 3: a bucket overflowed
};
__device__ __forceinline__ uint64_t coarse_base(const CoarseView& cv, uint32_t b) {
  return cv.uniform ? (uint64_t)b * cv.uniform : cv.base[b];
}
__device__ __forceinline__ uint64_t region_base(const PartView& pv, uint32_t p) {
  return pv.uniform ? (uint64_t)p * pv.uniform : pv.base[p];
}

template <int NL>
size_t coarse_smem() {
  constexpr uint32_t kSlots = coarse_slots<NL>();
  return (size_t)kSlots * NL * 8 + kSlots * (1 + 1 + 2 + 2) + kCoarse * (4 + 4 + 8);
}

template <int NL>
__global__ void __launch_bounds__(kCoarseBlock, 2) k_part_coarse(ReadsView R, unsigned k, PartView pv,
                                                                 CoarseView cv,
                                                                 unsigned long long* __restrict__ occ_out) {
  extern __shared__ __align__(16) unsigned char cs_smem[];
  constexpr uint32_t kCoarseSlots = coarse_slots<NL>();
  constexpr int kCoarseW = coarse_w<NL>();
  uint64_t* ks = (uint64_t*)cs_smem;                       // keys by slot
  unsigned long long* gbase = (unsigned long long*)(ks + kCoarseSlots * NL);
  uint32_t* hist = (uint32_t*)(gbase + kCoarse);
  uint32_t* start = hist + kCoarse;
  uint16_t* rk = (uint16_t*)(start + kCoarse);             // rank of a slot in its bucket
  uint16_t* perm = rk + kCoarseSlots;                      // slot of a sorted position
  uint8_t* bk = (uint8_t*)(perm + kCoarseSlots);           // bucket of a slot (0xFF: none)
  uint8_t* sb = bk + kCoarseSlots;                         // bucket of a sorted position
  const unsigned topsh = 2 * k - 2 - 64 * (NL - 1);
  const uint64_t topmask = (2 * k - 64 * (NL - 1)) >= 64 ? ~0ULL : ((1ULL << (2 * k - 64 * (NL - 1))) - 1);
  const unsigned lane = threadIdx.x & 31;
  const uint32_t lp = pv.log2parts - pv.log2groups;        // span index bits within a group
  const uint32_t fshift = lp - kCoarseBits;                // group's span index -> bucket
  if (threadIdx.x < kCoarse) hist[threadIdx.x] = 0;
  uint64_t occ = 0;
  const uint64_t ntiles = (R.n_reads + blockDim.x - 1) / blockDim.x;
  for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const uint64_t r = tile * blockDim.x + threadIdx.x;
    uint32_t np = 0;
    uint64_t bit0 = 0;
    if (r < R.n_reads) {
      const uint32_t len = __ldg(R.lengths + r);
      const uint64_t off = __ldg(R.offsets + r);
      if (off + ((uint64_t)len + 3) / 4 > R.data_len) {  // src/packed_reads.rs:600-602
        atomicOr(R.err, 4);
      } else if (len >= k) {
        np = len - k + 1;
        bit0 = 8ull * (R.byte_base + off);
      }
    }
    Seq<NL> V, Rc;
    if (np) {
      V = extract<NL>(R.words, bit0, k);
      Rc = revcomp<NL>(V, k);
    }
    uint64_t buf = 0, nextbit = bit0 + 2ull * k;
    unsigned bleft = 0;
    uint32_t i = 0;
    while (__syncthreads_or(i < np)) {
      // ---- roll up to kCoarseW windows into the tile ----
#pragma unroll
      for (int w = 0; w < kCoarseW; w++) {
        const uint32_t slot = w * kCoarseBlock + threadIdx.x;  // consecutive lanes, consecutive slots
        uint8_t b = 0xFF;
        if (i < np) {
          if (i > 0) {
            if (bleft == 0) {
              buf = extract<1>(R.words, nextbit, 32).v[0];
              bleft = 32;
            }
            const uint64_t bb = buf >> 62;
            buf <<= 2;
            bleft--;
            nextbit += 2;
            if (NL == 1) {
              V.v[0] = ((V.v[0] << 2) | bb) & topmask;
              Rc.v[0] = (Rc.v[0] >> 2) | ((3 - bb) << topsh);
            } else {
              // the window moves one base: V left by 2 bits, Rc right by 2
#pragma unroll
              for (int j = NL - 1; j >= 1; j--) V.v[j] = (V.v[j] << 2) | (V.v[j - 1] >> 62);
              V.v[0] = (V.v[0] << 2) | bb;
              V.v[NL - 1] &= topmask;
#pragma unroll
              for (int j = 0; j < NL - 1; j++) Rc.v[j] = (Rc.v[j] >> 2) | (Rc.v[j + 1] << 62);
              Rc.v[NL - 1] = (Rc.v[NL - 1] >> 2) | ((3 - bb) << topsh);
            }
          }
          Seq<NL> C = seq_le<NL>(V, Rc) ? V : Rc;  // canonical, src/dna.rs:185-192
          i++;
          occ += pv.group == 0;  // every occurrence once over the groups' passes
          uint64_t w4[4];
          kmer256_limbs<NL>(C, k, w4);
          const uint64_t raw0 = hash_seed(hash_pre(w4), kSeed1);
          const uint32_t p = (uint32_t)(raw0 >> (64 - pv.log2parts));  // log2parts > kCoarseBits
          if (pv.packed_home)
            C.v[NL - 1] |= (raw0 << pv.log2parts) >> (64 - kHomeBits) << (64 - kHomeBits);
          if ((p >> lp) == pv.group) {  // else another pass's
            b = (uint8_t)((p & ((1u << lp) - 1)) >> fshift);
            key_put<NL>(ks, slot, C);
            rk[slot] = (uint16_t)atomicAdd(&hist[b], 1u);
          }
        }
        bk[slot] = b;
      }
      __syncthreads();
      // ---- bucket starts in the tile, and one reservation per bucket ----
      if (threadIdx.x < 32) {
        const uint32_t h0 = hist[2 * lane], h1 = hist[2 * lane + 1];
        uint32_t x = h0 + h1;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
          if ((int)lane >= d) x += y;
        }
        const uint32_t ex = x - h0 - h1;
        start[2 * lane] = ex;
        start[2 * lane + 1] = ex + h0;
        gbase[2 * lane] = h0 ? coarse_base(cv, 2 * lane) + atomicAdd(cv.fill + (uint64_t)(2 * lane) * kFillStride, h0) : 0;
        gbase[2 * lane + 1] =
            h1 ? coarse_base(cv, 2 * lane + 1) + atomicAdd(cv.fill + (uint64_t)(2 * lane + 1) * kFillStride, h1) : 0;
      }
      __syncthreads();
      for (uint32_t slot = threadIdx.x; slot < kCoarseSlots; slot += blockDim.x) {
        const uint8_t b = bk[slot];
        if (b == 0xFF) continue;
        const uint32_t pos = start[b] + rk[slot];
        perm[pos] = (uint16_t)slot;
        sb[pos] = b;
      }
      __syncthreads();
      // ---- contiguous runs out ----
      const uint32_t total = start[kCoarse - 1] + hist[kCoarse - 1];
      for (uint32_t j = threadIdx.x; j < total; j += blockDim.x) {
        const uint32_t b = sb[j];
        const uint64_t gi = gbase[b] + (j - start[b]);
        const uint64_t end = cv.uniform ? (uint64_t)(b + 1) * cv.uniform : cv.base[b + 1];
        if (gi < end) {
          key_copy<NL>(cv.keys, gi, ks, perm[j]);
        } else {
          atomicOr(cv.err, (int)kErrRegion);
        }
      }
      __syncthreads();
      if (threadIdx.x < kCoarse) hist[threadIdx.x] = 0;
    }
  }
  warp_add_u64(occ_out, occ);
}

// Keys in coarse bucket b: its fill, at most its capacity (a bucket that
// overflowed holds only what fits; the overflow flag sends the job back).
__device__ __forceinline__ uint64_t coarse_len(const CoarseView& cv, uint32_t b) {
  const uint64_t capb = cv.uniform ? cv.uniform : cv.base[b + 1] - cv.base[b];
  return min((uint64_t)cv.fill[(uint64_t)b * kFillStride], capb);
}

// cfirst[b] = the first chunk of bucket b (`chunk` keys per chunk);
// cfirst[kCoarse] = the number of chunks.  One warp.
__global__ void k_coarse_chunks(CoarseView cv, uint32_t chunk, uint32_t* __restrict__ cfirst) {
  const unsigned lane = threadIdx.x & 31;
  const uint32_t c0 = (uint32_t)((coarse_len(cv, 2 * lane) + chunk - 1) / chunk);
  const uint32_t c1 = (uint32_t)((coarse_len(cv, 2 * lane + 1) + chunk - 1) / chunk);
  uint32_t x = c0 + c1;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
    if ((int)lane >= d) x += y;
  }
  cfirst[2 * lane] = x - c0 - c1;
  cfirst[2 * lane + 1] = x - c1;
  if (lane == 31) cfirst[kCoarse] = x;
}

// ---- bulk copies into shared memory (the fine pass's staged chunks) ----
// One thread issues cp.async.bulk (the TMA's untiled copy: 16-byte aligned
// addresses, a multiple of 16 bytes) from this GPU's global memory into the
// CTA's shared memory, completing on an mbarrier; the threads wait on the
// barrier's phase with a bounded number of polls.  Each copy lands in this
// CTA's shared memory alone, from this GPU's own memory.
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* m, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(m)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// Orders this thread's earlier generic-proxy accesses of shared memory (after
// a barrier: the CTA's) before later bulk-copy writes into it.
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* m) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(m)), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(m))
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* m, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(m)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Polls of a staged copy's barrier before the kernel gives up (a copy of a
// chunk takes microseconds; this is tens of milliseconds).
constexpr uint32_t kStageSpinLimit = 1u << 20;
constexpr uint32_t kErrStage = 32;  // a staged copy never completed (the job fails)
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* m, uint32_t parity) {
  for (uint32_t i = 0; i < kStageSpinLimit; i++)
    if (mbar_try_wait(m, parity)) return true;
  return false;
}

template <int NL>
size_t fine_smem(uint32_t nfine) {
  constexpr uint32_t kChunk = fine_chunk<NL>();
  // two chunk buffers, then per key: span, rank, sorted slot, span of a sorted position
  return (size_t)kChunk * NL * 8 * 2 + (size_t)kChunk * (2 + 2 + 2 + 2) + (size_t)nfine * (8 + 4 + 4) + 64;
}

// Chunk c of the coarse buckets: its bucket, first key and length.
struct FineChunkAt {
  uint32_t b;
  uint64_t s0;
  uint32_t n;
};
__device__ __forceinline__ FineChunkAt fine_chunk_at(const CoarseView& cv, const uint32_t* cfirst, uint32_t c,
                                                     uint32_t chunk) {
  uint32_t b = 0;  // cfirst[b] <= c < cfirst[b + 1]
  for (uint32_t step = kCoarse >> 1; step; step >>= 1)
    if (cfirst[b + step] <= c) b += step;
  const uint64_t bb = coarse_base(cv, b);
  const uint64_t bend = bb + coarse_len(cv, b);
  const uint64_t s0 = bb + (uint64_t)(c - cfirst[b]) * chunk;
  return FineChunkAt{b, s0, (uint32_t)min((uint64_t)chunk, bend - s0)};
}

// k_part_fine: chunks of each coarse bucket (kFineChunk keys) are sorted by
// span and written to the span regions.  Each CTA walks its chunks with two
// shared-memory buffers: while it ranks and writes out one chunk, the bulk
// copy of its next chunk lands in the other buffer (a chunk whose start or
// size is not a multiple of 16 bytes is loaded by the threads instead).  The
// keys are ranked within their span, and the write-out reads them in span
// order through a permutation, so every global store is part of a contiguous
// run of one span.
template <int NL>
__global__ void __launch_bounds__(kFineBlock, 2) k_part_fine(CoarseView cv, const uint32_t* __restrict__ cfirst,
                                                             PartView pv, unsigned k) {
  extern __shared__ __align__(16) unsigned char fs_smem[];
  constexpr uint32_t kFineChunk = fine_chunk<NL>();
  const uint32_t fbits = pv.log2parts - pv.log2groups - kCoarseBits, nfine = 1u << fbits;
  uint64_t* const kbuf0 = (uint64_t*)fs_smem;
  uint64_t* const kbuf1 = kbuf0 + kFineChunk * NL;
  unsigned long long* gbase = (unsigned long long*)(kbuf1 + kFineChunk * NL);
  uint32_t* hist = (uint32_t*)(gbase + nfine);
  uint32_t* start = hist + nfine;
  uint16_t* fb = (uint16_t*)(start + nfine);  // span (in the bucket) of a loaded key
  uint16_t* rk = fb + kFineChunk;             // its rank in that span
  uint16_t* perm = rk + kFineChunk;           // the loaded key at a sorted position
  uint16_t* sf = perm + kFineChunk;           // span of a sorted position
  __shared__ uint32_t wsum[kFineBlock / 32];
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t staged[2];  // the chunk in buffer i comes by bulk copy
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t nchunks = cfirst[kCoarse];
  // (thread 0) the bulk copy of chunk c into buffer i, if its bytes allow one
  auto issue = [&](uint32_t c, int i) {
    const FineChunkAt ch = fine_chunk_at(cv, cfirst, c, kFineChunk);
    const uint64_t* src = cv.keys + ch.s0 * NL;
    const uint32_t bytes = ch.n * (uint32_t)(NL * 8);
    const bool ok = ((uintptr_t)src & 15) == 0 && (bytes & 15) == 0 && bytes > 0;
    staged[i] = ok;
    if (ok) {
      fence_proxy_async_smem();  // the buffer's last chunk was read before the barrier
      bulk_g2s(i ? kbuf1 : kbuf0, src, bytes, &mbar[i]);
    }
  };
  if (threadIdx.x == 0) {
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
    fence_mbar_init();
    staged[0] = staged[1] = 0;
    if (blockIdx.x < nchunks) issue(blockIdx.x, 0);
  }
  __syncthreads();
  uint32_t ph0 = 0, ph1 = 0;  // phase to wait for on each buffer's barrier
  int buf = 0;
  for (uint32_t c = blockIdx.x; c < nchunks; c += gridDim.x, buf ^= 1) {
    // the next chunk's copy into the other buffer, whose chunk was finished
    // before the barrier that ended the last round
    if (threadIdx.x == 0 && c + gridDim.x < nchunks) issue(c + gridDim.x, buf ^ 1);
    const FineChunkAt ch = fine_chunk_at(cv, cfirst, c, kFineChunk);
    const uint32_t b = ch.b, n = ch.n;
    uint64_t* ks = buf ? kbuf1 : kbuf0;
    for (uint32_t f = threadIdx.x; f < nfine; f += blockDim.x) hist[f] = 0;
    bool ok = true;
    if (staged[buf]) {
      ok = mbar_wait_bounded(&mbar[buf], buf ? ph1 : ph0);
      if (buf) ph1 ^= 1;
      else ph0 ^= 1;
    } else {
      for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) key_put<NL>(ks, j, key_get_cs<NL>(cv.keys, ch.s0 + j));
    }
    if (__syncthreads_or(!ok)) {
      // A copy that never completed: report it, give the other buffer's copy
      // (if one was issued) a bounded wait, and stop.
      if (threadIdx.x == 0) {
        atomicOr(pv.err, (int)kErrStage);
        if (c + gridDim.x < nchunks && staged[buf ^ 1]) mbar_wait_bounded(&mbar[buf ^ 1], buf ? ph0 : ph1);
      }
      return;
    }
    // rank every key within its span
    for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) {
      Seq<NL> C = key_get<NL>(ks, j);
      if (pv.packed_home) C.v[NL - 1] &= ~0ULL >> kHomeBits;
      uint64_t w4[4];
      kmer256_limbs<NL>(C, k, w4);
      const uint32_t p = (uint32_t)(hash_seed(hash_pre(w4), kSeed1) >> (64 - pv.log2parts));
      const uint32_t f = p & (nfine - 1);
      fb[j] = (uint16_t)f;
      rk[j] = (uint16_t)atomicAdd(&hist[f], 1u);
    }
    __syncthreads();
    // exclusive scan of hist (each thread a run of consecutive spans), and
    // one reservation per span in its region
    const uint32_t per = (nfine + blockDim.x - 1) / blockDim.x;
    const uint32_t f0 = min(nfine, threadIdx.x * per), f1 = min(nfine, f0 + per);
    uint32_t run = 0;
    for (uint32_t f = f0; f < f1; f++) run += hist[f];
    uint32_t x = run;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
      if ((int)lane >= d) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    uint32_t before = x - run;
    for (unsigned w = 0; w < warp; w++) before += wsum[w];
    for (uint32_t f = f0; f < f1; f++) {
      const uint32_t h = hist[f];
      start[f] = before;
      before += h;
      const uint32_t pg = (b << fbits) | f;
      gbase[f] = h ? region_base(pv, pg) + atomicAdd(pv.fill + (uint64_t)pg * kFillStride, h) : 0ULL;
    }
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) {
      const uint32_t f = fb[j];
      const uint32_t pos = start[f] + rk[j];
      perm[pos] = (uint16_t)j;
      sf[pos] = (uint16_t)f;
    }
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) {
      const uint32_t f = sf[j];
      const uint32_t pg = (b << fbits) | f;
      const uint64_t gi = gbase[f] + (j - start[f]);
      const uint64_t end = pv.uniform ? (uint64_t)(pg + 1) * pv.uniform : pv.base[pg + 1];
      if (gi < end) {
        key_put<NL>(pv.keys, gi, key_get<NL>(ks, perm[j]));
      } else {
        atomicOr(pv.err, (int)kErrRegion);
      }
    }
    __syncthreads();
  }
}

// Shared-memory slots of one span: keys (8 or 16 bytes) then u32 counts.
template <int NL>
struct SpanKey;
template <>
struct SpanKey<1> {
  typedef unsigned long long T;
};
template <>
struct SpanKey<2> {
  typedef U128 T;
};
template <int NL>
struct WideKey {
  unsigned long long v[NL];
};
template <>
struct SpanKey<3> {
  typedef WideKey<3> T;
};
template <>
struct SpanKey<4> {
  typedef WideKey<4> T;
};
// k > 64: a slot's count word is also its state.  0: empty; kSpanClaimed:
// its claimer is writing the key (it publishes the key and sets the count to
// 1 in the same step, so the state never outlasts that step); else settled,
// and the count.
constexpr uint32_t kSpanClaimed = 0xFFFFFFFFu;

// One probe step at slot s of the shared-memory span: 1 when the
// occurrence of C is counted there (C found, or s empty and claimed for C),
// 0 when s holds another key, 2 when s is being claimed (k > 64: look again).
template <int NL>
__device__ __forceinline__ int span_step(typename SpanKey<NL>::T* keys, uint32_t* cnt, uint32_t s,
                                         const Seq<NL>& C) {
  if constexpr (NL == 1) {
    unsigned long long* kp = (unsigned long long*)&keys[s];
    const unsigned long long cur = *(volatile unsigned long long*)kp;
    if (cur == C.v[0]) { atomicAdd(cnt + s, 1u); return 1; }
    if (cur == kEmpty) {
      const unsigned long long old = atomicCAS(kp, kEmpty, (unsigned long long)C.v[0]);
      if (old == kEmpty || old == C.v[0]) { atomicAdd(cnt + s, 1u); return 1; }
    }
    return 0;
  } else if constexpr (NL == 2) {
    U128* kp = (U128*)&keys[s];
    U128 cur;
    cur.x = ((volatile unsigned long long*)kp)[0];
    cur.y = ((volatile unsigned long long*)kp)[1];
    if (cur.x != kEmpty && cur.y != kEmpty) {
      // settled (a slot changes once, from empty to its key; a read that
      // overlaps that change has an empty half and takes the CAS below)
      if (cur.x == C.v[0] && cur.y == C.v[NL - 1]) { atomicAdd(cnt + s, 1u); return 1; }
      return 0;
    }
    const U128 e{kEmpty, kEmpty}, mine{C.v[0], C.v[NL - 1]};
    const U128 old = atomicCAS(kp, e, mine);
    if ((old.x == kEmpty && old.y == kEmpty) || (old.x == mine.x && old.y == mine.y)) {
      atomicAdd(cnt + s, 1u);
      return 1;
    }
    return 0;
  } else {
    uint32_t c = *(volatile uint32_t*)(cnt + s);
    if (c == 0) {
      c = atomicCAS(cnt + s, 0u, kSpanClaimed);
      if (c == 0) {
        volatile unsigned long long* kp = keys[s].v;
#pragma unroll
        for (int j = 0; j < NL; j++) kp[j] = C.v[j];
        __threadfence_block();
        atomicExch(cnt + s, 1u);
        return 1;
      }
    }
    if (c == kSpanClaimed) return 2;
    __threadfence_block();  // the settled key was written before its count
    const volatile unsigned long long* kp = keys[s].v;
    bool eq = true;
#pragma unroll
    for (int j = 0; j < NL; j++) eq &= kp[j] == C.v[j];
    if (!eq) return 0;
    atomicAdd(cnt + s, 1u);
    return 1;
  }
}

// Bloom operations binned by range (2^kLog2Range bits of both tiers).
struct RangeView {
  uint32_t* ops;             // op = (bit offset in the range << 1) | (k-mer count >= 2)
  const uint64_t* base;      // range r holds ops [base[r], base[r + 1]) (when uniform == 0)
  unsigned int* fill;        // ops appended to range r: fill[r * kFillStride]
  uint64_t uniform;          // > 0: every range holds `uniform` ops, base[r] = r * uniform
  uint32_t nranges;
  int* err;                  // bit 4: some range overflowed
};
constexpr uint32_t kLog2Range = 19;        // 64 KiB of each tier per range
constexpr uint32_t kMaxRanges = 4096;      // shared-memory bins of k_part_count
constexpr uint32_t kErrRange = 16;

__device__ __forceinline__ uint64_t range_base(const RangeView& rv, uint32_t r) {
  return rv.uniform ? (uint64_t)r * rv.uniform : rv.base[r];
}

// Sorted emission of a span's Bloom operations (k <= 64).  Written one by
// one, the ~3 operations per distinct k-mer are 4-byte stores scattered over
// all ranges, and they cost the span pass about a third of its time.  Here
// they are sorted by range in shared memory first: the per-range counts become
// starts (an exclusive scan), and the operations are placed in groups of
// ranges whose operations fit the span's count array (free once the span is
// written out), then each group goes out in contiguous runs.  A group holds
// the ranges whose first operation falls in a window of S minus the largest
// range count, so its operations fit the S entries; a span whose largest
// range count exceeds S/2 is emitted directly instead.
#ifndef SPK_SORTED_OPS
#define SPK_SORTED_OPS 1
#endif
constexpr bool kSortedOps = SPK_SORTED_OPS;

template <int NL>
__device__ __forceinline__ void span_emit_sorted(const typename SpanKey<NL>::T* keys, uint32_t* buf, uint32_t S,
                                                 uint32_t* rs, uint32_t* rcur,
                                                 const unsigned long long* rbase, const RangeView& rv) {
  __shared__ uint32_t wpart[32], wmax[32], bnd[8];
  __shared__ uint32_t s_total, s_maxc;
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const uint32_t nr = rv.nranges;
  const uint32_t mask = (1u << kLog2Range) - 1u;
  // counts -> starts (exclusive scan in place), their total and largest count
  const uint32_t per = (nr + blockDim.x - 1) / blockDim.x;
  const uint32_t r0 = min(nr, threadIdx.x * per), r1 = min(nr, r0 + per);
  uint32_t sum = 0, mx = 0;
  for (uint32_t r = r0; r < r1; r++) {
    const uint32_t c = rs[r];
    sum += c;
    mx = max(mx, c);
  }
  uint32_t x = sum;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
    if ((int)lane >= d) x += y;
  }
  const uint32_t wm = __reduce_max_sync(0xffffffffu, mx);
  if (lane == 31) wpart[warp] = x;
  if (lane == 0) wmax[warp] = wm;
  __syncthreads();
  uint32_t before = x - sum;
  for (unsigned w = 0; w < warp; w++) before += wpart[w];
  for (uint32_t r = r0; r < r1; r++) {
    const uint32_t c = rs[r];
    rs[r] = before;
    before += c;
  }
  if (threadIdx.x == 0) {
    uint32_t tt = 0, mm = 0;
    for (unsigned w = 0; w < nwarps; w++) {
      tt += wpart[w];
      mm = max(mm, wmax[w]);
    }
    s_total = tt;
    s_maxc = mm;
  }
  __syncthreads();
  // groups of ranges starting within a window of H positions span at most
  // H + (largest count) <= S positions of the buffer
  const uint32_t total = s_total, H = s_maxc <= (S >> 1) ? S - s_maxc : 0u;
  if (H == 0) {
    // direct emission (a range holds more than half a span's worth)
    for (uint32_t s = threadIdx.x; s < S; s += blockDim.x) {
      const uint32_t* st = (const uint32_t*)&keys[s];
      if (st[1] == 0xFFFFFFFFu) continue;  // empty slot
      const uint32_t flag = st[0] >> 31;
      const uint32_t pk[3] = {st[0] & 0x7FFFFFFFu, st[1], st[2]};
#pragma unroll
      for (int j = 0; j < 3; j++) {
        const uint32_t r = pk[j] >> kLog2Range;
        const uint64_t i = rbase[r] + atomicAdd(rcur + r, 1u);
        const uint64_t end = rv.uniform ? (uint64_t)(r + 1) * rv.uniform : rv.base[r + 1];
        if (i < end) rv.ops[i] = ((pk[j] & mask) << 1) | flag;
        else atomicOr(rv.err, (int)kErrRange);
      }
    }
    __syncthreads();
    return;
  }
  const uint32_t G = (total + H - 1) / H;  // <= 6: at most 3 S operations, H >= S / 2
  if (threadIdx.x <= G) {
    // bnd[g] = the first range start at or after g H (total if none)
    const uint32_t xv = threadIdx.x * H;
    uint32_t lo = 0, hi = nr;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (rs[mid] < xv) lo = mid + 1;
      else hi = mid;
    }
    bnd[threadIdx.x] = (xv >= total || lo == nr) ? total : rs[lo];
  }
  __syncthreads();
  for (uint32_t g = 0; g < G; g++) {
    const uint32_t gb = g * H;
    for (uint32_t s = threadIdx.x; s < S; s += blockDim.x) {
      const uint32_t* st = (const uint32_t*)&keys[s];
      if (st[1] == 0xFFFFFFFFu) continue;  // empty slot
      const uint32_t flag = st[0] >> 31;
      const uint32_t pk[3] = {st[0] & 0x7FFFFFFFu, st[1], st[2]};
#pragma unroll
      for (int j = 0; j < 3; j++) {
        const uint32_t r = pk[j] >> kLog2Range;
        const uint32_t a = rs[r];
        if (a < gb || a - gb >= H) continue;  // another group's range
        const uint32_t pos = a + atomicAdd(rcur + r, 1u);
        buf[pos - gb] = (r << 20) | ((pk[j] & mask) << 1) | flag;
      }
    }
    __syncthreads();
    const uint32_t lo = bnd[g], hi = bnd[g + 1];
    for (uint32_t q = lo + threadIdx.x; q < hi; q += blockDim.x) {
      const uint32_t v = buf[q - gb];
      const uint32_t r = v >> 20;
      const uint64_t i = rbase[r] + (q - rs[r]);
      const uint64_t end = rv.uniform ? (uint64_t)(r + 1) * rv.uniform : rv.base[r + 1];
      if (i < end) rv.ops[i] = v & 0xFFFFFu;
      else atomicOr(rv.err, (int)kErrRange);
    }
    __syncthreads();
  }
}

// Output of the span count when the count table is not kept: the span's
// k-mers counted at least lmin times (at least twice) go straight to the
// k-mer list, and those counted once to a buffer of keys that singleton
// admission reads after the Bloom tiers are built.  Both hold every distinct
// k-mer at most once, so cap (the table's slot count) bounds each.
constexpr int kHistBins = 256;  // counts >= 255 share the last bin
struct ListOut {
  uint64_t* l[4];               // list: limbs 0..NL-1 (SoA)
  uint32_t* cnt;                // list: counts (nullptr: the table is written instead)
  uint64_t* s[4];               // singletons: limbs 0..NL-1
  uint64_t cap;                 // list entries
  uint64_t scap;                // singleton keys
  uint32_t lmin;                // smallest count listed (>= 2 here; singletons are listed
                                // by admission when lmin is 1)
  unsigned long long* fill;     // [0] list entries, [1] singletons
  unsigned long long* hist;     // kHistBins counts of the k-mers counted >= 2 times
  unsigned long long* occ2;     // occurrences of the k-mers counted >= 2 times
};

template <int NL, bool OPS>
__global__ void __launch_bounds__(kPartBlock, kPartCtasPerSm) k_part_count(PartView pv, TableView t, unsigned k,
                                                            FastMod fm, U128* __restrict__ tiers,
                                                            RangeView rv, ListOut lo) {
  typedef typename SpanKey<NL>::T KeyT;
  extern __shared__ __align__(16) unsigned char span_smem[];
  // list output: per (write-out round, warp) entry counts of the list and of
  // the singletons, their exclusive prefixes, and the span's two reservations
  constexpr int kWarps = kPartBlock / 32;
  constexpr int kRounds = (1 << kHomeBits) / kPartBlock > 0 ? (1 << kHomeBits) / kPartBlock : 1;
  __shared__ uint32_t lw[2][kRounds * kWarps];
  __shared__ unsigned long long lbase[2];
  __shared__ unsigned s_hist[kHistBins];
  __shared__ int s_full;  // this span, or an earlier one of the launch, ran out of slots
  const bool to_list = lo.cnt != nullptr;
  const uint32_t lmin = lo.lmin < 2 ? 2u : lo.lmin;
  uint64_t occ2 = 0;
  if (to_list)
    for (int i = threadIdx.x; i < kHistBins; i += blockDim.x) s_hist[i] = 0;
  const uint32_t S = 1u << t.log2span;
  KeyT* keys = (KeyT*)span_smem;
  uint32_t* cnt = (uint32_t*)(span_smem + (size_t)S * sizeof(KeyT));
  // OPS: per-range op counts (then the ops emitted so far), and the global
  // index reserved for each range's ops of this span
  uint32_t* rhist = cnt + S;
  // k <= 64 with sorted emission: a cursor per range (the ops placed so far)
  uint32_t* rcur = rhist + ((rv.nranges + 1) & ~1u);
  unsigned long long* rbase =
      (unsigned long long*)(rcur + ((NL >= 2 && kSortedOps) ? ((rv.nranges + 1) & ~1u) : 0u));
  const uint32_t nparts = 1u << (pv.log2parts - pv.log2groups);  // this group's spans
  for (uint32_t p = blockIdx.x; p < nparts; p += gridDim.x) {
    // A span that ran out of slots sends the job back with more slots: the
    // spans after it are skipped (their counts would be dropped).
    if (threadIdx.x == 0) s_full = *(volatile int*)t.err & 1;
    __syncthreads();
    if (s_full) break;
    for (uint32_t s = threadIdx.x; s < S; s += blockDim.x) {
      if constexpr (NL == 1) {
        ((unsigned long long*)keys)[s] = kEmpty;
      } else if constexpr (NL == 2) {
        ((U128*)keys)[s] = U128{kEmpty, kEmpty};
      } else {
        // (k > 64: the count marks empty slots; all-ones keys mark them for
        // the sorted emission of the Bloom operations)
#pragma unroll
        for (int j = 0; j < NL; j++) keys[s].v[j] = kEmpty;
      }
      cnt[s] = 0;
    }
    if (OPS)
      for (uint32_t r = threadIdx.x; r < rv.nranges; r += blockDim.x) {
        rhist[r] = 0;
        if (NL >= 2 && kSortedOps) rcur[r] = 0;
      }
    __syncthreads();
    const uint64_t b = pv.base[p];
    const uint64_t e = min(pv.base[p + 1], b + (uint64_t)pv.fill[(uint64_t)p * kFillStride]);
    // Each thread keeps one key in flight and makes one probe step per
    // iteration, taking its next key as soon as the current one is placed:
    // a warp's steps are then not held back by its longest probe sequence.
    bool full = false;
    {
      uint64_t i = b + threadIdx.x;
      bool have = false;
      Seq<NL> C;
      uint32_t home = 0, step = 0, waits = 0;
      for (;;) {
        if (!have) {
          if (i >= e || *(volatile int*)&s_full) break;
          C = key_get_cs<NL>(pv.keys, i);
          i += blockDim.x;
#if SPK_COUNT_PREFETCH
          // the key this lane takes next, on its way to L1 while this one is placed
          if (i < e) asm volatile("prefetch.global.L1 [%0];" ::"l"(pv.keys + (uint64_t)NL * i));
#endif
          if (pv.packed_home) {
            const uint64_t top = C.v[NL - 1];
            home = (uint32_t)(top >> (64 - kHomeBits)) >> (kHomeBits - t.log2span);
            C.v[NL - 1] = top & (~0ULL >> kHomeBits);
          } else {
            uint64_t w4[4];
            kmer256_limbs<NL>(C, k, w4);
            home = (uint32_t)(table_home(t, hash_seed(hash_pre(w4), kSeed1)) & (S - 1));
          }
          have = true;
          step = 0;
          waits = 0;
        }
        const int got = span_step<NL>(keys, cnt, (home + step) & (S - 1), C);
        if (got == 1) {
          have = false;
        } else if (got == 0) {
          if (++step == S) {
            full = true;  // every slot probed
            have = false;
            s_full = 1;
          }
        } else if (++waits > kSpinLimit) {
          atomicOr(t.err, 2);  // a claim that never settled: the job fails
          have = false;
        }
      }
    }
    if (full) atomicOr(t.err, 1);  // span full: the host regrows the table
    __syncthreads();
    if (s_full) break;
    const uint64_t g0 = ((uint64_t)pv.group << (pv.log2parts - pv.log2groups) | p) << t.log2span;
    if (OPS && to_list) {
      // Entries of each (round, warp) of the write-out loop below: a ballot
      // per round, then one reservation per span for the list and one for
      // the singletons, so that each warp's entries of a round are
      // contiguous in both.
      const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
      const uint32_t rounds = (S + blockDim.x - 1) / blockDim.x;
      for (uint32_t r = 0; r < rounds; r++) {
        const uint32_t s = r * blockDim.x + threadIdx.x;
        const uint32_t c = s < S ? cnt[s] : 0u;
        const unsigned bl = __ballot_sync(FULL, c >= lmin), bs = __ballot_sync(FULL, c == 1);
        if (lane == 0) {
          lw[0][r * kWarps + warp] = __popc(bl);
          lw[1][r * kWarps + warp] = __popc(bs);
        }
        if (c >= 2) {
          atomicAdd(&s_hist[c < kHistBins - 1 ? c : kHistBins - 1], 1u);
          occ2 += c;
        }
      }
      __syncthreads();
      if (warp < 2) {
        // exclusive scan of the (round, warp) counts of list `warp`
        const uint32_t n = ((S + blockDim.x - 1) / blockDim.x) * kWarps;
        uint32_t carry = 0;
        for (uint32_t b = 0; b < n; b += 32) {
          const uint32_t v = b + lane < n ? lw[warp][b + lane] : 0u;
          uint32_t x = v;
#pragma unroll
          for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(FULL, x, d);
            if ((int)lane >= d) x += y;
          }
          if (b + lane < n) lw[warp][b + lane] = carry + x - v;
          carry += __shfl_sync(FULL, x, 31);
        }
        if (lane == 0) lbase[warp] = carry ? atomicAdd(lo.fill + warp, (unsigned long long)carry) : 0ULL;
      }
      __syncthreads();
    }
    if (OPS) {
      // Write the span out (to the table, or to the list and the singleton
      // keys) and count its Bloom operations per range.
      const unsigned warp = threadIdx.x >> 5;
      const uint32_t rounds = (S + blockDim.x - 1) / blockDim.x;
      for (uint32_t r = 0; r < rounds; r++) {
        const uint32_t s = r * blockDim.x + threadIdx.x;
        if (!to_list && s >= S) continue;
        const uint32_t c = s < S ? cnt[s] : 0u;
        Seq<NL> C;
        if constexpr (NL == 1) {
          C.v[0] = c ? ((unsigned long long*)keys)[s] : kEmpty;
          if (!to_list) {
            ulonglong2* gp = (ulonglong2*)slot_key<NL>(t, g0 + s);
            *gp = make_ulonglong2(C.v[0], (unsigned long long)c);
          }
        } else if constexpr (NL == 2) {
          const U128 kv = c ? ((U128*)keys)[s] : U128{kEmpty, kEmpty};
          C.v[0] = kv.x;
          C.v[NL - 1] = kv.y;
          if (!to_list) {
            ulonglong2* gp = (ulonglong2*)slot_key<NL>(t, g0 + s);
            gp[0] = make_ulonglong2(kv.x, kv.y);
            gp[1] = make_ulonglong2((unsigned long long)c, 0ULL);
          }
        } else {
          // k > 64 runs in list mode only
#pragma unroll
          for (int j = 0; j < NL; j++) C.v[j] = c ? keys[s].v[j] : kEmpty;
        }
        if (to_list) {
          // (lanes past the span's end have c == 0 and take part in the ballots only)
          const unsigned bl = __ballot_sync(FULL, c >= lmin), bs = __ballot_sync(FULL, c == 1);
          if (c >= lmin) {
            const uint64_t q = lbase[0] + lw[0][r * kWarps + warp] + __popc(bl & lanemask_lt());
            if (q < lo.cap) {
#pragma unroll
              for (int j = 0; j < NL; j++) lo.l[j][q] = C.v[j];
              lo.cnt[q] = c;
            }
          } else if (c == 1) {
            const uint64_t q = lbase[1] + lw[1][r * kWarps + warp] + __popc(bs & lanemask_lt());
            if (q < lo.scap) {
#pragma unroll
              for (int j = 0; j < NL; j++) lo.s[j][q] = C.v[j];
            }
          }
        }
        if (!c) continue;
        uint64_t raw[3], pos[3];
        bloom_positions<NL>(C, k, fm, raw, pos);
#pragma unroll
        for (int j = 0; j < 3; j++) {
          atomicAdd(rhist + (uint32_t)(pos[j] >> kLog2Range), 1u);
          // k > 32: the written-out key's slot keeps the three positions as
          // (range << kLog2Range | offset), at most 31 bits each
          if (NL >= 2) ((uint32_t*)&keys[s])[j] = (uint32_t)pos[j];
        }
        // with the sorted emission the count array is reused: the slot's
        // stash keeps "count >= 2" in bit 31 of its first position (positions
        // are below 2^31 since there are at most 2^12 ranges); an empty
        // slot's stash stays all ones
        if (NL >= 2 && kSortedOps && c >= 2) ((uint32_t*)&keys[s])[0] |= 0x80000000u;
      }
      __syncthreads();
      // One reservation per non-empty range; rhist then counts the span's
      // ops emitted into each range.
      for (uint32_t r = threadIdx.x; r < rv.nranges; r += blockDim.x) {
        const uint32_t n = rhist[r];
        rbase[r] = n ? range_base(rv, r) + atomicAdd(rv.fill + (uint64_t)r * kFillStride, n) : 0ULL;
        if (!(NL >= 2 && kSortedOps)) rhist[r] = 0;
      }
      __syncthreads();
      if (NL >= 2 && kSortedOps) {
        span_emit_sorted<NL>(keys, cnt, S, rhist, rcur, rbase, rv);
      } else {
      // Emit the operations.
      for (uint32_t s = threadIdx.x; s < S; s += blockDim.x) {
        const uint32_t c = cnt[s];
        if (!c) continue;
        uint32_t pk[3];
        if (NL >= 2) {
#pragma unroll
          for (int j = 0; j < 3; j++) pk[j] = ((const uint32_t*)&keys[s])[j];
        } else {
          Seq<NL> C;
          C.v[0] = ((unsigned long long*)keys)[s];
          uint64_t raw[3], pos[3];
          bloom_positions<NL>(C, k, fm, raw, pos);
#pragma unroll
          for (int j = 0; j < 3; j++) pk[j] = (uint32_t)pos[j];
        }
#pragma unroll
        for (int j = 0; j < 3; j++) {
          const uint32_t r = pk[j] >> kLog2Range;
          const uint64_t i = rbase[r] + atomicAdd(rhist + r, 1u);
          const uint64_t end = rv.uniform ? (uint64_t)(r + 1) * rv.uniform : rv.base[r + 1];
          if (i < end)
            rv.ops[i] = ((pk[j] & ((1u << kLog2Range) - 1)) << 1) | (c >= 2 ? 1u : 0u);
          else
            atomicOr(rv.err, (int)kErrRange);
        }
      }
      __syncthreads();
      }
      continue;
    }
    if constexpr (NL <= 2) {
    constexpr int U = kSpanBatch;
    for (uint32_t s0 = threadIdx.x; s0 < S; s0 += U * blockDim.x) {
      uint32_t c[U];
      uint64_t pos[U][3];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const uint32_t s = s0 + u * blockDim.x;
        c[u] = 0;
        pos[u][0] = pos[u][1] = pos[u][2] = 0;
        if (s >= S) continue;
        c[u] = cnt[s];
        Seq<NL> C;
        if (NL == 1) {
          C.v[0] = c[u] ? ((unsigned long long*)keys)[s] : kEmpty;
          ulonglong2* gp = (ulonglong2*)slot_key<NL>(t, g0 + s);
          *gp = make_ulonglong2(C.v[0], (unsigned long long)c[u]);
        } else {
          const U128 kv = c[u] ? ((U128*)keys)[s] : U128{kEmpty, kEmpty};
          C.v[0] = kv.x;
          C.v[NL - 1] = kv.y;
          ulonglong2* gp = (ulonglong2*)slot_key<NL>(t, g0 + s);
          gp[0] = make_ulonglong2(kv.x, kv.y);
          gp[1] = make_ulonglong2((unsigned long long)c[u], 0ULL);
        }
        if (c[u]) {
          uint64_t raw[3];
          bloom_positions<NL>(C, k, fm, raw, pos[u]);
        }
      }
      // The Bloom operations of these k-mers (see k_bloom_from_table).
      bloom_ops_distinct<U>(tiers, pos, c);
    }
    }
    __syncthreads();
  }
  if (to_list) {
    warp_add_u64(lo.occ2, occ2);
    __syncthreads();
    for (int i = threadIdx.x; i < kHistBins; i += blockDim.x)
      if (s_hist[i]) atomicAdd(lo.hist + i, (unsigned long long)s_hist[i]);
  }
}

// Exact regions after an overflow: base[p] = sum of fill[0..p), base[P] = total.
// One block of 1024 threads.
__global__ void __launch_bounds__(1024) k_part_bases(const unsigned int* __restrict__ fill,
                                                     uint32_t n, uint64_t* __restrict__ base) {
  __shared__ unsigned long long part[1024];
  const uint32_t per = (n + blockDim.x - 1) / blockDim.x;
  const uint32_t lo = min(n, threadIdx.x * per), hi = min(n, lo + per);
  unsigned long long s = 0;
  for (uint32_t i = lo; i < hi; i++) s += fill[(uint64_t)i * kFillStride];
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long run = 0;
    for (uint32_t j = 0; j < blockDim.x; j++) {
      const unsigned long long v = part[j];
      part[j] = run;
      run += v;
    }
    base[n] = run;
  }
  __syncthreads();
  unsigned long long run = part[threadIdx.x];
  for (uint32_t i = lo; i < hi; i++) {
    base[i] = run;
    run += fill[(uint64_t)i * kFillStride];
  }
}

// Uniform regions: base[p] = p * cap for p = 0..n.
__global__ void k_part_uniform(uint32_t n, uint64_t cap, uint64_t* __restrict__ base) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i <= n;
       i += (uint64_t)gridDim.x * blockDim.x)
    base[i] = i * cap;
}

// Applies the operations of each Bloom range in shared memory (one u32 word
// per 32 bits of each tier) and writes the range's seen and twice words,
// with their popcounts.  An operation of a k-mer seen twice sets both bits;
// an operation of a k-mer seen once sets its seen bit and, if that bit was
// already set, its twice bit -- the same tiers as applying every occurrence.
constexpr int kApplyBlock = 1024;
__global__ void __launch_bounds__(kApplyBlock) k_bloom_apply(RangeView rv, uint64_t num_words,
                                                             uint64_t* __restrict__ seen,
                                                             uint64_t* __restrict__ twice,
                                                             unsigned long long* __restrict__ pops) {
  extern __shared__ __align__(16) uint32_t range_smem[];
  constexpr uint32_t W32 = (1u << kLog2Range) / 32;  // u32 words per tier and range
  uint32_t* s_seen = range_smem;
  uint32_t* s_twice = range_smem + W32;
  uint64_t cs = 0, ct = 0;
  for (uint32_t r = blockIdx.x; r < rv.nranges; r += gridDim.x) {
    for (uint32_t i = threadIdx.x; i < 2 * W32; i += blockDim.x) range_smem[i] = 0;
    __syncthreads();
    const uint64_t b = range_base(rv, r);
    const uint64_t end = rv.uniform ? (uint64_t)(r + 1) * rv.uniform : rv.base[r + 1];
    const uint64_t e = min(end, b + (uint64_t)rv.fill[(uint64_t)r * kFillStride]);
    auto apply = [&](uint32_t op) {
      const uint32_t off = op >> 1;
      const uint32_t w = off >> 5, bit = 1u << (off & 31);
      if (op & 1) {
        atomicOr(s_seen + w, bit);
        atomicOr(s_twice + w, bit);
      } else if (atomicOr(s_seen + w, bit) & bit) {
        atomicOr(s_twice + w, bit);
      }
    };
    // The operations stream in as 16-byte loads, two per thread in flight
    // (one 4-byte load per thread kept too few bytes in flight: the pass ran
    // at the latency of its loads); the unaligned head and the tail one by one.
    const uint64_t a0 = min(e, (uint64_t)((b + 3) & ~3ULL)), a1 = max(a0, (uint64_t)(e & ~3ULL));
    for (uint64_t i = b + threadIdx.x; i < a0; i += blockDim.x) apply(__ldcs(rv.ops + i));
    const uint4* v = (const uint4*)(rv.ops + a0);
    const uint64_t nv = (a1 - a0) / 4;
    uint64_t q = threadIdx.x;
    for (; q + blockDim.x < nv; q += 2 * blockDim.x) {
      const uint4 x = __ldcs(v + q), y = __ldcs(v + q + blockDim.x);
      apply(x.x);
      apply(x.y);
      apply(x.z);
      apply(x.w);
      apply(y.x);
      apply(y.y);
      apply(y.z);
      apply(y.w);
    }
    for (; q < nv; q += blockDim.x) {
      const uint4 x = __ldcs(v + q);
      apply(x.x);
      apply(x.y);
      apply(x.z);
      apply(x.w);
    }
    for (uint64_t i = a1 + threadIdx.x; i < e; i += blockDim.x) apply(__ldcs(rv.ops + i));
    __syncthreads();
    const uint64_t g0 = (uint64_t)r * (W32 / 2);
    for (uint32_t i = threadIdx.x; i < W32 / 2 && g0 + i < num_words; i += blockDim.x) {
      const uint64_t sv = (uint64_t)s_seen[2 * i] | ((uint64_t)s_seen[2 * i + 1] << 32);
      const uint64_t tv = (uint64_t)s_twice[2 * i] | ((uint64_t)s_twice[2 * i + 1] << 32);
      seen[g0 + i] = sv;
      twice[g0 + i] = tv;
      cs += __popcll(sv);
      ct += __popcll(tv);
    }
    __syncthreads();
  }
  warp_add_u64(pops + 0, cs);
  warp_add_u64(pops + 1, ct);
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
// A table slot: its count, and its key in C (keys of empty slots are junk).
template <int NL>
__device__ __forceinline__ uint32_t load_slot(const TableView& t, uint64_t s, Seq<NL>& C) {
  if (NL == 1) {
    const ulonglong2 v = __ldcs((const ulonglong2*)slot_key<NL>(t, s));
    C.v[0] = v.x;
    return (uint32_t)v.y;
  }
  if (NL == 2) {
    const ulonglong2* q = (const ulonglong2*)slot_key<NL>(t, s);
    const ulonglong2 a = __ldcs(q), b = __ldcs(q + 1);
    C.v[0] = a.x;
    C.v[NL - 1] = a.y;
    return (uint32_t)b.x;
  }
  const uint32_t c = *slot_count<NL>(t, s);
  const uint64_t* kp = slot_key<NL>(t, s);
#pragma unroll
  for (int j = 0; j < NL; j++) C.v[j] = c ? kp[j] : 0;
  return c;
}

constexpr int kAdmitBatch = 2;  // slots per lane in flight

template <int NL>
__global__ void __launch_bounds__(kBlock, 4) k_admit_compact(TableView t, unsigned k, FastMod fm,
                                                          const uint64_t* __restrict__ twice,
                                                          int check_singletons, uint32_t lmin,
                                                          uint64_t* o0, uint64_t* o1, uint64_t* o2,
                                                          uint64_t* o3, uint32_t* __restrict__ ocnt,
                                                          uint64_t out_cap,
                                                          unsigned long long* __restrict__ hist,
                                                          unsigned long long* __restrict__ sums,
                                                          unsigned long long* __restrict__ rejected) {
  constexpr int U = kAdmitBatch;
  constexpr int NW = kBlock / 32;
  constexpr uint64_t CHUNK = (uint64_t)kBlock * U;
  __shared__ unsigned sh[kHistBins];
  __shared__ unsigned wkeep[NW];
  __shared__ unsigned long long cta_base;
  for (int i = threadIdx.x; i < kHistBins; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint64_t n_adm = 0, n_one = 0, occ = 0, n_rej = 0;
  // A CTA scans CHUNK consecutive slots at a time (warp w: 32U of them) and
  // reserves its list entries with one atomic per chunk.
  for (uint64_t chunk0 = blockIdx.x * CHUNK; chunk0 < t.capacity; chunk0 += (uint64_t)gridDim.x * CHUNK) {
    const uint64_t chunk = chunk0 + (uint64_t)warp * 32 * U;
    uint32_t c[U];
    Seq<NL> C[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const uint64_t s = chunk + 32 * u + lane;
      c[u] = s < t.capacity ? load_slot<NL>(t, s, C[u]) : 0u;
      if (c[u] & kRejected) {  // rejected by an earlier admission pass
        c[u] = 0;
        n_rej++;
      }
    }
    // Singletons: a k-mer seen once is admitted when its three twice bits are
    // set; the twice words of every slot in flight are loaded together.
    uint64_t pos[U][3], tw[U][3];
#pragma unroll
    for (int u = 0; u < U; u++) {
      if (c[u] == 1 && check_singletons) {
        uint64_t raw[3];
        bloom_positions<NL>(C[u], k, fm, raw, pos[u]);
#pragma unroll
        for (int j = 0; j < 3; j++) tw[u][j] = __ldg(twice + (pos[u][j] >> 6));
      }
    }
    unsigned km[U];
    unsigned nkeep = 0;
#pragma unroll
    for (int u = 0; u < U; u++) {
      const bool admit = !(c[u] == 1 && check_singletons) ||
                         ((tw[u][0] >> (pos[u][0] & 63)) & (tw[u][1] >> (pos[u][1] & 63)) &
                          (tw[u][2] >> (pos[u][2] & 63)) & 1);
      if (!admit) {
        *slot_count<NL>(t, chunk + 32 * u + lane) = 1u | kRejected;
        c[u] = 0;
        n_rej++;
      }
      if (c[u]) {
        n_adm++;
        n_one += c[u] == 1;
        occ += c[u];
        atomicAdd(&sh[c[u] < kHistBins - 1 ? c[u] : kHistBins - 1], 1u);
      }
      km[u] = __ballot_sync(FULL, c[u] != 0 && c[u] >= lmin);
      nkeep += __popc(km[u]);
    }
    if (lane == 0) wkeep[warp] = nkeep;
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned tot = 0;
      for (int w = 0; w < NW; w++) tot += wkeep[w];
      cta_base = tot ? atomicAdd(sums + 3, (unsigned long long)tot) : 0ULL;
    }
    __syncthreads();
    uint64_t p0 = cta_base;
    for (unsigned w = 0; w < warp; w++) p0 += wkeep[w];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const uint64_t p = p0 + __popc(km[u] & lanemask_lt());
      if (((km[u] >> lane) & 1) && p < out_cap) {
        o0[p] = C[u].v[0];
        if (NL > 1) o1[p] = C[u].v[NL > 1 ? 1 : 0];
        if (NL > 2) o2[p] = C[u].v[NL > 2 ? 2 : 0];
        if (NL > 3) o3[p] = C[u].v[NL > 3 ? 3 : 0];
        ocnt[p] = c[u];
      }
      p0 += __popc(km[u]);
    }
    __syncthreads();  // wkeep and cta_base are reused by the next chunk
  }
  warp_add_u64(sums + 0, n_adm);
  warp_add_u64(sums + 1, n_one);
  warp_add_u64(sums + 2, occ);
  warp_add_u64(rejected, n_rej);
  __syncthreads();
  for (int i = threadIdx.x; i < kHistBins; i += blockDim.x)
    if (sh[i]) atomicAdd(hist + i, (unsigned long long)sh[i]);
}

// Singleton admission when the span count wrote the list instead of the
// table: a k-mer counted once is admitted when its three twice bits are set
// (a k-mer counted twice always has them).  Admitted singletons add to the
// count histogram's bin 1 and, when the list keeps count-1 k-mers (lmin 1),
// are appended to the list after the span count's entries, one reservation
// per warp.  sums: [0] admitted singletons.
template <int NL>
__global__ void __launch_bounds__(kBlock) k_admit_singletons(ListOut lo, unsigned k, FastMod fm,
                                                              const uint64_t* __restrict__ twice,
                                                              unsigned long long* __restrict__ sums) {
  const unsigned lane = threadIdx.x & 31;
  const uint64_t n = min((uint64_t)lo.fill[1], lo.scap);
  uint64_t adm = 0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = blockIdx.x * (uint64_t)blockDim.x; base < n; base += stride) {
    const uint64_t i = base + threadIdx.x;
    bool admit = false;
    Seq<NL> C;
    if (i < n) {
#pragma unroll
      for (int j = 0; j < NL; j++) C.v[j] = __ldcs(lo.s[j] + i);
      uint64_t raw[3], pos[3];
      bloom_positions<NL>(C, k, fm, raw, pos);
      const uint64_t a = __ldg(twice + (pos[0] >> 6)), b = __ldg(twice + (pos[1] >> 6)),
                     c = __ldg(twice + (pos[2] >> 6));
      admit = (a >> (pos[0] & 63)) & (b >> (pos[1] & 63)) & (c >> (pos[2] & 63)) & 1;
    }
    adm += admit;
    if (lo.lmin <= 1) {
      const unsigned m = __ballot_sync(FULL, admit);
      if (m) {
        unsigned long long wb = 0;
        if (lane == 0) wb = atomicAdd(lo.fill, (unsigned long long)__popc(m));
        const uint64_t q = __shfl_sync(FULL, wb, 0) + __popc(m & lanemask_lt());
        if (admit && q < lo.cap) {
#pragma unroll
          for (int j = 0; j < NL; j++) lo.l[j][q] = C.v[j];
          lo.cnt[q] = 1;
        }
      }
    }
  }
  warp_add_u64(sums, adm);
  warp_add_u64(lo.hist + 1, adm);
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
// rc(X.extend_right(b)) as a (k+1)-mer: comp(b) in front of RC = revcomp(X).
template <int NL, int NLE>
__device__ __forceinline__ Seq<NLE> prepend_wide(const Seq<NL>& RC, unsigned c, unsigned k) {
  Seq<NLE> R;
#pragma unroll
  for (int i = 0; i < NLE; i++) R.v[i] = i < NL ? RC.v[i] : 0;
  const unsigned top = 2u * k;  // bit of the first base of the (k+1)-mer
#pragma unroll
  for (int i = 0; i < NLE; i++)
    if ((unsigned)i == (top >> 6)) R.v[i] |= (uint64_t)c << (top & 63);
  return R;
}

// The solid k-mers (count >= cutoff) of a list as a set: open addressing with
// linear probing over 2^log2cap slots of NL key limbs (k <= 64), all-ones =
// empty (never a canonical k-mer: all-ones full limbs would be poly-T, whose
// reverse complement poly-A is smaller, and a partial top limb never has its
// unused bits set).  Home slot: hash_kmer256(key, seed 1) >> (64 - log2cap).
// Probed 8 times per solid k-mer by k_edges, it is small enough to stay
// mostly in L2, unlike the count table.  A bit filter of 2^log2filter bits
// (bit: the low hash bits of each solid k-mer) answers most lookups of
// k-mers that are not solid with one L2-resident bit.
struct SetView {
  uint64_t* keys;
  uint32_t log2cap;
  uint32_t log2filter;
  uint32_t* filter;
};
__device__ __forceinline__ uint64_t filter_bit(const SetView& sv, uint64_t raw0) {
  return raw0 & ((1ULL << sv.log2filter) - 1);
}

// Wide keys (k > 64) take a slot with a CAS on their top limb and then write
// the others: the keys inserted are distinct, and lookups run in a later
// kernel.  The top limb of a key with 2k < 64 NL has unused high bits, so it
// is never all-ones (k = 96 fills it and does not use the set).
struct ListCols {
  const uint64_t* p[4];
};
template <int NL>
__global__ void __launch_bounds__(kBlock) k_solid_set(ListCols L, const uint32_t* __restrict__ cnt, uint64_t n,
                                                       const uint32_t* __restrict__ thr, unsigned k,
                                                       SetView sv) {
  const uint32_t cutoff = thr[0];
  const uint64_t mask = (1ULL << sv.log2cap) - 1;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    if (cnt[i] < cutoff) continue;
    Seq<NL> C;
#pragma unroll
    for (int j = 0; j < NL; j++) C.v[j] = L.p[j][i];
    uint64_t w4[4];
    kmer256_limbs<NL>(C, k, w4);
    const uint64_t raw0 = hash_seed(hash_pre(w4), kSeed1);
    const uint64_t fb = filter_bit(sv, raw0);
    atomicOr(sv.filter + (fb >> 5), 1u << (fb & 31));
    uint64_t h = raw0 >> (64 - sv.log2cap);
    // keys are distinct and the set is at most 2/3 full, so a free slot is found
    for (uint64_t probe = 0; probe <= mask; probe++, h = (h + 1) & mask) {
      if constexpr (NL == 1) {
        if (atomicCAS((unsigned long long*)sv.keys + h, kEmpty, (unsigned long long)C.v[0]) == kEmpty)
          break;
      } else if constexpr (NL == 2) {
        const U128 old = atomicCAS((U128*)sv.keys + h, U128{kEmpty, kEmpty}, U128{C.v[0], C.v[NL - 1]});
        if (old.x == kEmpty && old.y == kEmpty) break;
      } else {
        uint64_t* kp = sv.keys + (uint64_t)NL * h;
        if (atomicCAS((unsigned long long*)(kp + NL - 1), kEmpty, (unsigned long long)C.v[NL - 1]) == kEmpty) {
#pragma unroll
          for (int j = 0; j < NL - 1; j++) kp[j] = C.v[j];
          break;
        }
      }
    }
  }
}

template <int NL>
__device__ __forceinline__ bool set_has(const SetView& sv, const Seq<NL>& C, uint64_t raw0) {
  const uint64_t fb = filter_bit(sv, raw0);
  if (!((__ldg(sv.filter + (fb >> 5)) >> (fb & 31)) & 1u)) return false;
  const uint64_t mask = (1ULL << sv.log2cap) - 1;
  uint64_t h = raw0 >> (64 - sv.log2cap);
  for (uint64_t probe = 0; probe <= mask; probe++, h = (h + 1) & mask) {
    if constexpr (NL == 1) {
      const uint64_t v = __ldg(sv.keys + h);
      if (v == C.v[0]) return true;
      if (v == kEmpty) return false;
    } else if constexpr (NL == 2) {
      const ulonglong2 v = __ldg((const ulonglong2*)sv.keys + h);
      if (v.x == C.v[0] && v.y == C.v[NL - 1]) return true;
      if (v.x == kEmpty && v.y == kEmpty) return false;
    } else {
      const uint64_t* kp = sv.keys + (uint64_t)NL * h;
      const uint64_t top = __ldg(kp + NL - 1);
      if (top == kEmpty) return false;
      bool eq = top == C.v[NL - 1];
#pragma unroll
      for (int j = 0; j < NL - 1; j++) eq &= __ldg(kp + j) == C.v[j];
      if (eq) return true;
    }
  }
  return false;
}

template <int NL, int NLE, bool SET>
__global__ void __launch_bounds__(kBlock) k_edges(const uint64_t* l0, const uint64_t* l1,
                                                   const uint64_t* l2, const uint64_t* l3,
                                                   const uint32_t* __restrict__ cnt, uint64_t n,
                                                   const uint32_t* __restrict__ thr, TableView t,
                                                   SetView sv, unsigned k, uint64_t* e0, uint64_t* e1,
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
    uint32_t emits = 0;  // bit 4o + b: the edge of orientation o and base b
    Seq<NL> RS;
    if (solid) RS = revcomp<NL>(S, k);
    for (int o = 0; o < 2; o++) {
      // the oriented k-mer and its reverse complement
      const Seq<NL> EX = o ? RS : S;
      const Seq<NL> RX = o ? S : RS;
      bool ok = solid;
      if (o == 1 && ok) ok = !seq_eq<NL>(RS, S);  // a palindromic k-mer (even k) has one orientation
      for (unsigned b = 0; b < 4; b++) {
        bool emit = false;
        if (ok) {
          const Seq<NL> NB = shl_append<NL>(EX, b, k);
          const Seq<NL> RB = shr_prepend<NL>(RX, 3u - b, k);
          const Seq<NL> CN = seq_le<NL>(NB, RB) ? NB : RB;  // canonical, src/dna.rs:185-192
          uint64_t w4[4];
          kmer256_limbs<NL>(CN, k, w4);
          const HashPre hp = hash_pre(w4);
          const uint64_t raw0 = hash_seed(hp, kSeed1);
          bool solid_nb;
          if (SET) {
            solid_nb = set_has<NL>(sv, CN, raw0);
          } else {
            const uint32_t c = table_find<NL>(t, CN, table_home(t, raw0));
            solid_nb = c && !(c & kRejected) && c >= cutoff;
          }
          if (solid_nb) {
            const Seq<NLE> E = widen_append<NL, NLE>(EX, b);
            emit = seq_le<NLE>(E, prepend_wide<NL, NLE>(RX, 3u - b, k));
          }
        }
        if (emit) emits |= 1u << (4 * o + b);
      }
    }
    // One reservation per warp for all its edges, then write them (the
    // edge (k+1)-mer is rebuilt from the oriented k-mer and the base).
    const uint32_t ne = __popc(emits);
    uint32_t incl = ne;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t v = __shfl_up_sync(FULL, incl, d);
      if ((int)lane >= d) incl += v;
    }
    const uint32_t wtot = __shfl_sync(FULL, incl, 31);
    if (!wtot) continue;
    unsigned long long wb = 0;
    if (lane == 0) wb = atomicAdd(counter, (unsigned long long)wtot);
    uint64_t p = __shfl_sync(FULL, wb, 0) + incl - ne;
    for (int o = 0; o < 2; o++) {
      if (!(emits >> (4 * o) & 15u)) continue;
      const Seq<NL> EX = o ? revcomp<NL>(S, k) : S;
      for (unsigned b = 0; b < 4; b++) {
        if (!(emits >> (4 * o + b) & 1u)) continue;
        const Seq<NLE> E = widen_append<NL, NLE>(EX, b);
        if (p < out_cap) {
          e0[p] = E.v[0];
          if (NLE > 1) e1[p] = E.v[NLE > 1 ? 1 : 0];
          if (NLE > 2) e2[p] = E.v[NLE > 2 ? 2 : 0];
          if (NLE > 3) e3[p] = E.v[NLE > 3 ? 3 : 0];
        }
        p++;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Prior and trusted contigs (src/assemble.rs:267-283): every k-window of a
// contig that Kmer256::from_bytes accepts (every byte A/C/G/T in either case,
// src/dna.rs:11-37, 299-321) adds `boost` to its canonical k-mer.  Runs after
// singleton admission: a singleton the Bloom rejected is not in the
// reference's map, so its count restarts from the boost; a k-mer the table
// lacks is inserted with it.  One warp per contig, lanes over its windows.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int ascii_base(uint8_t c) {
  switch (c) {
    case 'A': case 'a': return 0;
    case 'C': case 'c': return 1;
    case 'G': case 'g': return 2;
    case 'T': case 't': return 3;
    default: return -1;
  }
}

// The slot holding key C (probe sequence from home), or ~0 if absent.
template <int NL>
__device__ __forceinline__ uint64_t table_slot_of(const TableView& t, const Seq<NL>& C, uint64_t home) {
  for (uint32_t i = 0; i < t.max_probe; i++) {
    const uint64_t s = probe_slot(t, home, i);
    const uint32_t c = *(volatile uint32_t*)slot_count<NL>(t, s);
    if (c == 0) return ~0ULL;  // an empty slot ends the probe sequence
    const volatile uint64_t* kp = slot_key<NL>(t, s);
    bool eq = true;
#pragma unroll
    for (int j = 0; j < NL; j++) eq &= kp[j] == C.v[j];
    if (eq) return s;
  }
  return ~0ULL;
}

template <int NL>
__global__ void __launch_bounds__(kBlock) k_prior_inject(const uint8_t* __restrict__ seqs,
                                                          const uint64_t* __restrict__ offs,
                                                          const uint32_t* __restrict__ lens, uint64_t n,
                                                          unsigned k, uint32_t boost, TableView t) {
  const unsigned lane = threadIdx.x & 31;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t c = warp; c < n; c += nwarps) {
    const uint8_t* sq = seqs + offs[c];
    const uint32_t L = lens[c];
    if (L < k) continue;  // src/assemble.rs:273-275
    for (uint32_t i = lane; i + k <= L; i += 32) {
      Seq<NL> V;
#pragma unroll
      for (int j = 0; j < NL; j++) V.v[j] = 0;
      bool ok = true;
      for (unsigned j = 0; j < k && ok; j++) {
        const int b = ascii_base(sq[i + j]);
        if (b < 0) ok = false;
        else V = shl_append<NL>(V, (unsigned)b, k);
      }
      if (!ok) continue;
      const Seq<NL> C = canonical<NL>(V, k);
      uint64_t w4[4];
      kmer256_limbs<NL>(C, k, w4);
      const uint64_t home = table_home(t, hash_seed(hash_pre(w4), kSeed1));
      const uint64_t s = table_slot_of<NL>(t, C, home);
      if (s == ~0ULL) {
        table_add<NL>(t, C, home, boost);  // absent: inserted with the boost
        continue;
      }
      uint32_t* cp = slot_count<NL>(t, s);
      uint32_t cur = *(volatile uint32_t*)cp;
      for (;;) {
        const uint32_t nv = (cur & kRejected) ? boost : cur + boost;
        const uint32_t old = atomicCAS(cp, cur, nv);
        if (old == cur) break;
        cur = old;
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

// flag = 1 if some read starts before the end of the read before it (the
// chunked upload then cannot hand reads to the first pass piece by piece).
__global__ void __launch_bounds__(kBlock) k_read_order(const uint64_t* __restrict__ offsets,
                                                      const uint32_t* __restrict__ lengths, uint64_t n,
                                                      unsigned long long* __restrict__ flag) {
  bool bad = false;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i + 1 < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    bad |= offsets[i] + (lengths[i] + 3ull) / 4 > offsets[i + 1];
  if (__any_sync(FULL, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1ull);
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
static int grid_for(spk_ctx* ctx, int blocks_per_sm) { return ctx->sm_count * blocks_per_sm; }

// F<NL>(args...) for the key width nl at run time (F returns a status).
#define SPK_NL_CALL(nl, F, ...)                                                              \
  ((nl) == 1 ? F<1>(__VA_ARGS__) : (nl) == 2 ? F<2>(__VA_ARGS__) : (nl) == 3 ? F<3>(__VA_ARGS__) \
                                                                             : F<4>(__VA_ARGS__))

#define SPK_DISPATCH_NL(nl, F, ...)                 \
  switch (nl) {                                     \
    case 1: F<1>(__VA_ARGS__); break;               \
    case 2: F<2>(__VA_ARGS__); break;               \
    case 3: F<3>(__VA_ARGS__); break;               \
    default: F<4>(__VA_ARGS__); break;              \
  }

template <int NL>
static void launch_admit_singletons(spk_ctx* ctx, cudaStream_t st, const ListOut& lo, unsigned k,
                                    const FastMod& fm, const uint64_t* twice, unsigned long long* sums) {
  k_admit_singletons<NL><<<grid_for(ctx, 8), kBlock, 0, st>>>(lo, k, fm, twice, sums);
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
static void launch_part_scatter(spk_ctx* ctx, cudaStream_t st, const ReadsView& rv, unsigned k,
                                const PartView& pv, unsigned long long* occ) {
  k_part_scatter<NL><<<grid_for(ctx, 8), kBlock, 0, st>>>(rv, k, pv, occ);
}
#ifndef SPK_TWO_LEVEL
#define SPK_TWO_LEVEL 1
#endif
template <int NL>
static int launch_part_coarse(spk_ctx* ctx, cudaStream_t st, const ReadsView& rv, unsigned k,
                              const PartView& pv, const CoarseView& cv, unsigned long long* occ) {
  const size_t smem = coarse_smem<NL>();
  int rc;
  if ((rc = raise_smem_limit((const void*)k_part_coarse<NL>, smem))) return rc;
  k_part_coarse<NL><<<grid_for(ctx, 2), kCoarseBlock, smem, st>>>(rv, k, pv, cv, occ);
  return SPK_OK;
}
template <int NL>
static int launch_part_fine(spk_ctx* ctx, cudaStream_t st, const CoarseView& cv, const uint32_t* cfirst,
                            const PartView& pv, unsigned k) {
  const size_t smem = fine_smem<NL>(1u << (pv.log2parts - pv.log2groups - kCoarseBits));
  int rc;
  if ((rc = raise_smem_limit((const void*)k_part_fine<NL>, smem))) return rc;
  k_part_fine<NL><<<grid_for(ctx, 2), kFineBlock, smem, st>>>(cv, cfirst, pv, k);
  return SPK_OK;
}
// rv.ops == nullptr: apply the Bloom operations to the interleaved tiers
// directly; else bin them by range into rv.
template <int NL>
static int launch_part_count(spk_ctx* ctx, cudaStream_t st, const PartView& pv, const TableView& t,
                             unsigned k, const FastMod& fm, U128* tiers, const RangeView& rv,
                             const ListOut& lo) {
  size_t smem = ((size_t)1 << t.log2span) * (sizeof(typename SpanKey<NL>::T) + 4);
  const uint64_t nparts = 1ULL << (pv.log2parts - pv.log2groups);
  const int grid = (int)std::min<uint64_t>(nparts, (uint64_t)ctx->sm_count * kPartCtasPerSm);
  if (rv.ops) {
    smem += ((rv.nranges + 1) & ~1u) * 4 + (size_t)rv.nranges * 8;
    if (NL >= 2 && kSortedOps) smem += ((rv.nranges + 1) & ~1u) * 4;  // range cursors
    int rc;
    if ((rc = raise_smem_limit((const void*)k_part_count<NL, true>, smem))) return rc;
    k_part_count<NL, true><<<grid, kPartBlock, smem, st>>>(pv, t, k, fm, tiers, rv, lo);
  } else if constexpr (NL <= 2) {
    int rc;
    if ((rc = raise_smem_limit((const void*)k_part_count<NL, false>, smem))) return rc;
    ListOut none{};  // the in-place Bloom form writes the table
    k_part_count<NL, false><<<grid, kPartBlock, smem, st>>>(pv, t, k, fm, tiers, rv, none);
  } else {
    return fail(SPK_E_INVALID_ARG, "k > 64 counts spans in list mode only");
  }
  return SPK_OK;
}
static int launch_bloom_apply(spk_ctx* ctx, cudaStream_t st, const RangeView& rv, uint64_t num_words,
                              uint64_t* seen, uint64_t* twice, unsigned long long* pops) {
  const size_t smem = (size_t)2 * ((1u << kLog2Range) / 32) * 4;
  int rc;
  if ((rc = raise_smem_limit((const void*)k_bloom_apply, smem))) return rc;
  const int grid = (int)std::min<uint64_t>(rv.nranges, (uint64_t)ctx->sm_count);
  k_bloom_apply<<<grid, kApplyBlock, smem, st>>>(rv, num_words, seen, twice, pops);
  return SPK_OK;
}
// Spans of the partitioned schedule: 8192 slots of 12 bytes (k <= 32), 4096
// of 20 bytes (k <= 64) or 2048 of 28 / 36 bytes (k <= 96 / 127) in shared
// memory, two CTAs per SM.
#ifndef SPK_PART_LOG2SPAN1
#define SPK_PART_LOG2SPAN1 13
#endif
#ifndef SPK_PART_LOG2SPAN2
#define SPK_PART_LOG2SPAN2 12
#endif
constexpr uint32_t kPartLog2Span1 = SPK_PART_LOG2SPAN1, kPartLog2Span2 = SPK_PART_LOG2SPAN2;
constexpr uint32_t kPartLog2SpanWide = 11;
static uint32_t part_log2span(int nl) {
  return nl == 1 ? kPartLog2Span1 : nl == 2 ? kPartLog2Span2 : kPartLog2SpanWide;
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
                         unsigned long long* sums, unsigned long long* rejected) {
  k_admit_compact<NL><<<grid_for(ctx, 8), kBlock, 0, st>>>(t, k, fm, twice, check, lmin, o[0], o[1],
                                                          o[2], o[3], oc, out_cap, hist, sums,
                                                          rejected);
}
template <int NL, int NLE>
static void launch_edges_t(spk_ctx* ctx, cudaStream_t st, uint64_t* l[4], const uint32_t* cnt,
                           uint64_t n, const uint32_t* thr, const TableView& t, const SetView* sv,
                           unsigned k, uint64_t* e[4], uint64_t out_cap,
                           unsigned long long* counter) {
  if (sv)
    k_edges<NL, NLE, true><<<grid_for(ctx, 8), kBlock, 0, st>>>(
        l[0], l[1], l[2], l[3], cnt, n, thr, t, *sv, k, e[0], e[1], e[2], e[3], out_cap, counter);
  else
    k_edges<NL, NLE, false><<<grid_for(ctx, 8), kBlock, 0, st>>>(
        l[0], l[1], l[2], l[3], cnt, n, thr, t, SetView{nullptr, 0, 0, nullptr}, k, e[0], e[1], e[2], e[3],
        out_cap, counter);
}
// sv: the solid set, or nullptr to probe the count table.
static void launch_edges(spk_ctx* ctx, cudaStream_t st, int nl, int nle, uint64_t* l[4],
                         const uint32_t* cnt, uint64_t n, const uint32_t* thr, const TableView& t,
                         const SetView* sv, unsigned k, uint64_t* e[4], uint64_t out_cap,
                         unsigned long long* counter) {
  if (nl == 1 && nle == 1) launch_edges_t<1, 1>(ctx, st, l, cnt, n, thr, t, sv, k, e, out_cap, counter);
  else if (nl == 1) launch_edges_t<1, 2>(ctx, st, l, cnt, n, thr, t, sv, k, e, out_cap, counter);
  else if (nl == 2 && nle == 2) launch_edges_t<2, 2>(ctx, st, l, cnt, n, thr, t, sv, k, e, out_cap, counter);
  else if (nl == 2) launch_edges_t<2, 3>(ctx, st, l, cnt, n, thr, t, sv, k, e, out_cap, counter);
  else if (nl == 3 && nle == 3) launch_edges_t<3, 3>(ctx, st, l, cnt, n, thr, t, sv, k, e, out_cap, counter);
  else if (nl == 3) launch_edges_t<3, 4>(ctx, st, l, cnt, n, thr, t, sv, k, e, out_cap, counter);
  else launch_edges_t<4, 4>(ctx, st, l, cnt, n, thr, t, sv, k, e, out_cap, counter);
}
static void launch_solid_set(spk_ctx* ctx, cudaStream_t st, int nl, uint64_t* const l[4], const uint32_t* cnt,
                             uint64_t n, const uint32_t* thr, unsigned k, const SetView& sv) {
  const ListCols L{{l[0], l[1], l[2], l[3]}};
  const int g = grid_for(ctx, 8);
  switch (nl) {
    case 1: k_solid_set<1><<<g, kBlock, 0, st>>>(L, cnt, n, thr, k, sv); break;
    case 2: k_solid_set<2><<<g, kBlock, 0, st>>>(L, cnt, n, thr, k, sv); break;
    case 3: k_solid_set<3><<<g, kBlock, 0, st>>>(L, cnt, n, thr, k, sv); break;
    default: k_solid_set<4><<<g, kBlock, 0, st>>>(L, cnt, n, thr, k, sv); break;
  }
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
// Slots of the span count: the distinct share of the occurrences grows with
// k (a read has fewer windows, a sequencing error makes more new k-mers),
// from 0.11 at k = 21 to 0.27 at k = 55, 0.36 at k = 77, 0.44 at k = 99 and
// 0.56 at k = 127 on 150 bp reads at 100x with 1% errors.
static uint64_t list_capacity(uint64_t occ, int nl) {
  return nl <= 2 ? fused_capacity(occ) : std::max<uint64_t>(next_pow2(occ * 9 / 20 + 1), 1024);
}

struct Ev {
  cudaEvent_t e = nullptr;
  Ev() : e(pooled_event(true)) {}
  ~Ev() { pooled_event_put(e, true); }
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

// A table of cap slots (a power of two) probed within spans of 2^log2span
// slots (0: the whole table).  init = false leaves the slots unwritten for a
// pass that writes every slot itself.
static int alloc_table(spk_ctx* ctx, KResult& kr, cudaStream_t st, uint64_t cap,
                       uint32_t log2span = 0, bool init = true, bool with_slots = true) {
  const uint32_t sb = slot_bytes(kr.nl);
  int rc;
  if (!with_slots) kr.tslots.release();
  else if ((rc = kr.tslots.alloc(cap * sb, st))) return rc;
  if (init && with_slots) {
    SPK_DISPATCH_NL(kr.nl, launch_init, ctx, st, kr.tslots.as<uint8_t>(), cap);
    SPK_CUDA(cudaGetLastError());
  }
  TableView& t = kr.table;
  t.slots = kr.tslots.as<uint8_t>();
  t.capacity = cap;
  t.log2cap = 0;
  while ((1ULL << t.log2cap) < cap) t.log2cap++;
  t.log2span = (log2span && log2span < t.log2cap) ? log2span : t.log2cap;
  t.slot_bytes = sb;
  t.max_probe = (uint32_t)std::min<uint64_t>(kMaxProbe, 1ULL << t.log2span);
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
  S_REJ = 12,            /* singletons the twice tier rejected */
  S_LFILL = 13,          /* 2 words: list entries, singletons (span count to the list) */
  S_OCC2 = 15,           /* occurrences of the k-mers counted at least twice */
  S_HIST = 16,           /* 256 words */
  S_WORDS = 16 + kHistBins
};

// The span count's list output over kr's list buffers and the singleton key
// buffers sgl (kr.nl limbs each), with the fills and histogram in scratch.
static ListOut list_out(KResult& kr, DevBuf* sgl, uint64_t lcap, uint64_t scap, uint32_t lmin,
                        unsigned long long* su) {
  ListOut lo{};
  for (int j = 0; j < kr.nl; j++) {
    lo.l[j] = kr.list[j].as<uint64_t>();
    lo.s[j] = sgl[j].as<uint64_t>();
  }
  lo.cnt = kr.list[4].as<uint32_t>();
  lo.cap = lcap;
  lo.scap = scap;
  lo.lmin = lmin;
  lo.fill = su + S_LFILL;
  lo.hist = su + S_HIST;
  lo.occ2 = su + S_OCC2;
  return lo;
}

// What a finished job keeps: the list and edge buffers cut to what they hold
// (they were sized by bounds: table slots, eight edges per solid k-mer), and
// the count table only when SPK_F_KEEP_TABLE asks for it.  Results stay
// resident (serving, batches), so their size decides how many fit.
static int shrink_to(DevBuf& b, uint64_t used, cudaStream_t st) {
  used = std::max<uint64_t>(used, 16);
  if (!b.p || b.bytes <= used + used / 4 + (1u << 20)) return SPK_OK;
  DevBuf n;
  int rc;
  if ((rc = n.alloc_keep(used, st))) return rc;
  SPK_CUDA(cudaMemcpyAsync(n.p, b.p, used, cudaMemcpyDeviceToDevice, st));
  b = std::move(n);  // the old buffer is freed after the copy, in stream order
  return SPK_OK;
}
static int keep_results(KResult& kr, cudaStream_t st, uint32_t flags) {
  int rc;
  for (int j = 0; j < kr.nl; j++)
    if ((rc = shrink_to(kr.list[j], kr.list_len * 8, st))) return rc;
  if ((rc = shrink_to(kr.list[4], kr.list_len * 4, st))) return rc;
  for (int j = 0; j < kr.nle; j++)
    if ((rc = shrink_to(kr.edges[j], kr.info.n_edges * 8, st))) return rc;
  if (!(flags & SPK_F_KEEP_TABLE)) {
    kr.tslots.release();
    kr.table.slots = nullptr;
  }
  return SPK_OK;
}

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
  const bool correct = (o.flags & SPK_F_CORRECT) != 0;
  const bool gated = (o.flags & SPK_F_GATED) != 0 || correct;
  // The reference-semantics solid tier depends on the order of the inserts,
  // so it needs the per-occurrence Bloom of the fused pass.
  const bool count_first = !gated && !ref;
  bool partitioned = count_first && nl <= 2 && !(o.flags & SPK_F_DIRECT);
  const bool priors = o.n_prior > 0 && o.prior_seqs && o.prior_offsets && o.prior_lengths;
  // The partitioned span count writes the k-mer list itself unless the count
  // table is asked for (its view, or prior contigs that update it).
  const bool table_wanted = priors || (o.flags & SPK_F_KEEP_TABLE);
  // Thresholds of the list (src/assemble.rs:286-292, 693-694).
  uint32_t fixed = o.min_count;
  if (!fixed && o.min_coverage > 5.0) {
    double v = std::max(o.min_coverage * 0.35, 2.0);
    fixed = v >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)v;
  }
  const uint32_t list_min = o.list_min_count ? o.list_min_count : 2;
  // The list keeps counts >= min(cutoff, list_min).  The adaptive cutoff is
  // never below 2, so compacting counts >= min(2 or the fixed cutoff,
  // list_min) keeps a superset; the exact threshold filters downloads.
  const uint32_t lmin_pre = std::max(1u, std::min(fixed ? fixed : 2u, list_min));

  Ev e0, e1, e2, e3, e4, e5, e6, kb0, kb1, kc0, kc1, ks0, ks1, ec0, ec1;
  uint32_t launches = 0;
  SPK_CUDA(cudaEventRecord(e0.e, st));

  // Bloom tiers as interleaved (seen, twice) word pairs, for the schedules
  // that update them in place (allocated on first use).
  if (ref && (rc = kr.ref_solid.alloc(kr.num_words * 8, st))) return rc;
  U128* tiers = nullptr;
  unsigned long long* refp = ref ? kr.ref_solid.as<unsigned long long>() : nullptr;
  auto reset_tiers = [&]() -> int {
    int r2;
    if (!kr.tiers.p && (r2 = kr.tiers.alloc(kr.num_words * 16, st))) return r2;
    tiers = kr.tiers.as<U128>();
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
    if ((int)host[S_ERR] & (int)kErrStage) return fail(SPK_E_TIMEOUT, "partition: a staged copy never completed");
    return SPK_OK;
  };

  uint64_t cap = 0;
  // Partitioned schedule: Bloom operations binned by range when the ranges'
  // bins fit in shared memory (else applied in place, as k_bloom_from_table).
  const uint64_t nranges = (size_bits + (1ULL << kLog2Range) - 1) >> kLog2Range;
  const bool use_ops = nranges <= kMaxRanges;
  DevBuf rbase, rfill, ops;
  RangeView bv{nullptr, nullptr, nullptr, 0, (uint32_t)nranges, errp};
  bool list_mode = false;  // the span count wrote the list (no table)
  ListOut lo{};
  DevBuf sgl[4];           // list mode: keys of the k-mers counted once
  if (!gated) {
    // ---- fused: Bloom and the count of every k-mer in one pass ----
    k_occ<<<grid_for(ctx, 2), kBlock, 0, st>>>(rv.lengths, rv.n_reads, k, su + S_OCC0);
    SPK_CUDA(cudaGetLastError());
    launches++;
    if ((rc = fetch(S_OCC0 + 1))) return rc;
    const uint64_t occ0 = host[S_OCC0];
    cap = o.table_log2 ? (1ULL << std::min<uint32_t>(o.table_log2, 40)) : list_capacity(occ0, nl);
    bool two_level_fits = false;
    if (partitioned) {
      // Regions hold 1.5x the mean share of occurrences per span: keep them
      // within a quarter of the device memory, else count with global atomics.
      // The two-level pass also holds the coarse buckets (1.125x) meanwhile.
      const uint64_t tot = ctx->total_mem;
      partitioned = (occ0 + (occ0 >> 1) + (1u << 20)) * (uint64_t)nl * 8 <= tot / 4;
      two_level_fits = (occ0 * 3 + (1u << 22)) * (uint64_t)nl * 8 <= tot / 4;
    }
    for (int attempt = 0; partitioned; attempt++) {
      if (!use_ops && (rc = reset_tiers())) return rc;
      list_mode = use_ops && !table_wanted;
      if ((rc = alloc_table(ctx, kr, st, cap, nl == 1 ? kPartLog2Span1 : kPartLog2Span2, false,
                            !list_mode)))
        return rc;
      lo = ListOut{};
      if (list_mode) {
        // the list (entries counted >= lmin times) and the singleton keys,
        // each at most one entry per table slot
        for (int j = 0; j < nl; j++)
          if ((rc = kr.list[j].alloc(cap * 8, st)) || (rc = sgl[j].alloc(cap * 8, st))) return rc;
        if ((rc = kr.list[4].alloc(cap * 4, st))) return rc;
        SPK_CUDA(cudaMemsetAsync(sw + S_LFILL, 0, 3 * 8, st));  // fills and S_OCC2
        SPK_CUDA(cudaMemsetAsync(sw + S_HIST, 0, kHistBins * 8, st));
        lo = list_out(kr, sgl, cap, cap, lmin_pre, su);
      }
      TableView& t = kr.table;
      t.err = errp;
      SPK_CUDA(cudaMemsetAsync(sw, 0, (S_ERR + 1) * 8, st));
      const uint32_t log2parts = t.log2cap - t.log2span;
      const uint64_t nparts = 1ULL << log2parts;
      DevBuf base, fill, region;
      if ((rc = base.alloc((nparts + 1) * 8, st)) || (rc = fill.alloc(nparts * 4 * kFillStride, st)))
        return rc;
      const uint64_t per = occ0 / nparts;
      const uint64_t capu = per + (per >> 1) + 256;
      if ((rc = region.alloc(nparts * capu * nl * 8, st))) return rc;
      k_part_uniform<<<64, kBlock, 0, st>>>((uint32_t)nparts, capu, base.as<uint64_t>());
      SPK_CUDA(cudaMemsetAsync(fill.p, 0, nparts * 4 * kFillStride, st));
      PartView pv{region.as<uint64_t>(), base.as<uint64_t>(), fill.as<unsigned int>(), capu, log2parts,
                  home_fits(k, nl) ? 1u : 0u, errp};
      SPK_CUDA(cudaEventRecord(ks0.e, st));
      const bool two_level = SPK_TWO_LEVEL && two_level_fits && log2parts > kCoarseBits &&
                             log2parts - kCoarseBits <= kFineMaxBits;
      info.part_passes = two_level ? 2 : 1;
      if (two_level) {
        // ---- coarse buckets, then spans (k_part_coarse, k_part_fine) ----
        DevBuf cbase, cfill, cregion, cfirst;
        const uint64_t cper = occ0 / kCoarse;
        const uint64_t ccap = (cper + (cper >> 3) + 8192 + 1) & ~1ULL;  // even: chunks start 16-byte aligned
        if ((rc = cbase.alloc((kCoarse + 1) * 8, st)) || (rc = cfill.alloc(kCoarse * 4 * kFillStride, st)) ||
            (rc = cregion.alloc(kCoarse * ccap * nl * 8, st)) || (rc = cfirst.alloc((kCoarse + 1) * 4, st)))
          return rc;
        k_part_uniform<<<1, 128, 0, st>>>(kCoarse, ccap, cbase.as<uint64_t>());
        SPK_CUDA(cudaMemsetAsync(cfill.p, 0, kCoarse * 4 * kFillStride, st));
        CoarseView cv{cregion.as<uint64_t>(), cbase.as<uint64_t>(), cfill.as<unsigned int>(), ccap, errp};
        if (nl == 1) rc = launch_part_coarse<1>(ctx, st, rv, k, pv, cv, su + S_OCC);
        else rc = launch_part_coarse<2>(ctx, st, rv, k, pv, cv, su + S_OCC);
        if (rc) return rc;
        SPK_CUDA(cudaGetLastError());
        launches += 2;  // k_part_uniform, k_part_coarse
        if ((rc = fetch(S_ERR + 1))) return rc;
        if ((int)host[S_ERR] & kErrRegion) {
          // A bucket outgrew its share: exact buckets from the fill counts.
          k_part_bases<<<1, 1024, 0, st>>>(cfill.as<unsigned int>(), kCoarse, cbase.as<uint64_t>());
          SPK_CUDA(cudaMemcpyAsync(host + S_WORDS, cbase.as<uint64_t>() + kCoarse, 8, cudaMemcpyDeviceToHost, st));
          SPK_CUDA(cudaStreamSynchronize(st));
          if ((rc = cregion.alloc(std::max<uint64_t>(host[S_WORDS], 1) * nl * 8, st))) return rc;
          cv.keys = cregion.as<uint64_t>();
          cv.uniform = 0;
          SPK_CUDA(cudaMemsetAsync(cfill.p, 0, kCoarse * 4 * kFillStride, st));
          SPK_CUDA(cudaMemsetAsync(sw, 0, (S_ERR + 1) * 8, st));
          if (nl == 1) rc = launch_part_coarse<1>(ctx, st, rv, k, pv, cv, su + S_OCC);
          else rc = launch_part_coarse<2>(ctx, st, rv, k, pv, cv, su + S_OCC);
          if (rc) return rc;
          SPK_CUDA(cudaGetLastError());
          launches += 2;
          info.part_rescatters++;
          if ((rc = fetch(S_ERR + 1))) return rc;
          if ((int)host[S_ERR] & kErrRegion) return fail(SPK_E_CUDA, "coarse bucket overflow after resizing");
        }
        k_coarse_chunks<<<1, 32, 0, st>>>(cv, fine_chunk<2>(), cfirst.as<uint32_t>());
        if (nl == 1) rc = launch_part_fine<1>(ctx, st, cv, cfirst.as<uint32_t>(), pv, k);
        else rc = launch_part_fine<2>(ctx, st, cv, cfirst.as<uint32_t>(), pv, k);
        if (rc) return rc;
        SPK_CUDA(cudaGetLastError());
        launches += 2;  // k_coarse_chunks, k_part_fine
        if ((rc = fetch(S_ERR + 1))) return rc;
        if ((int)host[S_ERR] & kErrRegion) {
          // Skewed spans: exact regions from the span fill counts, fine pass again.
          k_part_bases<<<1, 1024, 0, st>>>(fill.as<unsigned int>(), (uint32_t)nparts, base.as<uint64_t>());
          SPK_CUDA(cudaMemcpyAsync(host + S_WORDS, base.as<uint64_t>() + nparts, 8, cudaMemcpyDeviceToHost, st));
          SPK_CUDA(cudaStreamSynchronize(st));
          if ((rc = region.alloc(std::max<uint64_t>(host[S_WORDS], 1) * nl * 8, st))) return rc;
          pv.keys = region.as<uint64_t>();
          pv.uniform = 0;
          SPK_CUDA(cudaMemsetAsync(fill.p, 0, nparts * 4 * kFillStride, st));
          SPK_CUDA(cudaMemsetAsync(errp, 0, 4, st));
          if (nl == 1) rc = launch_part_fine<1>(ctx, st, cv, cfirst.as<uint32_t>(), pv, k);
          else rc = launch_part_fine<2>(ctx, st, cv, cfirst.as<uint32_t>(), pv, k);
          if (rc) return rc;
          SPK_CUDA(cudaGetLastError());
          launches += 2;
          info.part_rescatters++;
          if ((rc = fetch(S_ERR + 1))) return rc;
          if ((int)host[S_ERR] & kErrRegion) return fail(SPK_E_CUDA, "span region overflow after resizing");
        }
      } else {
      if (nl == 1) launch_part_scatter<1>(ctx, st, rv, k, pv, su + S_OCC);
      else launch_part_scatter<2>(ctx, st, rv, k, pv, su + S_OCC);
      SPK_CUDA(cudaGetLastError());
      launches += 2;  // k_part_uniform, k_part_scatter
      if ((rc = fetch(S_ERR + 1))) return rc;
      if ((int)host[S_ERR] & kErrRegion) {
        // Skewed spans: the fill counters are the exact sizes.  Lay the
        // regions out by them and scatter again (this cannot overflow).
        k_part_bases<<<1, 1024, 0, st>>>(fill.as<unsigned int>(), (uint32_t)nparts, base.as<uint64_t>());
        SPK_CUDA(cudaMemcpyAsync(host + S_WORDS, base.as<uint64_t>() + nparts, 8,
                                 cudaMemcpyDeviceToHost, st));
        SPK_CUDA(cudaStreamSynchronize(st));
        if ((rc = region.alloc(std::max<uint64_t>(host[S_WORDS], 1) * nl * 8, st))) return rc;
        pv.keys = region.as<uint64_t>();
        pv.uniform = 0;
        SPK_CUDA(cudaMemsetAsync(fill.p, 0, nparts * 4 * kFillStride, st));
        SPK_CUDA(cudaMemsetAsync(sw, 0, (S_ERR + 1) * 8, st));
        if (nl == 1) launch_part_scatter<1>(ctx, st, rv, k, pv, su + S_OCC);
        else launch_part_scatter<2>(ctx, st, rv, k, pv, su + S_OCC);
        SPK_CUDA(cudaGetLastError());
        launches += 2;  // k_part_bases, k_part_scatter
        info.part_rescatters++;
      }
      }
      SPK_CUDA(cudaEventRecord(ks1.e, st));
      if (use_ops) {
        // At most three operations per table slot; each range gets 1.25x its
        // share of that bound (Bloom positions are uniform over the ranges).
        const uint64_t share = 3 * cap / nranges + 1;
        const uint64_t rcap = share + (share >> 2) + 1024;
        if ((rc = rbase.alloc((nranges + 1) * 8, st)) ||
            (rc = rfill.alloc(nranges * 4 * kFillStride, st)) || (rc = ops.alloc(nranges * rcap * 4, st)))
          return rc;
        SPK_CUDA(cudaMemsetAsync(rfill.p, 0, nranges * 4 * kFillStride, st));
        bv = RangeView{ops.as<uint32_t>(), rbase.as<uint64_t>(), rfill.as<unsigned int>(), rcap,
                       (uint32_t)nranges, errp};
      }
      SPK_CUDA(cudaEventRecord(kc0.e, st));
      if (nl == 1) rc = launch_part_count<1>(ctx, st, pv, t, k, kr.fm, tiers, bv, lo);
      else rc = launch_part_count<2>(ctx, st, pv, t, k, kr.fm, tiers, bv, lo);
      if (rc) return rc;
      SPK_CUDA(cudaGetLastError());
      SPK_CUDA(cudaEventRecord(kc1.e, st));
      launches++;
      if ((rc = fetch(S_ERR + 1))) return rc;
      if ((int)host[S_ERR] & kErrRegion) return fail(SPK_E_CUDA, "partition region overflow after resizing");
      if ((int)host[S_ERR] & 1) {
        if (attempt >= 24) return fail(SPK_E_TABLE_FULL, "count table overflow after regrow attempts");
        cap *= 2;
        info.table_regrows++;
        continue;
      }
      if (use_ops && ((int)host[S_ERR] & kErrRange)) {
        // A range outgrew its share: lay the ranges out by their exact
        // counts and count the spans again (the table comes out the same).
        k_part_bases<<<1, 1024, 0, st>>>(rfill.as<unsigned int>(), (uint32_t)nranges,
                                         rbase.as<uint64_t>());
        SPK_CUDA(cudaMemcpyAsync(host + S_WORDS, rbase.as<uint64_t>() + nranges, 8,
                                 cudaMemcpyDeviceToHost, st));
        SPK_CUDA(cudaStreamSynchronize(st));
        if ((rc = ops.alloc(std::max<uint64_t>(host[S_WORDS], 1) * 4, st))) return rc;
        SPK_CUDA(cudaMemsetAsync(rfill.p, 0, nranges * 4 * kFillStride, st));
        SPK_CUDA(cudaMemsetAsync(errp, 0, 4, st));
        bv = RangeView{ops.as<uint32_t>(), rbase.as<uint64_t>(), rfill.as<unsigned int>(), 0,
                       (uint32_t)nranges, errp};
        if (list_mode) {
          SPK_CUDA(cudaMemsetAsync(sw + S_LFILL, 0, 3 * 8, st));
          SPK_CUDA(cudaMemsetAsync(sw + S_HIST, 0, kHistBins * 8, st));
        }
        if (nl == 1) rc = launch_part_count<1>(ctx, st, pv, t, k, kr.fm, tiers, bv, lo);
        else rc = launch_part_count<2>(ctx, st, pv, t, k, kr.fm, tiers, bv, lo);
        if (rc) return rc;
        SPK_CUDA(cudaGetLastError());
        launches += 2;  // k_part_bases, k_part_count
        info.part_rescatters++;
        if ((rc = fetch(S_ERR + 1))) return rc;
        if ((int)host[S_ERR] & (kErrRange | 1)) return fail(SPK_E_CUDA, "Bloom range overflow after resizing");
      }
      break;
    }
    for (int attempt = 0; !partitioned; attempt++) {
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
    if (count_first && !partitioned) {
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
  // the compact tiers (every schedule)
  if ((rc = kr.seen.alloc(kr.num_words * 8, st))) return rc;
  if ((rc = kr.twice.alloc(kr.num_words * 8, st))) return rc;
  if (bv.ops) {
    // partitioned: apply the binned operations range by range
    SPK_CUDA(cudaEventRecord(kb0.e, st));
    if ((rc = launch_bloom_apply(ctx, st, bv, kr.num_words, kr.seen.as<uint64_t>(),
                                 kr.twice.as<uint64_t>(), su + S_POPS)))
      return rc;
    SPK_CUDA(cudaGetLastError());
    SPK_CUDA(cudaEventRecord(kb1.e, st));
    launches++;
    ops.release();
  } else {
    k_tier_finish<<<grid_for(ctx, 4), kBlock, 0, st>>>(tiers, kr.num_words, kr.seen.as<uint64_t>(),
                                                      kr.twice.as<uint64_t>(), su + S_POPS);
    SPK_CUDA(cudaGetLastError());
    launches++;
    kr.tiers.release();
  }
  SPK_CUDA(cudaEventRecord(e1.e, st));
  if ((rc = fetch(S_POPS + 2))) return rc;
  info.occurrences = host[S_OCC];
  info.seen_popcount = host[S_POPS];
  info.twice_popcount = host[S_POPS + 1];

  DevBuf cdata;  // SPK_F_CORRECT: the corrected copy of the packed reads
  if (correct) {
    // ---- Stage 3 error correction (src/assemble.rs:183-191) into a copy ----
    if ((rc = cdata.alloc(rv.data_len + 128, st))) return rc;
    SPK_CUDA(cudaMemsetAsync(cdata.as<uint8_t>() + rv.data_len, 0, 128, st));
    SPK_CUDA(cudaEventRecord(ec0.e, st));
    uint64_t nc = 0;
    if ((rc = correct_reads(ctx, st, k, (const unsigned long long*)kr.twice.as<uint64_t>(), kr.fm,
                            (const uint8_t*)rv.words + rv.byte_base, rv.data_len, rv.offsets, rv.lengths,
                            rv.n_reads, cdata.as<uint8_t>(), nullptr, &nc, &launches)))
      return rc;
    SPK_CUDA(cudaEventRecord(ec1.e, st));
    info.n_corrected_reads = nc;
    rv.words = cdata.as<uint64_t>();
    rv.byte_base = 0;
  }
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

  // ---- prior contigs (src/assemble.rs:244-284), after singleton admission ----
  if (priors) {
    // Mark the rejected singletons (nothing is listed), then inject.
    DevBuf junk;
    if ((rc = junk.alloc((kHistBins + 8) * 8, st))) return rc;
    SPK_CUDA(cudaMemsetAsync(junk.p, 0, (kHistBins + 8) * 8, st));
    unsigned long long* jw = junk.as<unsigned long long>();
    uint64_t* none[4] = {nullptr, nullptr, nullptr, nullptr};
    SPK_DISPATCH_NL(nl, launch_admit, ctx, st, kr.table, k, kr.fm, kr.twice.as<uint64_t>(),
                    gated ? 0 : 1, 0xFFFFFFFFu, none, nullptr, 0, jw, jw + kHistBins,
                    jw + kHistBins + 4);
    SPK_CUDA(cudaGetLastError());
    launches++;
    uint64_t total = 0;
    for (uint64_t i = 0; i < o.n_prior; i++) total = std::max(total, o.prior_offsets[i] + o.prior_lengths[i]);
    DevBuf pseq, poff, plen;
    if ((rc = pseq.alloc(std::max<uint64_t>(total, 1), st)) || (rc = poff.alloc(o.n_prior * 8, st)) ||
        (rc = plen.alloc(o.n_prior * 4, st)))
      return rc;
    if (total) SPK_CUDA(cudaMemcpyAsync(pseq.p, o.prior_seqs, total, cudaMemcpyHostToDevice, st));
    SPK_CUDA(cudaMemcpyAsync(poff.p, o.prior_offsets, o.n_prior * 8, cudaMemcpyHostToDevice, st));
    SPK_CUDA(cudaMemcpyAsync(plen.p, o.prior_lengths, o.n_prior * 4, cudaMemcpyHostToDevice, st));
    const uint32_t mc = o.min_coverage >= 4294967295.0 ? 0xFFFFFFFFu
                        : o.min_coverage > 0 ? (uint32_t)o.min_coverage : 0u;
    const uint32_t boost = std::max<uint32_t>(mc * 4u, 50u);  // src/assemble.rs:272
    SPK_CUDA(cudaMemsetAsync(errp, 0, 4, st));
    switch (nl) {
      case 1: k_prior_inject<1><<<grid_for(ctx, 4), kBlock, 0, st>>>(pseq.as<uint8_t>(), poff.as<uint64_t>(), plen.as<uint32_t>(), o.n_prior, k, boost, kr.table); break;
      case 2: k_prior_inject<2><<<grid_for(ctx, 4), kBlock, 0, st>>>(pseq.as<uint8_t>(), poff.as<uint64_t>(), plen.as<uint32_t>(), o.n_prior, k, boost, kr.table); break;
      case 3: k_prior_inject<3><<<grid_for(ctx, 4), kBlock, 0, st>>>(pseq.as<uint8_t>(), poff.as<uint64_t>(), plen.as<uint32_t>(), o.n_prior, k, boost, kr.table); break;
      default: k_prior_inject<4><<<grid_for(ctx, 4), kBlock, 0, st>>>(pseq.as<uint8_t>(), poff.as<uint64_t>(), plen.as<uint32_t>(), o.n_prior, k, boost, kr.table); break;
    }
    SPK_CUDA(cudaGetLastError());
    launches++;
    if ((rc = fetch(S_ERR + 1))) return rc;
    if ((int)host[S_ERR] & 1)
      return fail(SPK_E_TABLE_FULL, "count table: no free slot for a prior contig k-mer");
  }

  // ---- admission of singletons, histogram, compaction, cutoff ----
  kr.list_min = lmin_pre;
  uint64_t* lp[4] = {nullptr, nullptr, nullptr, nullptr};
  if (list_mode) {
    // The span count listed the k-mers counted >= lmin times and histogrammed
    // those counted twice or more; admission adds the singletons.
    SPK_CUDA(cudaMemsetAsync(sw + S_SUMS, 0, 4 * 8, st));
    SPK_CUDA(cudaMemsetAsync(sw + S_REJ, 0, 8, st));
    if (nl == 1)
      k_admit_singletons<1><<<grid_for(ctx, 8), kBlock, 0, st>>>(lo, k, kr.fm, kr.twice.as<uint64_t>(),
                                                                 su + S_SUMS + 1);
    else
      k_admit_singletons<2><<<grid_for(ctx, 8), kBlock, 0, st>>>(lo, k, kr.fm, kr.twice.as<uint64_t>(),
                                                                 su + S_SUMS + 1);
    SPK_CUDA(cudaGetLastError());
    launches++;
    for (int j = 0; j < nl; j++) lp[j] = kr.list[j].as<uint64_t>();
  }
  // List capacity from the Bloom: k-mers seen at least twice (twice-tier
  // estimate, an overestimate), plus admitted singletons if they are listed.
  uint64_t lcap = 0;
  if (!list_mode) {
    const double md = (double)size_bits;
    const double fs = std::min((double)info.seen_popcount / md, 0.999999);
    const double ft = std::min((double)info.twice_popcount / md, 0.999999);
    const double n_all = -(md / 3.0) * std::log1p(-fs);
    const double n2 = -(md / 3.0) * std::log1p(-ft);
    double est = n2 * 1.25 + 65536;
    if (kr.list_min <= 1) est += std::max(n_all - n2, 0.0) * ft * ft * ft * 1.5 + 65536;
    lcap = std::min<uint64_t>((uint64_t)est, cap);
  }
  for (int pass = 0; !list_mode; pass++) {
    for (int j = 0; j < nl; j++) {
      if ((rc = kr.list[j].alloc(std::max<uint64_t>(lcap, 1) * 8, st))) return rc;
      lp[j] = kr.list[j].as<uint64_t>();
    }
    if ((rc = kr.list[4].alloc(std::max<uint64_t>(lcap, 1) * 4, st))) return rc;
    SPK_CUDA(cudaMemsetAsync(sw + S_SUMS, 0, 4 * 8, st));
    SPK_CUDA(cudaMemsetAsync(sw + S_REJ, 0, 8, st));
    SPK_CUDA(cudaMemsetAsync(sw + S_HIST, 0, kHistBins * 8, st));
    SPK_DISPATCH_NL(nl, launch_admit, ctx, st, kr.table, k, kr.fm, kr.twice.as<uint64_t>(),
                    (gated || priors) ? 0 : 1, lmin_pre, lp, kr.list[4].as<uint32_t>(), lcap, su + S_HIST,
                    su + S_SUMS, su + S_REJ);
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
  if (list_mode) {
    uint64_t n2 = 0;
    for (int c = 2; c < kHistBins; c++) n2 += host[S_HIST + c];
    const uint64_t adm1 = host[S_SUMS + 1];
    info.n_table = n2 + adm1;
    info.n_singletons = adm1;
    info.n_distinct = n2 + host[S_LFILL + 1];
    info.admitted_occurrences = host[S_OCC2] + adm1;
    kr.list_len = host[S_LFILL];
    if (kr.list_len > cap || host[S_LFILL + 1] > cap)
      return fail(SPK_E_CUDA, "k-mer list larger than the table it came from");
  } else {
    info.n_table = host[S_SUMS + 0];
    info.n_singletons = host[S_SUMS + 1];
    info.n_distinct = host[S_SUMS + 0] + host[S_REJ];
    info.admitted_occurrences = host[S_SUMS + 2];
    kr.list_len = host[S_SUMS + 3];
  }
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
  if ((rc = sort_bufs(st, nl, kr.list_len, 2 * k, kr.list, &kr.list[4], host, &launches))) return rc;
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
    // For k <= 64 the neighbours are looked up in a set of the solid k-mers
    // (at most 2/3 full), built from the list; wider keys probe the table.
    DevBuf set, filt;
    SetView sv{nullptr, 0, 0, nullptr};
    if (nl <= 2) {
      uint32_t lg = 10, lf = 20;
      while ((1ULL << lg) < info.n_solid + (info.n_solid >> 1) + 1) lg++;
      while (lf < 30 && (1ULL << lf) < info.n_solid * 16) lf++;  // ~1/16 false positives
      if ((rc = set.alloc((1ULL << lg) * nl * 8, st)) || (rc = filt.alloc((1ULL << lf) / 8, st)))
        return rc;
      SPK_CUDA(cudaMemsetAsync(set.p, 0xFF, (1ULL << lg) * nl * 8, st));
      SPK_CUDA(cudaMemsetAsync(filt.p, 0, (1ULL << lf) / 8, st));
      sv = SetView{set.as<uint64_t>(), lg, lf, filt.as<uint32_t>()};
      launch_solid_set(ctx, st, nl, lp, kr.list[4].as<uint32_t>(), kr.list_len, thr, k, sv);
      SPK_CUDA(cudaGetLastError());
      launches++;
    }
    launch_edges(ctx, st, nl, kr.nle, lp, kr.list[4].as<uint32_t>(), kr.list_len, thr, kr.table,
                 nl <= 2 ? &sv : nullptr, k, ep, ecap, su + S_EDGES);
    SPK_CUDA(cudaGetLastError());
    launches++;
    if ((rc = fetch(S_EDGES + 1))) return rc;
    info.n_edges = host[S_EDGES];
    if (info.n_edges > ecap) return fail(SPK_E_CUDA, "edge list larger than its bound");
    if ((rc = sort_bufs(st, kr.nle, info.n_edges, 2 * (k + 1), kr.edges, nullptr, host, &launches)))
      return rc;
  }
  SPK_CUDA(cudaEventRecord(e5.e, st));
  if (!(o.flags & SPK_F_KEEP_BLOOM)) {
    kr.seen.release();
    kr.twice.release();
  }
  if ((rc = keep_results(kr, st, o.flags))) return rc;
  SPK_CUDA(cudaEventRecord(e6.e, st));
  SPK_CUDA(cudaStreamSynchronize(st));
  info.ms_bloom = ms_between(e0, e1);
  info.ms_correct = correct ? ms_between(ec0, ec1) : 0.f;
  info.ms_count = ms_between(e1, e2);
  info.ms_finish = ms_between(e2, e3);
  info.ms_sort = ms_between(e3, e4);
  info.ms_edges = ms_between(e4, e5);
  info.ms_total = ms_between(e0, e6);
  info.ms_bloom_kernel = ms_between(kb0, kb1);
  info.ms_count_kernel = (gated || count_first) ? ms_between(kc0, kc1) : 0.f;
  info.ms_scatter_kernel = partitioned ? ms_between(ks0, ks1) : 0.f;
  info.kernel_launches = launches;
  info.schedule = gated         ? SPK_SCHEDULE_GATED
                  : partitioned ? SPK_SCHEDULE_PARTITIONED
                  : count_first ? SPK_SCHEDULE_COUNT_FIRST
                                : SPK_SCHEDULE_FUSED;
  return SPK_OK;
}

// ---------------------------------------------------------------------------
// The default job for 12 <= k <= 64 with few host round trips.  It runs the
// partitioned schedule with the two-level read partition and the span count
// writing the k-mer list (no table), and reads device values back three
// times: the occurrence count that sizes the table, one block of counters
// after the cutoff (sizes of the lists, the histogram, the overflow flags),
// and the edge count at the end.  Region, bucket and range overflows (skewed
// inputs) and full spans are only checked at the mid-job readback: the
// kernels keep every access inside its buffer, and on any overflow the job is
// counted again by count_one_k, which lays the buffers out exactly.
// Returns kNotThisPath when the inputs need another layout (count_one_k
// handles them), kRedo after an overflow, else the status.
// ---------------------------------------------------------------------------
constexpr int kNotThisPath = -100, kRedo = -101, kGrow = -102;
constexpr uint32_t kMaxLog2Groups = 4;  // at most 16 passes over the reads

// A second stream of one job, joined back to the job's stream by events.
struct SideStream {
  cudaStream_t s = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  int open() {
    s = pooled_stream();
    fork = pooled_event(false);
    join = pooled_event(false);
    if (!s || !fork || !join) return fail(SPK_E_CUDA, "side stream or events");
    return SPK_OK;
  }
  ~SideStream() {
    pooled_stream_put(s);  // work still queued on it runs before its next user's
    pooled_event_put(fork, false);
    pooled_event_put(join, false);
  }
};

int count_one_k_list(spk_ctx* ctx, cudaStream_t st, uint64_t* host, const ReadsView& rv_in, unsigned k,
                     const spk_count_opts& o, KResult& kr) {
  const int nl = (int)((k + 31) / 32);
  // (k = 96 fills its top limb, which the solid set's empty mark needs free)
  if (k < 12 || (nl >= 3 && 2 * k == 64u * nl)) return kNotThisPath;
  if (o.flags & (SPK_F_GATED | SPK_F_CORRECT | SPK_F_REF_SOLID | SPK_F_DIRECT | SPK_F_KEEP_TABLE))
    return kNotThisPath;
  if (o.n_prior > 0 && o.prior_seqs && o.prior_offsets && o.prior_lengths) return kNotThisPath;
  const uint64_t bloom_bits = o.bloom_bits ? o.bloom_bits : (512ULL << 20);
  const uint64_t num_words = std::max<uint64_t>((bloom_bits + 63) / 64, 1);  // src/bloom.rs:27
  const uint64_t size_bits = num_words * 64;                                  // src/bloom.rs:28
  const uint64_t nranges = (size_bits + (1ULL << kLog2Range) - 1) >> kLog2Range;
  if (nranges > kMaxRanges) return kNotThisPath;
  int rc;
  DevBuf scratch;
  constexpr int S_ORDER = S_WORDS;  // reads out of order (chunked upload)
  if ((rc = scratch.alloc((S_WORDS + 1) * 8, st))) return rc;
  uint64_t* sw = scratch.as<uint64_t>();
  SPK_CUDA(cudaMemsetAsync(sw, 0, (S_WORDS + 1) * 8, st));
  unsigned long long* su = (unsigned long long*)sw;
  // ---- the first readback: occurrences, which size the table ----
  Ev e0, e1, e2, e3, e4, e5, e6, kb0, kb1, kc0, kc1, ks0, ks1, ksm;
  SPK_CUDA(cudaEventRecord(e0.e, st));
  k_occ<<<grid_for(ctx, 2), kBlock, 0, st>>>(rv_in.lengths, rv_in.n_reads, k, su + S_OCC0);
  SPK_CUDA(cudaGetLastError());
  if (rv_in.chunks) {
    k_read_order<<<grid_for(ctx, 2), kBlock, 0, st>>>(rv_in.offsets, rv_in.lengths, rv_in.n_reads, su + S_ORDER);
    SPK_CUDA(cudaGetLastError());
    SPK_CUDA(cudaMemcpyAsync(host + S_ORDER, sw + S_ORDER, 8, cudaMemcpyDeviceToHost, st));
  }
  SPK_CUDA(cudaMemcpyAsync(host + S_OCC0, sw + S_OCC0, 8, cudaMemcpyDeviceToHost, st));
  SPK_CUDA(cudaStreamSynchronize(st));
  const uint64_t occ0 = host[S_OCC0];
  const bool per_chunk = rv_in.chunks && host[S_ORDER] == 0;
  uint64_t cap = o.table_log2 ? (1ULL << std::min<uint32_t>(o.table_log2, 40)) : list_capacity(occ0, nl);
  const uint32_t log2span = part_log2span(nl);
  uint32_t log2cap = 0;
  while ((1ULL << log2cap) < cap) log2cap++;
  if (log2cap <= log2span) return kNotThisPath;
  const uint32_t log2parts = log2cap - log2span;
  // Span groups: a read set whose partition buffers (span regions and coarse
  // buckets, 2.6 keys per occurrence) would pass a quarter of the device is
  // partitioned and counted in 2^lg passes, each keeping the keys of one group
  // of spans (the reads are streamed once per pass).
  // Span regions hold 1.5x their mean share of occurrences, 2x for the
  // smaller spans of keys wider than 64 bits (fewer k-mers per span, so its
  // share varies more); the coarse buckets 1.125x.
  const uint64_t part_keys4 = nl >= 3 ? 13 : 11;  // regions + buckets, in quarter keys per occurrence
  auto part_bytes = [&](uint32_t g) { return ((occ0 >> g) * part_keys4 / 4 + (1u << 22)) * (uint64_t)nl * 8; };
  uint32_t lg = std::min<uint32_t>(o.span_groups_log2, kMaxLog2Groups);
  while (lg < kMaxLog2Groups && part_bytes(lg) > ctx->total_mem / 4) lg++;
  if (part_bytes(lg) > ctx->total_mem / 4) return kNotThisPath;
  while (lg > 0 && log2parts - lg <= kCoarseBits) lg--;
  if (!SPK_TWO_LEVEL || log2parts - lg <= kCoarseBits || log2parts - lg - kCoarseBits > kFineMaxBits ||
      part_bytes(lg) > ctx->total_mem / 4)
    return kNotThisPath;
  // The span count holds at most one distinct k-mer per slot (a full span
  // sends the job back), so the singleton keys and the list, up to one entry
  // per slot each, cannot overflow.  With several groups (large read sets)
  // the list gets half the slots: k-mers counted twice or more are a small
  // share of the distinct ones (the mid-job readback sends the job back if
  // it overflowed).
  const uint64_t lcap_ = lg ? cap >> 1 : cap, scap_ = cap;

  kr.k = k;
  kr.nl = nl;
  kr.num_words = num_words;
  kr.fm = make_fastmod(size_bits);
  spk_result_info& info = kr.info;
  memset(&info, 0, sizeof info);
  info.k = k;
  info.bloom_size_bits = size_bits;
  int* errp = (int*)(sw + S_ERR);
  ReadsView rv = rv_in;
  rv.err = errp;
  uint32_t fixed = o.min_count;
  if (!fixed && o.min_coverage > 5.0) {  // src/assemble.rs:693-694
    double v = std::max(o.min_coverage * 0.35, 2.0);
    fixed = v >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)v;
  }
  const uint32_t list_min = o.list_min_count ? o.list_min_count : 2;
  const uint32_t lmin_pre = std::max(1u, std::min(fixed ? fixed : 2u, list_min));
  kr.list_min = lmin_pre;

  uint32_t launches = 1;  // k_occ
  if ((rc = alloc_table(ctx, kr, st, cap, log2span, false, false))) return rc;
  TableView& t = kr.table;
  t.err = errp;
  const uint64_t nparts = 1ULL << log2parts;
  const uint64_t nparts_g = nparts >> lg;  // spans of one group

  // Buffers of the span count, filled over every group's pass (allocated
  // after the first group's partition, when a single group has freed its
  // coarse buckets, so that they never coexist).
  const bool early_sort = lmin_pre >= 2;
  SideStream side;
  if (early_sort && (rc = side.open())) return rc;
  DevSort lsort, esort;  // after `side`: its buffers are freed on that stream first
  DevBuf rbase, rfill, ops, sgl[4];
  RangeView bv{};
  ListOut lo{};
  auto alloc_count_buffers = [&]() -> int {
    int r2;
    const uint64_t share = 3 * cap / nranges + 1;  // three per distinct k-mer
    const uint64_t rcap = share + (share >> 2) + 1024;
    if ((r2 = rbase.alloc((nranges + 1) * 8, st)) || (r2 = rfill.alloc(nranges * 4 * kFillStride, st)) ||
        (r2 = ops.alloc(nranges * rcap * 4, st)))
      return r2;
    SPK_CUDA(cudaMemsetAsync(rfill.p, 0, nranges * 4 * kFillStride, st));
    bv = RangeView{ops.as<uint32_t>(), rbase.as<uint64_t>(), rfill.as<unsigned int>(), rcap, (uint32_t)nranges,
                   errp};
    for (int j = 0; j < nl; j++)
      if ((r2 = kr.list[j].alloc(lcap_ * 8, st)) || (r2 = sgl[j].alloc(scap_ * 8, st))) return r2;
    if ((r2 = kr.list[4].alloc(lcap_ * 4, st))) return r2;
    lo = list_out(kr, sgl, lcap_, scap_, lmin_pre, su);
    return SPK_OK;
  };

  // ---- two-level read partition (k_part_coarse, k_part_fine) and span
  // count, once per group of spans ----
  DevBuf base, fill, region;
  const uint64_t per = occ0 / nparts;
  const uint64_t capu = nl >= 3 ? 2 * per + 512 : per + (per >> 1) + 256;
  if ((rc = base.alloc((nparts_g + 1) * 8, st)) || (rc = fill.alloc(nparts_g * 4 * kFillStride, st)) ||
      (rc = region.alloc(nparts_g * capu * nl * 8, st)))
    return rc;
  k_part_uniform<<<64, kBlock, 0, st>>>((uint32_t)nparts_g, capu, base.as<uint64_t>());
  DevBuf cbase, cfill, cregion, cfirst;
  const uint64_t cper = (occ0 >> lg) / kCoarse;
  const uint64_t ccap = (cper + (cper >> 3) + 8192 + 1) & ~1ULL;  // even: chunks start 16-byte aligned
  if ((rc = cbase.alloc((kCoarse + 1) * 8, st)) || (rc = cfill.alloc(kCoarse * 4 * kFillStride, st)) ||
      (rc = cregion.alloc(kCoarse * ccap * nl * 8, st)) || (rc = cfirst.alloc((kCoarse + 1) * 4, st)))
    return rc;
  k_part_uniform<<<1, 128, 0, st>>>(kCoarse, ccap, cbase.as<uint64_t>());
  info.part_passes = 2;
  info.span_groups = 1u << lg;
  SPK_CUDA(cudaEventRecord(ks0.e, st));
  for (uint32_t g = 0; g < (1u << lg); g++) {
  SPK_CUDA(cudaMemsetAsync(fill.p, 0, nparts_g * 4 * kFillStride, st));
  PartView pv{region.as<uint64_t>(), base.as<uint64_t>(), fill.as<unsigned int>(), capu, log2parts,
              home_fits(k, nl) ? 1u : 0u, errp, lg, g};
  {
    SPK_CUDA(cudaMemsetAsync(cfill.p, 0, kCoarse * 4 * kFillStride, st));
    CoarseView cv{cregion.as<uint64_t>(), cbase.as<uint64_t>(), cfill.as<unsigned int>(), ccap, errp};
    if (per_chunk && g == 0) {
      // the reads of each uploaded piece as soon as it is on the device
      uint64_t r0 = 0;
      for (int c = 0; c < rv.chunks->n; c++) {
        SPK_CUDA(cudaStreamWaitEvent(st, rv.chunks->ready[c], 0));
        const uint64_t r1 = std::min<uint64_t>(std::max<uint64_t>(rv.chunks->read_end[c], r0), rv.n_reads);
        if (r1 > r0) {
          ReadsView rc_ = rv;
          rc_.offsets += r0;
          rc_.lengths += r0;
          rc_.n_reads = r1 - r0;
          rc = SPK_NL_CALL(nl, launch_part_coarse, ctx, st, rc_, k, pv, cv, su + S_OCC);
          if (rc) return rc;
          launches++;
        }
        r0 = r1;
      }
      launches--;  // counted below
    } else {
      if (rv.chunks) SPK_CUDA(cudaStreamWaitEvent(st, rv.chunks->ready[rv.chunks->n - 1], 0));
      rc = SPK_NL_CALL(nl, launch_part_coarse, ctx, st, rv, k, pv, cv, su + S_OCC);
      if (rc) return rc;
    }
    if (lg == 0) SPK_CUDA(cudaEventRecord(ksm.e, st));
    k_coarse_chunks<<<1, 32, 0, st>>>(cv, nl <= 2 ? fine_chunk<2>() : fine_chunk<4>(), cfirst.as<uint32_t>());
    rc = SPK_NL_CALL(nl, launch_part_fine, ctx, st, cv, cfirst.as<uint32_t>(), pv, k);
    if (rc) return rc;
    SPK_CUDA(cudaGetLastError());
    launches += 3;  // k_part_coarse, k_coarse_chunks, k_part_fine
  }
  if (g + 1 == (1u << lg)) SPK_CUDA(cudaEventRecord(ks1.e, st));
  if (lg == 0) {  // one group: its coarse buckets are done with
    cregion.release();
    cbase.release();
    cfill.release();
    cfirst.release();
  }
  if (g == 0 && (rc = alloc_count_buffers())) return rc;

  // ---- span count of this group: the list, the singleton keys and the binned Bloom ops ----
  if (g == 0) SPK_CUDA(cudaEventRecord(kc0.e, st));
  rc = SPK_NL_CALL(nl, launch_part_count, ctx, st, pv, t, k, kr.fm, nullptr, bv, lo);
  if (rc) return rc;
  SPK_CUDA(cudaGetLastError());
  launches++;
  }  // span groups
  launches += 2;  // k_part_uniform x 2
  cregion.release();
  cbase.release();
  cfill.release();
  cfirst.release();
  {
    SPK_CUDA(cudaEventRecord(kc1.e, st));
    if (early_sort) {
      // The list is final once the spans are counted (singletons are not
      // listed): sort it on the side stream while the job's stream builds
      // the Bloom tiers, admits the singletons and finds the cutoff.
      SPK_CUDA(cudaEventRecord(side.fork, st));
      SPK_CUDA(cudaStreamWaitEvent(side.s, side.fork, 0));
      if ((rc = sort_dev_enqueue(side.s, nl, lcap_, su + S_LFILL, 2 * k, kr.list, &kr.list[4], nullptr, lsort,
                                 &launches)))
        return rc;
      SPK_CUDA(cudaEventRecord(side.join, side.s));
    }
    region.release();
    base.release();
    fill.release();
    // ---- Bloom tiers from the binned operations ----
    if ((rc = kr.seen.alloc(num_words * 8, st)) || (rc = kr.twice.alloc(num_words * 8, st))) return rc;
    SPK_CUDA(cudaEventRecord(kb0.e, st));
    if ((rc = launch_bloom_apply(ctx, st, bv, num_words, kr.seen.as<uint64_t>(), kr.twice.as<uint64_t>(),
                                 su + S_POPS)))
      return rc;
    SPK_CUDA(cudaGetLastError());
    SPK_CUDA(cudaEventRecord(kb1.e, st));
    ops.release();
    rbase.release();
    rfill.release();
    launches += 1;
    SPK_CUDA(cudaEventRecord(e1.e, st));
    SPK_CUDA(cudaEventRecord(e2.e, st));
    // ---- singleton admission, histogram, cutoff ----
    SPK_DISPATCH_NL(nl, launch_admit_singletons, ctx, st, lo, k, kr.fm, kr.twice.as<uint64_t>(),
                    su + S_SUMS + 1);
    SPK_CUDA(cudaGetLastError());
    launches++;
  }
  uint32_t* thr = (uint32_t*)(sw + S_THR);
  k_cutoff<<<1, 32, 0, st>>>(su + S_HIST, fixed, list_min, thr);
  SPK_CUDA(cudaGetLastError());
  launches++;
  // ---- the one mid-job readback ----
  if (early_sort) SPK_CUDA(cudaStreamWaitEvent(st, side.join, 0));
  SPK_CUDA(cudaMemcpyAsync(host, sw, S_WORDS * 8, cudaMemcpyDeviceToHost, st));
  SPK_CUDA(cudaStreamSynchronize(st));
  const int err = (int)host[S_ERR];
  if (err & 4) return fail(SPK_E_INVALID_ARG, "a read extends past the end of the packed data");
  if (err & 2) return fail(SPK_E_TIMEOUT, "count table: claim wait timed out");
  if (err & (int)kErrStage) return fail(SPK_E_TIMEOUT, "partition: a staged copy never completed");
  if (err & (kErrRegion | kErrRange)) return kRedo;  // an overflowed region
  if (err & 1) return kGrow;                           // a span with more distinct k-mers than slots
  info.occurrences = host[S_OCC];
  info.seen_popcount = host[S_POPS];
  info.twice_popcount = host[S_POPS + 1];
  info.table_capacity = cap;
  const uint32_t* hthr = (const uint32_t*)(host + S_THR);
  info.cutoff = hthr[0];
  kr.list_min = hthr[1];
  uint64_t n2 = 0;
  for (int c = 2; c < kHistBins; c++) n2 += host[S_HIST + c];
  const uint64_t adm1 = host[S_SUMS + 1];
  info.n_table = n2 + adm1;
  info.n_singletons = adm1;
  info.n_distinct = n2 + host[S_LFILL + 1];
  info.admitted_occurrences = host[S_OCC2] + adm1;
  kr.list_len = host[S_LFILL];
  if (kr.list_len > lcap_ || host[S_LFILL + 1] > scap_) {
    if (lg) return kRedo;  // a share of the slots was too small
    return fail(SPK_E_CUDA, "k-mer list larger than the table it came from");
  }
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
    k_count_solid<<<grid_for(ctx, 2), 256, 0, st>>>(kr.list[4].as<uint32_t>(), kr.list_len, thr, su + S_CNT);
    SPK_CUDA(cudaGetLastError());
    launches++;
    SPK_CUDA(cudaMemcpyAsync(host + S_CNT, sw + S_CNT, 8, cudaMemcpyDeviceToHost, st));
    SPK_CUDA(cudaStreamSynchronize(st));
    info.n_solid = host[S_CNT];
  }
  SPK_CUDA(cudaEventRecord(e3.e, st));

  // ---- sort of the list, unless it ran early (the singleton buffers, read by
  // admission, are its temporaries here) ----
  if (!early_sort &&
      (rc = sort_dev_enqueue(st, nl, kr.list_len, nullptr, 2 * k, kr.list, &kr.list[4], sgl, lsort, &launches)))
    return rc;
  uint64_t* lp[4] = {nullptr, nullptr, nullptr, nullptr};
  for (int j = 0; j < nl; j++) lp[j] = kr.list[j].as<uint64_t>();
  SPK_CUDA(cudaEventRecord(e4.e, st));

  // ---- the solid list for the caller's host buffers: converted here, copied
  // on a side stream while the edges are built ----
  const bool want_solid = (o.solid_keys_out || o.solid_counts_out) && info.n_solid <= o.solid_capacity;
  SideStream cpy;
  if (want_solid) {
    uint64_t m = 0;
    if ((rc = cpy.open())) return rc;
    if ((rc = ordered_convert(st, nl, kr.list_len, k, kr.list, kr.list[4].as<uint32_t>(), info.cutoff,
                              &kr.conv.keys, &kr.conv.cnt, host, &m, info.n_solid)))
      return rc;
    kr.conv.kind = 0;  // what spk_result_solid converts (kept for later downloads)
    kr.conv.minc = info.cutoff;
    kr.conv.n = m;
    launches += 4;     // k_oc_count, the scan's two kernels, k_oc_write
    SPK_CUDA(cudaEventRecord(cpy.fork, st));
    SPK_CUDA(cudaStreamWaitEvent(cpy.s, cpy.fork, 0));
  }

  // ---- edges ----
  kr.nle = (int)((k + 1 + 31) / 32);
  uint64_t ecap = 0;
  DevBuf set, filt;
  if ((o.flags & SPK_F_EDGES) && info.n_solid > 0) {
    uint64_t* ep[4] = {nullptr, nullptr, nullptr, nullptr};
    ecap = info.n_solid * 8;  // at most 8 canonical edges per solid k-mer
    for (int j = 0; j < kr.nle; j++) {
      if ((rc = kr.edges[j].alloc(ecap * 8, st))) return rc;
      ep[j] = kr.edges[j].as<uint64_t>();
    }
    uint32_t lg = 10, lf = 20;
    while ((1ULL << lg) < info.n_solid + (info.n_solid >> 1) + 1) lg++;
    while (lf < 30 && (1ULL << lf) < info.n_solid * 16) lf++;  // ~1/16 false positives
    if ((rc = set.alloc((1ULL << lg) * nl * 8, st)) || (rc = filt.alloc((1ULL << lf) / 8, st))) return rc;
    SPK_CUDA(cudaMemsetAsync(set.p, 0xFF, (1ULL << lg) * nl * 8, st));
    SPK_CUDA(cudaMemsetAsync(filt.p, 0, (1ULL << lf) / 8, st));
    SetView sv{set.as<uint64_t>(), lg, lf, filt.as<uint32_t>()};
    launch_solid_set(ctx, st, nl, lp, kr.list[4].as<uint32_t>(), kr.list_len, thr, k, sv);
    SPK_CUDA(cudaGetLastError());
    launch_edges(ctx, st, nl, kr.nle, lp, kr.list[4].as<uint32_t>(), kr.list_len, thr, kr.table, &sv, k, ep,
                 ecap, su + S_EDGES);
    SPK_CUDA(cudaGetLastError());
    launches += 2;
    set.release();
    filt.release();
    if ((rc = sort_dev_enqueue(st, kr.nle, ecap, su + S_EDGES, 2 * (k + 1), kr.edges, nullptr, nullptr, esort,
                               &launches)))
      return rc;
  }
  SPK_CUDA(cudaEventRecord(e5.e, st));
  if (want_solid) {
    // (the host waits here for the copy while the device builds the edges)
    const uint64_t m = kr.conv.n;
    if (m && o.solid_keys_out && (rc = xfer_d2h(ctx, o.solid_keys_out, kr.conv.keys.p, m * nl * 8, cpy.s)))
      return rc;
    if (m && o.solid_counts_out && (rc = xfer_d2h(ctx, o.solid_counts_out, kr.conv.cnt.p, m * 4, cpy.s)))
      return rc;
    SPK_CUDA(cudaStreamSynchronize(cpy.s));
    info.solid_copied = 1;
  }
  if (!(o.flags & SPK_F_KEEP_BLOOM)) {
    kr.seen.release();
    kr.twice.release();
  }
  // ---- the final readback: edge count and the buckets left to sort ----
  SPK_CUDA(cudaMemcpyAsync(host + S_EDGES, sw + S_EDGES, 8, cudaMemcpyDeviceToHost, st));
  uint32_t* hb = (uint32_t*)(host + S_WORDS);
  SPK_CUDA(cudaMemcpyAsync(hb, sort_dev_nbig(lsort), 4, cudaMemcpyDeviceToHost, st));
  if (esort.pending) SPK_CUDA(cudaMemcpyAsync(hb + 1, sort_dev_nbig(esort), 4, cudaMemcpyDeviceToHost, st));
  else hb[1] = 0;
  SPK_CUDA(cudaStreamSynchronize(st));
  info.n_edges = ecap ? host[S_EDGES] : 0;
  if (info.n_edges > ecap) return fail(SPK_E_CUDA, "edge list larger than its bound");
  const unsigned nbig_l = hb[0], nbig_e = hb[1];
  if ((rc = sort_dev_finish(st, lsort, kr.list, &kr.list[4], kr.list_len, nbig_l, host, &launches))) return rc;
  if ((rc = sort_dev_finish(st, esort, kr.edges, nullptr, info.n_edges, nbig_e, host, &launches))) return rc;
  if ((rc = keep_results(kr, st, o.flags))) return rc;
  SPK_CUDA(cudaEventRecord(e6.e, st));
  SPK_CUDA(cudaStreamSynchronize(st));
  info.ms_bloom = ms_between(e0, e1);
  info.ms_count = ms_between(e1, e2);
  info.ms_finish = ms_between(e2, e3);
  info.ms_sort = ms_between(e3, e4);
  info.ms_edges = ms_between(e4, e5);
  info.ms_total = ms_between(e0, e6);
  info.ms_bloom_kernel = ms_between(kb0, kb1);
  info.ms_count_kernel = ms_between(kc0, kc1);
  info.ms_scatter_kernel = ms_between(ks0, ks1);
  info.ms_coarse_kernel = lg == 0 ? ms_between(ks0, ksm) : 0.f;
  info.kernel_launches = launches;
  info.schedule = SPK_SCHEDULE_PARTITIONED;
  return SPK_OK;
}

// Device buffers of a k allocated on another stream: stream-ordered frees
// go to `s` from now on (the allocating stream has been synchronised).
static void rehome(KResult& kr, cudaStream_t s) {
  DevBuf* bufs[] = {&kr.tiers, &kr.seen, &kr.twice, &kr.ref_solid, &kr.tslots, &kr.conv.keys,
                    &kr.conv.cnt};
  for (DevBuf* b : bufs) b->st = s;
  for (DevBuf& b : kr.list) b.st = s;
  for (DevBuf& b : kr.edges) b.st = s;
}
// Every buffer of a finished result (its work on its old stream ordered
// before `s`): frees go to `s` from now on.
void rehome_result(spk_result* res, cudaStream_t s) {
  for (auto& kr : res->ks) rehome(*kr, s);
  res->reads.st = res->offs.st = res->lens.st = s;
}

// The solid list into the caller's host buffers (spk_count_opts.solid_*_out)
// after a job that did not copy it during the count.
static int solid_copy_after(spk_ctx* ctx, cudaStream_t st, uint64_t* host, KResult& kr,
                            const spk_count_opts& o) {
  if (!(o.solid_keys_out || o.solid_counts_out) || kr.info.solid_copied || kr.info.n_solid > o.solid_capacity)
    return SPK_OK;
  KResult::Conv& cv = kr.conv;
  uint64_t m = 0;
  int rc = ordered_convert(st, kr.nl, kr.list_len, kr.k, kr.list, kr.list[4].as<uint32_t>(), kr.info.cutoff,
                           &cv.keys, &cv.cnt, host, &m);
  if (rc) return rc;
  cv.kind = 0;
  cv.minc = kr.info.cutoff;
  cv.n = m;
  if (m > o.solid_capacity) return SPK_OK;
  if (m && o.solid_keys_out && (rc = xfer_d2h(ctx, o.solid_keys_out, cv.keys.p, m * kr.nl * 8, st))) return rc;
  if (m && o.solid_counts_out && (rc = xfer_d2h(ctx, o.solid_counts_out, cv.cnt.p, m * 4, st))) return rc;
  SPK_CUDA(cudaStreamSynchronize(st));
  kr.info.solid_copied = 1;
  return SPK_OK;
}

static int count_k_job(spk_ctx* ctx, cudaStream_t st, uint64_t* host, const ReadsView& rv, unsigned k,
                       const spk_count_opts& o, KResult& kr);
// One k, and the copy of its solid list to the caller's buffers if asked for.
static int count_k(spk_ctx* ctx, cudaStream_t st, uint64_t* host, const ReadsView& rv, unsigned k,
                   const spk_count_opts& o, KResult& kr) {
  const int rc = count_k_job(ctx, st, host, rv, k, o, kr);
  if (rc) return rc;
  return solid_copy_after(ctx, st, host, kr, o);
}

// One k: the job with few round trips where it applies, else (or after an
// overflow there) the general one.
static int count_k_job(spk_ctx* ctx, cudaStream_t st, uint64_t* host, const ReadsView& rv, unsigned k,
                       const spk_count_opts& o, KResult& kr) {
  int rc = count_one_k_list(ctx, st, host, rv, k, o, kr);
  // A span with more distinct k-mers than slots: twice the slots, twice at most.
  for (uint32_t grow = 1; rc == kGrow && grow <= 2; grow++) {
    SPK_CUDA(cudaStreamSynchronize(st));  // the abandoned job's buffers are freed in stream order
    spk_count_opts og = o;
    og.table_log2 = kr.table.log2cap + 1;
    kr = KResult();
    rc = count_one_k_list(ctx, st, host, rv, k, og, kr);
    if (rc == SPK_OK) {
      kr.info.table_regrows = grow;
      return SPK_OK;
    }
    if (rc == SPK_E_OOM) rc = kRedo;  // the general path instead
  }
  if (rc == kGrow) rc = kRedo;
  if (rc != kNotThisPath && rc != kRedo) return rc;
  // every uploaded piece of the reads, before the general path reads them
  if (rv.chunks) SPK_CUDA(cudaStreamWaitEvent(st, rv.chunks->ready[rv.chunks->n - 1], 0));
  SPK_CUDA(cudaStreamSynchronize(st));  // the abandoned job's buffers are freed in stream order
  kr = KResult();
  const int rc2 = count_one_k(ctx, st, host, rv, k, o, kr);
  if (!rc2 && rc == kRedo) kr.info.part_rescatters++;  // the first layout overflowed
  return rc2;
}

uint64_t job_estimate(const spk_job& j, uint64_t total_mem);

int count_pipeline(spk_ctx* ctx, cudaStream_t st, const ReadsView& rv, uint32_t max_len,
                   const uint32_t* ks, int n_k, const spk_count_opts& o, spk_result* res) {
  (void)max_len;
  if (n_k == 1) {
    auto kr = std::make_unique<KResult>();
    int rc = count_k(ctx, st, res->h_staging, rv, ks[0], o, *kr);
    if (rc) return rc;
    res->ks.push_back(std::move(kr));
    return SPK_OK;
  }
  // Several k (run_multik_assembly's per-k loop, src/multik.rs:109-178): the
  // k values are independent.  Each fills the device on a read set of useful
  // size, and jobs side by side then only contend for the memory pool (the
  // 5 Mb x 100x reads at k in {21, 33, 55, 77}: 85.7 ms side by side, 82.6 ms
  // one after another), so they count one after another on st unless together
  // they need at most an eighth of the device memory; then each counts
  // concurrently on its own stream and staging block over the same
  // read-only reads, once the reads that st uploads are ready.
  {
    uint64_t need = 0;
    for (int i = 0; i < n_k; i++) {
      spk_job j{};
      j.data_len = rv.data_len;
      j.n_reads = rv.n_reads;
      j.ks = &ks[i];
      j.n_k = 1;
      j.opts = o;
      need += job_estimate(j, ctx->total_mem);
    }
    if (need > ctx->total_mem / 8) {
      for (int i = 0; i < n_k; i++) {
        spk_count_opts oi = o;
        if (i > 0) {  // the caller's solid buffers are the first k's
          oi.solid_keys_out = nullptr;
          oi.solid_counts_out = nullptr;
        }
        auto kr = std::make_unique<KResult>();
        const int rc = count_k(ctx, st, res->h_staging, rv, ks[i], oi, *kr);
        if (rc) return fail(rc, "k=" + std::to_string(ks[i]) + ": " + spk_last_error());
        res->ks.push_back(std::move(kr));
      }
      return SPK_OK;
    }
  }
  cudaEvent_t ready = pooled_event(false);
  if (!ready) return fail(SPK_E_CUDA, "event");
  SPK_CUDA(cudaEventRecord(ready, st));
  std::vector<std::unique_ptr<KResult>> krs(n_k);
  std::vector<int> rcs(n_k, SPK_OK);
  std::vector<std::string> errs(n_k);
  std::vector<std::thread> th;
  for (int i = 0; i < n_k; i++) {
    th.emplace_back([&, i] {
      cudaSetDevice(ctx->device);
      cudaStream_t s2 = nullptr;
      uint64_t* h = staging_acquire(ctx);
      int rc = SPK_OK;
      if (!h) rc = fail(SPK_E_OOM, "pinned host staging allocation failed");
      else if (!(s2 = pooled_stream()))
        rc = fail(SPK_E_CUDA, "per-k stream");
      auto kr = std::make_unique<KResult>();
      if (!rc && cudaStreamWaitEvent(s2, ready, 0) != cudaSuccess) rc = cuda_fail(cudaGetLastError(), "wait");
      spk_count_opts oi = o;
      if (i > 0) {  // the caller's solid buffers are the first k's
        oi.solid_keys_out = nullptr;
        oi.solid_counts_out = nullptr;
      }
      if (!rc) rc = count_k(ctx, s2, h, rv, ks[i], oi, *kr);
      if (s2) {
        cudaStreamSynchronize(s2);
        rehome(*kr, st);
        pooled_stream_put(s2);
      }
      staging_release(ctx, h);
      if (rc) errs[i] = spk_last_error();
      rcs[i] = rc;
      krs[i] = std::move(kr);
    });
  }
  for (auto& t : th) t.join();
  pooled_event_put(ready, false);
  for (int i = 0; i < n_k; i++)
    if (rcs[i]) return fail(rcs[i], "k=" + std::to_string(ks[i]) + ": " + errs[i]);
  for (int i = 0; i < n_k; i++) res->ks.push_back(std::move(krs[i]));
  return SPK_OK;
}

// ---------------------------------------------------------------------------
// Downloads
// ---------------------------------------------------------------------------
// The converted list (Kmer256 limbs, kept counts) of the last download of a
// kind is cached in the result, so that a size query followed by the copy
// converts once.
static int copy_out(spk_result* res, KResult& kr, int kind, int nl, DevBuf* limbs, const uint32_t* cin,
                    uint64_t n, unsigned k, uint32_t minc, uint64_t* keys, uint32_t* counts,
                    size_t* n_inout) {
  cudaStream_t st = res->stream;
  KResult::Conv& cv = kr.conv;
  if (cv.kind != kind || cv.minc != minc) {
    cv.kind = -1;
    int rc = ordered_convert(st, nl, n, k, limbs, cin, minc, &cv.keys, cin ? &cv.cnt : nullptr,
                             res->h_staging, &cv.n);
    if (rc) return rc;
    cv.kind = kind;
    cv.minc = minc;
  }
  const uint64_t m = cv.n;
  if (!keys && !counts) {
    *n_inout = m;
    return SPK_OK;
  }
  if (*n_inout < m) {
    *n_inout = m;
    return fail(SPK_E_INVALID_ARG, "output buffer too small");
  }
  int rc;
  if (m && keys && (rc = xfer_d2h(res->ctx, keys, cv.keys.p, m * nl * 8, st))) return rc;
  if (m && counts && cin && (rc = xfer_d2h(res->ctx, counts, cv.cnt.p, m * 4, st))) return rc;
  SPK_CUDA(cudaStreamSynchronize(st));
  *n_inout = m;
  return SPK_OK;
}

int download_list(spk_result* res, int ki, uint32_t min_count, bool solid_only, uint64_t* keys,
                  uint32_t* counts, size_t* n_inout) {
  KResult& kr = *res->ks[ki];
  const uint32_t minc = solid_only ? kr.info.cutoff : std::max(min_count, kr.list_min);
  return copy_out(res, kr, 0, kr.nl, kr.list, kr.list[4].as<uint32_t>(), kr.list_len, kr.k, minc,
                  keys, counts, n_inout);
}

int download_edges(spk_result* res, int ki, uint64_t* out, size_t* n_inout) {
  KResult& kr = *res->ks[ki];
  return copy_out(res, kr, 1, kr.nle, kr.edges, nullptr, kr.info.n_edges, kr.k + 1, 0, out, nullptr,
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

// ---------------------------------------------------------------------------
// Diagnostic of the bounded claim wait of wide keys (table_add, NL >= 3).
// A writer that claims a slot publishes its key and marks the slot ready
// right after; a slot that stays claimed (a writer gone mid-claim) would stall
// every reader of it.  Here one thread leaves the home slot of a k-mer
// claimed and then counts that k-mer: its wait runs out after kSpinLimit
// polls (a fraction of a second), sets error bit 1 and returns.
// ---------------------------------------------------------------------------
template <int NL>
__global__ void k_stuck_claim(TableView t, Seq<NL> C, unsigned k) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  uint64_t w4[4];
  kmer256_limbs<NL>(C, k, w4);
  const uint64_t home = table_home(t, hash_seed(hash_pre(w4), kSeed1));
  atomicExch(slot_state<NL>(t, home), 1u);  // claimed, never published
  __threadfence();
  table_add<NL>(t, C, home, 1);
}

int stuck_claim(spk_ctx* ctx, uint32_t k) {
  if (k < 65 || k > 127) return fail(SPK_E_INVALID_K, "the claim wait serves keys of k = 65..127");
  cudaStream_t st = ctx->stream;
  KResult kr;
  kr.nl = (int)((k + 31) / 32);
  int rc;
  DevBuf errw;
  if ((rc = errw.alloc(8, st))) return rc;
  SPK_CUDA(cudaMemsetAsync(errw.p, 0, 8, st));
  if ((rc = alloc_table(ctx, kr, st, 1024))) return rc;
  kr.table.err = errw.as<int>();
  // any k-mer of k bases: limb j holds bases 32j.. in its low bits
  Seq<4> C4{};
  for (int j = 0; j < 4; j++) C4.v[j] = 0x9e3779b97f4a7c15ULL * (j + 1);
  const unsigned top = 2 * k - 64 * (kr.nl - 1);
  if (top < 64) C4.v[kr.nl - 1] &= (1ULL << top) - 1;
  if (kr.nl == 3) {
    Seq<3> C;
    for (int j = 0; j < 3; j++) C.v[j] = C4.v[j];
    k_stuck_claim<3><<<1, 32, 0, st>>>(kr.table, C, k);
  } else {
    k_stuck_claim<4><<<1, 32, 0, st>>>(kr.table, C4, k);
  }
  SPK_CUDA(cudaGetLastError());
  int host_err = 0;
  SPK_CUDA(cudaMemcpyAsync(&host_err, errw.p, 4, cudaMemcpyDeviceToHost, st));
  SPK_CUDA(cudaStreamSynchronize(st));
  if (host_err & 2) return fail(SPK_E_TIMEOUT, "count table: claim wait timed out (slot left claimed)");
  return fail(SPK_E_CUDA, "the claim wait ended without its timeout");
}

}  // namespace spk
