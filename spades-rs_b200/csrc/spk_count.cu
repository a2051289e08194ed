// spk_count.cu -- the k-mer counting pipeline on one B200.
//
// Replaces Stages 2-3 of run_assembly_with_packed_reads (src/assemble.rs:
// 129-292) and the implicit edge probes of CompactedGraph::build
// (src/graph.rs:78-102).  Per k:
//   1. k_bloom_pass   Stage 2: every canonical k-mer occurrence sets its three
//                     Bloom bits (src/bloom.rs:83-97).  Seen and twice tiers
//                     are interleaved per 64-bit word so one 16-byte access
//                     serves both.
//   2. k_tier_finish  splits out the compact twice tier, popcounts.
//   3. k_count_pass   Stage 3: occurrences whose three twice bits are set
//                     are counted in an open-addressing table in HBM
//                     (src/assemble.rs:193-207), warp-aggregated.
//   4. k_table_hist + k_cutoff   src/assemble.rs:692-735 on the device.
//   5. k_compact      stream compaction of the table into the k-mer list.
//   6. radix sort     the sorted (k-mer, count) list.
//   7. k_edges        (k+1)-mer edges between solid k-mers (src/graph.rs:78-102),
//                     then their sort.
//
// Admission rule.  The reference promotes a k-mer to its solid tier only when
// an insert finds all three seen bits already set, which depends on the
// order of the rayon chunks (src/bloom.rs:95-106).  The GPU keeps an
// order-free twice tier instead: a seen-tier fetch_or that finds its bit set
// also sets that bit in the twice tier.  Every k-mer that occurs at least
// twice gets all three twice bits, so the count >= 2 list is exact and equals
// the reference's.  The reference-semantics solid tier is still produced on
// request (SPK_F_REF_SOLID).
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
// Occurrences per streamed chunk of the partitioned Stage 2 (4 bytes of
// staged operation per Bloom bit: 12 bytes per occurrence).
constexpr uint64_t kMaxChunkOcc = 1ULL << 30;

struct alignas(16) U128 {
  unsigned long long x, y;
};

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

// ---------------------------------------------------------------------------
// 1. Stage 2: Bloom population (src/assemble.rs:141-157, src/bloom.rs:83-107)
// ---------------------------------------------------------------------------
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
    if (REF && allprev) {  // src/bloom.rs:99-103
#pragma unroll
      for (int i = 0; i < 3; i++) {
        const unsigned long long bit = 1ULL << (pos[i] & 63);
        unsigned long long* a = ref_solid + (pos[i] >> 6);
        if (!(*a & bit)) atomicOr(a, bit);
      }
    }
  };
  foreach_position(R, k, fn);
  warp_add_u64(occ_out, occ);
}

// ---------------------------------------------------------------------------
// 2. Split the compact twice tier out of the word pairs; popcount both tiers.
// ---------------------------------------------------------------------------
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
// 3. Stage 3: count table (src/assemble.rs:175-219)
// ---------------------------------------------------------------------------
template <int NL>
__device__ __forceinline__ uint64_t table_home(const TableView& t, uint64_t raw0) {
  return raw0 >> (64 - t.log2cap);
}

// Adds n to key C.  Keys of <= 128 bits are claimed with one 64- or 128-bit
// CAS against the all-ones sentinel, which no canonical k-mer can equal (for
// k < 32 / k < 64 the top bits are unused; for k = 32 / 64 all-ones is
// poly-T, whose reverse complement poly-A is smaller).  Wider keys claim the
// slot through a state word and publish the key before marking it ready.
template <int NL>
__device__ __forceinline__ void table_add(const TableView& t, const Seq<NL>& C, uint64_t home,
                                          uint32_t n) {
  const uint64_t mask = t.capacity - 1;
  for (uint32_t i = 0; i < t.max_probe; i++) {
    const uint64_t s = (home + i) & mask;
    if (NL == 1) {
      unsigned long long* kp = (unsigned long long*)(t.keys + s);
      unsigned long long cur = __ldcg(kp);
      if (cur == C.v[0]) { atomicAdd(t.counts + s, n); return; }
      if (cur == kEmpty) {
        unsigned long long old = atomicCAS(kp, kEmpty, (unsigned long long)C.v[0]);
        if (old == kEmpty || old == C.v[0]) { atomicAdd(t.counts + s, n); return; }
      }
    } else if (NL == 2) {
      U128* kp = (U128*)(t.keys + 2 * s);
      ulonglong2 cur = __ldcg((const ulonglong2*)kp);
      if (cur.x != kEmpty && cur.y != kEmpty) {
        // A settled key (a 16-byte load may tear only while a slot is being
        // claimed, and a claimed slot never changes afterwards).
        if (cur.x == C.v[0] && cur.y == C.v[NL - 1]) { atomicAdd(t.counts + s, n); return; }
        continue;
      }
      U128 e{kEmpty, kEmpty}, mine{C.v[0], C.v[NL - 1]};
      U128 old = atomicCAS(kp, e, mine);
      if ((old.x == kEmpty && old.y == kEmpty) || (old.x == mine.x && old.y == mine.y)) {
        atomicAdd(t.counts + s, n);
        return;
      }
    } else {
      uint32_t st = __ldcg(t.state + s);
      if (st == 0) {
        uint32_t old = atomicCAS(t.state + s, 0u, 1u);
        if (old == 0) {
          uint64_t* kp = t.keys + (uint64_t)t.stride * s;
#pragma unroll
          for (int j = 0; j < NL; j++) __stcg(kp + j, C.v[j]);
          atomicAdd(t.counts + s, n);
          __threadfence();
          atomicExch(t.state + s, 2u);
          return;
        }
        st = old;
      }
      if (st == 1) {
        int spins = 0;
        while ((st = ((volatile uint32_t*)t.state)[s]) != 2u) {
          if (++spins > kSpinLimit) { atomicOr(t.err, 2); return; }
          __nanosleep(64);
        }
        __threadfence();
      }
      const uint64_t* kp = t.keys + (uint64_t)t.stride * s;
      bool eq = true;
#pragma unroll
      for (int j = 0; j < NL; j++) eq &= __ldcg(kp + j) == C.v[j];
      if (eq) { atomicAdd(t.counts + s, n); return; }
    }
  }
  atomicOr(t.err, 1);  // probe limit: the host regrows the table and recounts
}

template <int NL>
__device__ __forceinline__ bool table_find(const TableView& t, const Seq<NL>& C, uint64_t home,
                                           uint32_t* count) {
  const uint64_t mask = t.capacity - 1;
  for (uint32_t i = 0; i < t.max_probe; i++) {
    const uint64_t s = (home + i) & mask;
    const uint32_t c = __ldg(t.counts + s);
    if (c == 0) return false;  // empty slot ends the probe sequence
    const uint64_t* kp = t.keys + (uint64_t)t.stride * s;
    bool eq = true;
#pragma unroll
    for (int j = 0; j < NL; j++) eq &= __ldg(kp + j) == C.v[j];
    if (eq) { *count = c; return true; }
  }
  return false;
}

template <int NL>
__global__ void __launch_bounds__(kBlock) k_count_pass(ReadsView R, unsigned k, FastMod fm,
                                                        const uint64_t* __restrict__ twice,
                                                        TableView t,
                                                        unsigned long long* __restrict__ adm_out) {
  uint64_t adm = 0;
  const unsigned lane = threadIdx.x & 31;
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
    const unsigned am = __ballot_sync(FULL, admitted);
    if (admitted) {
      adm++;
      // Equal keys in the warp (repeats, hot k-mers) become one atomic add.
      unsigned peers = am;
#pragma unroll
      for (int j = 0; j < NL; j++) peers &= __match_any_sync(am, (unsigned long long)C.v[j]);
      if (lane == (unsigned)(__ffs(peers) - 1)) table_add<NL>(t, C, table_home<NL>(t, raw0), __popc(peers));
    }
  };
  foreach_position(R, k, fn);
  warp_add_u64(adm_out, adm);
}

// ---------------------------------------------------------------------------
// 4. Count histogram and the adaptive cutoff (src/assemble.rs:692-735)
// ---------------------------------------------------------------------------
constexpr int kHistBins = 256;  // counts >= 255 share the last bin

__global__ void __launch_bounds__(kBlock) k_table_hist(const uint32_t* __restrict__ counts,
                                                        uint64_t cap,
                                                        unsigned long long* __restrict__ hist) {
  __shared__ unsigned sh[kHistBins];
  for (int i = threadIdx.x; i < kHistBins; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < cap;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t c = counts[i];
    if (c) atomicAdd(&sh[c < kHistBins - 1 ? c : kHistBins - 1], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kHistBins; i += blockDim.x)
    if (sh[i]) atomicAdd(hist + i, (unsigned long long)sh[i]);
}

// params: [0] fixed cutoff (0 = adaptive), [1] list_min_count
// out:    [0] cutoff, [1] list threshold
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
// 5. Stream compaction of the table into the SoA k-mer list.
// counters: [0] list length, [1] solid (>= cutoff), [2] count == 1, [3] occupied
// ---------------------------------------------------------------------------
template <int NL>
__global__ void __launch_bounds__(kBlock) k_compact(TableView t, const uint32_t* __restrict__ thr,
                                                     uint64_t* o0, uint64_t* o1, uint64_t* o2,
                                                     uint64_t* o3, uint32_t* __restrict__ ocnt,
                                                     unsigned long long* __restrict__ counters) {
  const uint32_t cutoff = thr[0], lmin = thr[1];
  const unsigned lane = threadIdx.x & 31;
  uint64_t nsolid = 0, nsingle = 0, nocc = 0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  // Uniform trip count per warp so the ballot below sees every lane.
  const uint64_t start = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  for (uint64_t base = start - lane; base < t.capacity; base += stride) {
    const uint64_t s = base + lane;
    const uint32_t c = s < t.capacity ? t.counts[s] : 0u;
    nocc += c != 0;
    nsolid += c >= cutoff && c != 0;
    nsingle += c == 1;
    const bool keep = c != 0 && c >= lmin;
    const unsigned m = __ballot_sync(FULL, keep);
    if (!m) continue;
    unsigned long long pos0 = 0;
    if (lane == (unsigned)(__ffs(m) - 1)) pos0 = atomicAdd(counters + 0, (unsigned long long)__popc(m));
    pos0 = __shfl_sync(FULL, pos0, __ffs(m) - 1);
    if (keep) {
      const uint64_t p = pos0 + __popc(m & lanemask_lt());
      const uint64_t* kp = t.keys + (uint64_t)t.stride * s;
      o0[p] = kp[0];
      if (NL > 1) o1[p] = kp[1];
      if (NL > 2) o2[p] = kp[2];
      if (NL > 3) o3[p] = kp[3];
      ocnt[p] = c;
    }
  }
  warp_add_u64(counters + 1, nsolid);
  warp_add_u64(counters + 2, nsingle);
  warp_add_u64(counters + 3, nocc);
}

// ---------------------------------------------------------------------------
// 7. (k+1)-mer edges (src/graph.rs:78-102 with OrientedKmer::explicit_seq
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
                                                   unsigned k, FastMod fm, uint64_t* e0,
                                                   uint64_t* e1, uint64_t* e2, uint64_t* e3,
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
      if (NL > 1) S.v[1] = l1[i];
      if (NL > 2) S.v[2] = l2[i];
      if (NL > 3) S.v[3] = l3[i];
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
          uint64_t raw[3], pos[3];
          uint64_t w4[4];
          kmer256_limbs<NL>(CN, k, w4);
          HashPre hp = hash_pre(w4);
          raw[0] = hash_seed(hp, kSeed1);
          (void)pos; (void)fm;
          uint32_t c = 0;
          if (table_find<NL>(t, CN, table_home<NL>(t, raw[0]), &c) && c >= cutoff) {
            E = widen_append<NL, NLE>(EX, b);
            emit = seq_le<NLE>(E, revcomp<NLE>(E, k + 1));
          }
        }
        const unsigned m = __ballot_sync(FULL, emit);
        if (!m) continue;
        unsigned long long p0 = 0;
        if (lane == (unsigned)(__ffs(m) - 1)) p0 = atomicAdd(counter, (unsigned long long)__popc(m));
        p0 = __shfl_sync(FULL, p0, __ffs(m) - 1);
        if (emit) {
          const uint64_t p = p0 + __popc(m & lanemask_lt());
          e0[p] = E.v[0];
          if (NLE > 1) e1[p] = E.v[1];
          if (NLE > 2) e2[p] = E.v[2];
          if (NLE > 3) e3[p] = E.v[3];
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
static int grid_for(spk_ctx* ctx, int blocks_per_sm) { return ctx->sm_count * blocks_per_sm; }

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
                         const FastMod& fm, const uint64_t* twice, const TableView& t,
                         unsigned long long* adm) {
  k_count_pass<NL><<<grid_for(ctx, 8), kBlock, 0, st>>>(rv, k, fm, twice, t, adm);
}
template <int NL>
static void launch_compact(spk_ctx* ctx, cudaStream_t st, const TableView& t, const uint32_t* thr,
                           uint64_t* o[4], uint32_t* oc, unsigned long long* counters) {
  k_compact<NL><<<grid_for(ctx, 8), kBlock, 0, st>>>(t, thr, o[0], o[1], o[2], o[3], oc, counters);
}
template <int NL, int NLE>
static void launch_edges_t(spk_ctx* ctx, cudaStream_t st, uint64_t* l[4], const uint32_t* cnt,
                           uint64_t n, const uint32_t* thr, const TableView& t, unsigned k,
                           const FastMod& fm, uint64_t* e[4], unsigned long long* counter) {
  k_edges<NL, NLE><<<grid_for(ctx, 8), kBlock, 0, st>>>(l[0], l[1], l[2], l[3], cnt, n, thr, t, k,
                                                       fm, e[0], e[1], e[2], e[3], counter);
}
static void launch_edges(spk_ctx* ctx, cudaStream_t st, int nl, int nle, uint64_t* l[4],
                         const uint32_t* cnt, uint64_t n, const uint32_t* thr, const TableView& t,
                         unsigned k, const FastMod& fm, uint64_t* e[4],
                         unsigned long long* counter) {
  if (nl == 1 && nle == 1) launch_edges_t<1, 1>(ctx, st, l, cnt, n, thr, t, k, fm, e, counter);
  else if (nl == 1) launch_edges_t<1, 2>(ctx, st, l, cnt, n, thr, t, k, fm, e, counter);
  else if (nl == 2 && nle == 2) launch_edges_t<2, 2>(ctx, st, l, cnt, n, thr, t, k, fm, e, counter);
  else if (nl == 2) launch_edges_t<2, 3>(ctx, st, l, cnt, n, thr, t, k, fm, e, counter);
  else if (nl == 3 && nle == 3) launch_edges_t<3, 3>(ctx, st, l, cnt, n, thr, t, k, fm, e, counter);
  else if (nl == 3) launch_edges_t<3, 4>(ctx, st, l, cnt, n, thr, t, k, fm, e, counter);
  else launch_edges_t<4, 4>(ctx, st, l, cnt, n, thr, t, k, fm, e, counter);
}

static uint64_t next_pow2(uint64_t x) {
  uint64_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

// Table capacity from the Bloom fill.  With m bits and 3 hashes a filter
// holding n items has fill 1 - exp(-3n/m), so n = -(m/3) ln(1 - fill).  The
// twice tier estimates the k-mers seen at least twice (plus collisions, an
// overestimate); singletons admitted by chance add (twice fill)^3 of the
// rest.  Sized for a load factor of at most 1/2.
static uint64_t table_capacity(uint64_t m, uint64_t pop_seen, uint64_t pop_twice) {
  const double md = (double)m;
  const double fs = std::min((double)pop_seen / md, 0.999999);
  const double ft = std::min((double)pop_twice / md, 0.999999);
  const double n_all = -(md / 3.0) * std::log1p(-fs);
  const double n2 = -(md / 3.0) * std::log1p(-ft);
  const double est = n2 + std::max(n_all - n2, 0.0) * ft * ft * ft;
  const uint64_t want = (uint64_t)(est * 2.0) + 1024;
  return std::max<uint64_t>(next_pow2(want), 1024);
}

struct Ev {
  cudaEvent_t e = nullptr;
  Ev() { cudaEventCreate(&e); }
  ~Ev() { if (e) cudaEventDestroy(e); }
};
static float ms_between(const Ev& a, const Ev& b) {
  float ms = 0;
  if (cudaEventElapsedTime(&ms, a.e, b.e) != cudaSuccess) ms = 0;
  return ms;
}

static int alloc_table(KResult& kr, cudaStream_t st, uint64_t cap) {
  const int nl = kr.nl;
  const uint32_t stride = nl == 3 ? 4 : nl;
  int rc;
  if ((rc = kr.tkeys.alloc(cap * stride * 8, st))) return rc;
  if ((rc = kr.tcounts.alloc(cap * 4, st))) return rc;
  SPK_CUDA(cudaMemsetAsync(kr.tkeys.p, 0xFF, cap * stride * 8, st));
  SPK_CUDA(cudaMemsetAsync(kr.tcounts.p, 0, cap * 4, st));
  if (nl >= 3) {
    if ((rc = kr.tstate.alloc(cap * 4, st))) return rc;
    SPK_CUDA(cudaMemsetAsync(kr.tstate.p, 0, cap * 4, st));
  } else {
    kr.tstate.release();
  }
  TableView& t = kr.table;
  t.keys = kr.tkeys.as<uint64_t>();
  t.counts = kr.tcounts.as<uint32_t>();
  t.state = nl >= 3 ? kr.tstate.as<uint32_t>() : nullptr;
  t.capacity = cap;
  t.log2cap = 0;
  while ((1ULL << t.log2cap) < cap) t.log2cap++;
  t.stride = stride;
  t.max_probe = (uint32_t)std::min<uint64_t>(kMaxProbe, cap);
  return SPK_OK;
}

// Scratch layout (u64 words) in the per-k scratch buffer.
enum {
  S_OCC = 0, S_ADM = 1, S_POPS = 2,  /* 2 words */
  S_ERR = 4,                          /* int */
  S_THR = 5,                          /* 2 x u32 */
  S_CNT = 6,                          /* 4 words: list, solid, single, occupied */
  S_EDGES = 10,
  S_HIST = 16,                        /* 256 words */
  S_WORDS = 16 + kHistBins
};

int count_one_k(spk_ctx* ctx, cudaStream_t st, const ReadsView& rv_in, unsigned k,
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
  uint64_t* host = ctx->h_pinned;
  int* errp = (int*)(sw + S_ERR);
  ReadsView rv = rv_in;
  rv.err = errp;

  Ev e0, e1, e2, e3, e4, e5, e6, kb0, kb1, kc0, kc1;
  uint32_t launches = 0;
  SPK_CUDA(cudaEventRecord(e0.e, st));
  // ---- Stage 2 ----
  const bool ref = (o.flags & SPK_F_REF_SOLID) != 0;
  auto stage2 = [&](bool partitioned) -> int {
    int rc2;
    kr.partitioned = partitioned;
    SPK_CUDA(cudaMemsetAsync(sw, 0, 8 * 8, st));  // occ, adm, pops, err
    if (partitioned) {
      SPK_CUDA(cudaEventRecord(kb0.e, st));
      if ((rc2 = bloom_partitioned(ctx, st, rv, k, kr, su + S_OCC, su + S_POPS, errp, host,
                                   &launches, o.max_chunk_occ ? o.max_chunk_occ : kMaxChunkOcc)))
        return rc2;
      SPK_CUDA(cudaEventRecord(kb1.e, st));
    } else {
      if ((rc2 = kr.tiers.alloc(kr.num_words * 16, st))) return rc2;
      SPK_CUDA(cudaMemsetAsync(kr.tiers.p, 0, kr.num_words * 16, st));
      if (ref) {
        if ((rc2 = kr.ref_solid.alloc(kr.num_words * 8, st))) return rc2;
        SPK_CUDA(cudaMemsetAsync(kr.ref_solid.p, 0, kr.num_words * 8, st));
      }
      U128* tiers = kr.tiers.as<U128>();
      unsigned long long* refp = ref ? kr.ref_solid.as<unsigned long long>() : nullptr;
      SPK_CUDA(cudaEventRecord(kb0.e, st));
      switch (nl) {
        case 1: launch_bloom<1>(ctx, st, rv, k, kr.fm, tiers, refp, su + S_OCC); break;
        case 2: launch_bloom<2>(ctx, st, rv, k, kr.fm, tiers, refp, su + S_OCC); break;
        case 3: launch_bloom<3>(ctx, st, rv, k, kr.fm, tiers, refp, su + S_OCC); break;
        default: launch_bloom<4>(ctx, st, rv, k, kr.fm, tiers, refp, su + S_OCC); break;
      }
      SPK_CUDA(cudaGetLastError());
      SPK_CUDA(cudaEventRecord(kb1.e, st));
      if ((rc2 = kr.seen.alloc(kr.num_words * 8, st))) return rc2;
      if ((rc2 = kr.twice.alloc(kr.num_words * 8, st))) return rc2;
      k_tier_finish<<<grid_for(ctx, 4), kBlock, 0, st>>>(tiers, kr.num_words, kr.seen.as<uint64_t>(),
                                                        kr.twice.as<uint64_t>(), su + S_POPS);
      SPK_CUDA(cudaGetLastError());
      kr.tiers.release();
      launches += 2;
    }
    SPK_CUDA(cudaMemcpyAsync(host, sw, 5 * 8, cudaMemcpyDeviceToHost, st));
    SPK_CUDA(cudaStreamSynchronize(st));
    return SPK_OK;
  };
  const bool want_part = !ref && !(o.flags & SPK_F_DIRECT) && partitioned_bloom_ok(kr.num_words);
  if ((rc = stage2(want_part))) return rc;
  if (want_part && ((int)host[S_ERR] & 8)) {
    // A partition received more operations than its region holds (a few
    // k-mers with huge multiplicity): redo Stage 2 with the direct kernel.
    info.stage2_fallback = 1;
    if ((rc = stage2(false))) return rc;
  }
  SPK_CUDA(cudaEventRecord(e1.e, st));
  if ((int)host[S_ERR] & 4)
    return fail(SPK_E_INVALID_ARG, "a read extends past the end of the packed data");
  info.stage2_partitioned = kr.partitioned ? 1 : 0;
  info.occurrences = host[S_OCC];
  info.seen_popcount = host[S_POPS];
  info.twice_popcount = host[S_POPS + 1];

  // ---- Stage 3 ----
  uint64_t cap = o.table_log2 ? (1ULL << std::min<uint32_t>(o.table_log2, 40))
                              : table_capacity(size_bits, info.seen_popcount, info.twice_popcount);
  for (int attempt = 0;; attempt++) {
    if ((rc = alloc_table(kr, st, cap))) return rc;
    kr.table.err = errp;
    SPK_CUDA(cudaMemsetAsync(sw + S_ADM, 0, 8, st));
    SPK_CUDA(cudaMemsetAsync(errp, 0, 8, st));
    SPK_CUDA(cudaEventRecord(kc0.e, st));
    switch (nl) {
      case 1: launch_count<1>(ctx, st, rv, k, kr.fm, kr.twice.as<uint64_t>(), kr.table, su + S_ADM); break;
      case 2: launch_count<2>(ctx, st, rv, k, kr.fm, kr.twice.as<uint64_t>(), kr.table, su + S_ADM); break;
      case 3: launch_count<3>(ctx, st, rv, k, kr.fm, kr.twice.as<uint64_t>(), kr.table, su + S_ADM); break;
      default: launch_count<4>(ctx, st, rv, k, kr.fm, kr.twice.as<uint64_t>(), kr.table, su + S_ADM); break;
    }
    SPK_CUDA(cudaGetLastError());
    SPK_CUDA(cudaEventRecord(kc1.e, st));
    launches++;
    SPK_CUDA(cudaMemcpyAsync(host, sw, 5 * 8, cudaMemcpyDeviceToHost, st));
    SPK_CUDA(cudaStreamSynchronize(st));
    const int err = (int)host[S_ERR];
    if (err & 2) return fail(SPK_E_TIMEOUT, "count table: claim wait timed out");
    if (!(err & 1)) break;
    if (attempt >= 24) return fail(SPK_E_TABLE_FULL, "count table overflow after regrow attempts");
    cap *= 2;
    info.table_regrows++;
  }
  info.admitted_occurrences = host[S_ADM];
  info.table_capacity = cap;
  SPK_CUDA(cudaEventRecord(e2.e, st));

  // ---- cutoff + compaction ----
  k_table_hist<<<grid_for(ctx, 4), kBlock, 0, st>>>(kr.table.counts, cap, su + S_HIST);
  uint32_t fixed = o.min_count;
  if (!fixed && o.min_coverage > 5.0) {  // src/assemble.rs:693-694
    double v = std::max(o.min_coverage * 0.35, 2.0);
    fixed = v >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)v;
  }
  uint32_t* thr = (uint32_t*)(sw + S_THR);
  k_cutoff<<<1, 32, 0, st>>>(su + S_HIST, fixed, o.list_min_count ? o.list_min_count : 2, thr);
  uint64_t* lp[4] = {nullptr, nullptr, nullptr, nullptr};
  for (int j = 0; j < nl; j++) {
    if ((rc = kr.list[j].alloc(cap * 8, st))) return rc;
    lp[j] = kr.list[j].as<uint64_t>();
  }
  if ((rc = kr.list[4].alloc(cap * 4, st))) return rc;
  switch (nl) {
    case 1: launch_compact<1>(ctx, st, kr.table, thr, lp, kr.list[4].as<uint32_t>(), su + S_CNT); break;
    case 2: launch_compact<2>(ctx, st, kr.table, thr, lp, kr.list[4].as<uint32_t>(), su + S_CNT); break;
    case 3: launch_compact<3>(ctx, st, kr.table, thr, lp, kr.list[4].as<uint32_t>(), su + S_CNT); break;
    default: launch_compact<4>(ctx, st, kr.table, thr, lp, kr.list[4].as<uint32_t>(), su + S_CNT); break;
  }
  SPK_CUDA(cudaGetLastError());
  launches += 3;
  SPK_CUDA(cudaEventRecord(e3.e, st));
  SPK_CUDA(cudaMemcpyAsync(host, sw, S_EDGES * 8, cudaMemcpyDeviceToHost, st));
  SPK_CUDA(cudaStreamSynchronize(st));
  const uint32_t* hthr = (const uint32_t*)(host + S_THR);
  info.cutoff = hthr[0];
  kr.list_min = hthr[1];
  info.n_list = host[S_CNT + 0];
  info.n_solid = host[S_CNT + 1];
  info.n_singletons = host[S_CNT + 2];
  info.n_table = host[S_CNT + 3];

  // ---- sort ----
  if ((rc = radix_sort_bufs(st, nl, info.n_list, 2 * k, kr.list, &kr.list[4], &launches))) return rc;
  for (int j = 0; j < nl; j++) lp[j] = kr.list[j].as<uint64_t>();
  SPK_CUDA(cudaEventRecord(e4.e, st));

  // ---- edges ----
  kr.nle = (int)((k + 1 + 31) / 32);
  if ((o.flags & SPK_F_EDGES) && info.n_solid > 0) {
    uint64_t* ep[4] = {nullptr, nullptr, nullptr, nullptr};
    const uint64_t ecap = info.n_solid * 8;
    for (int j = 0; j < kr.nle; j++) {
      if ((rc = kr.edges[j].alloc(ecap * 8, st))) return rc;
      ep[j] = kr.edges[j].as<uint64_t>();
    }
    launch_edges(ctx, st, nl, kr.nle, lp, kr.list[4].as<uint32_t>(), info.n_list, thr, kr.table, k,
                 kr.fm, ep, su + S_EDGES);
    SPK_CUDA(cudaGetLastError());
    launches++;
    SPK_CUDA(cudaMemcpyAsync(host + S_EDGES, sw + S_EDGES, 8, cudaMemcpyDeviceToHost, st));
    SPK_CUDA(cudaStreamSynchronize(st));
    info.n_edges = host[S_EDGES];
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
  info.ms_count_kernel = ms_between(kc0, kc1);
  info.kernel_launches = launches;
  return SPK_OK;
}

int count_pipeline(spk_ctx* ctx, cudaStream_t st, const ReadsView& rv, uint32_t max_len,
                   const uint32_t* ks, int n_k, const spk_count_opts& o, spk_result* res) {
  (void)max_len;
  for (int i = 0; i < n_k; i++) {
    auto kr = std::make_unique<KResult>();
    int rc = count_one_k(ctx, st, rv, ks[i], o, *kr);
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
                           res->ctx->h_pinned, &m);
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
  return copy_out(res, kr.nl, kr.list, kr.list[4].as<uint32_t>(), kr.info.n_list, kr.k, minc,
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
