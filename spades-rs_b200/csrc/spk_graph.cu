// spk_graph.cu -- unitigs of the solid k-mers on the device:
// CompactedGraph::build (src/graph.rs:65-235), compacting the de Bruijn graph
// of the solid k-mers into maximal non-branching paths.
//
// Nodes are oriented solid k-mers, v = 2i + o for solid k-mer i (sorted list
// order) in orientation o (0: the canonical sequence, 1: its reverse
// complement; OrientedKmer, src/graph.rs:14-40).  The successors of a node
// are the solid k-mers of its four right extensions (src/graph.rs:78-90); the
// predecessors of v are the twins of the successors of its twin (v ^ 1).
// The reference extends a path from u to w while u has one successor w, w has
// one predecessor and w is a k-mer not yet on a path (src/graph.rs:104-157).
// Those links (u -> w with w a different k-mer) give every node at most one
// link in and out, so the linked components are chains and cycles, and every
// chain comes with its twin (the reverse-complement chain).  The reference
// outputs one of each twin pair; an isolated cycle is cut where its walk
// starts (src/graph.rs:219-231).
//
// Device steps: solid list -> successors by binary search in the sorted list
// -> links -> list ranking by pointer jumping (head and rank of every node)
// -> cycles found, cut at their smallest k-mer in forward orientation (where
// the reference's walk in sorted order starts) and their twins dropped ->
// one chain per twin pair -> sequences spelled in place.  The host then puts
// each unitig in the orientation not greater than its reverse complement and
// sorts them by sequence (the reference's order depends on its hasher).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "spk_internal.h"

namespace spk {

constexpr uint32_t kNil = 0xFFFFFFFFu;
constexpr int kUgBlock = 256;

struct SolidView {
  const uint64_t* l[4];  // key limbs (sequence values, SoA), sorted
  const uint32_t* cnt;
  uint32_t n;
  const uint32_t* first;  // first list index of every bucket (top `bbits` bits), 2^bbits + 1
  uint32_t bbits;
};

// Bucket of a sequence value: its top bbits bits of 2k.
template <int NL>
__device__ __forceinline__ uint32_t ug_bucket(const Seq<NL>& V, unsigned k, unsigned bbits) {
  const uint64_t top = 2u * k >= 64u ? bits64<NL>(V, 2u * k - 64u) : (V.v[0] << (64u - 2u * k));
  return (uint32_t)(top >> (64u - bbits));
}

// Index of key C in the sorted solid list, or kNil: a binary search inside
// the bucket of C.
template <int NL>
__device__ __forceinline__ uint32_t ug_find(const SolidView& S, const Seq<NL>& C, unsigned k) {
  const uint32_t b = ug_bucket<NL>(C, k, S.bbits);
  uint32_t lo = __ldg(S.first + b), hi = __ldg(S.first + b + 1);
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    int cmp = 0;  // key(mid) vs C, most significant limb first
#pragma unroll
    for (int j = NL - 1; j >= 0; j--) {
      if (cmp == 0) {
        const uint64_t a = __ldg(S.l[j] + mid);
        cmp = a < C.v[j] ? -1 : (a > C.v[j] ? 1 : 0);
      }
    }
    if (cmp == 0) return mid;
    if (cmp < 0) lo = mid + 1;
    else hi = mid;
  }
  return kNil;
}

template <int NL>
__device__ __forceinline__ Seq<NL> ug_key(const SolidView& S, uint32_t i) {
  Seq<NL> K;
#pragma unroll
  for (int j = 0; j < NL; j++) K.v[j] = __ldg(S.l[j] + i);
  return K;
}

// The solid entries (count >= cutoff) of the sorted list, in order.
__global__ void k_ug_flags(const uint32_t* __restrict__ cnt, uint64_t n, uint32_t cutoff,
                           uint32_t* __restrict__ pos) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    pos[i] = cnt[i] >= cutoff ? 1u : 0u;
}
template <int NL>
__global__ void k_ug_compact(const uint64_t* l0, const uint64_t* l1, const uint64_t* l2, const uint64_t* l3,
                             const uint32_t* __restrict__ cnt, uint64_t n, uint32_t cutoff,
                             const uint32_t* __restrict__ pos, uint64_t* s0, uint64_t* s1, uint64_t* s2,
                             uint64_t* s3, uint32_t* __restrict__ scnt) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    if (cnt[i] < cutoff) continue;
    const uint32_t p = pos[i];
    s0[p] = l0[i];
    if (NL > 1) s1[p] = l1[i];
    if (NL > 2) s2[p] = l2[i];
    if (NL > 3) s3[p] = l3[i];
    scnt[p] = cnt[i];
  }
}

// first[b] = the first index whose bucket is >= b, for b in [0, 2^bbits].
template <int NL>
__global__ void k_ug_buckets(SolidView S, unsigned k, uint32_t* __restrict__ first) {
  const uint32_t nb = 1u << S.bbits;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i <= S.n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t hi = i < S.n ? ug_bucket<NL>(ug_key<NL>(S, (uint32_t)i), k, S.bbits) : nb;
    const uint32_t lo = i > 0 ? ug_bucket<NL>(ug_key<NL>(S, (uint32_t)(i - 1)), k, S.bbits) + 1 : 0;
    for (uint32_t b = lo; b <= hi; b++) first[b] = (uint32_t)i;
  }
}

// Successor count and, when it is one, the successor of every node
// (src/graph.rs:78-90 with canonical(), src/dna.rs:185-192: ties keep fwd).
template <int NL>
__global__ void __launch_bounds__(kUgBlock) k_ug_succ(SolidView S, unsigned k, uint8_t* __restrict__ nsucc,
                                                       uint32_t* __restrict__ succ) {
  const uint64_t n2 = 2ull * S.n;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n2;
       v += (uint64_t)gridDim.x * blockDim.x) {
    const Seq<NL> K = ug_key<NL>(S, (uint32_t)(v >> 1));
    const Seq<NL> RK = revcomp<NL>(K, k);
    const Seq<NL> X = (v & 1) ? RK : K;   // explicit_seq, src/graph.rs:24-30
    const Seq<NL> RX = (v & 1) ? K : RK;
    uint32_t c = 0, t = kNil;
    for (unsigned b = 0; b < 4; b++) {
      const Seq<NL> NB = shl_append<NL>(X, b, k);
      const Seq<NL> RB = shr_prepend<NL>(RX, 3u - b, k);
      const bool rc = !seq_le<NL>(NB, RB);
      const uint32_t j = ug_find<NL>(S, rc ? RB : NB, k);
      if (j != kNil) {
        c++;
        t = 2 * j + (rc ? 1u : 0u);
      }
    }
    nsucc[v] = (uint8_t)c;
    succ[v] = c == 1 ? t : kNil;
  }
}

// Links u -> w: u's only successor is w, w's only predecessor is u (the
// predecessors of w are the twins of the successors of w ^ 1), and w is
// another k-mer.  prev must be all kNil before.
__global__ void k_ug_links(const uint8_t* __restrict__ nsucc, const uint32_t* __restrict__ succ, uint64_t n2,
                           uint32_t* __restrict__ next, uint32_t* __restrict__ prev) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n2;
       v += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t w = succ[v];
    if (w != kNil && (w >> 1) != (uint32_t)(v >> 1) && nsucc[w ^ 1u] == 1) {
      next[v] = w;
      prev[w] = (uint32_t)v;
    } else {
      next[v] = kNil;
    }
  }
}

// List ranking by pointer jumping.  One 16-byte record per node (x: jump
// pointer towards the head, y: distance covered, z: the farthest node
// reached, which is the head once x is kNil), so a round gathers one record.
__global__ void k_ug_rank_init(const uint32_t* __restrict__ prev, uint64_t n2, uint4* __restrict__ A) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n2;
       v += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t p = prev[v];
    A[v] = make_uint4(p, p != kNil ? 1u : 0u, p != kNil ? p : (uint32_t)v, 0u);
  }
}
__global__ void k_ug_rank_step(const uint4* __restrict__ A, uint64_t n2, uint4* __restrict__ B) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n2;
       v += (uint64_t)gridDim.x * blockDim.x) {
    uint4 r = A[v];
    if (r.x != kNil) {
      const uint4 q = A[r.x];
      r = make_uint4(q.x, r.y + q.y, q.z, 0u);
    }
    B[v] = r;
  }
}

// Cycles: nodes whose jump pointer is still set after enough rounds.  Per
// node (x: the smallest node seen so far, y: the node 2^r steps ahead along
// next), by pointer jumping along next; *ncyc counts the nodes on cycles.
__global__ void k_ug_cyc_init(const uint4* __restrict__ A, const uint32_t* __restrict__ next, uint64_t n2,
                              uint2* __restrict__ MC, unsigned long long* __restrict__ ncyc) {
  uint32_t c = 0;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n2;
       v += (uint64_t)gridDim.x * blockDim.x) {
    const bool cyc = A[v].x != kNil;
    MC[v] = cyc ? make_uint2((uint32_t)v, next[v]) : make_uint2(kNil, kNil);
    c += cyc;
  }
  c = __reduce_add_sync(0xffffffffu, c);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(ncyc, (unsigned long long)c);
}
__global__ void k_ug_cyc_step(const uint2* __restrict__ MC, uint64_t n2, uint2* __restrict__ MC2) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n2;
       v += (uint64_t)gridDim.x * blockDim.x) {
    uint2 m = MC[v];
    if (m.y != kNil) {
      const uint2 q = MC[m.y];
      m = make_uint2(min(m.x, q.x), q.y);
    }
    MC2[v] = m;
  }
}
// Cut every cycle before its smallest node; a cycle whose smallest node is a
// reverse orientation is the twin of the cycle holding the forward one and is
// dropped.  flags bit 0: on a cycle, bit 1: dropped.
__global__ void k_ug_cut(const uint2* __restrict__ MC, uint64_t n2, uint32_t* __restrict__ next,
                         uint32_t* __restrict__ prev, uint8_t* __restrict__ flags) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n2;
       v += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t m = MC[v].x;
    if (m == kNil) {
      flags[v] = 0;
      continue;
    }
    flags[v] = (uint8_t)(1u | ((m & 1u) ? 2u : 0u));
    if (m == (uint32_t)v) {
      next[prev[v]] = kNil;
      prev[v] = kNil;
    }
  }
}

// Tails: the kept chains (one per twin pair: the chain whose head is not
// greater than the twin of its tail; cut cycles that were not dropped) and
// their lengths, recorded at their heads.
__global__ void k_ug_tails(const uint32_t* __restrict__ next, const uint4* __restrict__ A,
                           const uint8_t* __restrict__ flags, uint64_t n2, unsigned k,
                           uint32_t* __restrict__ bytes, uint32_t* __restrict__ keep,
                           uint32_t* __restrict__ len) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n2;
       v += (uint64_t)gridDim.x * blockDim.x) {
    if (next[v] != kNil) continue;
    const uint4 a = A[v];
    const uint32_t h = a.z;
    const bool cyc = flags[v] & 1u;
    const bool kept = cyc ? !(flags[v] & 2u) : h <= ((uint32_t)v ^ 1u);
    if (!kept) continue;
    keep[h] = 1;
    len[h] = a.y + 1;
    bytes[h] = a.y + k;
  }
}

// Spell every kept chain in place: node v (at rank D[v]) writes the last base
// of its sequence at offset(head) + k - 1 + D[v]; the head also writes its
// first k - 1 bases (build_unitig, src/graph.rs:159-177).  Coverage sums per
// unitig (kmer_cov of each k-mer, src/graph.rs:162-168).
template <int NL>
__global__ void __launch_bounds__(kUgBlock) k_ug_spell(SolidView S, unsigned k, const uint4* __restrict__ A,
                                                        const uint32_t* __restrict__ keep,
                                                        const uint32_t* __restrict__ off,
                                                        const uint32_t* __restrict__ uidx,
                                                        const uint32_t* __restrict__ len, uint64_t n2,
                                                        char* __restrict__ seq,
                                                        unsigned long long* __restrict__ cov,
                                                        uint32_t* __restrict__ ulen) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n2;
       v += (uint64_t)gridDim.x * blockDim.x) {
    const uint4 a = A[v];
    const uint32_t h = a.z;
    if (!keep[h]) continue;
    const uint32_t i = (uint32_t)(v >> 1);
    const Seq<NL> K = ug_key<NL>(S, i);
    const Seq<NL> X = (v & 1) ? revcomp<NL>(K, k) : K;
    const uint32_t o = off[h];
    seq[o + k - 1 + a.y] = "ACGT"[X.v[0] & 3];
    if (h == (uint32_t)v) {
      ulen[uidx[h]] = len[h];
      for (unsigned p = 0; p + 1 < k; p++) {
        const unsigned sh = 2u * (k - 1 - p);  // bit of base p
        uint64_t w = 0;
#pragma unroll
        for (int j = 0; j < NL; j++)
          if ((unsigned)j == (sh >> 6)) w = X.v[j];
        seq[o + p] = "ACGT"[(w >> (sh & 63)) & 3];
      }
    }
    atomicAdd(cov + uidx[h], (unsigned long long)__ldg(S.cnt + i));
  }
}

static unsigned ug_grid(spk_ctx* ctx) { return (unsigned)ctx->sm_count * 8; }

template <int NL>
static int ug_run(spk_ctx* ctx, cudaStream_t st, KResult& kr, uint32_t* launches, UnitigSet& out,
                  cudaEvent_t e_end) {
  const unsigned k = kr.k;
  const uint32_t cutoff = kr.info.cutoff;
  const uint64_t nl_list = kr.list_len;
  const unsigned g = ug_grid(ctx);
  int rc;
  // ---- solid list ----
  DevBuf pos, sums;
  if ((rc = pos.alloc(std::max<uint64_t>(nl_list, 1) * 4 + 4, st))) return rc;
  SPK_CUDA(cudaMemsetAsync(pos.p, 0, std::max<uint64_t>(nl_list, 1) * 4 + 4, st));
  k_ug_flags<<<g, kUgBlock, 0, st>>>(kr.list[4].as<uint32_t>(), nl_list, cutoff, pos.as<uint32_t>());
  if ((rc = scan_u32(st, pos.as<uint32_t>(), nl_list + 1, sums, launches))) return rc;
  uint32_t hn = 0;
  SPK_CUDA(cudaMemcpyAsync(&hn, pos.as<uint32_t>() + nl_list, 4, cudaMemcpyDeviceToHost, st));
  SPK_CUDA(cudaStreamSynchronize(st));
  const uint64_t n = hn;
  if (n == 0) {
    SPK_CUDA(cudaEventRecord(e_end, st));
    return SPK_OK;
  }
  if (2 * n >= kNil) return fail(SPK_E_INVALID_ARG, "unitigs: more than 2^31 solid k-mers");
  DevBuf sl[4], scnt;
  for (int j = 0; j < NL; j++)
    if ((rc = sl[j].alloc(n * 8, st))) return rc;
  if ((rc = scnt.alloc(n * 4, st))) return rc;
  uint64_t* lp[4] = {nullptr, nullptr, nullptr, nullptr};
  uint64_t* sp[4] = {nullptr, nullptr, nullptr, nullptr};
  for (int j = 0; j < NL; j++) {
    lp[j] = kr.list[j].as<uint64_t>();
    sp[j] = sl[j].as<uint64_t>();
  }
  k_ug_compact<NL><<<g, kUgBlock, 0, st>>>(lp[0], lp[1], lp[2], lp[3], kr.list[4].as<uint32_t>(), nl_list,
                                          cutoff, pos.as<uint32_t>(), sp[0], sp[1], sp[2], sp[3],
                                          scnt.as<uint32_t>());
  pos.release();
  // about one k-mer per bucket, 2^8..2^24 buckets
  unsigned bbits = 8;
  while (bbits < 24 && bbits < 2 * k && (1ull << bbits) < n) bbits++;
  DevBuf first;
  if ((rc = first.alloc(((1ull << bbits) + 1) * 4, st))) return rc;
  SolidView S{{sp[0], sp[1], sp[2], sp[3]}, scnt.as<uint32_t>(), (uint32_t)n, first.as<uint32_t>(), bbits};
  k_ug_buckets<NL><<<g, kUgBlock, 0, st>>>(S, k, first.as<uint32_t>());
  // ---- successors and links ----
  const uint64_t n2 = 2 * n;
  DevBuf nsucc, succ, next, prev;
  if ((rc = nsucc.alloc(n2, st)) || (rc = succ.alloc(n2 * 4, st)) || (rc = next.alloc(n2 * 4, st)) ||
      (rc = prev.alloc(n2 * 4, st)))
    return rc;
  k_ug_succ<NL><<<g, kUgBlock, 0, st>>>(S, k, nsucc.as<uint8_t>(), succ.as<uint32_t>());
  first.release();
  SPK_CUDA(cudaMemsetAsync(prev.p, 0xFF, n2 * 4, st));
  k_ug_links<<<g, kUgBlock, 0, st>>>(nsucc.as<uint8_t>(), succ.as<uint32_t>(), n2, next.as<uint32_t>(),
                                     prev.as<uint32_t>());
  nsucc.release();
  succ.release();
  if (launches) *launches += 6;
  // ---- list ranking; cycles found, cut and ranked again ----
  DevBuf A[2];
  for (int b = 0; b < 2; b++)
    if ((rc = A[b].alloc(n2 * 16, st))) return rc;
  int rounds = 1;
  while ((1ull << rounds) < n2) rounds++;
  rounds += 1;
  int cur = 0;
  auto rank = [&]() {
    k_ug_rank_init<<<g, kUgBlock, 0, st>>>(prev.as<uint32_t>(), n2, A[0].as<uint4>());
    cur = 0;
    for (int r = 0; r < rounds; r++) {
      k_ug_rank_step<<<g, kUgBlock, 0, st>>>(A[cur].as<uint4>(), n2, A[cur ^ 1].as<uint4>());
      cur ^= 1;
    }
    if (launches) *launches += 1 + rounds;
  };
  rank();
  DevBuf flags;
  if ((rc = flags.alloc(n2, st))) return rc;
  {
    // A[cur].x != kNil marks the nodes on cycles; find each cycle's smallest node.
    DevBuf MC[2], ncyc;
    for (int b = 0; b < 2; b++)
      if ((rc = MC[b].alloc(n2 * 8, st))) return rc;
    if ((rc = ncyc.alloc(8, st))) return rc;
    SPK_CUDA(cudaMemsetAsync(ncyc.p, 0, 8, st));
    k_ug_cyc_init<<<g, kUgBlock, 0, st>>>(A[cur].as<uint4>(), next.as<uint32_t>(), n2, MC[0].as<uint2>(),
                                          ncyc.as<unsigned long long>());
    unsigned long long hc = 0;
    SPK_CUDA(cudaMemcpyAsync(&hc, ncyc.p, 8, cudaMemcpyDeviceToHost, st));
    SPK_CUDA(cudaStreamSynchronize(st));
    if (launches) *launches += 1;
    if (hc == 0) {
      SPK_CUDA(cudaMemsetAsync(flags.p, 0, n2, st));  // no cycles: the ranking stands
    } else {
      int c = 0;
      for (int r = 0; r < rounds; r++) {
        k_ug_cyc_step<<<g, kUgBlock, 0, st>>>(MC[c].as<uint2>(), n2, MC[c ^ 1].as<uint2>());
        c ^= 1;
      }
      k_ug_cut<<<g, kUgBlock, 0, st>>>(MC[c].as<uint2>(), n2, next.as<uint32_t>(), prev.as<uint32_t>(),
                                       flags.as<uint8_t>());
      if (launches) *launches += 1 + rounds;
      rank();
    }
  }
  // ---- kept chains, offsets, spelling ----
  DevBuf bytes, keep, len, uidx;
  if ((rc = bytes.alloc(n2 * 4 + 4, st)) || (rc = keep.alloc(n2 * 4 + 4, st)) || (rc = len.alloc(n2 * 4, st)) ||
      (rc = uidx.alloc(n2 * 4 + 4, st)))
    return rc;
  SPK_CUDA(cudaMemsetAsync(bytes.p, 0, n2 * 4 + 4, st));
  SPK_CUDA(cudaMemsetAsync(keep.p, 0, n2 * 4 + 4, st));
  k_ug_tails<<<g, kUgBlock, 0, st>>>(next.as<uint32_t>(), A[cur].as<uint4>(), flags.as<uint8_t>(), n2, k,
                                     bytes.as<uint32_t>(), keep.as<uint32_t>(), len.as<uint32_t>());
  SPK_CUDA(cudaMemcpyAsync(uidx.p, keep.p, n2 * 4 + 4, cudaMemcpyDeviceToDevice, st));
  if ((rc = scan_u32(st, uidx.as<uint32_t>(), n2 + 1, sums, launches))) return rc;
  uint32_t hv[2] = {0, 0};
  SPK_CUDA(cudaMemcpyAsync(hv, uidx.as<uint32_t>() + n2, 4, cudaMemcpyDeviceToHost, st));
  SPK_CUDA(cudaStreamSynchronize(st));
  const uint64_t nu = hv[0];
  // Spelled bytes: every k-mer adds one base, every unitig k - 1 more.
  const uint64_t total = n + nu * (k - 1);
  if (total >= (1ull << 32)) return fail(SPK_E_INVALID_ARG, "unitigs: more than 2^32 spelled bases");
  if ((rc = scan_u32(st, bytes.as<uint32_t>(), n2 + 1, sums, launches))) return rc;
  DevBuf seq, cov, ulen;
  if ((rc = seq.alloc(std::max<uint64_t>(total, 1), st)) || (rc = cov.alloc(std::max<uint64_t>(nu, 1) * 8, st)) ||
      (rc = ulen.alloc(std::max<uint64_t>(nu, 1) * 4, st)))
    return rc;
  SPK_CUDA(cudaMemsetAsync(cov.p, 0, std::max<uint64_t>(nu, 1) * 8, st));
  k_ug_spell<NL><<<g, kUgBlock, 0, st>>>(S, k, A[cur].as<uint4>(), keep.as<uint32_t>(), bytes.as<uint32_t>(), uidx.as<uint32_t>(),
                                        len.as<uint32_t>(), n2, seq.as<char>(), cov.as<unsigned long long>(),
                                        ulen.as<uint32_t>());
  SPK_CUDA(cudaGetLastError());
  if (launches) *launches += 3;
  // ---- to the host; each unitig in the orientation not greater than its
  // reverse complement, sorted by sequence ----
  std::vector<uint32_t> h_len(nu);
  std::string h_seq(total, '\0');
  std::vector<unsigned long long> h_cov(nu);
  if (nu) {
    SPK_CUDA(cudaMemcpyAsync(h_len.data(), ulen.p, nu * 4, cudaMemcpyDeviceToHost, st));
    SPK_CUDA(cudaMemcpyAsync(&h_seq[0], seq.p, total, cudaMemcpyDeviceToHost, st));
    SPK_CUDA(cudaMemcpyAsync(h_cov.data(), cov.p, nu * 8, cudaMemcpyDeviceToHost, st));
  }
  SPK_CUDA(cudaEventRecord(e_end, st));
  SPK_CUDA(cudaStreamSynchronize(st));
  const auto t0 = std::chrono::steady_clock::now();
  std::vector<uint64_t> off(nu + 1, 0);
  for (uint64_t u = 0; u < nu; u++) off[u + 1] = off[u] + h_len[u] + k - 1;
  if (off[nu] != total) return fail(SPK_E_CUDA, "unitigs: spelled length mismatch");
  char kComp[256] = {};
  kComp['A'] = 'T';
  kComp['C'] = 'G';
  kComp['G'] = 'C';
  kComp['T'] = 'A';
  std::vector<std::string> seqs(nu);
  for (uint64_t u = 0; u < nu; u++) {
    const char* f = h_seq.data() + off[u];
    const size_t L = off[u + 1] - off[u];
    // compare the sequence with its reverse complement without building it
    int c = 0;
    for (size_t i = 0; i < L && c == 0; i++) {
      const char r = kComp[(unsigned char)f[L - 1 - i]];
      c = r < f[i] ? -1 : (r > f[i] ? 1 : 0);
    }
    if (c < 0) {
      seqs[u].resize(L);
      for (size_t i = 0; i < L; i++) seqs[u][i] = kComp[(unsigned char)f[L - 1 - i]];
    } else {
      seqs[u].assign(f, L);
    }
  }
  std::vector<size_t> ord(nu);
  std::iota(ord.begin(), ord.end(), 0);
  std::sort(ord.begin(), ord.end(), [&](size_t a, size_t b) { return seqs[a] < seqs[b]; });
  out.seq.clear();
  out.seq.reserve(total);
  out.lengths.assign(nu, 0);
  out.cov.assign(nu, 0.0);
  out.kmers.assign(nu, 0);
  for (uint64_t r = 0; r < nu; r++) {
    const size_t u = ord[r];
    out.seq += seqs[u];
    out.lengths[r] = seqs[u].size();
    out.kmers[r] = h_len[u];
    out.cov[r] = (double)h_cov[u] / (double)h_len[u];
  }
  out.ms_host = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return SPK_OK;
}

int build_unitigs(spk_result* res, int ki) {
  KResult& kr = *res->ks[ki];
  if (kr.unitigs.ready) return SPK_OK;
  if ((kr.k & 1) == 0) return fail(SPK_E_INVALID_ARG, "unitigs need an odd k");
  cudaStream_t st = res->stream;
  cudaEvent_t e0, e1;
  SPK_CUDA(cudaEventCreate(&e0));
  SPK_CUDA(cudaEventCreate(&e1));
  UnitigSet u;
  int rc = SPK_OK;
  if (cudaEventRecord(e0, st) != cudaSuccess) rc = fail(SPK_E_CUDA, "event record");
  if (!rc) {
    switch (kr.nl) {
      case 1: rc = ug_run<1>(res->ctx, st, kr, &u.launches, u, e1); break;
      case 2: rc = ug_run<2>(res->ctx, st, kr, &u.launches, u, e1); break;
      case 3: rc = ug_run<3>(res->ctx, st, kr, &u.launches, u, e1); break;
      default: rc = ug_run<4>(res->ctx, st, kr, &u.launches, u, e1); break;
    }
  }
  if (!rc && cudaEventSynchronize(e1) == cudaSuccess) cudaEventElapsedTime(&u.ms_device, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  u.ready = true;
  kr.unitigs = std::move(u);
  return SPK_OK;
}

}  // namespace spk

using namespace spk;

extern "C" int spk_result_unitigs(spk_result* res, int k_index, char* seqs, uint64_t* seq_bytes,
                                  uint64_t* lengths, double* mean_coverage, uint64_t* kmers_count,
                                  uint64_t* n_inout) {
  if (!res) return fail(SPK_E_INVALID_ARG, "null result");
  if (k_index < 0 || k_index >= (int)res->ks.size()) return fail(SPK_E_INVALID_ARG, "k index out of range");
  if (!n_inout || !seq_bytes) return fail(SPK_E_INVALID_ARG, "null size pointer");
  SPK_CUDA(cudaSetDevice(res->ctx->device));
  int rc = build_unitigs(res, k_index);
  if (rc) return rc;
  const UnitigSet& u = res->ks[k_index]->unitigs;
  const uint64_t n = u.lengths.size(), b = u.seq.size();
  if (!seqs && !lengths && !mean_coverage && !kmers_count) {
    *n_inout = n;
    *seq_bytes = b;
    return SPK_OK;
  }
  if (*n_inout < n || (seqs && *seq_bytes < b)) {
    *n_inout = n;
    *seq_bytes = b;
    return fail(SPK_E_INVALID_ARG, "output buffer too small");
  }
  if (seqs && b) memcpy(seqs, u.seq.data(), b);
  if (lengths) memcpy(lengths, u.lengths.data(), n * 8);
  if (mean_coverage) memcpy(mean_coverage, u.cov.data(), n * 8);
  if (kmers_count) memcpy(kmers_count, u.kmers.data(), n * 8);
  *n_inout = n;
  *seq_bytes = b;
  return SPK_OK;
}
