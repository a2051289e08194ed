// spk_part.cu -- Stage 2 (Bloom population) as partition-and-apply.
//
// The reference sets three Bloom bits per k-mer occurrence with random 64-bit
// fetch_or on two 64 MiB tiers (src/bloom.rs:95-106).  On B200 those random
// accesses miss L2 and cost one DRAM sector each.  Here the work is split in
// two streaming kernels:
//   k_stream_ops   walks the reads once, computes the three bit positions of
//                  every canonical k-mer and appends them, staged in shared
//                  memory, to one of P partitions (8192 words = 512 Ki bits of
//                  the filter each);
//   k_bloom_apply  gives each partition to one CTA, which builds the seen and
//                  twice words of its 8192-word slice in shared memory and
//                  writes them out once.
// The seen/twice state of a bit depends only on how many operations hit it
// (at least one / at least two), not on their order, so applying the
// operations grouped by partition gives exactly the tiers of the serial
// insertion order (the seen tier bit-exact with the reference).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "spk_internal.h"

namespace spk {

constexpr unsigned FULLP = 0xffffffffu;
constexpr int SO_BLOCK = 512;
constexpr uint32_t kPartBits = 19;                 // 512 Ki bits per partition
constexpr uint32_t kPartWords = 1u << (kPartBits - 6);
constexpr uint32_t kNoOp = 0xFFFFFFFFu;
constexpr uint32_t kChunk = 64;                    // slots a CTA claims per partition at a time
constexpr uint32_t kMaxParts = 4096;
constexpr int AP_BLOCK = 1024;

struct OpSink {
  uint32_t* ops;              // P regions of `cap` operations
  unsigned long long* cur;    // per-partition claimed slots (relative)
  uint64_t cap;
  uint32_t parts;
  int* err;                   // bit 3: a partition region overflowed
};

// Per-CTA bump allocation of partition slots.  s_cur[b]/s_end[b] delimit the
// CTA's current chunk of partition b.  An operation takes a slot with one
// shared atomic and stores straight to global memory; the L2 merges the
// 4-byte stores of all CTAs into full sectors.  Operations that find their
// chunk exhausted go to a small overflow list and are placed at the next
// CTA-wide refill, which claims `overflow + kChunk` slots at once.
struct Bump {
  uint32_t* s_cur;   // parts
  uint32_t* s_end;   // parts
  uint32_t* s_ovf;   // overflow ops (partition << 32 | bit offset packed as two u32)
  uint32_t* s_ovn;   // [0] overflow count
};

__device__ __forceinline__ void bump_put(const OpSink& S, const Bump& B, uint32_t pos, uint32_t ovf_cap) {
  const uint32_t b = pos >> kPartBits;
  const uint32_t payload = pos & ((1u << kPartBits) - 1);
  const uint32_t r = atomicAdd(&B.s_cur[b], 1u);
  if (r < B.s_end[b]) {
    S.ops[(uint64_t)b * S.cap + r] = payload;
  } else {
    const uint32_t q = atomicAdd(B.s_ovn, 1u);
    if (q < ovf_cap) {
      B.s_ovf[2 * q] = b;
      B.s_ovf[2 * q + 1] = payload;
    } else {
      atomicOr(S.err, 8);  // cannot happen with ovf_cap >= ops per round
    }
  }
}

// CTA-wide: claim new chunks for exhausted partitions, then place the
// overflow list.  Dead partitions (region full) keep s_end = 0 and drop ops.
__device__ __forceinline__ void bump_refill(const OpSink& S, const Bump& B, uint32_t* s_base) {
  __syncthreads();
  const uint32_t nov = min(*B.s_ovn, (uint32_t)(3 * SO_BLOCK));
  if (nov) {
    for (uint32_t b = threadIdx.x; b < S.parts; b += blockDim.x) {
      const uint32_t c = B.s_cur[b], e = B.s_end[b];
      if (c > e) {  // exhausted with (c - e) overflowed operations
        const uint32_t need = c - e;
        const unsigned long long base = atomicAdd(S.cur + b, (unsigned long long)(need + kChunk));
        if (base + need + kChunk > S.cap) {
          atomicOr(S.err, 8);
          s_base[b] = kNoOp;
          B.s_cur[b] = 0;
          B.s_end[b] = 0;
        } else {
          s_base[b] = (uint32_t)base;  // overflow ops take [base, base + need)
          B.s_cur[b] = (uint32_t)base + need;
          B.s_end[b] = (uint32_t)(base + need + kChunk);
        }
      }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < nov; i += blockDim.x) {
      const uint32_t b = B.s_ovf[2 * i], payload = B.s_ovf[2 * i + 1];
      if (s_base[b] == kNoOp) continue;
      const uint32_t r = atomicAdd(&s_base[b], 1u);
      S.ops[(uint64_t)b * S.cap + r] = payload;
    }
    __syncthreads();
    if (threadIdx.x == 0) *B.s_ovn = 0;
  }
  __syncthreads();
}

// One pass over the reads: three Bloom operations per k-mer occurrence.  The
// CTA walks groups of SO_BLOCK reads; each warp scans its 32 reads and all
// warps step through positions in lockstep rounds (so refills can be
// CTA-wide).
template <int NL>
__global__ void __launch_bounds__(SO_BLOCK) k_stream_ops(ReadsView R, unsigned k, FastMod fm,
                                                         OpSink S,
                                                         unsigned long long* __restrict__ occ_out) {
  extern __shared__ uint32_t smem[];
  Bump B;
  B.s_cur = smem;
  B.s_end = smem + S.parts;
  uint32_t* s_base = smem + 2 * S.parts;
  B.s_ovf = smem + 3 * S.parts;               // 2 * 3 * SO_BLOCK
  B.s_ovn = smem + 3 * S.parts + 6 * SO_BLOCK;
  __shared__ uint32_t s_rounds;
  for (uint32_t b = threadIdx.x; b < S.parts; b += blockDim.x) {
    B.s_cur[b] = 0;
    B.s_end[b] = 0;
  }
  if (threadIdx.x == 0) *B.s_ovn = 0;
  __syncthreads();
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint64_t occ = 0;
  for (uint64_t g = (uint64_t)blockIdx.x * SO_BLOCK; g < R.n_reads; g += (uint64_t)gridDim.x * SO_BLOCK) {
    const uint64_t r = g + warp * 32 + lane;
    uint32_t len = 0;
    uint64_t off = 0;
    if (r < R.n_reads) {
      len = __ldg(R.lengths + r);
      off = __ldg(R.offsets + r);
      if (off + ((uint64_t)len + 3) / 4 > R.data_len) {
        atomicOr(R.err, 4);
        len = 0;
      }
    }
    const uint32_t np = len >= k ? len - k + 1 : 0;
    uint32_t incl = np;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      uint32_t t = __shfl_up_sync(FULLP, incl, d);
      if ((int)lane >= d) incl += t;
    }
    const uint32_t excl = incl - np;
    const uint32_t total = __shfl_sync(FULLP, incl, 31);
    if (threadIdx.x == 0) s_rounds = 0;
    __syncthreads();
    if (lane == 0) atomicMax(&s_rounds, (total + 31) / 32);
    __syncthreads();
    const uint32_t rounds = s_rounds;
    for (uint32_t it = 0; it < rounds; it++) {
      const uint32_t p = it * 32 + lane;
      unsigned j = 0;
#pragma unroll
      for (unsigned step = 16; step >= 1; step >>= 1) {
        uint32_t c = __shfl_sync(FULLP, incl, j + step - 1);
        if (p >= c) j += step;
      }
      const uint64_t o = __shfl_sync(FULLP, off, j);
      const uint32_t e = __shfl_sync(FULLP, excl, j);
      if (p < total) {
        occ++;
        const uint64_t bitpos = 8ull * (R.byte_base + o) + 2ull * (uint64_t)(p - e);
        const Seq<NL> V = extract<NL>(R.words, bitpos, k);
        const Seq<NL> C = canonical<NL>(V, k);
        uint64_t w4[4];
        kmer256_limbs<NL>(C, k, w4);
        const HashPre hp = hash_pre(w4);
        // bit positions < 2^31: partition in bits 19..30, bit offset below
        bump_put(S, B, (uint32_t)fastmod(fm, hash_seed(hp, kSeed1)), 3 * SO_BLOCK);
        bump_put(S, B, (uint32_t)fastmod(fm, hash_seed(hp, kSeed2)), 3 * SO_BLOCK);
        bump_put(S, B, (uint32_t)fastmod(fm, hash_seed(hp, kSeed3)), 3 * SO_BLOCK);
      }
      bump_refill(S, B, s_base);
    }
  }
  // mark the unused tail of every claimed chunk
  for (uint32_t b = threadIdx.x; b < S.parts; b += blockDim.x) {
    const uint32_t c = B.s_cur[b], e = B.s_end[b];
    for (uint32_t q = c; q < e; q++) S.ops[(uint64_t)b * S.cap + q] = kNoOp;
  }
#pragma unroll
  for (int d = 16; d >= 1; d >>= 1) occ += __shfl_xor_sync(FULLP, occ, d);
  if (lane == 0 && occ) atomicAdd(occ_out, (unsigned long long)occ);
}

// Applies every operation of one partition in shared memory and writes the
// partition's seen and twice words (compact arrays) and their popcounts.
// With `accumulate`, the words already in seen/twice are loaded first, so a
// read set may be streamed in several chunks.
__global__ void __launch_bounds__(AP_BLOCK) k_bloom_apply(const uint32_t* __restrict__ ops,
                                                          const unsigned long long* __restrict__ cur,
                                                          uint64_t cap, uint32_t parts,
                                                          uint64_t num_words, int accumulate,
                                                          unsigned long long* __restrict__ seen,
                                                          unsigned long long* __restrict__ twice,
                                                          unsigned long long* __restrict__ pops,
                                                          const int* __restrict__ err) {
  extern __shared__ uint32_t sm[];
  // After an overflow some reserved slots were never written; the host
  // discards this pass and reruns Stage 2 directly, so do nothing here.
  if (*err & 8) return;
  uint32_t* s_seen = sm;                    // 2 * kPartWords u32
  uint32_t* s_twice = sm + 2 * kPartWords;  // 2 * kPartWords u32
  uint64_t cs = 0, ct = 0;
  for (uint32_t b = blockIdx.x; b < parts; b += gridDim.x) {
    const uint64_t w0 = (uint64_t)b * kPartWords;
    const uint64_t left = num_words - w0;
    const uint32_t nw = left < kPartWords ? (uint32_t)left : kPartWords;
    for (uint32_t i = threadIdx.x; i < nw; i += blockDim.x) {
      uint64_t s = 0, t = 0;
      if (accumulate) {
        s = seen[w0 + i];
        t = twice[w0 + i];
      }
      s_seen[2 * i] = (uint32_t)s;
      s_seen[2 * i + 1] = (uint32_t)(s >> 32);
      s_twice[2 * i] = (uint32_t)t;
      s_twice[2 * i + 1] = (uint32_t)(t >> 32);
    }
    __syncthreads();
    const uint64_t n = cur[b] < cap ? (uint64_t)cur[b] : cap;
    const uint32_t* po = ops + (uint64_t)b * cap;
    for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) {
      const uint32_t raw = __ldcs(po + i);
      if (raw == kNoOp) continue;  // unused tail of a claimed chunk
      const uint32_t v = raw & ((1u << kPartBits) - 1);
      const uint32_t bit = 1u << (v & 31);
      const uint32_t prev = atomicOr(&s_seen[v >> 5], bit);
      if (prev & bit) atomicOr(&s_twice[v >> 5], bit);
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < nw; i += blockDim.x) {
      const uint64_t s = (uint64_t)s_seen[2 * i] | ((uint64_t)s_seen[2 * i + 1] << 32);
      const uint64_t t = (uint64_t)s_twice[2 * i] | ((uint64_t)s_twice[2 * i + 1] << 32);
      seen[w0 + i] = s;
      twice[w0 + i] = t;
      cs += __popcll(s);
      ct += __popcll(t);
    }
    __syncthreads();
  }
#pragma unroll
  for (int d = 16; d >= 1; d >>= 1) {
    cs += __shfl_xor_sync(FULLP, cs, d);
    ct += __shfl_xor_sync(FULLP, ct, d);
  }
  if ((threadIdx.x & 31) == 0 && pops) {
    if (cs) atomicAdd(pops + 0, (unsigned long long)cs);
    if (ct) atomicAdd(pops + 1, (unsigned long long)ct);
  }
}

// k-mer occurrences of each unit of `unit` reads (for chunk planning).
__global__ void __launch_bounds__(256) k_occ_units(const uint32_t* __restrict__ lengths,
                                                    uint64_t n_reads, unsigned k, uint64_t unit,
                                                    unsigned long long* __restrict__ out) {
  uint64_t s = 0;
  const uint64_t u = blockIdx.x;
  const uint64_t r0 = u * unit, r1 = min(r0 + unit, n_reads);
  for (uint64_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
    const uint32_t len = lengths[r];
    s += len >= k ? len - k + 1 : 0;
  }
#pragma unroll
  for (int d = 16; d >= 1; d >>= 1) s += __shfl_xor_sync(FULLP, s, d);
  if ((threadIdx.x & 31) == 0 && s) atomicAdd(out + u, (unsigned long long)s);
}

// ---------------------------------------------------------------------------
size_t stream_ops_smem(uint32_t parts) { return (3 * (size_t)parts + 6 * SO_BLOCK + 1) * 4; }

uint32_t bloom_parts(uint64_t num_words) {
  return (uint32_t)((num_words + kPartWords - 1) / kPartWords);
}

// Largest filter the partitioned path takes (the staging histogram must fit
// next to the staging buffer): 4096 partitions = 2 Gi bits per tier.
bool partitioned_bloom_ok(uint64_t num_words) { return bloom_parts(num_words) <= kMaxParts; }

template <int NL>
static int launch_stream(spk_ctx* ctx, cudaStream_t st, const ReadsView& rv, unsigned k,
                         const FastMod& fm, const OpSink& S, unsigned long long* occ) {
  const size_t smem = stream_ops_smem(S.parts);
  SPK_CUDA(cudaFuncSetAttribute(k_stream_ops<NL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem));
  int per_sm = 0;
  SPK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_stream_ops<NL>, SO_BLOCK, smem));
  const uint64_t groups = (rv.n_reads + SO_BLOCK - 1) / SO_BLOCK;
  const uint64_t grid = std::max<uint64_t>(1, std::min<uint64_t>(groups, (uint64_t)ctx->sm_count * std::max(per_sm, 1)));
  k_stream_ops<NL><<<(unsigned)grid, SO_BLOCK, smem, st>>>(rv, k, fm, S, occ);
  SPK_CUDA(cudaGetLastError());
  return SPK_OK;
}

// Stage 2 over device-resident reads: fills kr.seen / kr.twice (compact) and
// the popcounts in pops[0..1]; occurrences are added to *occ.
int bloom_partitioned(spk_ctx* ctx, cudaStream_t st, const ReadsView& rv, unsigned k,
                      KResult& kr, unsigned long long* occ, unsigned long long* pops, int* errp,
                      uint64_t* host, uint32_t* launches, uint64_t max_chunk_occ) {
  const uint32_t parts = bloom_parts(kr.num_words);
  int rc;
  // occurrences per unit of reads -> chunk plan
  const uint64_t unit = 1 << 16;
  const uint64_t nunits = std::max<uint64_t>((rv.n_reads + unit - 1) / unit, 1);
  DevBuf uocc;
  if ((rc = uocc.alloc(nunits * 8, st))) return rc;
  SPK_CUDA(cudaMemsetAsync(uocc.p, 0, nunits * 8, st));
  if (rv.n_reads)
    k_occ_units<<<(unsigned)nunits, 256, 0, st>>>(rv.lengths, rv.n_reads, k, unit,
                                                 uocc.as<unsigned long long>());
  SPK_CUDA(cudaGetLastError());
  std::vector<uint64_t> uo(nunits);
  SPK_CUDA(cudaMemcpyAsync(uo.data(), uocc.p, nunits * 8, cudaMemcpyDeviceToHost, st));
  SPK_CUDA(cudaStreamSynchronize(st));
  *launches += 1;
  // group units into chunks of at most max_chunk_occ occurrences
  std::vector<std::pair<uint64_t, uint64_t>> chunks;  // [unit begin, unit end)
  std::vector<uint64_t> chunk_occ;
  uint64_t acc = 0, ub = 0;
  for (uint64_t u = 0; u < nunits; u++) {
    if (acc && acc + uo[u] > max_chunk_occ) {
      chunks.push_back({ub, u});
      chunk_occ.push_back(acc);
      ub = u;
      acc = 0;
    }
    acc += uo[u];
  }
  chunks.push_back({ub, nunits});
  chunk_occ.push_back(acc);
  uint64_t max_occ = 0;
  for (uint64_t c : chunk_occ) max_occ = std::max(max_occ, c);
  // A full partition receives 3 occ * kPartWords / num_words operations on
  // average (the last one may be shorter).  Genomic k-mers arrive in clumps
  // of ~coverage occurrences, so the spread is far above Poisson: allow 25%,
  // plus one claimed-but-unfilled chunk per CTA.  A region that still
  // overflows makes the host redo Stage 2 with the direct kernel.
  const double mean = 3.0 * (double)max_occ * std::min<double>(1.0, (double)kPartWords / (double)kr.num_words);
  const uint64_t cap = (uint64_t)(mean * 1.25) + (uint64_t)ctx->sm_count * 4 * kChunk * 2 + 65536;
  DevBuf ops, cur;
  if ((rc = ops.alloc(cap * parts * 4, st))) return rc;
  if ((rc = cur.alloc((uint64_t)parts * 8, st))) return rc;
  if ((rc = kr.seen.alloc(kr.num_words * 8, st))) return rc;
  if ((rc = kr.twice.alloc(kr.num_words * 8, st))) return rc;
  OpSink S{ops.as<uint32_t>(), cur.as<unsigned long long>(), cap, parts, errp};
  SPK_CUDA(cudaFuncSetAttribute(k_bloom_apply, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(4 * kPartWords * 4)));
  for (size_t c = 0; c < chunks.size(); c++) {
    ReadsView cv = rv;
    const uint64_t r0 = chunks[c].first * unit;
    const uint64_t r1 = std::min<uint64_t>(chunks[c].second * unit, rv.n_reads);
    cv.offsets = rv.offsets + r0;
    cv.lengths = rv.lengths + r0;
    cv.n_reads = r1 - r0;
    SPK_CUDA(cudaMemsetAsync(cur.p, 0, (uint64_t)parts * 8, st));
    switch (kr.nl) {
      case 1: rc = launch_stream<1>(ctx, st, cv, k, kr.fm, S, occ); break;
      case 2: rc = launch_stream<2>(ctx, st, cv, k, kr.fm, S, occ); break;
      case 3: rc = launch_stream<3>(ctx, st, cv, k, kr.fm, S, occ); break;
      default: rc = launch_stream<4>(ctx, st, cv, k, kr.fm, S, occ); break;
    }
    if (rc) return rc;
    const bool last = c + 1 == chunks.size();
    if (last) SPK_CUDA(cudaMemsetAsync(pops, 0, 16, st));
    const unsigned grid = (unsigned)std::min<uint64_t>(parts, (uint64_t)ctx->sm_count);
    k_bloom_apply<<<grid, AP_BLOCK, 4 * kPartWords * 4, st>>>(
        ops.as<uint32_t>(), cur.as<unsigned long long>(), cap, parts, kr.num_words, c > 0 ? 1 : 0,
        kr.seen.as<unsigned long long>(), kr.twice.as<unsigned long long>(),
        last ? pops : nullptr, errp);
    SPK_CUDA(cudaGetLastError());
    *launches += 2;
  }
  return SPK_OK;
}

}  // namespace spk
