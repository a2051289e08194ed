// spk_correct.cu -- single-base read error correction against the solid tier
// of a TwoTierFilter: ErrorCorrector::correct_read_in_place (src/hammer.rs:
// 34-121), as Stage 3 applies it to every packed read before counting
// (src/assemble.rs:183-191).
//
// One warp per read.  The read's 2-bit bases sit in shared memory as 64-bit
// big-endian words (the packed layout), with one bit per k-window: solid or
// not under the current bases.  The reference walks the windows in order and
// at an unsolid window i tries every single substitution inside it, keeping
// the one whose window i becomes solid and that gains the most solid windows
// over the windows covering the substituted base (first offset, then A<C<G<T,
// wins ties).  Its "base_solid" count (windows covering the base before the
// substitution, window i excluded) is a popcount of the window bits here, so
// a trial costs one Bloom query plus, when window i turns solid, one query
// per covering window; the lanes split the 3k trials of a window.  After a
// substitution the bits of the windows covering it are recomputed, so each
// later window is judged on the corrected bases, as the reference's scratch
// buffer does.
#include <cuda_runtime.h>

#include <algorithm>

#include "spk_internal.h"

namespace spk {

constexpr int kCorrWarps = 8;                     // warps (reads in flight) per CTA
constexpr uint32_t kCorrMaxLen = 8192;            // bases per read
constexpr int kCorrWords = kCorrMaxLen / 32 + 8;  // u64 base words (+ room for a window's tail)
constexpr int kCorrFlagWords = kCorrMaxLen / 32;  // u32 window-bit words

struct CorrTier {
  const unsigned long long* solid;
  FastMod fm;
};

// The window of k bases starting at base s of the shared words.
template <int NL>
__device__ __forceinline__ Seq<NL> corr_window(const uint64_t* W, uint32_t s, unsigned k) {
  const uint32_t bit = 2u * s;
  const uint64_t* p = W + (bit >> 6);
  const unsigned sh = bit & 63u;
  uint64_t U[NL + 1];
#pragma unroll
  for (int j = 0; j <= NL; j++) U[j] = p[j];
  uint64_t X[NL];
#pragma unroll
  for (int j = 0; j < NL; j++) X[NL - 1 - j] = shl2(U[j], U[j + 1], sh);
  const unsigned r = 64u * NL - 2u * k;
  Seq<NL> V;
#pragma unroll
  for (int i = 0; i < NL; i++) V.v[i] = (i + 1 < NL) ? shr2(X[i + 1], X[i], r) : (X[i] >> r);
  return V;
}

// V with its base q (0-based from the window start) replaced by c.
template <int NL>
__device__ __forceinline__ Seq<NL> corr_patch(Seq<NL> V, unsigned q, unsigned c, unsigned k) {
  const unsigned bit = 2u * (k - 1u - q);
#pragma unroll
  for (int j = 0; j < NL; j++)
    if ((unsigned)j == (bit >> 6)) V.v[j] = (V.v[j] & ~(3ULL << (bit & 63))) | ((uint64_t)c << (bit & 63));
  return V;
}

// is_solid_kmer256(canonical(V)) (src/bloom.rs:111-126, src/dna.rs:185-192).
template <int NL>
__device__ __forceinline__ bool corr_solid(const CorrTier& T, const Seq<NL>& V, unsigned k) {
  const Seq<NL> C = canonical<NL>(V, k);
  uint64_t w[4];
  kmer256_limbs<NL>(C, k, w);
  const HashPre hp = hash_pre(w);
  const uint64_t p0 = fastmod(T.fm, hash_seed(hp, kSeed1));
  const uint64_t p1 = fastmod(T.fm, hash_seed(hp, kSeed2));
  const uint64_t p2 = fastmod(T.fm, hash_seed(hp, kSeed3));
  return ((__ldg(T.solid + (p0 >> 6)) >> (p0 & 63)) & 1) && ((__ldg(T.solid + (p1 >> 6)) >> (p1 & 63)) & 1) &&
         ((__ldg(T.solid + (p2 >> 6)) >> (p2 & 63)) & 1);
}

__device__ __forceinline__ unsigned corr_base(const uint64_t* W, uint32_t s) {
  return (unsigned)(W[s >> 5] >> (62u - 2u * (s & 31u))) & 3u;
}

// Solid windows among [a, b] (inclusive, a <= b).
__device__ __forceinline__ uint32_t corr_count(const uint32_t* F, uint32_t a, uint32_t b) {
  uint32_t n = 0;
  for (uint32_t w = a >> 5; w <= (b >> 5); w++) {
    uint32_t m = F[w];
    if (w == (a >> 5)) m &= ~0u << (a & 31u);
    if (w == (b >> 5) && (b & 31u) != 31u) m &= (1u << ((b & 31u) + 1u)) - 1u;
    n += __popc(m);
  }
  return n;
}

template <int NL>
__global__ void __launch_bounds__(kCorrWarps * 32) k_correct(const uint8_t* __restrict__ data, uint64_t data_len,
                                                             const uint64_t* __restrict__ offsets,
                                                             const uint32_t* __restrict__ lengths, uint64_t n_reads,
                                                             unsigned k, CorrTier T, uint8_t* __restrict__ out,
                                                             uint8_t* __restrict__ corrected,
                                                             unsigned long long* __restrict__ n_corrected,
                                                             int* __restrict__ err) {
  __shared__ uint64_t sW[kCorrWarps][kCorrWords];
  __shared__ uint32_t sF[kCorrWarps][kCorrFlagWords];
  const unsigned lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
  uint64_t* W = sW[wib];
  uint32_t* F = sF[wib];
  const uint64_t nwarps = (uint64_t)gridDim.x * kCorrWarps;
  for (uint64_t r = blockIdx.x * (uint64_t)kCorrWarps + wib; r < n_reads; r += nwarps) {
    const uint32_t L = lengths[r];
    const uint64_t off = offsets[r];
    const uint64_t nbytes = (L + 3u) / 4u;
    if (off > data_len || nbytes > data_len - off) {
      if (lane == 0) atomicOr(err, 4);
      continue;
    }
    if (L > kCorrMaxLen) {
      if (lane == 0) atomicOr(err, 32);
      continue;
    }
    bool modified = false;
    if (k > 0 && L >= k) {
      // ---- bases into shared words, zero beyond the read ----
      const uint32_t nW = (uint32_t)((nbytes + 7) / 8);
      const uint32_t nZ = min((uint32_t)kCorrWords, nW + NL + 1u);
      for (uint32_t w = lane; w < nZ; w += 32) {
        uint64_t x = 0;
        if (w < nW) {
#pragma unroll
          for (int b = 0; b < 8; b++) {
            const uint64_t j = 8ull * w + b;
            if (j < nbytes) x |= (uint64_t)data[off + j] << (56 - 8 * b);
          }
        }
        W[w] = x;
      }
      __syncwarp();
      // ---- one bit per window ----
      const uint32_t nw = L - k + 1;
      for (uint32_t s0 = 0; s0 < nw; s0 += 32) {
        const uint32_t s = s0 + lane;
        const bool ok = s < nw && corr_solid<NL>(T, corr_window<NL>(W, s, k), k);
        const uint32_t m = __ballot_sync(0xffffffffu, ok);
        if (lane == 0) F[s0 >> 5] = m;
      }
      __syncwarp();
      const uint32_t nfw = (nw + 31) / 32;
      uint32_t i = 0;
      while (i < nw) {
        // next unsolid window at or after i
        uint32_t next = nw;
        for (uint32_t w = i >> 5; w < nfw; w++) {
          uint32_t z = ~F[w];
          if (w == (i >> 5)) z &= ~0u << (i & 31u);
          if (w == nfw - 1 && (nw & 31u)) z &= (1u << (nw & 31u)) - 1u;
          if (z) {
            next = 32u * w + (__ffs(z) - 1);
            break;
          }
        }
        if (next >= nw) break;
        i = next;
        // trials t = 4 * offset + base, base != the current one: the lanes
        // split the trials; the trials that make window i solid are then
        // scored one by one, the lanes splitting the windows that cover the
        // substituted base
        const Seq<NL> Vi = corr_window<NL>(W, i, k);
        uint32_t best = 0;
        for (uint32_t t0 = 0; t0 < 4u * k; t0 += 32) {
          const uint32_t t = t0 + lane;
          bool hit = false;
          if (t < 4u * k) {
            const uint32_t o = t >> 2, c = t & 3u;
            hit = c != corr_base(W, i + o) && corr_solid<NL>(T, corr_patch<NL>(Vi, o, c, k), k);
          }
          uint32_t hits = __ballot_sync(0xffffffffu, hit);
          while (hits) {
            const uint32_t tt = t0 + (__ffs(hits) - 1);
            hits &= hits - 1;
            const uint32_t pos = i + (tt >> 2), c = tt & 3u;
            const uint32_t a = pos >= k - 1 ? pos - (k - 1) : 0;
            const uint32_t b = min(pos, nw - 1);
            uint32_t cnt = 0;
            for (uint32_t s = a + lane; s <= b; s += 32) {
              if (s == i) continue;
              cnt += corr_solid<NL>(T, corr_patch<NL>(corr_window<NL>(W, s, k), pos - s, c, k), k) ? 1u : 0u;
            }
            cnt = __reduce_add_sync(0xffffffffu, cnt) + 1u;  // + window i, solid by the trial
            const uint32_t base = corr_count(F, a, b);       // window i is unsolid: not counted
            if (cnt > base) best = max(best, ((cnt - base) << 12) | (4095u - tt));
          }
        }
        if (best) {
          const uint32_t t = 4095u - (best & 4095u);
          const uint32_t pos = i + (t >> 2), c = t & 3u;
          __syncwarp();
          if (lane == 0) {
            const unsigned sh = 62u - 2u * (pos & 31u);
            W[pos >> 5] = (W[pos >> 5] & ~(3ULL << sh)) | ((uint64_t)c << sh);
          }
          __syncwarp();
          modified = true;
          const uint32_t a = pos >= k - 1 ? pos - (k - 1) : 0;
          const uint32_t b = min(pos, nw - 1);
          for (uint32_t s = a + lane; s <= b; s += 32) {
            const bool ok = corr_solid<NL>(T, corr_window<NL>(W, s, k), k);
            if (ok) atomicOr(&F[s >> 5], 1u << (s & 31u));
            else atomicAnd(&F[s >> 5], ~(1u << (s & 31u)));
          }
          __syncwarp();
        }
        i++;
      }
      if (modified) {
        for (uint64_t j = lane; j < nbytes; j += 32)
          out[off + j] = (uint8_t)(W[j >> 3] >> (56 - 8 * (j & 7)));
      }
      __syncwarp();
    }
    if (lane == 0) {
      if (corrected) corrected[r] = modified ? 1 : 0;
      if (modified) atomicAdd(n_corrected, 1ULL);
    }
  }
}

int correct_reads(spk_ctx* ctx, cudaStream_t st, unsigned k, const unsigned long long* tier, const FastMod& fm,
                  const uint8_t* d_data, uint64_t data_len, const uint64_t* d_off, const uint32_t* d_len,
                  uint64_t n, uint8_t* d_out, uint8_t* d_corr, uint64_t* nc, uint32_t* launches) {
  if (k > 127) return fail(SPK_E_INVALID_K, "error correction supports k up to 127");
  if (d_out != d_data && data_len) SPK_CUDA(cudaMemcpyAsync(d_out, d_data, data_len, cudaMemcpyDeviceToDevice, st));
  DevBuf cnt;
  int rc;
  if ((rc = cnt.alloc(16, st))) return rc;
  SPK_CUDA(cudaMemsetAsync(cnt.p, 0, 16, st));
  unsigned long long* d_nc = cnt.as<unsigned long long>();
  int* d_err = (int*)(d_nc + 1);
  if (n) {
    const CorrTier T{tier, fm};
    const unsigned grid = (unsigned)std::max<uint64_t>(
        1, std::min<uint64_t>((n + kCorrWarps - 1) / kCorrWarps, (uint64_t)ctx->sm_count * 8));
    const unsigned nl = k ? (k + 31) / 32 : 1;
#define SPK_CORR(NL_)                                                                                   \
  k_correct<NL_><<<grid, kCorrWarps * 32, 0, st>>>(d_data, data_len, d_off, d_len, n, k, T, d_out, d_corr, \
                                                   d_nc, d_err)
    switch (nl) {
      case 1: SPK_CORR(1); break;
      case 2: SPK_CORR(2); break;
      case 3: SPK_CORR(3); break;
      default: SPK_CORR(4); break;
    }
#undef SPK_CORR
    SPK_CUDA(cudaGetLastError());
    if (launches) ++*launches;
  }
  uint64_t h[2] = {0, 0};
  SPK_CUDA(cudaMemcpyAsync(h, cnt.p, 16, cudaMemcpyDeviceToHost, st));
  SPK_CUDA(cudaStreamSynchronize(st));
  const int e = (int)h[1];
  if (e & 4) return fail(SPK_E_INVALID_ARG, "a read lies outside the packed data");
  if (e & 32) return fail(SPK_E_INVALID_ARG, "error correction takes reads of at most 8192 bases");
  if (nc) *nc = h[0];
  return SPK_OK;
}

static int correct_device(spk_bloom* b, unsigned k, const uint8_t* d_data, uint64_t data_len,
                          const uint64_t* d_off, const uint32_t* d_len, uint64_t n, uint8_t* d_out,
                          uint8_t* d_corr, uint64_t* nc) {
  return correct_reads(b->ctx, b->ctx->stream, k, b->solid.as<unsigned long long>(), b->fm, d_data, data_len,
                       d_off, d_len, n, d_out, d_corr, nc, nullptr);
}

}  // namespace spk

using namespace spk;

extern "C" int spk_bloom_correct_reads_device(spk_bloom* bloom, uint32_t k, const uint8_t* d_data, size_t data_len,
                                              const uint64_t* d_offsets, const uint32_t* d_lengths, size_t n_reads,
                                              uint8_t* d_data_out, uint8_t* d_corrected, uint64_t* n_corrected) {
  if (!bloom) return fail(SPK_E_INVALID_ARG, "null filter");
  if (n_reads && (!d_offsets || !d_lengths)) return fail(SPK_E_INVALID_ARG, "null read arrays");
  if (data_len && (!d_data || !d_data_out)) return fail(SPK_E_INVALID_ARG, "null data");
  SPK_CUDA(cudaSetDevice(bloom->ctx->device));
  return correct_device(bloom, k, d_data, data_len, d_offsets, d_lengths, n_reads, d_data_out, d_corrected,
                        n_corrected);
}

extern "C" int spk_bloom_correct_reads(spk_bloom* bloom, uint32_t k, const uint8_t* data, size_t data_len,
                                       const uint64_t* offsets, const uint32_t* lengths, size_t n_reads,
                                       uint8_t* data_out, uint8_t* corrected, uint64_t* n_corrected) {
  if (!bloom) return fail(SPK_E_INVALID_ARG, "null filter");
  if (n_reads && (!offsets || !lengths)) return fail(SPK_E_INVALID_ARG, "null read arrays");
  if (data_len && (!data || !data_out)) return fail(SPK_E_INVALID_ARG, "null data");
  spk_ctx* ctx = bloom->ctx;
  SPK_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  DevBuf dd, dout, doff, dlen, dcor;
  int rc;
  if ((rc = dd.alloc(std::max<size_t>(data_len, 1) + 64, st)) ||
      (rc = dout.alloc(std::max<size_t>(data_len, 1) + 64, st)) ||
      (rc = doff.alloc(std::max<size_t>(n_reads, 1) * 8, st)) ||
      (rc = dlen.alloc(std::max<size_t>(n_reads, 1) * 4, st)) || (rc = dcor.alloc(std::max<size_t>(n_reads, 1), st)))
    return rc;
  if (data_len) SPK_CUDA(cudaMemcpyAsync(dd.p, data, data_len, cudaMemcpyHostToDevice, st));
  if (n_reads) {
    SPK_CUDA(cudaMemcpyAsync(doff.p, offsets, n_reads * 8, cudaMemcpyHostToDevice, st));
    SPK_CUDA(cudaMemcpyAsync(dlen.p, lengths, n_reads * 4, cudaMemcpyHostToDevice, st));
  }
  uint64_t nc = 0;
  if ((rc = correct_device(bloom, k, dd.as<uint8_t>(), data_len, doff.as<uint64_t>(), dlen.as<uint32_t>(), n_reads,
                           dout.as<uint8_t>(), dcor.as<uint8_t>(), &nc)))
    return rc;
  if (data_len) SPK_CUDA(cudaMemcpyAsync(data_out, dout.p, data_len, cudaMemcpyDeviceToHost, st));
  if (corrected && n_reads) SPK_CUDA(cudaMemcpyAsync(corrected, dcor.p, n_reads, cudaMemcpyDeviceToHost, st));
  SPK_CUDA(cudaStreamSynchronize(st));
  if (n_corrected) *n_corrected = nc;
  return SPK_OK;
}
