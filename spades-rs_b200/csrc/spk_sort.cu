// spk_sort.cu -- LSD radix sort of multi-limb keys (SoA) and an ordered
// stream compaction, both written for this library.
//
// Sort: 8-bit digits, one pass per digit of the significant bits.  Each pass
// is a tile histogram, one exclusive scan over (digit, tile) and a stable
// scatter.  Inside a tile, items are ranked per warp with __match_any_sync on
// the digit, then offset by the per-warp prefix of each digit, so equal
// digits keep their input order (stability across passes).
#include <cuda_runtime.h>

#include <algorithm>
#include <utility>
#include <vector>

#include "spk_internal.h"

namespace spk {

constexpr unsigned FULLM = 0xffffffffu;
constexpr int RS_BLOCK = 256;
constexpr int RS_WARPS = RS_BLOCK / 32;
constexpr int RS_IPT = 8;
constexpr int RS_TILE = RS_BLOCK * RS_IPT;  // 2048 items

__global__ void __launch_bounds__(RS_BLOCK) k_rs_hist(const uint64_t* __restrict__ limb, uint64_t n,
                                                       unsigned sh, uint32_t* __restrict__ hist,
                                                       uint32_t ntiles) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const uint64_t base = (uint64_t)blockIdx.x * RS_TILE;
#pragma unroll
  for (int j = 0; j < RS_IPT; j++) {
    const uint64_t i = base + j * RS_BLOCK + threadIdx.x;
    if (i < n) atomicAdd(&h[(unsigned)(__ldg(limb + i) >> sh) & 255u], 1u);
  }
  __syncthreads();
  hist[(uint64_t)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

// Exclusive scan of n u32 values in place, one block of 1024 threads.  Used
// for short arrays (the per-chunk sums of scan_u32).
__global__ void __launch_bounds__(1024) k_scan_u32(uint32_t* __restrict__ a, uint64_t n) {
  __shared__ uint32_t ws[32];
  __shared__ uint32_t carry_s;
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry_s = 0;
  __syncthreads();
  for (uint64_t base = 0; base < n; base += 1024) {
    const uint64_t i = base + threadIdx.x;
    const uint32_t v = i < n ? a[i] : 0u;
    uint32_t x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      uint32_t t = __shfl_up_sync(FULLM, x, d);
      if ((int)lane >= d) x += t;
    }
    if (lane == 31) ws[warp] = x;
    __syncthreads();
    if (warp == 0) {
      uint32_t y = ws[lane];
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        uint32_t t = __shfl_up_sync(FULLM, y, d);
        if ((int)lane >= d) y += t;
      }
      ws[lane] = y;
    }
    __syncthreads();
    const uint32_t carry = carry_s;
    const uint32_t excl = carry + (warp ? ws[warp - 1] : 0u) + x - v;
    if (i < n) a[i] = excl;
    __syncthreads();
    if (threadIdx.x == 1023) carry_s = carry + ws[31];
    __syncthreads();
  }
}

// Multi-block exclusive scan: chunk sums, a scan of the sums, then a
// block-wide scan of every chunk with its offset.
constexpr int SC_BLOCK = 256, SC_IPT = 16, SC_CHUNK = SC_BLOCK * SC_IPT;

__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* ws, uint32_t* total) {
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    uint32_t t = __shfl_up_sync(FULLM, x, d);
    if ((int)lane >= d) x += t;
  }
  if (lane == 31) ws[warp] = x;
  __syncthreads();
  uint32_t pre = 0, tot = 0;
  for (unsigned w = 0; w < blockDim.x / 32; w++) {
    const uint32_t s = ws[w];
    if (w < warp) pre += s;
    tot += s;
  }
  __syncthreads();
  if (total) *total = tot;
  return pre + x - v;
}

__global__ void __launch_bounds__(SC_BLOCK) k_scan_reduce(const uint32_t* __restrict__ a, uint64_t n,
                                                           uint32_t* __restrict__ sums) {
  __shared__ uint32_t ws[SC_BLOCK / 32];
  const uint64_t base = (uint64_t)blockIdx.x * SC_CHUNK;
  uint32_t s = 0;
#pragma unroll
  for (int j = 0; j < SC_IPT; j++) {
    const uint64_t i = base + j * SC_BLOCK + threadIdx.x;
    if (i < n) s += a[i];
  }
  uint32_t tot;
  block_excl_scan(s, ws, &tot);
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(SC_BLOCK) k_scan_apply(uint32_t* __restrict__ a, uint64_t n,
                                                          const uint32_t* __restrict__ sums) {
  __shared__ uint32_t ws[SC_BLOCK / 32];
  // Thread t owns the contiguous items [t*IPT, t*IPT + IPT) of the chunk.
  const uint64_t base = (uint64_t)blockIdx.x * SC_CHUNK + (uint64_t)threadIdx.x * SC_IPT;
  uint32_t v[SC_IPT];
  uint32_t s = 0;
#pragma unroll
  for (int j = 0; j < SC_IPT; j++) {
    v[j] = base + j < n ? a[base + j] : 0u;
    s += v[j];
  }
  uint32_t run = sums[blockIdx.x] + block_excl_scan(s, ws, nullptr);
#pragma unroll
  for (int j = 0; j < SC_IPT; j++) {
    if (base + j < n) a[base + j] = run;
    run += v[j];
  }
}

int scan_u32(cudaStream_t st, uint32_t* a, uint64_t n, DevBuf& sums, uint32_t* launches) {
  const uint64_t nb = (n + SC_CHUNK - 1) / SC_CHUNK;
  int rc;
  if (sums.bytes < nb * 4 && (rc = sums.alloc(nb * 4, st))) return rc;
  k_scan_reduce<<<(unsigned)nb, SC_BLOCK, 0, st>>>(a, n, sums.as<uint32_t>());
  k_scan_u32<<<1, 1024, 0, st>>>(sums.as<uint32_t>(), nb);
  k_scan_apply<<<(unsigned)nb, SC_BLOCK, 0, st>>>(a, n, sums.as<uint32_t>());
  SPK_CUDA(cudaGetLastError());
  if (launches) *launches += 3;
  return SPK_OK;
}

template <int NL, bool HASV>
__global__ void __launch_bounds__(RS_BLOCK) k_rs_scatter(
    const uint64_t* __restrict__ s0, const uint64_t* __restrict__ s1, const uint64_t* __restrict__ s2,
    const uint64_t* __restrict__ s3, const uint32_t* __restrict__ sv, uint64_t* __restrict__ d0,
    uint64_t* __restrict__ d1, uint64_t* __restrict__ d2, uint64_t* __restrict__ d3,
    uint32_t* __restrict__ dv, uint64_t n, unsigned dlimb, unsigned sh,
    const uint32_t* __restrict__ offs, uint32_t ntiles) {
  __shared__ uint32_t wh[RS_WARPS][256];
  __shared__ uint32_t goff[256];
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned lt = lanemask_lt();
  const uint64_t base = (uint64_t)blockIdx.x * RS_TILE + warp * (32 * RS_IPT);

  uint64_t key[RS_IPT][NL];
  uint32_t val[RS_IPT], dig[RS_IPT], rank[RS_IPT];
#pragma unroll
  for (int r = 0; r < RS_IPT; r++) {
    const uint64_t i = base + r * 32 + lane;
    const bool ok = i < n;
#pragma unroll
    for (int j = 0; j < NL; j++) {
      const uint64_t* s = j == 0 ? s0 : j == 1 ? s1 : j == 2 ? s2 : s3;
      key[r][j] = ok ? __ldg(s + i) : 0;
    }
    val[r] = (HASV && ok) ? __ldg(sv + i) : 0u;
    uint64_t dl = 0;
#pragma unroll
    for (int j = 0; j < NL; j++)
      if ((unsigned)j == dlimb) dl = key[r][j];
    dig[r] = ok ? (unsigned)(dl >> sh) & 255u : 0xFFFFFFFFu;
  }
  for (int j = threadIdx.x; j < RS_WARPS * 256; j += RS_BLOCK) (&wh[0][0])[j] = 0;
  goff[threadIdx.x] = offs[(uint64_t)threadIdx.x * ntiles + blockIdx.x];
  __syncthreads();
#pragma unroll
  for (int r = 0; r < RS_IPT; r++) {
    const bool ok = dig[r] != 0xFFFFFFFFu;
    const unsigned vm = __ballot_sync(FULLM, ok);
    unsigned peers = 0;
    if (ok) {
      peers = __match_any_sync(vm, dig[r]);
      rank[r] = wh[warp][dig[r]] + __popc(peers & lt);
    }
    __syncwarp();
    if (ok && lane == (unsigned)(__ffs(peers) - 1)) wh[warp][dig[r]] += __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  {
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < RS_WARPS; w++) {
      const uint32_t x = wh[w][threadIdx.x];
      wh[w][threadIdx.x] = run;
      run += x;
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < RS_IPT; r++) {
    if (dig[r] == 0xFFFFFFFFu) continue;
    const uint64_t p = (uint64_t)goff[dig[r]] + wh[warp][dig[r]] + rank[r];
    d0[p] = key[r][0];
    if (NL > 1) d1[p] = key[r][NL > 1 ? 1 : 0];
    if (NL > 2) d2[p] = key[r][NL > 2 ? 2 : 0];
    if (NL > 3) d3[p] = key[r][NL > 3 ? 3 : 0];
    if (HASV) dv[p] = val[r];
  }
}

template <int NL>
static void launch_scatter(cudaStream_t st, uint64_t* src[4], uint32_t* sv, uint64_t* dst[4],
                           uint32_t* dv, uint64_t n, unsigned dlimb, unsigned sh,
                           const uint32_t* offs, uint32_t ntiles) {
  if (sv)
    k_rs_scatter<NL, true><<<ntiles, RS_BLOCK, 0, st>>>(src[0], src[1], src[2], src[3], sv, dst[0],
                                                      dst[1], dst[2], dst[3], dv, n, dlimb, sh,
                                                      offs, ntiles);
  else
    k_rs_scatter<NL, false><<<ntiles, RS_BLOCK, 0, st>>>(src[0], src[1], src[2], src[3], nullptr,
                                                       dst[0], dst[1], dst[2], dst[3], nullptr, n,
                                                       dlimb, sh, offs, ntiles);
}

int radix_sort_bufs(cudaStream_t st, int nl, uint64_t n, unsigned nbits, DevBuf* keys,
                    DevBuf* vals, uint32_t* launches) {
  if (n <= 1) return SPK_OK;
  if (n >= (1ULL << 32)) return fail(SPK_E_INVALID_ARG, "sort: more than 2^32 items");
  const uint32_t ntiles = (uint32_t)((n + RS_TILE - 1) / RS_TILE);
  int rc;
  DevBuf tk[4], tv, hist, sums;
  for (int j = 0; j < nl; j++)
    if ((rc = tk[j].alloc(n * 8, st))) return rc;
  if (vals && (rc = tv.alloc(n * 4, st))) return rc;
  if ((rc = hist.alloc((uint64_t)256 * ntiles * 4, st))) return rc;
  uint64_t* a[4] = {nullptr, nullptr, nullptr, nullptr};
  uint64_t* b[4] = {nullptr, nullptr, nullptr, nullptr};
  for (int j = 0; j < nl; j++) { a[j] = keys[j].as<uint64_t>(); b[j] = tk[j].as<uint64_t>(); }
  uint32_t* av = vals ? vals->as<uint32_t>() : nullptr;
  uint32_t* bv = vals ? tv.as<uint32_t>() : nullptr;
  const unsigned passes = (nbits + 7) / 8;
  for (unsigned p = 0; p < passes; p++) {
    const unsigned bit = 8 * p, dlimb = bit / 64, sh = bit % 64;
    k_rs_hist<<<ntiles, RS_BLOCK, 0, st>>>(a[dlimb], n, sh, hist.as<uint32_t>(), ntiles);
    if ((rc = scan_u32(st, hist.as<uint32_t>(), (uint64_t)256 * ntiles, sums, launches))) return rc;
    if (launches) *launches += 2;
    switch (nl) {
      case 1: launch_scatter<1>(st, a, av, b, bv, n, dlimb, sh, hist.as<uint32_t>(), ntiles); break;
      case 2: launch_scatter<2>(st, a, av, b, bv, n, dlimb, sh, hist.as<uint32_t>(), ntiles); break;
      case 3: launch_scatter<3>(st, a, av, b, bv, n, dlimb, sh, hist.as<uint32_t>(), ntiles); break;
      default: launch_scatter<4>(st, a, av, b, bv, n, dlimb, sh, hist.as<uint32_t>(), ntiles); break;
    }
    SPK_CUDA(cudaGetLastError());
    for (int j = 0; j < nl; j++) std::swap(a[j], b[j]);
    std::swap(av, bv);
  }
  if (passes & 1) {  // sorted data sits in the temporaries: hand them over
    for (int j = 0; j < nl; j++) std::swap(keys[j], tk[j]);
    if (vals) std::swap(*vals, tv);
  }
  return SPK_OK;
}

// ---------------------------------------------------------------------------
// Bucket sort: an MSD split on the top b significant bits of the key into 2^b
// buckets (b chosen for ~128 items per bucket, 8 <= b <= 16), then a bitonic
// sort of each bucket in shared memory.  The top bits of canonical k-mers
// and (k+1)-mers spread their lists over the buckets; a bucket larger than
// BS_LOCAL items is sorted by the LSD radix sort above instead.  Equal keys
// do not occur (the lists hold distinct k-mers), so stability is not needed.
// ---------------------------------------------------------------------------
constexpr uint32_t BS_MAX_BITS = 16;
constexpr uint32_t BS_LOCAL = 2048;
constexpr int BS_BLOCK = 256;
constexpr uint32_t BS_MAX_BIG = 4096;
constexpr uint64_t BS_STAGE_WORDS = 1024;  // big-bucket list offset in the host staging block

struct Limbs {
  uint64_t* p[4];
};

template <int NL>
__device__ __forceinline__ uint32_t bs_digit(const Limbs& L, uint64_t i, unsigned limb, unsigned sh,
                                             uint32_t nb) {
  uint64_t lo = 0, hi = 0;
#pragma unroll
  for (int j = 0; j < NL; j++) {
    if ((unsigned)j == limb) lo = L.p[j][i];
    if ((unsigned)j == limb + 1) hi = L.p[j][i];
  }
  return (uint32_t)(((lo >> sh) | ((hi << 1) << (63 - sh))) & (nb - 1));
}

// n_dev (nullable): the item count in device memory, at most n.
template <int NL>
__global__ void __launch_bounds__(BS_BLOCK) k_bs_hist(Limbs L, uint64_t n, const unsigned long long* n_dev,
                                                       unsigned limb, unsigned sh, uint32_t nb,
                                                       uint32_t* __restrict__ hist) {
  if (n_dev) n = min(n, (uint64_t)*n_dev);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    atomicAdd(hist + bs_digit<NL>(L, i, limb, sh, nb), 1u);
}

template <int NL, bool HASV>
__global__ void __launch_bounds__(BS_BLOCK) k_bs_scatter(Limbs S, const uint32_t* __restrict__ sv, Limbs D,
                                                          uint32_t* __restrict__ dv, uint64_t n,
                                                          const unsigned long long* n_dev,
                                                          unsigned limb, unsigned sh, uint32_t nb,
                                                          uint32_t* __restrict__ cur) {
  if (n_dev) n = min(n, (uint64_t)*n_dev);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t p = atomicAdd(cur + bs_digit<NL>(S, i, limb, sh, nb), 1u);
#pragma unroll
    for (int j = 0; j < NL; j++) D.p[j][p] = S.p[j][i];
    if (HASV) dv[p] = sv[i];
  }
}

// A bitonic sort of P (a power of two, <= BS_WARP) items in one warp's
// shared-memory region, ascending on the limbs (most significant last).
constexpr uint32_t BS_WARP = 256;  // largest bucket one warp sorts
template <int NL, bool HASV>
__device__ __forceinline__ void warp_bitonic(uint64_t* sk, uint32_t* svl, uint32_t P) {
  const unsigned lane = threadIdx.x & 31;
  for (uint32_t kk = 2; kk <= P; kk <<= 1) {
    for (uint32_t j = kk >> 1; j > 0; j >>= 1) {
      for (uint32_t i = lane; i < P; i += 32) {
        const uint32_t x = i ^ j;
        if (x <= i) continue;
        bool gt = false, eq = true;
#pragma unroll
        for (int q = NL - 1; q >= 0; q--) {
          const uint64_t u = sk[q * BS_WARP + i], v = sk[q * BS_WARP + x];
          if (eq && u != v) {
            gt = u > v;
            eq = false;
          }
        }
        if (gt == ((i & kk) == 0) && !eq) {
#pragma unroll
          for (int q = 0; q < NL; q++) {
            const uint64_t t = sk[q * BS_WARP + i];
            sk[q * BS_WARP + i] = sk[q * BS_WARP + x];
            sk[q * BS_WARP + x] = t;
          }
          if (HASV) {
            const uint32_t t = svl[i];
            svl[i] = svl[x];
            svl[x] = t;
          }
        }
      }
      __syncwarp();
    }
  }
}

// Sorts every bucket of at most BS_LOCAL items from T into D: buckets of at
// most BS_WARP items one per warp, the others one per CTA.  Larger buckets
// are copied to D unsorted and listed in big[3i..3i+2] = (bucket, offset,
// size) for the host, which sorts them from T.
template <int NL, bool HASV>
__global__ void __launch_bounds__(BS_BLOCK) k_bs_local(Limbs T, const uint32_t* __restrict__ tv, Limbs D,
                                                        uint32_t* __restrict__ dv,
                                                        const uint32_t* __restrict__ off,
                                                        const uint32_t* __restrict__ size, uint32_t nb,
                                                        uint32_t* __restrict__ big,
                                                        unsigned* __restrict__ nbig) {
  extern __shared__ __align__(16) uint64_t bs_smem[];
  // Warp phase: warp w sorts the small buckets b = its global warp index +
  // j * (all warps), in its own region of BS_WARP items.
  {
    const unsigned lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint64_t* wk = bs_smem + (size_t)w * BS_WARP * (NL + (HASV ? 1 : 0));
    uint32_t* wv = (uint32_t*)(wk + NL * BS_WARP);
    const uint32_t gw = blockIdx.x * (BS_BLOCK / 32) + w, nw = gridDim.x * (BS_BLOCK / 32);
    for (uint32_t b = gw; b < nb; b += nw) {
      const uint32_t m = size[b];
      if (m == 0 || m > BS_WARP) continue;
      const uint32_t o = off[b];
      if (m == 1) {
        if (lane == 0) {
#pragma unroll
          for (int j = 0; j < NL; j++) D.p[j][o] = T.p[j][o];
          if (HASV) dv[o] = tv[o];
        }
        continue;
      }
      uint32_t P = 2;
      while (P < m) P <<= 1;
      for (uint32_t i = lane; i < P; i += 32) {
        const bool in = i < m;
#pragma unroll
        for (int j = 0; j < NL; j++) wk[j * BS_WARP + i] = in ? T.p[j][o + i] : ~0ULL;
        if (HASV) wv[i] = in ? tv[o + i] : 0u;
      }
      __syncwarp();
      warp_bitonic<NL, HASV>(wk, wv, P);
      for (uint32_t i = lane; i < m; i += 32) {
#pragma unroll
        for (int j = 0; j < NL; j++) D.p[j][o + i] = wk[j * BS_WARP + i];
        if (HASV) dv[o + i] = wv[i];
      }
      __syncwarp();
    }
  }
  __syncthreads();
  // CTA phase: the buckets of BS_WARP < items <= BS_LOCAL.
  uint64_t* sk = bs_smem;                              // NL arrays of BS_LOCAL limbs
  uint32_t* svl = (uint32_t*)(bs_smem + NL * BS_LOCAL);  // values
  for (uint32_t b = blockIdx.x; b < nb; b += gridDim.x) {
    const uint32_t m = size[b];
    if (m <= BS_WARP) continue;
    const uint32_t o = off[b];
    if (m > BS_LOCAL) {
      if (threadIdx.x == 0) {
        const unsigned q = atomicAdd(nbig, 1u);
        if (q < BS_MAX_BIG) {
          big[3 * q] = b;
          big[3 * q + 1] = o;
          big[3 * q + 2] = m;
        }
      }
      // The bucket goes to its place unsorted, so that D holds the whole
      // list (in every bucket's range) before the host sorts this range.
      for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
#pragma unroll
        for (int j = 0; j < NL; j++) D.p[j][o + i] = T.p[j][o + i];
        if (HASV) dv[o + i] = tv[o + i];
      }
      continue;
    }
    uint32_t P = 1;
    while (P < m) P <<= 1;
    for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) {
      const bool in = i < m;
#pragma unroll
      for (int j = 0; j < NL; j++) sk[j * BS_LOCAL + i] = in ? T.p[j][o + i] : ~0ULL;
      if (HASV) svl[i] = in ? tv[o + i] : 0u;
    }
    __syncthreads();
    for (uint32_t kk = 2; kk <= P; kk <<= 1) {
      for (uint32_t j = kk >> 1; j > 0; j >>= 1) {
        for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) {
          const uint32_t x = i ^ j;
          if (x <= i) continue;
          // a > b on the limbs, most significant first
          bool gt = false, eq = true;
#pragma unroll
          for (int q = NL - 1; q >= 0; q--) {
            const uint64_t u = sk[q * BS_LOCAL + i], v = sk[q * BS_LOCAL + x];
            if (eq && u != v) {
              gt = u > v;
              eq = false;
            }
          }
          const bool up = (i & kk) == 0;
          if (gt == up && !eq) {
#pragma unroll
            for (int q = 0; q < NL; q++) {
              const uint64_t t = sk[q * BS_LOCAL + i];
              sk[q * BS_LOCAL + i] = sk[q * BS_LOCAL + x];
              sk[q * BS_LOCAL + x] = t;
            }
            if (HASV) {
              const uint32_t t = svl[i];
              svl[i] = svl[x];
              svl[x] = t;
            }
          }
        }
        __syncthreads();
      }
    }
    for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
#pragma unroll
      for (int j = 0; j < NL; j++) D.p[j][o + i] = sk[j * BS_LOCAL + i];
      if (HASV) dv[o + i] = svl[i];
    }
    __syncthreads();
  }
}

// The buckets k_bs_local left unsorted, side by side: seg[3i..3i+2] = (offset
// in the concatenation C, offset in the list L, size).  Gathers L's segments
// into C (back = false) or writes C's back into L; one CTA per segment.
template <int NL, bool HASV>
__global__ void __launch_bounds__(BS_BLOCK) k_bs_segments(Limbs L, uint32_t* lv, Limbs C, uint32_t* cv,
                                                           const uint32_t* __restrict__ seg, bool back) {
  const uint32_t co = seg[3 * blockIdx.x], lo = seg[3 * blockIdx.x + 1], m = seg[3 * blockIdx.x + 2];
  for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
#pragma unroll
    for (int j = 0; j < NL; j++) {
      if (back) L.p[j][lo + i] = C.p[j][co + i];
      else C.p[j][co + i] = L.p[j][lo + i];
    }
    if (HASV) {
      if (back) lv[lo + i] = cv[co + i];
      else cv[co + i] = lv[lo + i];
    }
  }
}
template <int NL>
static void launch_segments(cudaStream_t st, bool hasv, Limbs L, uint32_t* lv, Limbs C, uint32_t* cv,
                            const uint32_t* seg, uint32_t nseg, bool back) {
  if (hasv) k_bs_segments<NL, true><<<nseg, BS_BLOCK, 0, st>>>(L, lv, C, cv, seg, back);
  else k_bs_segments<NL, false><<<nseg, BS_BLOCK, 0, st>>>(L, lv, C, cv, seg, back);
}

template <int NL, bool HASV>
static int bs_launch(cudaStream_t st, Limbs K, uint32_t* v, Limbs T, uint32_t* tv, uint64_t n,
                     const unsigned long long* n_dev, unsigned limb, unsigned sh, uint32_t nb,
                     uint32_t* hist, uint32_t* off, uint32_t* cur, uint32_t* big, unsigned* nbig,
                     uint32_t* launches) {
  const int sms = current_sm_count();
  const unsigned g = (unsigned)std::max<uint64_t>(
      std::min<uint64_t>((n + BS_BLOCK - 1) / BS_BLOCK, (uint64_t)sms * 16), 1);
  k_bs_hist<NL><<<g, BS_BLOCK, 0, st>>>(K, n, n_dev, limb, sh, nb, hist);
  SPK_CUDA(cudaMemcpyAsync(off, hist, (size_t)nb * 4, cudaMemcpyDeviceToDevice, st));
  DevBuf sums;
  int rc;
  if ((rc = scan_u32(st, off, nb, sums, launches))) return rc;
  SPK_CUDA(cudaMemcpyAsync(cur, off, (size_t)nb * 4, cudaMemcpyDeviceToDevice, st));
  k_bs_scatter<NL, HASV><<<g, BS_BLOCK, 0, st>>>(K, v, T, tv, n, n_dev, limb, sh, nb, cur);
  const size_t smem = std::max<size_t>(BS_LOCAL * (NL * 8 + (HASV ? 4 : 0)),
                                       (size_t)(BS_BLOCK / 32) * BS_WARP * (NL + (HASV ? 1 : 0)) * 8);
  if ((rc = raise_smem_limit((const void*)k_bs_local<NL, HASV>, smem))) return rc;
  const unsigned gl = (unsigned)std::min<uint32_t>(nb, (uint32_t)sms * 4);
  k_bs_local<NL, HASV><<<gl, BS_BLOCK, smem, st>>>(T, tv, K, v, off, hist, nb, big, nbig);
  SPK_CUDA(cudaGetLastError());
  if (launches) *launches += 3;
  return SPK_OK;
}

int sort_bufs(cudaStream_t st, int nl, uint64_t n, unsigned nbits, DevBuf* keys, DevBuf* vals,
              uint64_t* h_staging, uint32_t* launches) {
  // ~128 items per bucket (a few bitonic stages each), 2^8 to 2^16 buckets
  uint32_t bbits = 8;
  while (bbits < BS_MAX_BITS && (n >> (bbits + 1)) >= 128) bbits++;
  const uint32_t nb = 1u << bbits;
  if (n < (1u << 18) || nbits < bbits + 8 || !h_staging)
    return radix_sort_bufs(st, nl, n, nbits, keys, vals, launches);
  if (n >= (1ULL << 32)) return fail(SPK_E_INVALID_ARG, "sort: more than 2^32 items");
  int rc;
  DevBuf tk[4], tv, hist, off, cur, big;
  Limbs K{}, T{};
  for (int j = 0; j < nl; j++) {
    if ((rc = tk[j].alloc(n * 8, st))) return rc;
    K.p[j] = keys[j].as<uint64_t>();
    T.p[j] = tk[j].as<uint64_t>();
  }
  if (vals && (rc = tv.alloc(n * 4, st))) return rc;
  if ((rc = hist.alloc(nb * 4, st)) || (rc = off.alloc(nb * 4, st)) || (rc = cur.alloc(nb * 4, st)) ||
      (rc = big.alloc((3 * BS_MAX_BIG + 1) * 4, st)))
    return rc;
  SPK_CUDA(cudaMemsetAsync(hist.p, 0, nb * 4, st));
  unsigned* nbig = (unsigned*)(big.as<uint32_t>() + 3 * BS_MAX_BIG);
  SPK_CUDA(cudaMemsetAsync(nbig, 0, 4, st));
  const unsigned hi_bit = nbits - bbits, limb = hi_bit / 64, sh = hi_bit % 64;
  uint32_t* v = vals ? vals->as<uint32_t>() : nullptr;
  uint32_t* tvp = vals ? tv.as<uint32_t>() : nullptr;
  uint32_t* H = hist.as<uint32_t>();
  uint32_t* O = off.as<uint32_t>();
  uint32_t* Cu = cur.as<uint32_t>();
  uint32_t* B = big.as<uint32_t>();
  switch (nl * 2 + (vals ? 1 : 0)) {
    case 2: rc = bs_launch<1, false>(st, K, v, T, tvp, n, nullptr, limb, sh, nb, H, O, Cu, B, nbig, launches); break;
    case 3: rc = bs_launch<1, true>(st, K, v, T, tvp, n, nullptr, limb, sh, nb, H, O, Cu, B, nbig, launches); break;
    case 4: rc = bs_launch<2, false>(st, K, v, T, tvp, n, nullptr, limb, sh, nb, H, O, Cu, B, nbig, launches); break;
    case 5: rc = bs_launch<2, true>(st, K, v, T, tvp, n, nullptr, limb, sh, nb, H, O, Cu, B, nbig, launches); break;
    case 6: rc = bs_launch<3, false>(st, K, v, T, tvp, n, nullptr, limb, sh, nb, H, O, Cu, B, nbig, launches); break;
    case 7: rc = bs_launch<3, true>(st, K, v, T, tvp, n, nullptr, limb, sh, nb, H, O, Cu, B, nbig, launches); break;
    case 8: rc = bs_launch<4, false>(st, K, v, T, tvp, n, nullptr, limb, sh, nb, H, O, Cu, B, nbig, launches); break;
    default: rc = bs_launch<4, true>(st, K, v, T, tvp, n, nullptr, limb, sh, nb, H, O, Cu, B, nbig, launches); break;
  }
  if (rc) return rc;
  uint64_t* hs = h_staging + BS_STAGE_WORDS;
  SPK_CUDA(cudaMemcpyAsync(hs, nbig, 4, cudaMemcpyDeviceToHost, st));
  SPK_CUDA(cudaStreamSynchronize(st));
  const unsigned nbig_h = ((unsigned*)hs)[0];
  if (nbig_h > BS_MAX_BIG) {
    // Too many large buckets: sort the bucketed copy as a whole instead.
    for (int j = 0; j < nl; j++)
      SPK_CUDA(cudaMemcpyAsync(K.p[j], T.p[j], n * 8, cudaMemcpyDeviceToDevice, st));
    if (vals) SPK_CUDA(cudaMemcpyAsync(v, tvp, n * 4, cudaMemcpyDeviceToDevice, st));
    return radix_sort_bufs(st, nl, n, nbits, keys, vals, launches);
  }
  if (nbig_h == 0) return SPK_OK;
  SPK_CUDA(cudaMemcpyAsync(hs, B, (size_t)nbig_h * 12, cudaMemcpyDeviceToHost, st));
  SPK_CUDA(cudaStreamSynchronize(st));
  std::vector<uint32_t> bl((const uint32_t*)hs, (const uint32_t*)hs + 3 * nbig_h);
  for (unsigned q = 0; q < nbig_h; q++) {
    const uint64_t o = bl[3 * q + 1], m = bl[3 * q + 2];
    DevBuf bk[4], bvv;
    for (int j = 0; j < nl; j++) {
      if ((rc = bk[j].alloc(m * 8, st))) return rc;
      SPK_CUDA(cudaMemcpyAsync(bk[j].p, T.p[j] + o, m * 8, cudaMemcpyDeviceToDevice, st));
    }
    if (vals) {
      if ((rc = bvv.alloc(m * 4, st))) return rc;
      SPK_CUDA(cudaMemcpyAsync(bvv.p, tvp + o, m * 4, cudaMemcpyDeviceToDevice, st));
    }
    if ((rc = radix_sort_bufs(st, nl, m, hi_bit, bk, vals ? &bvv : nullptr, launches))) return rc;
    for (int j = 0; j < nl; j++)
      SPK_CUDA(cudaMemcpyAsync(K.p[j] + o, bk[j].p, m * 8, cudaMemcpyDeviceToDevice, st));
    if (vals) SPK_CUDA(cudaMemcpyAsync(v + o, bvv.p, m * 4, cudaMemcpyDeviceToDevice, st));
  }
  return SPK_OK;
}

// Bucket sort of a list whose length is known only on the device (*n_dev, at
// most n_cap): the same split and shared-memory sorts, enqueued without
// reading anything back.  Buckets over BS_LOCAL items stay in the bucketed
// copy and are listed on the device; sort_dev_finish sorts them once the
// host has the counts.  Temporaries: tmp_keys (nullable, NL limb arrays of
// n_cap items that the caller no longer needs) or new allocations.
int sort_dev_enqueue(cudaStream_t st, int nl, uint64_t n_cap, const unsigned long long* n_dev,
                     unsigned nbits, DevBuf* keys, DevBuf* vals, DevBuf* tmp_keys, DevSort& ds,
                     uint32_t* launches) {
  uint32_t bbits = 8;
  while (bbits < BS_MAX_BITS && (n_cap >> (bbits + 1)) >= 128) bbits++;
  if (nbits < bbits + 8) return fail(SPK_E_INVALID_ARG, "device-count sort: keys too short");
  if (n_cap >= (1ULL << 32)) return fail(SPK_E_INVALID_ARG, "sort: more than 2^32 items");
  const uint32_t nb = 1u << bbits;
  ds.nl = nl;
  ds.nbits = nbits;
  ds.bbits = bbits;
  ds.n_cap = n_cap;
  ds.has_vals = vals != nullptr;
  int rc;
  Limbs K{}, T{};
  for (int j = 0; j < nl; j++) {
    if (tmp_keys) ds.tk[j] = std::move(tmp_keys[j]);
    else if ((rc = ds.tk[j].alloc(std::max<uint64_t>(n_cap, 1) * 8, st))) return rc;
    K.p[j] = keys[j].as<uint64_t>();
    T.p[j] = ds.tk[j].as<uint64_t>();
  }
  if (vals && (rc = ds.tv.alloc(std::max<uint64_t>(n_cap, 1) * 4, st))) return rc;
  if ((rc = ds.hist.alloc(nb * 4, st)) || (rc = ds.off.alloc(nb * 4, st)) || (rc = ds.cur.alloc(nb * 4, st)) ||
      (rc = ds.big.alloc((3 * BS_MAX_BIG + 1) * 4, st)))
    return rc;
  SPK_CUDA(cudaMemsetAsync(ds.hist.p, 0, nb * 4, st));
  unsigned* nbig = (unsigned*)(ds.big.as<uint32_t>() + 3 * BS_MAX_BIG);
  SPK_CUDA(cudaMemsetAsync(nbig, 0, 4, st));
  const unsigned hi_bit = nbits - bbits, limb = hi_bit / 64, sh = hi_bit % 64;
  uint32_t* v = vals ? vals->as<uint32_t>() : nullptr;
  uint32_t* tvp = vals ? ds.tv.as<uint32_t>() : nullptr;
  uint32_t* H = ds.hist.as<uint32_t>();
  uint32_t* O = ds.off.as<uint32_t>();
  uint32_t* Cu = ds.cur.as<uint32_t>();
  uint32_t* B = ds.big.as<uint32_t>();
  switch (nl * 2 + (vals ? 1 : 0)) {
    case 2: rc = bs_launch<1, false>(st, K, v, T, tvp, n_cap, n_dev, limb, sh, nb, H, O, Cu, B, nbig, launches); break;
    case 3: rc = bs_launch<1, true>(st, K, v, T, tvp, n_cap, n_dev, limb, sh, nb, H, O, Cu, B, nbig, launches); break;
    case 4: rc = bs_launch<2, false>(st, K, v, T, tvp, n_cap, n_dev, limb, sh, nb, H, O, Cu, B, nbig, launches); break;
    case 5: rc = bs_launch<2, true>(st, K, v, T, tvp, n_cap, n_dev, limb, sh, nb, H, O, Cu, B, nbig, launches); break;
    case 6: rc = bs_launch<3, false>(st, K, v, T, tvp, n_cap, n_dev, limb, sh, nb, H, O, Cu, B, nbig, launches); break;
    case 7: rc = bs_launch<3, true>(st, K, v, T, tvp, n_cap, n_dev, limb, sh, nb, H, O, Cu, B, nbig, launches); break;
    case 8: rc = bs_launch<4, false>(st, K, v, T, tvp, n_cap, n_dev, limb, sh, nb, H, O, Cu, B, nbig, launches); break;
    default: rc = bs_launch<4, true>(st, K, v, T, tvp, n_cap, n_dev, limb, sh, nb, H, O, Cu, B, nbig, launches); break;
  }
  if (rc) return rc;
  ds.pending = true;
  return SPK_OK;
}

const unsigned* sort_dev_nbig(const DevSort& ds) {
  return (const unsigned*)(ds.big.as<uint32_t>() + 3 * BS_MAX_BIG);
}

// Sorts the buckets sort_dev_enqueue left over (nbig_host of them, read
// back by the caller; n_host = the list length) and frees the temporaries.
int sort_dev_finish(cudaStream_t st, DevSort& ds, DevBuf* keys, DevBuf* vals, uint64_t n_host,
                    unsigned nbig_host, uint64_t* h_staging, uint32_t* launches) {
  if (!ds.pending) return SPK_OK;
  ds.pending = false;
  // The temporaries may come from another stream that `st` has joined; their
  // frees follow the work enqueued here.
  ds.rehome(st);
  const int nl = ds.nl;
  int rc;
  uint32_t* v = vals ? vals->as<uint32_t>() : nullptr;
  uint32_t* tvp = vals ? ds.tv.as<uint32_t>() : nullptr;
  if (nbig_host > BS_MAX_BIG) {
    // Too many large buckets: sort the bucketed copy as a whole instead.
    for (int j = 0; j < nl; j++)
      SPK_CUDA(cudaMemcpyAsync(keys[j].p, ds.tk[j].p, n_host * 8, cudaMemcpyDeviceToDevice, st));
    if (vals) SPK_CUDA(cudaMemcpyAsync(v, tvp, n_host * 4, cudaMemcpyDeviceToDevice, st));
    rc = radix_sort_bufs(st, nl, n_host, ds.nbits, keys, vals, launches);
  } else if (nbig_host > 0) {
    // The large buckets side by side, in list order, sorted as one array on
    // their whole keys (their top bits keep the buckets apart), then put
    // back: one sort however many buckets there are.
    uint32_t* hs = (uint32_t*)(h_staging + BS_STAGE_WORDS);
    SPK_CUDA(cudaMemcpyAsync(hs, ds.big.p, (size_t)nbig_host * 12, cudaMemcpyDeviceToHost, st));
    SPK_CUDA(cudaStreamSynchronize(st));
    std::vector<std::pair<uint32_t, uint32_t>> segs(nbig_host);  // (offset in the list, size)
    for (unsigned q = 0; q < nbig_host; q++) segs[q] = {hs[3 * q + 1], hs[3 * q + 2]};
    std::sort(segs.begin(), segs.end());
    uint64_t total = 0;
    for (unsigned q = 0; q < nbig_host; q++) {
      hs[3 * q] = (uint32_t)total;
      hs[3 * q + 1] = segs[q].first;
      hs[3 * q + 2] = segs[q].second;
      total += segs[q].second;
    }
    uint32_t* seg = ds.big.as<uint32_t>();
    SPK_CUDA(cudaMemcpyAsync(seg, hs, (size_t)nbig_host * 12, cudaMemcpyHostToDevice, st));
    DevBuf ck[4], cvb;
    Limbs L{}, Cc{};
    for (int j = 0; j < nl; j++) {
      if ((rc = ck[j].alloc(total * 8, st))) return rc;
      L.p[j] = keys[j].as<uint64_t>();
      Cc.p[j] = ck[j].as<uint64_t>();
    }
    if (vals && (rc = cvb.alloc(total * 4, st))) return rc;
    uint32_t* cvp = vals ? cvb.as<uint32_t>() : nullptr;
    switch (nl) {
      case 1: launch_segments<1>(st, vals, L, v, Cc, cvp, seg, nbig_host, false); break;
      case 2: launch_segments<2>(st, vals, L, v, Cc, cvp, seg, nbig_host, false); break;
      case 3: launch_segments<3>(st, vals, L, v, Cc, cvp, seg, nbig_host, false); break;
      default: launch_segments<4>(st, vals, L, v, Cc, cvp, seg, nbig_host, false); break;
    }
    SPK_CUDA(cudaGetLastError());
    if ((rc = radix_sort_bufs(st, nl, total, ds.nbits, ck, vals ? &cvb : nullptr, launches))) return rc;
    for (int j = 0; j < nl; j++) Cc.p[j] = ck[j].as<uint64_t>();  // the sort may have swapped buffers
    cvp = vals ? cvb.as<uint32_t>() : nullptr;
    switch (nl) {
      case 1: launch_segments<1>(st, vals, L, v, Cc, cvp, seg, nbig_host, true); break;
      case 2: launch_segments<2>(st, vals, L, v, Cc, cvp, seg, nbig_host, true); break;
      case 3: launch_segments<3>(st, vals, L, v, Cc, cvp, seg, nbig_host, true); break;
      default: launch_segments<4>(st, vals, L, v, Cc, cvp, seg, nbig_host, true); break;
    }
    SPK_CUDA(cudaGetLastError());
    if (launches) *launches += 2;
  } else {
    rc = SPK_OK;
  }
  ds.release();
  return rc;
}

// ---------------------------------------------------------------------------
// Ordered compaction with conversion of sequence values to Kmer256 limbs.
// Item i of a sorted SoA list is kept when cin == nullptr or cin[i] >=
// min_count; kept items are written in list order as AoS Kmer256 limbs.
// ---------------------------------------------------------------------------
constexpr int OC_BLOCK = 256, OC_IPT = 16, OC_TILE = OC_BLOCK * OC_IPT;

__global__ void __launch_bounds__(OC_BLOCK) k_oc_count(const uint32_t* __restrict__ cin, uint64_t n,
                                                        uint32_t min_count,
                                                        uint32_t* __restrict__ bc) {
  __shared__ uint32_t s;
  if (threadIdx.x == 0) s = 0;
  __syncthreads();
  uint32_t c = 0;
  const uint64_t base = (uint64_t)blockIdx.x * OC_TILE;
  for (int j = 0; j < OC_IPT; j++) {
    const uint64_t i = base + j * OC_BLOCK + threadIdx.x;
    c += i < n && (cin == nullptr || cin[i] >= min_count);
  }
  atomicAdd(&s, c);
  __syncthreads();
  if (threadIdx.x == 0) bc[blockIdx.x] = s;
}

template <int NL>
__global__ void __launch_bounds__(OC_BLOCK) k_oc_write(const uint64_t* l0, const uint64_t* l1,
                                                        const uint64_t* l2, const uint64_t* l3,
                                                        const uint32_t* __restrict__ cin, uint64_t n,
                                                        unsigned k, uint32_t min_count,
                                                        const uint32_t* __restrict__ bc,
                                                        uint64_t* __restrict__ out,
                                                        uint32_t* __restrict__ cout, uint64_t out_cap) {
  __shared__ uint32_t ws[OC_BLOCK / 32];
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // Thread t owns the contiguous items [t*IPT, t*IPT+IPT) of the tile.
  const uint64_t base = (uint64_t)blockIdx.x * OC_TILE + (uint64_t)threadIdx.x * OC_IPT;
  uint32_t keepmask = 0;
#pragma unroll
  for (int j = 0; j < OC_IPT; j++) {
    const uint64_t i = base + j;
    if (i < n && (cin == nullptr || cin[i] >= min_count)) keepmask |= 1u << j;
  }
  const uint32_t c = __popc(keepmask);
  uint32_t x = c;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    uint32_t t = __shfl_up_sync(FULLM, x, d);
    if ((int)lane >= d) x += t;
  }
  if (lane == 31) ws[warp] = x;
  __syncthreads();
  uint32_t wpre = 0;
  for (unsigned w = 0; w < warp; w++) wpre += ws[w];
  uint64_t p = (uint64_t)bc[blockIdx.x] + wpre + x - c;
#pragma unroll 1
  for (int j = 0; j < OC_IPT; j++) {
    if (!(keepmask & (1u << j))) continue;
    if (p >= out_cap) break;  // (a caller's count of the kept items that was short)
    const uint64_t i = base + j;
    Seq<NL> V;
    V.v[0] = l0[i];
    if (NL > 1) V.v[NL > 1 ? 1 : 0] = l1[i];
    if (NL > 2) V.v[NL > 2 ? 2 : 0] = l2[i];
    if (NL > 3) V.v[NL > 3 ? 3 : 0] = l3[i];
    uint64_t w[4];
    kmer256_limbs<NL>(V, k, w);
#pragma unroll
    for (int q = 0; q < NL; q++) out[p * NL + q] = w[q];
    if (cout) cout[p] = cin[i];
    p++;
  }
}

// Returns the number of kept items in *m (host value; synchronises st).
int ordered_convert(cudaStream_t st, int nl, uint64_t n, unsigned k, DevBuf* limbs,
                    const uint32_t* cin, uint32_t min_count, DevBuf* out, DevBuf* cout,
                    uint64_t* h_staging, uint64_t* m, uint64_t known_m) {
  int rc;
  const uint32_t nt = (uint32_t)std::max<uint64_t>((n + OC_TILE - 1) / OC_TILE, 1);
  DevBuf bc;
  if ((rc = bc.alloc((uint64_t)(nt + 1) * 4, st))) return rc;
  SPK_CUDA(cudaMemsetAsync(bc.p, 0, (uint64_t)(nt + 1) * 4, st));
  if (n) {
    k_oc_count<<<nt, OC_BLOCK, 0, st>>>(cin, n, min_count, bc.as<uint32_t>());
  }
  DevBuf sums;
  if ((rc = scan_u32(st, bc.as<uint32_t>(), nt + 1, sums))) return rc;
  if (known_m != ~0ULL) {
    *m = known_m;
  } else {
    SPK_CUDA(cudaMemcpyAsync(h_staging, bc.as<uint32_t>() + nt, 4, cudaMemcpyDeviceToHost, st));
    SPK_CUDA(cudaStreamSynchronize(st));
    *m = (uint64_t)((uint32_t*)h_staging)[0];
  }
  if ((rc = out->alloc_keep(std::max<uint64_t>(*m, 1) * nl * 8, st))) return rc;
  if (cout && (rc = cout->alloc_keep(std::max<uint64_t>(*m, 1) * 4, st))) return rc;
  if (n && *m) {
    const uint64_t* p[4] = {nullptr, nullptr, nullptr, nullptr};
    for (int j = 0; j < nl; j++) p[j] = limbs[j].as<uint64_t>();
    uint64_t* o = out->as<uint64_t>();
    uint32_t* oc = cout ? cout->as<uint32_t>() : nullptr;
    switch (nl) {
      case 1: k_oc_write<1><<<nt, OC_BLOCK, 0, st>>>(p[0], p[1], p[2], p[3], cin, n, k, min_count, bc.as<uint32_t>(), o, oc, *m); break;
      case 2: k_oc_write<2><<<nt, OC_BLOCK, 0, st>>>(p[0], p[1], p[2], p[3], cin, n, k, min_count, bc.as<uint32_t>(), o, oc, *m); break;
      case 3: k_oc_write<3><<<nt, OC_BLOCK, 0, st>>>(p[0], p[1], p[2], p[3], cin, n, k, min_count, bc.as<uint32_t>(), o, oc, *m); break;
      default: k_oc_write<4><<<nt, OC_BLOCK, 0, st>>>(p[0], p[1], p[2], p[3], cin, n, k, min_count, bc.as<uint32_t>(), o, oc, *m); break;
    }
    SPK_CUDA(cudaGetLastError());
  }
  return SPK_OK;
}

}  // namespace spk
