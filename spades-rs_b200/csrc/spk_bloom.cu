// spk_bloom.cu -- the reference TwoTierFilter (src/bloom.rs:13-131) on the GPU.
//
// Batched calls return exactly what calling the reference method once per key
// in array order returns.  The three fetch_or of insert_kmer256
// (src/bloom.rs:95-97) for key i are operations 3i, 3i+1, 3i+2 of one serial
// sequence; operation j finds its bit already set iff the bit was set before
// the batch or some operation j' < j of the batch targets the same bit.  The
// first operation per bit is found with an atomicMin into a small hash map
// keyed by bit position, so the whole batch runs in parallel and still has
// serial semantics, including the order-dependent solid tier.
#include <cuda_runtime.h>

#include <algorithm>

#include "spk_internal.h"

namespace spk {

constexpr int kB = 256;

struct BloomKeys {
  const uint64_t* keys;  // 4 limbs per key when wide, else 1
  uint64_t n;
  int wide;
};

__device__ __forceinline__ void key_limbs(const BloomKeys& K, uint64_t i, uint64_t w[4]) {
  if (K.wide) {
#pragma unroll
    for (int j = 0; j < 4; j++) w[j] = K.keys[4 * i + j];
  } else {
    w[0] = K.keys[i];  // insert(u64) == insert_kmer256(Kmer256(x as u128, 0)), src/bloom.rs:48-50
    w[1] = w[2] = w[3] = 0;
  }
}

__device__ __forceinline__ void key_positions(const BloomKeys& K, uint64_t i, const FastMod& fm,
                                              uint64_t pos[3]) {
  uint64_t w[4];
  key_limbs(K, i, w);
  HashPre hp = hash_pre(w);
  pos[0] = fastmod(fm, hash_seed(hp, kSeed1));
  pos[1] = fastmod(fm, hash_seed(hp, kSeed2));
  pos[2] = fastmod(fm, hash_seed(hp, kSeed3));
}

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x ^= x >> 31;
  x *= 0x7fb5d329728ea185ULL;
  x ^= x >> 27;
  x *= 0x81dadef4bc2dd44dULL;
  x ^= x >> 33;
  return x;
}

// Phase 1: positions, the bits as they were before the batch, and the first
// operation index per position.
__global__ void __launch_bounds__(kB) k_api_first(BloomKeys K, FastMod fm,
                                                  const unsigned long long* __restrict__ seen,
                                                  uint64_t* __restrict__ pos_out,
                                                  uint8_t* __restrict__ init_out,
                                                  unsigned long long* __restrict__ mkeys,
                                                  unsigned long long* __restrict__ mvals,
                                                  uint64_t mmask) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < K.n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t pos[3];
    key_positions(K, i, fm, pos);
#pragma unroll
    for (int s = 0; s < 3; s++) {
      const uint64_t op = 3 * i + s;
      pos_out[op] = pos[s];
      init_out[op] = (uint8_t)((seen[pos[s] >> 6] >> (pos[s] & 63)) & 1);
      uint64_t h = mix64(pos[s]) & mmask;
      // The map has at least twice as many slots as operations, so a free or
      // matching slot is always found within mmask + 1 probes.
      for (uint64_t probe = 0; probe <= mmask; probe++) {
        unsigned long long cur = mkeys[h];
        if (cur == ~0ULL) cur = atomicCAS(mkeys + h, ~0ULL, (unsigned long long)pos[s]);
        if (cur == ~0ULL || cur == pos[s]) {
          atomicMin(mvals + h, (unsigned long long)op);
          break;
        }
        h = (h + 1) & mmask;
      }
    }
  }
}

// Phase 2: resolve each key's promotion and apply its bits.
__global__ void __launch_bounds__(kB) k_api_apply(uint64_t n, const uint64_t* __restrict__ pos_in,
                                                  const uint8_t* __restrict__ init_in,
                                                  const unsigned long long* __restrict__ mkeys,
                                                  const unsigned long long* __restrict__ mvals,
                                                  uint64_t mmask, unsigned long long* __restrict__ seen,
                                                  unsigned long long* __restrict__ solid,
                                                  uint8_t* __restrict__ promoted) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    bool all = true;
    uint64_t pos[3];
#pragma unroll
    for (int s = 0; s < 3; s++) {
      const uint64_t op = 3 * i + s;
      pos[s] = pos_in[op];
      uint64_t h = mix64(pos[s]) & mmask;
      for (uint64_t probe = 0; probe <= mmask && mkeys[h] != pos[s]; probe++) h = (h + 1) & mmask;
      const bool before = init_in[op] || mvals[h] < op;
      all &= before;
    }
#pragma unroll
    for (int s = 0; s < 3; s++) atomicOr(seen + (pos[s] >> 6), 1ULL << (pos[s] & 63));
    if (all) {
#pragma unroll
      for (int s = 0; s < 3; s++) atomicOr(solid + (pos[s] >> 6), 1ULL << (pos[s] & 63));
    }
    if (promoted) promoted[i] = all ? 1 : 0;
  }
}

__global__ void __launch_bounds__(kB) k_api_query(BloomKeys K, FastMod fm,
                                                  const unsigned long long* __restrict__ solid,
                                                  uint8_t* __restrict__ out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < K.n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t pos[3];
    key_positions(K, i, fm, pos);
    bool ok = true;
#pragma unroll
    for (int s = 0; s < 3; s++) ok &= ((solid[pos[s] >> 6] >> (pos[s] & 63)) & 1) != 0;
    out[i] = ok ? 1 : 0;
  }
}

static unsigned grid_n(spk_ctx* ctx, uint64_t n) {
  const uint64_t want = (n + kB - 1) / kB;
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)ctx->sm_count * 8));
}

int bloom_create(spk_ctx* ctx, uint64_t capacity_bits, spk_bloom** out) {
  auto* b = new spk_bloom();
  b->ctx = ctx;
  b->num_words = std::max<uint64_t>((capacity_bits + 63) / 64, 1);  // src/bloom.rs:27
  b->size_bits = b->num_words * 64;                                 // src/bloom.rs:28
  b->fm = make_fastmod(b->size_bits);
  cudaStream_t st = ctx->stream;
  int rc;
  if ((rc = b->seen.alloc(b->num_words * 8, st)) || (rc = b->solid.alloc(b->num_words * 8, st))) {
    delete b;
    return rc;
  }
  cudaError_t e = cudaMemsetAsync(b->seen.p, 0, b->num_words * 8, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->solid.p, 0, b->num_words * 8, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    delete b;
    return cuda_fail(e, "bloom create");
  }
  *out = b;
  return SPK_OK;
}

int bloom_insert(spk_bloom* b, const uint64_t* keys, size_t n, int wide, uint8_t* promoted) {
  if (n == 0) return SPK_OK;
  spk_ctx* ctx = b->ctx;
  cudaStream_t st = ctx->stream;
  const uint64_t limbs = wide ? 4 : 1;
  const uint64_t ops = 3 * (uint64_t)n;
  uint64_t mcap = 1;
  while (mcap < 2 * ops) mcap <<= 1;
  DevBuf dk, dpos, dinit, mk, mv, dprom;
  int rc;
  if ((rc = dk.alloc(n * limbs * 8, st)) || (rc = dpos.alloc(ops * 8, st)) ||
      (rc = dinit.alloc(ops, st)) || (rc = mk.alloc(mcap * 8, st)) || (rc = mv.alloc(mcap * 8, st)) ||
      (rc = dprom.alloc(n, st)))
    return rc;
  SPK_CUDA(cudaMemcpyAsync(dk.p, keys, n * limbs * 8, cudaMemcpyHostToDevice, st));
  SPK_CUDA(cudaMemsetAsync(mk.p, 0xFF, mcap * 8, st));
  SPK_CUDA(cudaMemsetAsync(mv.p, 0xFF, mcap * 8, st));
  BloomKeys K{dk.as<uint64_t>(), n, wide};
  k_api_first<<<grid_n(ctx, n), kB, 0, st>>>(K, b->fm, b->seen.as<unsigned long long>(),
                                             dpos.as<uint64_t>(), dinit.as<uint8_t>(),
                                             mk.as<unsigned long long>(), mv.as<unsigned long long>(),
                                             mcap - 1);
  k_api_apply<<<grid_n(ctx, n), kB, 0, st>>>(n, dpos.as<uint64_t>(), dinit.as<uint8_t>(),
                                             mk.as<unsigned long long>(), mv.as<unsigned long long>(),
                                             mcap - 1, b->seen.as<unsigned long long>(),
                                             b->solid.as<unsigned long long>(), dprom.as<uint8_t>());
  SPK_CUDA(cudaGetLastError());
  if (promoted) SPK_CUDA(cudaMemcpyAsync(promoted, dprom.p, n, cudaMemcpyDeviceToHost, st));
  SPK_CUDA(cudaStreamSynchronize(st));
  return SPK_OK;
}

int bloom_query(spk_bloom* b, const uint64_t* keys, size_t n, int wide, uint8_t* out) {
  if (n == 0) return SPK_OK;
  spk_ctx* ctx = b->ctx;
  cudaStream_t st = ctx->stream;
  const uint64_t limbs = wide ? 4 : 1;
  DevBuf dk, dout;
  int rc;
  if ((rc = dk.alloc(n * limbs * 8, st)) || (rc = dout.alloc(n, st))) return rc;
  SPK_CUDA(cudaMemcpyAsync(dk.p, keys, n * limbs * 8, cudaMemcpyHostToDevice, st));
  BloomKeys K{dk.as<uint64_t>(), n, wide};
  k_api_query<<<grid_n(ctx, n), kB, 0, st>>>(K, b->fm, b->solid.as<unsigned long long>(),
                                             dout.as<uint8_t>());
  SPK_CUDA(cudaGetLastError());
  SPK_CUDA(cudaMemcpyAsync(out, dout.p, n, cudaMemcpyDeviceToHost, st));
  SPK_CUDA(cudaStreamSynchronize(st));
  return SPK_OK;
}

int bloom_download(spk_bloom* b, uint64_t* seen, uint64_t* solid) {
  cudaStream_t st = b->ctx->stream;
  if (seen) SPK_CUDA(cudaMemcpyAsync(seen, b->seen.p, b->num_words * 8, cudaMemcpyDeviceToHost, st));
  if (solid) SPK_CUDA(cudaMemcpyAsync(solid, b->solid.p, b->num_words * 8, cudaMemcpyDeviceToHost, st));
  SPK_CUDA(cudaStreamSynchronize(st));
  return SPK_OK;
}

}  // namespace spk

// ---------------------------------------------------------------------------
// spk_bloom_insert_k256_noalloc: the batched insert above with its scratch in
// a static device array instead of stream-ordered allocations, for callers
// that cannot allocate device memory (their HBM is committed elsewhere, or an
// allocation's implicit synchronisation would stall their other streams).
//
// Scratch layout for up to SPK_NOALLOC_MAX_KEYS keys (3 operations each):
//   [map keys: kNaMapSlots u64][map values: kNaMapSlots u64]
//   [positions: kNaOps u64][bits-before-the-batch flags: kNaOps u8]
// The map needs a power of two of at least 2 * operations slots, so that
// every probe sequence of k_api_first finds a free or matching slot.
// ---------------------------------------------------------------------------
namespace {
constexpr uint64_t kNaMaxKeys = SPK_NOALLOC_MAX_KEYS;
constexpr uint64_t kNaOps = 3 * kNaMaxKeys;
constexpr uint64_t kNaMapSlots = 524288;  // next power of two >= 2 * kNaOps
static_assert(kNaMapSlots >= 2 * kNaOps && (kNaMapSlots & (kNaMapSlots - 1)) == 0,
              "map must hold twice the operations");
constexpr size_t kNaKeysOff = 0;
constexpr size_t kNaValsOff = kNaKeysOff + kNaMapSlots * 8;
constexpr size_t kNaPosOff = kNaValsOff + kNaMapSlots * 8;
constexpr size_t kNaInitOff = kNaPosOff + kNaOps * 8;
constexpr size_t kNaBytes = (kNaInitOff + kNaOps + 255) & ~(size_t)255;  // 9.7 MiB
}  // namespace

// One copy per device, reserved when the library's device code is loaded on
// that device and held until the process exits.  Host code must not use this
// name as a pointer (on the host it is only a stand-in for the symbol); it
// passes the address from cudaGetSymbolAddress to the kernels instead.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

namespace {
constexpr int kNaMaxDevices = 64;
struct NaDevice {
  unsigned char* scratch = nullptr;  // device address of g_noalloc_scratch
  int sm_count = 0;
  bool ready = false;
};
std::mutex g_na_mu;
NaDevice g_na_dev[kNaMaxDevices];

// Once per device, with that device current: the scratch array's device
// address and the SM count used to size the grid.
int noalloc_setup(int dev, NaDevice** out) {
  std::lock_guard<std::mutex> l(g_na_mu);
  NaDevice& d = g_na_dev[dev];
  if (!d.ready) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return spk::cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    if (!p) return spk::fail(SPK_E_CUDA, "cudaGetSymbolAddress returned a null scratch address");
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return spk::cuda_fail(e, "cudaDeviceGetAttribute(multiProcessorCount)");
    d.scratch = static_cast<unsigned char*>(p);
    d.sm_count = sms;
    d.ready = true;
  }
  *out = &d;
  return SPK_OK;
}
}  // namespace

extern "C" int spk_bloom_insert_k256_noalloc(uint64_t* d_seen, uint64_t* d_solid, uint64_t num_words,
                                             const uint64_t* d_keys4, size_t n,
                                             uint8_t* d_out_promoted, void* cuda_stream) {
  using namespace spk;
  if (n > kNaMaxKeys)
    return fail(SPK_E_INVALID_ARG, "spk_bloom_insert_k256_noalloc: n = " + std::to_string(n) +
                                       " keys exceeds the maximum of " + std::to_string(kNaMaxKeys) +
                                       " per call (SPK_NOALLOC_MAX_KEYS)");
  if (!d_seen || !d_solid) return fail(SPK_E_INVALID_ARG, "null tier pointer");
  if (num_words == 0) return fail(SPK_E_INVALID_ARG, "num_words must be at least 1");
  if (num_words > (~0ULL >> 6)) return fail(SPK_E_INVALID_ARG, "num_words too large");
  if (n && !d_keys4) return fail(SPK_E_INVALID_ARG, "null keys");
  if (n == 0) return SPK_OK;
  int dev = 0;
  SPK_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNaMaxDevices) return fail(SPK_E_INVALID_ARG, "device ordinal above 63");
  NaDevice* d = nullptr;
  int rc = noalloc_setup(dev, &d);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
  const uint64_t ops = 3 * (uint64_t)n;
  uint64_t mcap = 1;
  while (mcap < 2 * ops) mcap <<= 1;  // <= kNaMapSlots because n <= kNaMaxKeys
  unsigned long long* mk = reinterpret_cast<unsigned long long*>(d->scratch + kNaKeysOff);
  unsigned long long* mv = reinterpret_cast<unsigned long long*>(d->scratch + kNaValsOff);
  uint64_t* pos = reinterpret_cast<uint64_t*>(d->scratch + kNaPosOff);
  uint8_t* init = d->scratch + kNaInitOff;
  // The previous call's map is still in the array: reset the part this call uses.
  SPK_CUDA(cudaMemsetAsync(mk, 0xFF, mcap * 8, st));
  SPK_CUDA(cudaMemsetAsync(mv, 0xFF, mcap * 8, st));
  const FastMod fm = make_fastmod(num_words * 64);  // src/bloom.rs:27-28
  BloomKeys K{d_keys4, (uint64_t)n, 1};
  const unsigned grid = (unsigned)std::max<uint64_t>(
      1, std::min<uint64_t>((n + kB - 1) / kB, (uint64_t)std::max(d->sm_count, 1) * 8));
  k_api_first<<<grid, kB, 0, st>>>(K, fm, reinterpret_cast<const unsigned long long*>(d_seen), pos,
                                   init, mk, mv, mcap - 1);
  k_api_apply<<<grid, kB, 0, st>>>((uint64_t)n, pos, init, mk, mv, mcap - 1,
                                   reinterpret_cast<unsigned long long*>(d_seen),
                                   reinterpret_cast<unsigned long long*>(d_solid), d_out_promoted);
  SPK_CUDA(cudaGetLastError());
  return SPK_OK;
}
