// spk_api.cu -- C ABI entry points of libspk (declared in include/spk.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <cstdio>
#include <cstring>
#include <string>

#include "spk_internal.h"

namespace spk {

// ---- errors -------------------------------------------------------------------
static thread_local std::string g_err;
void set_error(const std::string& msg) { g_err = msg; }
int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
int cuda_fail(cudaError_t e, const char* what) {
  g_err = std::string(what) + ": " + cudaGetErrorString(e);
  if (e == cudaErrorMemoryAllocation) return SPK_E_OOM;
  return SPK_E_CUDA;
}

int raise_smem_limit(const void* kernel, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, size_t> limits;
  int dev = 0;
  SPK_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  size_t& cur = limits[{kernel, dev}];
  if (bytes <= cur) return SPK_OK;
  SPK_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  cur = bytes;
  return SPK_OK;
}

int current_sm_count() {
  static std::mutex mu;
  static std::map<int, int> cache;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return 148;
  }
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find(dev);
  if (it != cache.end()) return it->second;
  int n = 0;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1) {
    cudaGetLastError();
    n = 148;
  }
  cache[dev] = n;
  return n;
}

namespace {
struct Pools {
  std::mutex mu;
  std::map<int, std::vector<cudaStream_t>> streams;
  std::map<int, std::vector<cudaEvent_t>> events[2];  // [timing]
};
Pools& pools() {
  static Pools* p = new Pools();  // kept to process exit: handles outlive contexts
  return *p;
}
int cur_device() {
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess) cudaGetLastError();
  return d;
}
}  // namespace

cudaStream_t pooled_stream() {
  const int d = cur_device();
  {
    std::lock_guard<std::mutex> l(pools().mu);
    auto& v = pools().streams[d];
    if (!v.empty()) {
      cudaStream_t s = v.back();
      v.pop_back();
      return s;
    }
  }
  cudaStream_t s = nullptr;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return s;
}
void pooled_stream_put(cudaStream_t s) {
  if (!s) return;
  std::lock_guard<std::mutex> l(pools().mu);
  pools().streams[cur_device()].push_back(s);
}
cudaEvent_t pooled_event(bool timing) {
  const int d = cur_device();
  {
    std::lock_guard<std::mutex> l(pools().mu);
    auto& v = pools().events[timing ? 1 : 0][d];
    if (!v.empty()) {
      cudaEvent_t e = v.back();
      v.pop_back();
      return e;
    }
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreateWithFlags(&e, timing ? cudaEventDefault : cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return e;
}
void pooled_event_put(cudaEvent_t e, bool timing) {
  if (!e) return;
  std::lock_guard<std::mutex> l(pools().mu);
  pools().events[timing ? 1 : 0][cur_device()].push_back(e);
}

// ---- FastMod constants (Granlund & Montgomery 1994, Fig. 4.1, N = 64) ---------
FastMod make_fastmod(uint64_t d) {
  FastMod f{};
  f.d = d;
  f.pow2 = (d & (d - 1)) == 0;
  f.mask = d - 1;
  unsigned l = 0;
  while (l < 64 && (1ULL << l) < d) l++;  // l = ceil(log2 d)
  typedef unsigned __int128 u128;
  const u128 two_l = (u128)1 << l;
  f.mprime = (uint64_t)((((u128)1 << 64) * (two_l - d)) / d + 1);
  f.sh1 = l < 1 ? l : 1;
  f.sh2 = l >= 1 ? l - 1 : 0;
  return f;
}

// ---- device memory --------------------------------------------------------------
int DevBuf::alloc(size_t n, cudaStream_t s) {
  release();
  if (n == 0) n = 16;
  // No trimming of the pool here: other jobs may be running on the same
  // pool, and giving its cached memory back would make all of them map it
  // again (tens of ms per GB).  A job that runs out reports SPK_E_OOM; the
  // batch runs it again alone after trimming (spk_count_batch).
  cudaError_t e = cudaMallocAsync(&p, n, s);
  if (e != cudaSuccess) {
    cudaGetLastError();
    p = nullptr;
    char msg[128];
    snprintf(msg, sizeof msg, "device allocation of %zu bytes failed", n);
    return fail(SPK_E_OOM, msg);
  }
  bytes = n;
  st = s;
  return SPK_OK;
}
// The results pool of the current device (created on first use; nullptr if
// the driver refuses one: results then come from the default pool).
static cudaMemPool_t results_pool() {
  static std::mutex mu;
  static std::map<int, cudaMemPool_t> pools;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  std::lock_guard<std::mutex> l(mu);
  auto it = pools.find(dev);
  if (it != pools.end()) return it->second;
  cudaMemPoolProps props = {};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = dev;
  cudaMemPool_t p = nullptr;
  if (cudaMemPoolCreate(&p, &props) != cudaSuccess) {
    cudaGetLastError();
    p = nullptr;
  } else {
    uint64_t thr = ~0ULL;  // keep freed blocks cached, as the default pool does
    cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  pools[dev] = p;
  return p;
}

int DevBuf::alloc_keep(size_t n, cudaStream_t s) {
  cudaMemPool_t pool = results_pool();
  if (!pool) return alloc(n, s);
  release();
  if (n == 0) n = 16;
  cudaError_t e = cudaMallocFromPoolAsync(&p, n, pool, s);
  if (e != cudaSuccess) {
    cudaGetLastError();
    p = nullptr;
    return alloc(n, s);  // the default pool may still have room
  }
  bytes = n;
  st = s;
  return SPK_OK;
}

void DevBuf::release() {
  if (p) cudaFreeAsync(p, st);
  p = nullptr;
  bytes = 0;
}

// ---- pinned staging blocks ----------------------------------------------------
uint64_t* staging_acquire(spk_ctx* ctx) {
  std::lock_guard<std::mutex> l(ctx->staging_mu);
  if (!ctx->staging_free.empty()) {
    uint64_t* b = ctx->staging_free.back();
    ctx->staging_free.pop_back();
    return b;
  }
  uint64_t* b = nullptr;
  if (cudaMallocHost((void**)&b, kStagingBytes) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  ctx->staging_all.push_back(b);
  return b;
}
void staging_release(spk_ctx* ctx, uint64_t* block) {
  if (!block) return;
  std::lock_guard<std::mutex> l(ctx->staging_mu);
  ctx->staging_free.push_back(block);
}
void pool_reserve(spk_ctx* ctx, uint64_t bytes) {
  if (!ctx->pool) return;
  std::lock_guard<std::mutex> l(ctx->pool_mu);
  if (bytes <= ctx->pool_reserved) return;
  if (cudaDeviceSynchronize() != cudaSuccess || cudaMemPoolTrimTo(ctx->pool, 0) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  size_t f = 0, t = 0;
  if (cudaMemGetInfo(&f, &t) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  const uint64_t room = (uint64_t)f > (1ull << 30) ? (uint64_t)f - (1ull << 30) : 0;  // leave 1 GiB to others
  const uint64_t n = std::min<uint64_t>(bytes, room);
  // (a request the device cannot hold in full is not retried until a larger one comes)
  ctx->pool_reserved = bytes;
  if (n < (2ull << 20)) return;
  void* p = nullptr;
  cudaStream_t st = ctx->own_stream;
  if (cudaMallocAsync(&p, n, st) != cudaSuccess || cudaFreeAsync(p, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    cudaGetLastError();  // a hint: without it the pool grows as the jobs need
  // The results' pool gets a block too (a sixteenth: lists and edges are a
  // few percent of a job's temporaries).
  if (cudaMemPool_t rp = results_pool()) {
    p = nullptr;
    if (cudaMallocFromPoolAsync(&p, n / 16 + (2ull << 20), rp, st) != cudaSuccess ||
        cudaFreeAsync(p, st) != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
      cudaGetLastError();
  }
}

void pool_trim(spk_ctx* ctx) {
  if (!ctx->pool) return;
  std::lock_guard<std::mutex> l(ctx->pool_mu);
  cudaMemPoolTrimTo(ctx->pool, 0);
  if (cudaMemPool_t rp = results_pool()) cudaMemPoolTrimTo(rp, 0);  // its unused blocks only
  ctx->pool_reserved = 0;
}

spk_result* result_new(spk_ctx* ctx, cudaStream_t st, bool own_stream) {
  uint64_t* h = staging_acquire(ctx);
  if (!h) {
    fail(SPK_E_OOM, "pinned host staging allocation failed");
    return nullptr;
  }
  auto* res = new spk_result();
  res->ctx = ctx;
  res->stream = st;
  res->own_stream = own_stream;
  res->h_staging = h;
  return res;
}

int bloom_create(spk_ctx* ctx, uint64_t capacity_bits, spk_bloom** out);
int bloom_insert(spk_bloom* b, const uint64_t* keys, size_t n, int wide, uint8_t* promoted);
int bloom_query(spk_bloom* b, const uint64_t* keys, size_t n, int wide, uint8_t* out);
int bloom_download(spk_bloom* b, uint64_t* seen, uint64_t* solid);
void serve_shutdown(spk_ctx* ctx);

static int use_device(spk_ctx* ctx) {
  if (!ctx) return fail(SPK_E_INVALID_ARG, "null context");
  SPK_CUDA(cudaSetDevice(ctx->device));
  return SPK_OK;
}

static int check_ks(const uint32_t* ks, int n_k) {
  if (!ks || n_k < 1) return fail(SPK_E_INVALID_ARG, "at least one k is required");
  for (int i = 0; i < n_k; i++)
    if (ks[i] < 1 || ks[i] > 127)
      return fail(SPK_E_INVALID_K, "k=" + std::to_string(ks[i]) + " is outside 1..=127");
  return SPK_OK;
}

// Copies packed reads to the device (data padded so that k-mer windows may
// read whole 64-bit words past the last byte).
constexpr uint64_t kChunkedUploadMin = 32ull << 20;  // bytes of packed data
constexpr int kUploadChunks = 4;

int upload_reads(spk_result* res, cudaStream_t st, const uint8_t* data, size_t data_len,
                 const uint64_t* offsets, const uint32_t* lengths, size_t n_reads, ReadsView* rv,
                 bool chunked) {
  int rc;
  const size_t padded = ((data_len + 7) / 8) * 8 + 64;
  if ((rc = res->reads.alloc(padded, st))) return rc;
  if ((rc = res->offs.alloc(std::max<size_t>(n_reads, 1) * 8, st))) return rc;
  if ((rc = res->lens.alloc(std::max<size_t>(n_reads, 1) * 4, st))) return rc;
  // Zero the tail from the last whole word of data to the end of the padding.
  const size_t tail = data_len & ~(size_t)7;
  SPK_CUDA(cudaMemsetAsync(res->reads.as<uint8_t>() + tail, 0, padded - tail, st));
  if (n_reads) {
    if ((rc = xfer_h2d(res->ctx, res->offs.p, offsets, n_reads * 8, st))) return rc;
    if ((rc = xfer_h2d(res->ctx, res->lens.p, lengths, n_reads * 4, st))) return rc;
  }
  rv->words = res->reads.as<uint64_t>();
  rv->offsets = res->offs.as<uint64_t>();
  rv->lengths = res->lens.as<uint32_t>();
  rv->n_reads = n_reads;
  rv->byte_base = 0;
  rv->data_len = data_len;
  rv->err = nullptr;
  rv->chunks = nullptr;
  if (!chunked || data_len < kChunkedUploadMin || n_reads < 2)
    return xfer_h2d(res->ctx, res->reads.p, data, data_len, st);
  // Large read sets: the data go up in kUploadChunks pieces on a copy stream,
  // so that the count's first pass works on the reads of a piece while the
  // next one is copied.  Reads [0, read_end[c]) end at least 64 bytes before
  // byte_end[c] (the word loads of a read reach past its last byte) if the
  // reads lie in order; the count checks that on the device and otherwise
  // waits for the last piece.
  ReadChunks& ch = res->chunks;
  res->copy_stream = pooled_stream();
  cudaEvent_t alloc_done = pooled_event(false);
  if (!res->copy_stream || !alloc_done) return fail(SPK_E_CUDA, "upload stream or event");
  cudaError_t e = cudaEventRecord(alloc_done, st);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(res->copy_stream, alloc_done, 0);
  pooled_event_put(alloc_done, false);
  if (e != cudaSuccess) return cuda_fail(e, "upload stream");
  ch.n = kUploadChunks;
  uint64_t b0 = 0;
  for (int c = 0; c < ch.n; c++) {
    uint64_t b1 = c + 1 == ch.n ? data_len : (data_len * (c + 1) / ch.n) & ~(uint64_t)7;
    if (b1 < b0) b1 = b0;
    ch.byte_end[c] = b1;
    if (c + 1 == ch.n) {
      ch.read_end[c] = n_reads;
    } else {
      // reads i with offsets[i + 1] <= b1 - 64 (offsets ascending when in order)
      const uint64_t lim = b1 >= 64 ? b1 - 64 : 0;
      const uint64_t j = (uint64_t)(std::upper_bound(offsets, offsets + n_reads, lim) - offsets);
      ch.read_end[c] = j > 0 ? j - 1 : 0;
    }
    ch.ready[c] = pooled_event(false);
    if (!ch.ready[c]) return fail(SPK_E_CUDA, "upload event");
    if (b1 > b0 && (rc = xfer_h2d(res->ctx, res->reads.as<uint8_t>() + b0, data + b0, b1 - b0, res->copy_stream)))
      return rc;
    SPK_CUDA(cudaEventRecord(ch.ready[c], res->copy_stream));
    b0 = b1;
  }
  rv->chunks = &ch;
  return SPK_OK;
}

int stuck_claim(spk_ctx* ctx, uint32_t k);

}  // namespace spk

using namespace spk;

extern "C" {

const char* spk_last_error(void) { return g_err.c_str(); }

int spk_diag_stuck_claim(spk_ctx* ctx, uint32_t k) {
  int rc = use_device(ctx);
  if (rc) return rc;
  return stuck_claim(ctx, k);
}
int spk_version(void) { return SPK_VERSION; }

// src/main.rs:11-30
int spk_validate_k(uint32_t k) {
  if (k < 11) return fail(SPK_E_INVALID_K, "k=" + std::to_string(k) + " is too small; minimum is 11");
  if (k > 127)
    return fail(SPK_E_INVALID_K, "k=" + std::to_string(k) + " exceeds maximum of 127 (Kmer256 limit)");
  if (k % 2 == 0)
    return fail(SPK_E_INVALID_K, "k=" + std::to_string(k) + " is even; SPAdes requires an odd k-mer size");
  return SPK_OK;
}

int spk_ctx_create(int device, spk_ctx** out) {
  if (!out) return fail(SPK_E_INVALID_ARG, "null output pointer");
  *out = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    return fail(SPK_E_NO_DEVICE, "no CUDA device is available");
  }
  if (device < 0 || device >= n) return fail(SPK_E_INVALID_ARG, "device index out of range");
  cudaDeviceProp prop;
  SPK_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10)
    return fail(SPK_E_NO_DEVICE, std::string("libspk is built for sm_100a; device is ") + prop.name);
  SPK_CUDA(cudaSetDevice(device));
  auto* c = new spk_ctx();
  c->device = device;
  c->sm_count = prop.multiProcessorCount;
  c->l2_bytes = prop.l2CacheSize;
  c->total_mem = prop.totalGlobalMem;
  e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
  c->stream = c->own_stream;
  if (e == cudaSuccess) e = cudaDeviceGetDefaultMemPool(&c->pool, device);
  if (e == cudaSuccess) {
    uint64_t thr = ~0ULL;  // keep freed blocks cached in the pool
    e = cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  // The hot kernels make random 8-32 byte accesses (Bloom words, table
  // slots); fetch only the 32-byte sector that was asked for.  This is a
  // limit of this process's context, not a device setting.
  if (e == cudaSuccess) {
    cudaError_t g = cudaDeviceSetLimit(cudaLimitMaxL2FetchGranularity, 32);
    if (g != cudaSuccess) cudaGetLastError();  // a hint; ignore if unsupported
  }
  if (e != cudaSuccess) {
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
    return cuda_fail(e, "context setup");
  }
  *out = c;
  return SPK_OK;
}

int spk_ctx_destroy(spk_ctx* ctx) {
  if (!ctx) return SPK_OK;
  cudaSetDevice(ctx->device);
  serve_shutdown(ctx);
  xfer_shutdown(ctx);
  ctx->scratch.release();
  cudaStreamSynchronize(ctx->stream);
  for (cudaStream_t& s : ctx->batch_streams)
    if (s) {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
      s = nullptr;
    }
  for (uint64_t* b : ctx->staging_all) cudaFreeHost(b);
  cudaStreamDestroy(ctx->own_stream);
  pool_trim(ctx);
  delete ctx;
  return SPK_OK;
}

int spk_ctx_memory(spk_ctx* ctx, uint64_t* reserved_bytes, uint64_t* free_bytes) {
  int rc;
  if ((rc = use_device(ctx))) return rc;
  if (reserved_bytes) {
    uint64_t v = 0;
    SPK_CUDA(cudaMemPoolGetAttribute(ctx->pool, cudaMemPoolAttrReservedMemCurrent, &v));
    *reserved_bytes = v;
  }
  if (free_bytes) {
    size_t f = 0, t = 0;
    SPK_CUDA(cudaMemGetInfo(&f, &t));
    *free_bytes = f;
  }
  return SPK_OK;
}

int spk_ctx_set_stream(spk_ctx* ctx, void* cuda_stream) {
  int rc;
  if ((rc = use_device(ctx))) return rc;
  SPK_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->stream = cuda_stream ? (cudaStream_t)cuda_stream : ctx->own_stream;
  return SPK_OK;
}

// ---- TwoTierFilter ------------------------------------------------------------
int spk_bloom_create(spk_ctx* ctx, uint64_t capacity_bits, spk_bloom** out) {
  int rc;
  if (!out) return fail(SPK_E_INVALID_ARG, "null output pointer");
  if ((rc = use_device(ctx))) return rc;
  return bloom_create(ctx, capacity_bits, out);
}
int spk_bloom_destroy(spk_bloom* b) {
  if (!b) return SPK_OK;
  cudaSetDevice(b->ctx->device);
  b->seen.release();
  b->solid.release();
  cudaStreamSynchronize(b->ctx->stream);
  delete b;
  return SPK_OK;
}
uint64_t spk_bloom_size_bits(const spk_bloom* b) { return b ? b->size_bits : 0; }
uint64_t spk_bloom_memory_usage_bytes(const spk_bloom* b) { return b ? b->num_words * 8 * 2 : 0; }

static int bloom_call(spk_bloom* b, const uint64_t* keys, size_t n, int wide, uint8_t* out,
                      bool insert) {
  int rc;
  if (!b) return fail(SPK_E_INVALID_ARG, "null filter");
  if (n && !keys) return fail(SPK_E_INVALID_ARG, "null keys");
  if (!insert && n && !out) return fail(SPK_E_INVALID_ARG, "null output");
  if ((rc = use_device(b->ctx))) return rc;
  return insert ? bloom_insert(b, keys, n, wide, out) : bloom_query(b, keys, n, wide, out);
}
int spk_bloom_insert_u64(spk_bloom* b, const uint64_t* keys, size_t n, uint8_t* out_promoted) {
  return bloom_call(b, keys, n, 0, out_promoted, true);
}
int spk_bloom_insert_k256(spk_bloom* b, const uint64_t* keys4, size_t n, uint8_t* out_promoted) {
  return bloom_call(b, keys4, n, 1, out_promoted, true);
}
int spk_bloom_is_solid_u64(spk_bloom* b, const uint64_t* keys, size_t n, uint8_t* out) {
  return bloom_call(b, keys, n, 0, out, false);
}
int spk_bloom_is_solid_k256(spk_bloom* b, const uint64_t* keys4, size_t n, uint8_t* out) {
  return bloom_call(b, keys4, n, 1, out, false);
}
int spk_bloom_download(spk_bloom* b, uint64_t* seen, uint64_t* solid) {
  int rc;
  if (!b) return fail(SPK_E_INVALID_ARG, "null filter");
  if ((rc = use_device(b->ctx))) return rc;
  return bloom_download(b, seen, solid);
}

// ---- counting -------------------------------------------------------------------
void spk_count_opts_default(spk_count_opts* o) {
  if (!o) return;
  memset(o, 0, sizeof *o);
  o->bloom_bits = 512ULL << 20;  // src/assemble.rs:84
  o->min_count = 0;
  o->list_min_count = 2;
  o->min_coverage = 5.0;         // src/assemble.rs:82
  o->flags = SPK_F_EDGES | SPK_F_KEEP_BLOOM;
}

static spk_count_opts resolve_opts(const spk_count_opts* o) {
  spk_count_opts r;
  spk_count_opts_default(&r);
  if (o) r = *o;
  if (!r.bloom_bits) r.bloom_bits = 512ULL << 20;
  if (!r.list_min_count) r.list_min_count = 2;
  return r;
}

int spk_count(spk_ctx* ctx, const uint8_t* data, size_t data_len, const uint64_t* offsets,
              const uint32_t* lengths, size_t n_reads, const uint32_t* ks, int n_k,
              const spk_count_opts* opts, spk_result** out) {
  int rc;
  if (!out) return fail(SPK_E_INVALID_ARG, "null output pointer");
  *out = nullptr;
  if ((rc = use_device(ctx))) return rc;
  if ((rc = check_ks(ks, n_k))) return rc;
  if (n_reads && (!offsets || !lengths)) return fail(SPK_E_INVALID_ARG, "null offsets/lengths");
  if (data_len && !data) return fail(SPK_E_INVALID_ARG, "null data");
  auto* res = result_new(ctx, ctx->stream, false);
  if (!res) return SPK_E_OOM;
  res->opts = resolve_opts(opts);
  ReadsView rv;
  rc = upload_reads(res, ctx->stream, data, data_len, offsets, lengths, n_reads, &rv, true);
  if (!rc) rc = count_pipeline(ctx, ctx->stream, rv, 0, ks, n_k, res->opts, res);
  if (res->chunks.n)  // the reads' buffer is freed after every piece has landed
    cudaStreamWaitEvent(ctx->stream, res->chunks.ready[res->chunks.n - 1], 0);
  if (rc) {
    spk_result_free(res);
    return rc;
  }
  // The reads are not needed after counting.
  res->reads.release();
  res->offs.release();
  res->lens.release();
  *out = res;
  return SPK_OK;
}

int spk_count_device(spk_ctx* ctx, const uint8_t* d_data, size_t data_len,
                     const uint64_t* d_offsets, const uint32_t* d_lengths, size_t n_reads,
                     const uint32_t* ks, int n_k, const spk_count_opts* opts, spk_result** out) {
  int rc;
  if (!out) return fail(SPK_E_INVALID_ARG, "null output pointer");
  *out = nullptr;
  if ((rc = use_device(ctx))) return rc;
  if ((rc = check_ks(ks, n_k))) return rc;
  if (n_reads && (!d_offsets || !d_lengths || !d_data))
    return fail(SPK_E_INVALID_ARG, "null device pointer");
  auto* res = result_new(ctx, ctx->stream, false);
  if (!res) return SPK_E_OOM;
  res->opts = resolve_opts(opts);
  ReadsView rv;
  const uintptr_t a = (uintptr_t)d_data;
  rv.words = (const uint64_t*)(a & ~(uintptr_t)7);
  rv.byte_base = a & 7;
  rv.offsets = d_offsets;
  rv.lengths = d_lengths;
  rv.n_reads = n_reads;
  rv.data_len = data_len;
  rv.err = nullptr;
  rv.chunks = nullptr;
  rc = count_pipeline(ctx, ctx->stream, rv, 0, ks, n_k, res->opts, res);
  if (rc) {
    spk_result_free(res);
    return rc;
  }
  *out = res;
  return SPK_OK;
}

static int get_k(const spk_result* res, int ki) {
  if (!res) return fail(SPK_E_INVALID_ARG, "null result");
  if (ki < 0 || ki >= (int)res->ks.size()) return fail(SPK_E_INVALID_ARG, "k index out of range");
  return use_device(res->ctx);
}

int spk_result_count(const spk_result* res, int* n_k) {
  if (!res || !n_k) return fail(SPK_E_INVALID_ARG, "null argument");
  *n_k = (int)res->ks.size();
  return SPK_OK;
}
int spk_result_info_get(const spk_result* res, int ki, spk_result_info* info) {
  int rc;
  if ((rc = get_k(res, ki))) return rc;
  if (!info) return fail(SPK_E_INVALID_ARG, "null info");
  *info = res->ks[ki]->info;
  const UnitigSet& u = res->ks[ki]->unitigs;
  if (u.ready) {
    info->ms_unitigs = u.ms_device;
    info->ms_unitigs_host = u.ms_host;
    info->unitig_launches = u.launches;
    info->n_unitigs = u.lengths.size();
  }
  return SPK_OK;
}
int spk_result_solid(spk_result* res, int ki, uint64_t* keys, uint32_t* counts, size_t* n) {
  int rc;
  if ((rc = get_k(res, ki))) return rc;
  if (!n) return fail(SPK_E_INVALID_ARG, "null size pointer");
  return download_list(res, ki, 0, true, keys, counts, n);
}
int spk_result_kmers(spk_result* res, int ki, uint32_t min_count, uint64_t* keys, uint32_t* counts,
                     size_t* n) {
  int rc;
  if ((rc = get_k(res, ki))) return rc;
  if (!n) return fail(SPK_E_INVALID_ARG, "null size pointer");
  return download_list(res, ki, min_count, false, keys, counts, n);
}
int spk_result_edges(spk_result* res, int ki, uint64_t* edges, size_t* n) {
  int rc;
  if ((rc = get_k(res, ki))) return rc;
  if (!n) return fail(SPK_E_INVALID_ARG, "null size pointer");
  return download_edges(res, ki, edges, n);
}
int spk_result_bloom(spk_result* res, int ki, uint64_t* seen, uint64_t* twice, uint64_t* ref_solid) {
  int rc;
  if ((rc = get_k(res, ki))) return rc;
  return download_bloom(res, ki, seen, twice, ref_solid);
}
int spk_result_table_view(spk_result* res, int ki, spk_table_view* v) {
  int rc;
  if ((rc = get_k(res, ki))) return rc;
  if (!v) return fail(SPK_E_INVALID_ARG, "null view");
  KResult& kr = *res->ks[ki];
  if (!kr.tslots.p)
    return fail(SPK_E_INVALID_ARG, "the count table was not kept (SPK_F_KEEP_TABLE)");
  v->slots = kr.table.slots;
  v->capacity = kr.table.capacity;
  v->key_limbs = (uint32_t)kr.nl;
  v->slot_bytes = kr.table.slot_bytes;
  v->k = kr.k;
  v->cutoff = kr.info.cutoff;
  v->log2span = kr.table.log2span;
  v->reserved = 0;
  return SPK_OK;
}
int spk_result_free(spk_result* res) {
  if (!res) return SPK_OK;
  cudaSetDevice(res->ctx->device);
  cudaStream_t st = res->stream;
  res->ks.clear();
  res->reads.release();
  res->offs.release();
  res->lens.release();
  cudaStreamSynchronize(st);
  staging_release(res->ctx, res->h_staging);
  if (res->own_stream) pooled_stream_put(st);  // synchronised above: idle
  delete res;
  return SPK_OK;
}

}  // extern "C"
