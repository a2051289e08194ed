// spk_internal.h -- host-side structures shared by the libspk translation units.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/spk.h"
#include "spk_device.cuh"

namespace spk {

// ---- errors -----------------------------------------------------------------
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);
#define SPK_CUDA(call)                                  \
  do {                                                  \
    cudaError_t _e = (call);                            \
    if (_e != cudaSuccess) return ::spk::cuda_fail(_e, #call); \
  } while (0)

// Host construction of the division constants of FastMod.
FastMod make_fastmod(uint64_t d);

// ---- device memory ------------------------------------------------------------
// Stream-ordered allocations from the device's memory pool (cudaMallocAsync),
// with the pool's release threshold raised so freed blocks stay cached
// between jobs instead of returning to the driver.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaStream_t st = nullptr;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept { *this = std::move(o); }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      release();
      p = o.p; bytes = o.bytes; st = o.st;
      o.p = nullptr; o.bytes = 0;
    }
    return *this;
  }
  ~DevBuf() { release(); }
  int alloc(size_t n, cudaStream_t s);
  // The same from a second pool of the device that holds only what results
  // keep (their lists, edges and converted downloads), so that buffers kept
  // past a job do not sit in the middle of the memory the next job's large
  // temporaries come from (that made the pool map new memory mid-job).
  int alloc_keep(size_t n, cudaStream_t s);
  void release();
  template <class T> T* as() const { return static_cast<T*>(p); }
};

// ---- packed reads on the device --------------------------------------------
// Packed data copied up in chunks on a copy stream (spk_count with host
// buffers): chunk c holds bytes [0, byte_end[c]) once ready[c] has fired,
// and, when the reads lie in order (each read at or after the end of the one
// before it, which the device checks), reads [0, read_end[c]) lie in it.
// Offsets and lengths are on the device before the count starts.
constexpr int kMaxReadChunks = 8;
struct ReadChunks {
  int n = 0;
  uint64_t byte_end[kMaxReadChunks] = {};
  uint64_t read_end[kMaxReadChunks] = {};
  cudaEvent_t ready[kMaxReadChunks] = {};
};

struct ReadsView {
  const uint64_t* words;    // packed bytes viewed as 64-bit words (8-byte aligned base)
  const uint64_t* offsets;  // byte offset of each read, relative to byte_base
  const uint32_t* lengths;  // bases per read
  uint64_t n_reads;
  uint64_t byte_base;       // byte offset of data[0] from `words`
  uint64_t data_len;        // bytes of packed data; reads beyond it are rejected
  int* err;                 // device error word: bit 2 set for an out-of-bounds read
  const ReadChunks* chunks; // host: the data still arriving in chunks, or nullptr
};

// ---- count table --------------------------------------------------------------
// Open addressing, linear probing; one slot of slot_bytes per entry: key limbs
// (sequence value V) first, then the u32 count (and a u32 state word for keys
// wider than 128 bits).  Count 0 marks an empty slot after counting.  The
// table is divided into spans of 2^log2span slots and a probe sequence wraps
// inside the span of its home slot (log2span == log2cap: the whole table).
struct TableView {
  uint8_t* slots;
  uint64_t capacity;  // power of two
  uint32_t log2cap;
  uint32_t slot_bytes;
  uint32_t max_probe;
  uint32_t log2span;
  int* err;           // device error word (bit 0: probe limit, bit 1: wait timeout)
};

// ---- per-k result ---------------------------------------------------------------
// Unitigs of the solid k-mers (spk_graph.cu), built on first request.
struct UnitigSet {
  bool ready = false;
  std::string seq;                // concatenated sequences
  std::vector<uint64_t> lengths;  // bases per unitig
  std::vector<double> cov;        // mean k-mer count
  std::vector<uint64_t> kmers;    // k-mers per unitig
  uint32_t launches = 0;          // kernels the build launched
  float ms_device = 0.f;          // device time of the build (kernels and copies)
  float ms_host = 0.f;            // host time of the orientation and sort
};

struct KResult {
  uint32_t k = 0;
  int nl = 0;
  spk_result_info info{};
  FastMod fm{};
  uint64_t num_words = 0;
  DevBuf tiers;       // (seen, twice) word pairs while counting
  DevBuf seen;        // compact seen tier, num_words * 8 bytes
  DevBuf twice;       // compact twice tier, num_words * 8 bytes
  DevBuf ref_solid;   // reference-semantics solid tier (SPK_F_REF_SOLID)
  DevBuf tslots;      // count table slots
  TableView table{};
  DevBuf list[5];     // sorted k-mer list: limbs 0..nl-1 (SoA), counts in list[4]
  DevBuf edges[4];    // sorted edge list: limbs (SoA)
  int nle = 0;        // limbs per edge key
  uint32_t list_min = 2;  // smallest count downloads of the list return
  uint64_t list_len = 0;  // entries in the list buffers (may include counts below list_min)
  // The last converted download (kind 0: k-mer list with counts >= minc, 1:
  // edges), kept for the copy that follows a size query.
  struct Conv {
    int kind = -1;
    uint32_t minc = 0;
    uint64_t n = 0;
    DevBuf keys, cnt;
  } conv;
  UnitigSet unitigs;
};

struct spk_result_impl;

// Non-blocking streams and events of the current device, reused across jobs
// (a job then makes no stream or event creation call, which can wait on
// other clients of the driver).  A stream handed back may still have work
// queued; its next user's work runs after it.
cudaStream_t pooled_stream();
void pooled_stream_put(cudaStream_t s);
cudaEvent_t pooled_event(bool timing);
void pooled_event_put(cudaEvent_t e, bool timing);

// Copies between host memory and the device on stream st (spk_xfer.cu).
// Pageable host memory goes through pinned chunks with several host threads;
// pinned memory is copied directly.  xfer_h2d returns once every piece is
// enqueued (the host source may be reused); xfer_d2h once the data is on the
// host.
struct XferPool;
int xfer_h2d(spk_ctx* ctx, void* dst, const void* src, size_t n, cudaStream_t st);
int xfer_d2h(spk_ctx* ctx, void* dst, const void* src, size_t n, cudaStream_t st);
void xfer_shutdown(spk_ctx* ctx);

}  // namespace spk

// ---- opaque handles --------------------------------------------------------------
struct spk_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;      // stream in use (own_stream or a caller's)
  cudaStream_t own_stream = nullptr;
  cudaMemPool_t pool = nullptr;
  int sm_count = 0;
  size_t l2_bytes = 0;
  size_t total_mem = 0;     // device memory (the partitioned passes size against it)
  spk::DevBuf scratch;      // small device scratch (counters, flags)
  // Pinned host staging blocks (kStagingBytes each) for counters read back
  // during a count.  Every result holds its own block, so jobs that run
  // concurrently (serving, batches) never share one.
  std::mutex staging_mu;
  std::vector<uint64_t*> staging_free, staging_all;
  // serving
  struct Server* server = nullptr;
  std::mutex serve_mu;
  // host threads and pinned chunks for copies from and to pageable memory
  // (created on first use)
  spk::XferPool* xfer = nullptr;
  std::mutex xfer_mu;
  // spk_count_batch: the upload stream and the lanes' streams (created on
  // first use, kept until the context is destroyed; batch results do their
  // later work on their lane's stream).  A fixed handful of streams, because
  // the device memory pool's allocations slow down with every stream that
  // has used it (measured: 1.4 us per allocation with 3 streams, 11 us after
  // a batch that gave every job streams of its own).
  cudaStream_t batch_streams[8] = {};
  std::mutex batch_mu;  // one batch at a time per context
  std::condition_variable batch_cv;
  bool batch_active = false;
  // Bytes of the one contiguous block the memory pool was last grown by
  // (spk::pool_reserve); 0 after the pool gave its cached memory back.
  uint64_t pool_reserved = 0;
  std::mutex pool_mu;
};

struct spk_bloom {
  spk_ctx* ctx = nullptr;
  uint64_t size_bits = 0, num_words = 0;
  spk::FastMod fm{};
  spk::DevBuf seen, solid;
};

struct spk_result {
  spk_ctx* ctx = nullptr;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  // chunked upload of the packed data (copy stream and its events), kept
  // until the count has used the reads
  spk::ReadChunks chunks;
  cudaStream_t copy_stream = nullptr;
  ~spk_result() {
    for (int c = 0; c < chunks.n; c++)
      if (chunks.ready[c]) spk::pooled_event_put(chunks.ready[c], false);
    if (copy_stream) spk::pooled_stream_put(copy_stream);
  }
  spk_count_opts opts{};
  std::vector<std::unique_ptr<spk::KResult>> ks;
  spk::DevBuf reads;  // device copy of the packed reads (when copied in by spk_count)
  spk::DevBuf offs, lens;
  uint64_t* h_staging = nullptr;  // pinned staging block of this result (from ctx)
};

namespace spk {
constexpr size_t kStagingBytes = 1 << 16;
// A pinned staging block for one result (nullptr if pinned memory is
// exhausted), and its return to the context's free list.
uint64_t* staging_acquire(spk_ctx* ctx);
void staging_release(spk_ctx* ctx, uint64_t* block);
// A new result on stream st with its own staging block, or nullptr (error set).
spk_result* result_new(spk_ctx* ctx, cudaStream_t st, bool own_stream);
// Grows the device memory pool by one contiguous block of at least `bytes`
// (capped by what the device has free), unless the last such block is as
// large already.  Jobs whose buffers come and go in sizes the pool has not
// seen make it map new memory piece by piece, in the middle of their kernels'
// work (about 8 ms per GB, and more when the pieces are fragmented); one
// block mapped up front serves them all.  It waits for the whole device and
// gives the pool's unused memory back first, so the caller makes sure no job
// of the context is running.
void pool_reserve(spk_ctx* ctx, uint64_t bytes);
// The pool's cached memory given back (a job that ran out of memory runs
// again): the reservation is gone too.
void pool_trim(spk_ctx* ctx);
// Count pipeline on device-resident reads (spk_count.cu).  `res` is filled
// with one KResult per k.
int count_pipeline(spk_ctx* ctx, cudaStream_t st, const ReadsView& rv, uint32_t max_len,
                   const uint32_t* ks, int n_k, const spk_count_opts& o, spk_result* res);
// Host copies of result lists (spk_count.cu).
int download_list(spk_result* res, int ki, uint32_t min_count, bool solid_only, uint64_t* keys,
                  uint32_t* counts, size_t* n_inout);
int download_edges(spk_result* res, int ki, uint64_t* out, size_t* n_inout);
int download_bloom(spk_result* res, int ki, uint64_t* seen, uint64_t* twice, uint64_t* ref_solid);

// Radix sort of SoA keys (spk_sort.cu): keys[0..nl) limbs (least significant
// first) and optional u32 values, sorted ascending by the low nbits of the
// key.  The buffers may be swapped with temporaries.
int radix_sort_bufs(cudaStream_t st, int nl, uint64_t n, unsigned nbits, DevBuf* keys,
                    DevBuf* vals, uint32_t* launches = nullptr);
// The same result with an MSD split into 65536 buckets by the top 16 bits and
// a shared-memory sort per bucket (large lists; falls back to the radix sort
// for short lists and for buckets too large for shared memory).  h_staging:
// a pinned host staging block (kStagingBytes).
int sort_bufs(cudaStream_t st, int nl, uint64_t n, unsigned nbits, DevBuf* keys, DevBuf* vals,
              uint64_t* h_staging, uint32_t* launches = nullptr);
// ErrorCorrector::correct_read_in_place on every read (spk_correct.cu), against
// a solid tier of size fm.d bits: d_out (data_len bytes, may equal d_data)
// gets the packed data with the corrected bases; d_corr (nullable) a flag per
// read; *nc the number of corrected reads.  Synchronises st.
int correct_reads(spk_ctx* ctx, cudaStream_t st, unsigned k, const unsigned long long* tier, const FastMod& fm,
                  const uint8_t* d_data, uint64_t data_len, const uint64_t* d_off, const uint32_t* d_len,
                  uint64_t n, uint8_t* d_out, uint8_t* d_corr, uint64_t* nc, uint32_t* launches = nullptr);
// Raises a kernel's dynamic shared-memory limit on the current device to at
// least `bytes`, and never lowers it (spk_api.cu).  Jobs on other host threads
// (batches, serving, multi-k) launch the same kernels with other sizes; a
// limit lowered between another thread's raise and its launch would make that
// launch fail.
int raise_smem_limit(const void* kernel, size_t bytes);
// Streaming multiprocessors of the current device (cached per device), for
// grid sizing in code that has no context at hand.
int current_sm_count();
// Bucket sort of a list whose length is in device memory (spk_sort.cu): the
// bucketed copy, offsets and the list of buckets too large for shared
// memory stay here between sort_dev_enqueue and sort_dev_finish.
struct DevSort {
  int nl = 0;
  unsigned nbits = 0;
  uint32_t bbits = 0;
  uint64_t n_cap = 0;
  bool has_vals = false;
  bool pending = false;
  DevBuf tk[4], tv, hist, off, cur, big;
  void rehome(cudaStream_t s) {
    for (DevBuf& b : tk) b.st = s;
    tv.st = hist.st = off.st = cur.st = big.st = s;
  }
  void release() {
    for (DevBuf& b : tk) b.release();
    tv.release();
    hist.release();
    off.release();
    cur.release();
    big.release();
  }
};
int sort_dev_enqueue(cudaStream_t st, int nl, uint64_t n_cap, const unsigned long long* n_dev,
                     unsigned nbits, DevBuf* keys, DevBuf* vals, DevBuf* tmp_keys, DevSort& ds,
                     uint32_t* launches = nullptr);
// Device word counting the buckets left for sort_dev_finish.
const unsigned* sort_dev_nbig(const DevSort& ds);
int sort_dev_finish(cudaStream_t st, DevSort& ds, DevBuf* keys, DevBuf* vals, uint64_t n_host,
                    unsigned nbig_host, uint64_t* h_staging, uint32_t* launches = nullptr);
// Exclusive scan of u32 in place (spk_sort.cu).
int scan_u32(cudaStream_t st, uint32_t* a, uint64_t n, DevBuf& sums, uint32_t* launches = nullptr);
// Ordered compaction of a sorted SoA list into AoS Kmer256 limbs; *m is the
// number of kept items (synchronises st to read it, unless the caller knows
// it already: known_m, which must be exact).
int ordered_convert(cudaStream_t st, int nl, uint64_t n, unsigned k, DevBuf* limbs,
                    const uint32_t* cin, uint32_t min_count, DevBuf* out, DevBuf* cout,
                    uint64_t* h_staging, uint64_t* m, uint64_t known_m = ~0ULL);
}  // namespace spk
