// spk_serve.cu -- serving loop: admission by HBM budget, concurrent jobs on
// separate streams, results kept resident until the caller takes them.
//
// spades-rs has no serving mode; this is the request loop around the counting
// path that keeps count tables resident for the downstream graph build
// (CompactedGraph::build, src/graph.rs:65-69).  The admission rule follows
// the reference's memory governor idea (src/memory.rs:25-92: budget a share
// of the available memory, size the Bloom to it), applied to HBM.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "spk_internal.h"
#include "spk_sched.h"

struct Server {
  // Shared with every caller inside spk_wait, so that a concurrent stop never
  // destroys the scheduler under a waiter.
  std::shared_ptr<spk::Scheduler> sched;
  uint64_t budget = 0;
};

namespace spk {

int upload_reads(spk_result* res, cudaStream_t st, const uint8_t* data, size_t data_len,
                 const uint64_t* offsets, const uint32_t* lengths, size_t n_reads, ReadsView* rv,
                 bool chunked);

static uint64_t next_pow2_u64(uint64_t x) {
  uint64_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

// Device bytes a job is expected to hold at its peak, per k (the k values of
// a job run concurrently, so their peaks add up), following the schedule
// spk_count picks:
//   occurrences      4 per packed byte less k - 1 per read (reads of >= k bases)
//   table capacity   next_pow2(0.3 occ), at least 1024 slots
//   default job      (12 <= k <= 64, partition within a quarter of the device)
//     first pass     span regions 1.5 occ keys + coarse buckets 1.125 occ keys
//     span count     regions + list and singleton keys (one entry per slot
//                    each) + Bloom operations (3.75 per slot) + the list's
//                    sort temporaries + both tiers
//   other schedules  the table (slots of 16/32/64 bytes), the interleaved
//                    tiers, and a list of a quarter of the slots with its sort
// Reads and outputs (list, edges, kept tiers) are added on top.  A job that
// outgrows the estimate still runs; the batch re-runs a job that ran out of
// memory alone after the others.
uint64_t job_estimate(const spk_job& j, uint64_t total_mem) {
  spk_count_opts o = j.opts;
  const uint64_t bloom_bits = o.bloom_bits ? o.bloom_bits : (512ULL << 20);
  const uint64_t words = std::max<uint64_t>((bloom_bits + 63) / 64, 1);
  const uint64_t nranges = (words * 64 + (1ULL << 19) - 1) >> 19;
  uint64_t bytes = j.data_len + 64 + j.n_reads * 12;
  const bool plain = !(o.flags & (SPK_F_GATED | SPK_F_CORRECT | SPK_F_REF_SOLID | SPK_F_DIRECT | SPK_F_KEEP_TABLE)) &&
                     !(o.n_prior > 0 && o.prior_seqs);
  for (int i = 0; i < j.n_k; i++) {
    const uint32_t k = j.ks ? j.ks[i] : 31;
    const uint64_t nl = (k + 31) / 32;
    const uint64_t b4 = (uint64_t)j.data_len * 4, sub = (uint64_t)j.n_reads * (k - 1);
    const uint64_t occ = b4 > sub ? b4 - sub : 0;
    // slots: 0.3 of the occurrences for k <= 64, 0.45 above (more distinct k-mers per read)
    const uint64_t cap = std::max<uint64_t>(next_pow2_u64(nl <= 2 ? occ * 3 / 10 + 1 : occ * 9 / 20 + 1), 1024);
    const uint64_t key = nl * 8, entry = nl * 8 + 4;
    const uint64_t tiers = words * 16 + (o.flags & SPK_F_REF_SOLID ? words * 8 : 0);
    uint64_t peak;
    // span groups: as many passes as keep the partition within a quarter of the device
    const uint64_t q4 = nl >= 3 ? 13 : 11;  // partition keys per occurrence, in quarters
    uint32_t lg = 0;
    while (lg < 4 && ((occ >> lg) * q4 / 4 + (1u << 22)) * key > total_mem / 4) lg++;
    if (plain && k >= 12 && !(nl >= 3 && 2 * k == 64 * nl) &&
        ((occ >> lg) * q4 / 4 + (1u << 22)) * key <= total_mem / 4) {
      const uint64_t og = occ >> lg;
      const uint64_t lcap = lg ? cap / 2 : cap, scap = cap;
      const uint64_t regions = (nl >= 3 ? 2 * og : og + og / 2) * key + (1u << 20) * key;
      const uint64_t first = regions + (og + og / 8 + 8192 * 64) * key;
      const uint64_t ops = (3 * cap * 5 / 4 + 1024 * nranges) * 4;
      const uint64_t count = regions + lcap * entry + scap * key + ops + lcap * entry + tiers;
      peak = std::max(first, count) + (lg ? count - regions : 0);
    } else {
      const uint64_t slot = nl == 1 ? 16 : (nl <= 3 ? 32 : 64);
      peak = cap * slot + tiers + (cap / 4) * entry * 2;
    }
    // outputs: the list and about one edge per listed k-mer
    peak += (cap / 4) * (entry + (k + 32) / 32 * 8);
    bytes += peak;
  }
  return bytes;
}

// Device memory a scheduler may budget: what the driver reports free plus
// what the stream-ordered pool holds cached but unused.
uint64_t usable_device_memory(spk_ctx* ctx) {
  size_t f = 0, t = 0;
  if (cudaMemGetInfo(&f, &t) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  uint64_t reserved = 0, used = 0;
  if (ctx->pool &&
      cudaMemPoolGetAttribute(ctx->pool, cudaMemPoolAttrReservedMemCurrent, &reserved) == cudaSuccess &&
      cudaMemPoolGetAttribute(ctx->pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess &&
      reserved > used)
    return f + (reserved - used);
  cudaGetLastError();
  return f;
}

int run_job(spk_ctx* ctx, const spk_job& j, const std::vector<uint32_t>& ks, void** out) {
  cudaSetDevice(ctx->device);
  cudaStream_t st = pooled_stream();
  if (!st) return fail(SPK_E_CUDA, "job stream");
  auto* res = result_new(ctx, st, true);
  if (!res) {
    pooled_stream_put(st);
    return SPK_E_OOM;
  }
  res->opts = j.opts;
  if (!res->opts.bloom_bits) res->opts.bloom_bits = 512ULL << 20;
  if (!res->opts.list_min_count) res->opts.list_min_count = 2;
  ReadsView rv;
  int rc = upload_reads(res, st, j.data, j.data_len, j.offsets, j.lengths, j.n_reads, &rv, true);
  if (!rc) rc = count_pipeline(ctx, st, rv, 0, ks.data(), (int)ks.size(), res->opts, res);
  if (res->chunks.n)  // the reads' buffer is freed after every piece has landed
    cudaStreamWaitEvent(st, res->chunks.ready[res->chunks.n - 1], 0);
  res->reads.release();
  res->offs.release();
  res->lens.release();
  if (rc) {
    spk_result_free(res);
    return rc;
  }
  *out = res;
  return SPK_OK;
}

void serve_shutdown(spk_ctx* ctx) {
  std::unique_lock<std::mutex> l(ctx->serve_mu);
  if (!ctx->server) return;
  // Queued jobs end cancelled, running ones finish, and the results nobody
  // waits for are freed; a caller already in spk_wait keeps the scheduler
  // alive until it returns.
  ctx->server->sched->stop();
  delete ctx->server;
  ctx->server = nullptr;
}

}  // namespace spk

using namespace spk;

extern "C" {

int spk_job_hbm_estimate(const spk_job* job, uint64_t* bytes) {
  if (!job || !bytes) return fail(SPK_E_INVALID_ARG, "null argument");
  if (!job->ks || job->n_k < 1) return fail(SPK_E_INVALID_ARG, "job has no k");
  int dev = 0;
  cudaDeviceProp prop;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
    cudaGetLastError();
    prop.totalGlobalMem = 0;
  }
  *bytes = job_estimate(*job, prop.totalGlobalMem ? prop.totalGlobalMem : (180ull << 30));
  return SPK_OK;
}

int spk_serve_start(spk_ctx* ctx, uint64_t hbm_budget_bytes, int max_inflight) {
  if (!ctx) return fail(SPK_E_INVALID_ARG, "null context");
  SPK_CUDA(cudaSetDevice(ctx->device));
  std::unique_lock<std::mutex> l(ctx->serve_mu);
  if (ctx->server) return fail(SPK_E_INVALID_ARG, "serving loop already running");
  if (!hbm_budget_bytes) hbm_budget_bytes = (uint64_t)(usable_device_memory(ctx) * 0.9);
  auto* s = new Server();
  s->budget = hbm_budget_bytes;
  // Jobs run side by side only while together they need at most a
  // sixteenth of the budget; a larger job runs alone.  Two jobs of 20-40 GB
  // side by side took 5-40 times their time alone (the memory pool maps new
  // memory for one while the other's buffers are in use), and jobs of 5-10 GB
  // side by side still took up to 50 times their time alone now and then.
  // At the arrival rates of a service a job takes a small share of the time
  // between arrivals, so running most jobs alone costs little queueing.
  // The jobs that run side by side share one block of the pool, mapped here
  // (several times their shared budget: their estimates leave out the list
  // sort's and the edges' temporaries, and blocks freed by one job in the
  // middle of another's are reused only once both are done).
  pool_reserve(ctx, hbm_budget_bytes / 4);
  s->sched = std::make_shared<Scheduler>(hbm_budget_bytes, max_inflight > 0 ? max_inflight : 4,
                                         [](void* r) { spk_result_free((spk_result*)r); },
                                         hbm_budget_bytes / 16);
  ctx->server = s;
  return SPK_OK;
}

int spk_serve_stop(spk_ctx* ctx) {
  if (!ctx) return fail(SPK_E_INVALID_ARG, "null context");
  serve_shutdown(ctx);
  return SPK_OK;
}

int spk_submit(spk_ctx* ctx, const spk_job* job, uint64_t* ticket) {
  if (!ctx || !job || !ticket) return fail(SPK_E_INVALID_ARG, "null argument");
  if (!job->ks || job->n_k < 1) return fail(SPK_E_INVALID_ARG, "job has no k");
  for (int i = 0; i < job->n_k; i++)
    if (job->ks[i] < 1 || job->ks[i] > 127) return fail(SPK_E_INVALID_K, "k outside 1..=127");
  std::unique_lock<std::mutex> l(ctx->serve_mu);
  if (!ctx->server) return fail(SPK_E_INVALID_ARG, "serving loop not started");
  spk_job j = *job;
  std::vector<uint32_t> ks(job->ks, job->ks + job->n_k);
  const uint64_t need = job_estimate(j, ctx->total_mem);
  // A job above the shared budget runs alone: the pool is first grown to
  // hold it in one block, if it has not been yet.
  const bool alone = need > ctx->server->budget / 16;
  // The job runs on a worker thread: its error message is taken there and
  // handed to the caller of spk_wait with the status.
  *ticket = ctx->server->sched->submit(need, [ctx, j, ks, need, alone](void** out, std::string* msg) {
    if (alone) pool_reserve(ctx, need + (need >> 3));
    const int rc = run_job(ctx, j, ks, out);
    if (rc) *msg = spk_last_error();
    return rc;
  });
  return SPK_OK;
}

int spk_poll(spk_ctx* ctx, uint64_t ticket, int* done) {
  if (!ctx || !done) return fail(SPK_E_INVALID_ARG, "null argument");
  std::unique_lock<std::mutex> l(ctx->serve_mu);
  if (!ctx->server) return fail(SPK_E_INVALID_ARG, "serving loop not started");
  int r = ctx->server->sched->poll(ticket);
  if (r < 0) return fail(SPK_E_NOT_FOUND, "unknown ticket");
  *done = r;
  return SPK_OK;
}

int spk_wait(spk_ctx* ctx, uint64_t ticket, int timeout_ms, spk_result** out, double* latency_ms) {
  if (!ctx || !out) return fail(SPK_E_INVALID_ARG, "null argument");
  *out = nullptr;
  std::shared_ptr<Scheduler> sched;
  {
    std::unique_lock<std::mutex> l(ctx->serve_mu);
    if (!ctx->server) return fail(SPK_E_INVALID_ARG, "serving loop not started");
    sched = ctx->server->sched;
  }
  int status = 0;
  void* r = nullptr;
  std::string msg;
  int w = sched->wait(ticket, timeout_ms, &status, &r, latency_ms, &msg);
  if (w < 0) return fail(SPK_E_NOT_FOUND, "unknown ticket");
  if (w == 0) return fail(SPK_E_NOT_READY, "job not finished");
  if (status == SPK_E_ADMISSION)
    return fail(SPK_E_ADMISSION, "job needs more device memory than the serving budget, "
                                 "or the serving loop stopped before admitting it");
  if (status) return fail(status, msg);
  *out = (spk_result*)r;
  return SPK_OK;
}

// Batched counting of independent samples.  Each sample gets its own Bloom
// and table; the samples run concurrently on a pool of streams.
int spk_count_batch(spk_ctx* ctx, const spk_job* jobs, int n_jobs, spk_result** results);

}  // extern "C"
