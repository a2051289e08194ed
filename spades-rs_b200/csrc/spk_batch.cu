// spk_batch.cu -- batched counting of independent samples (spk_batch_start /
// spk_batch_next / spk_batch_end, and spk_count_batch on top of them).
//
// The samples of a batch are independent jobs (their own Bloom tiers, table
// and lists).  Measured on one B200, a sample's device work already runs at
// the rate of one large sample (64 samples of 3-150 M occurrences: 142 ms of
// device time, 144 ms counted one after another from device memory), so what
// one-at-a-time counting from host buffers loses is the copies: every
// sample's packed reads go up before its count starts, its solid list comes
// down after it, and the device idles meanwhile.  The batch is therefore a
// pipeline:
//   uploader   one host thread enqueues each job's upload on one upload
//              stream (pageable memory through the context's pinned chunks),
//              up to kAhead jobs ahead of the counts;
//   lanes      kLanes (3) host threads take the jobs in order and run each count
//              on the lane's stream once its upload has landed, so one job's
//              copies overlap the counts of the jobs before it and a lane's
//              host readbacks overlap the other lanes' kernels;
//   results    a finished job's result moves to the batch's result stream,
//              and spk_batch_next hands the results out in job order as they
//              finish, so the caller's downloads of one result overlap the
//              counts of the jobs after it.
// A lane starts a job only while the estimated device memory of the jobs in
// flight (spk_job_hbm_estimate) fits 90% of the free HBM, or when nothing
// else is in flight; jobs count side by side only while together they need
// at most an eighth of that budget, and a larger job runs alone (its upload
// and the downloads of the results before it still overlap it).  A job that
// runs out of device memory anyway waits until no other job runs, gives the
// memory pool's cached blocks back and runs again alone.  The batch runs on
// a fixed handful of streams of the context (spk_ctx::batch_streams).  Every
// result is exactly spk_count's on that sample alone: the jobs share nothing
// but the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <condition_variable>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "spk_internal.h"

namespace spk {
int upload_reads(spk_result* res, cudaStream_t st, const uint8_t* data, size_t data_len,
                 const uint64_t* offsets, const uint32_t* lengths, size_t n_reads, ReadsView* rv,
                 bool chunked);
uint64_t job_estimate(const spk_job& j, uint64_t total_mem);
uint64_t usable_device_memory(spk_ctx* ctx);
void rehome_result(spk_result* res, cudaStream_t s);
// jobs counting at once (64 samples of 0.05-1.2 Mb: 132 ms per batch with
// two lanes, 125 ms with three, 126 ms with four)
constexpr int kLanes = 3;
constexpr int kAhead = 4;   // uploads enqueued ahead of the jobs counting
// spk_ctx::batch_streams: [0] uploads, [1, kLanes] the lanes, [kLanes + 1]
// the finished jobs' results
constexpr int kResultStream = kLanes + 1;
static_assert(kResultStream < 8, "spk_ctx::batch_streams holds eight streams");

namespace {
struct BatchSlot {
  spk_result* res = nullptr;
  ReadsView rv{};
  cudaEvent_t uploaded = nullptr;  // the job's copies are on the device
  int status = SPK_OK;
  std::string err;
  bool done = false;               // the lane finished with the job
};
}  // namespace
}  // namespace spk

struct spk_batch {
  spk_ctx* ctx = nullptr;
  std::vector<spk_job> jobs;
  std::vector<std::vector<uint32_t>> ks;
  std::vector<uint64_t> need;
  uint64_t budget = 0;
  std::vector<spk::BatchSlot> slot;
  std::mutex mu;
  std::condition_variable cv;
  int uploaded = 0;        // jobs whose upload is enqueued (or failed)
  int finished = 0;        // jobs the lanes are done with
  int next_start = 0;      // the job the lanes start next (in order)
  int next_out = 0;        // the job spk_batch_next hands out next
  uint64_t inflight = 0;   // estimated device bytes of the jobs counting
  int running = 0;         // jobs counting
  bool exclusive = false;  // a job runs alone: a large one, or one that ran out of memory
  int oom_waiting = 0;     // jobs waiting to run again alone (no job starts meanwhile)
  std::thread uploader;
  std::vector<std::thread> lanes;

  void upload_all();
  void lane(cudaStream_t st);
};

void spk_batch::upload_all() {
  using namespace spk;
  cudaSetDevice(ctx->device);
  cudaStream_t up = ctx->batch_streams[0];
  const int n = (int)jobs.size();
  for (int i = 0; i < n; i++) {
    {
      std::unique_lock<std::mutex> l(mu);
      cv.wait(l, [&] { return i - finished < kAhead + kLanes; });
    }
    BatchSlot& s = slot[i];
    const spk_job& j = jobs[i];
    int rc = SPK_OK;
    std::string err;
    spk_result* res = result_new(ctx, up, false);
    cudaEvent_t ev = pooled_event(false);
    if (!res) {
      rc = SPK_E_OOM;
    } else if (!ev) {
      rc = fail(SPK_E_CUDA, "upload event");
    } else {
      res->opts = j.opts;
      if (!res->opts.bloom_bits) res->opts.bloom_bits = 512ULL << 20;
      if (!res->opts.list_min_count) res->opts.list_min_count = 2;
      rc = upload_reads(res, up, j.data, j.data_len, j.offsets, j.lengths, j.n_reads, &s.rv, false);
      if (!rc && cudaEventRecord(ev, up) != cudaSuccess) rc = cuda_fail(cudaGetLastError(), "upload event");
    }
    if (rc) err = spk_last_error();
    {
      std::lock_guard<std::mutex> l(mu);
      s.res = res;
      s.uploaded = ev;
      s.status = rc;
      s.err = err;
      uploaded = i + 1;
    }
    cv.notify_all();
  }
}

void spk_batch::lane(cudaStream_t st) {
  using namespace spk;
  cudaSetDevice(ctx->device);
  const int n = (int)jobs.size();
  cudaStream_t out_st = ctx->batch_streams[kResultStream];
  for (;;) {
    int i;
    bool big;
    {
      std::unique_lock<std::mutex> l(mu);
      // Jobs start in order, and alone a job always starts.  Jobs count side
      // by side only while together they need at most an eighth of the
      // budget; a larger job runs alone.  (Two jobs of 20-40 GB side by side
      // took 5-40 times their time alone: the memory pool then maps new
      // memory for one job's buffers while the other's are in use.)
      cv.wait(l, [&] {
        if (next_start >= n) return true;
        if (exclusive || oom_waiting || uploaded <= next_start) return false;
        if (running == 0) return true;
        return inflight + need[next_start] <= budget / 8;
      });
      if (next_start >= n) return;
      i = next_start++;
      inflight += need[i];
      running++;
      big = need[i] > budget / 8;
      if (big) exclusive = true;
    }
    cv.notify_all();
    BatchSlot& s = slot[i];
    int rc = s.status;
    std::string err = s.err;
    spk_result* res = s.res;
    if (res) res->stream = st;
    if (!rc && cudaStreamWaitEvent(st, s.uploaded, 0) != cudaSuccess)
      rc = cuda_fail(cudaGetLastError(), "wait for the upload");
    if (s.uploaded) pooled_event_put(s.uploaded, false);
    bool counted = false, alone = false;
    if (!rc) {
      rc = count_pipeline(ctx, st, s.rv, 0, ks[i].data(), (int)ks[i].size(), res->opts, res);
      counted = true;
    }
    if (rc == SPK_E_OOM && counted) {
      // Run again once no other job is counting, with the pool's cached
      // blocks given back (fragments of the other jobs' buffers may be what
      // this one could not fit).  Lanes that run out together take turns.
      {
        std::unique_lock<std::mutex> l(mu);
        running--;
        if (big) exclusive = false;  // it ran alone already; it takes its turn below
        oom_waiting++;
        cv.notify_all();
        cv.wait(l, [&] { return !exclusive && running == 0; });
        oom_waiting--;
        exclusive = true;
        running++;
      }
      alone = true;
      cudaStreamSynchronize(st);
      cudaDeviceSynchronize();
      pool_trim(ctx);
      res->ks.clear();
      rc = count_pipeline(ctx, st, s.rv, 0, ks[i].data(), (int)ks[i].size(), res->opts, res);
    }
    if (rc) err = spk_last_error();
    if (res) {
      // The reads were allocated on the upload stream; their frees follow
      // this lane's count.  The result's later work (downloads, unitigs,
      // its frees) goes to the result stream, after this job's kernels.
      res->reads.st = res->offs.st = res->lens.st = st;
      res->reads.release();
      res->offs.release();
      res->lens.release();
      if (rc) {
        spk_result_free(res);
        res = nullptr;
      } else {
        cudaEvent_t done = pooled_event(false);
        if (!done || cudaEventRecord(done, st) != cudaSuccess ||
            cudaStreamWaitEvent(out_st, done, 0) != cudaSuccess) {
          cudaGetLastError();
          cudaStreamSynchronize(st);  // without the event: the job's work is complete once this returns
        }
        if (done) pooled_event_put(done, false);
        res->stream = out_st;
        rehome_result(res, out_st);
      }
    }
    {
      std::lock_guard<std::mutex> l(mu);
      s.res = res;
      s.status = rc;
      s.err = err;
      s.done = true;
      inflight -= need[i];
      running--;
      finished++;
      if (alone || big) exclusive = false;
    }
    cv.notify_all();
  }
}

using namespace spk;

extern "C" {

int spk_batch_start(spk_ctx* ctx, const spk_job* jobs, int n_jobs, spk_batch** out) {
  if (!out) return fail(SPK_E_INVALID_ARG, "null output pointer");
  *out = nullptr;
  if (!ctx || (n_jobs > 0 && !jobs)) return fail(SPK_E_INVALID_ARG, "null argument");
  if (n_jobs < 0) return fail(SPK_E_INVALID_ARG, "negative job count");
  for (int i = 0; i < n_jobs; i++) {
    const spk_job& j = jobs[i];
    if (!j.ks || j.n_k < 1) return fail(SPK_E_INVALID_ARG, "job has no k");
    for (int q = 0; q < j.n_k; q++)
      if (j.ks[q] < 1 || j.ks[q] > 127) return fail(SPK_E_INVALID_K, "k outside 1..=127");
    if (j.n_reads && (!j.offsets || !j.lengths)) return fail(SPK_E_INVALID_ARG, "null offsets/lengths");
    if (j.data_len && !j.data) return fail(SPK_E_INVALID_ARG, "null data");
  }
  SPK_CUDA(cudaSetDevice(ctx->device));
  {
    // one batch at a time on a context: its streams are the context's
    std::unique_lock<std::mutex> l(ctx->batch_mu);
    ctx->batch_cv.wait(l, [&] { return !ctx->batch_active; });
    for (int q = 0; q <= kResultStream; q++)
      if (!ctx->batch_streams[q] &&
          cudaStreamCreateWithFlags(&ctx->batch_streams[q], cudaStreamNonBlocking) != cudaSuccess)
        return cuda_fail(cudaGetLastError(), "batch streams");
    ctx->batch_active = true;
  }
  auto* b = new spk_batch();
  b->ctx = ctx;
  b->jobs.assign(jobs, jobs + n_jobs);
  b->ks.resize(n_jobs);
  b->need.resize(n_jobs);
  b->slot.resize(n_jobs);
  b->budget = (uint64_t)(usable_device_memory(ctx) * 0.9);
  uint64_t need_max = 0, small_max = 0, ahead = 0;
  for (int i = 0; i < n_jobs; i++) {
    b->ks[i].assign(jobs[i].ks, jobs[i].ks + jobs[i].n_k);
    b->jobs[i].ks = b->ks[i].data();
    b->need[i] = job_estimate(jobs[i], ctx->total_mem);
    need_max = std::max(need_max, b->need[i]);
    if (b->need[i] <= b->budget / 8) small_max = std::max(small_max, b->need[i]);
    ahead = std::max<uint64_t>(ahead, jobs[i].data_len + jobs[i].n_reads * 12 + 64);
  }
  // The most the batch holds at once: a large job alone, or small ones side
  // by side within an eighth of the budget, plus the uploads enqueued ahead.
  // The pool is grown to that in one block before the first job, so that no
  // job maps memory piece by piece mid-way (64 samples of 0.5-12 Mb: 1.28 s
  // steady with the block, 1.30-1.86 s without).
  if (n_jobs > 0) {
    const uint64_t side = small_max ? std::min<uint64_t>(b->budget / 8, kLanes * small_max) : 0;
    const uint64_t peak = std::max(need_max, side) + (need_max >> 3) + (uint64_t)(kAhead + kLanes) * ahead;
    pool_reserve(ctx, std::min<uint64_t>(peak, b->budget));
  }
  if (n_jobs > 0) {
    b->uploader = std::thread([b] { b->upload_all(); });
    for (int q = 0; q < std::min(kLanes, n_jobs); q++)
      b->lanes.emplace_back([b, q] { b->lane(b->ctx->batch_streams[1 + q]); });
  }
  *out = b;
  return SPK_OK;
}

int spk_batch_next(spk_batch* b, int* index, spk_result** result) {
  if (!b || !index || !result) return fail(SPK_E_INVALID_ARG, "null argument");
  *result = nullptr;
  *index = -1;
  std::unique_lock<std::mutex> l(b->mu);
  const int n = (int)b->jobs.size();
  if (b->next_out >= n) return fail(SPK_E_NOT_FOUND, "every job of the batch was handed out");
  const int i = b->next_out;
  b->cv.wait(l, [&] { return b->slot[i].done; });
  b->next_out++;
  BatchSlot& s = b->slot[i];
  *index = i;
  if (s.status) return fail(s.status, "job " + std::to_string(i) + " of the batch failed: " + s.err);
  *result = s.res;
  s.res = nullptr;  // the caller owns it now
  return SPK_OK;
}

int spk_batch_end(spk_batch* b) {
  if (!b) return SPK_OK;
  spk_ctx* ctx = b->ctx;
  cudaSetDevice(ctx->device);
  if (b->uploader.joinable()) b->uploader.join();
  for (std::thread& t : b->lanes) t.join();
  for (BatchSlot& s : b->slot) spk_result_free(s.res);  // results never handed out
  delete b;
  {
    std::lock_guard<std::mutex> l(ctx->batch_mu);
    ctx->batch_active = false;
  }
  ctx->batch_cv.notify_all();
  return SPK_OK;
}

int spk_count_batch(spk_ctx* ctx, const spk_job* jobs, int n_jobs, spk_result** results) {
  if (!ctx || (n_jobs > 0 && (!jobs || !results))) return fail(SPK_E_INVALID_ARG, "null argument");
  for (int i = 0; i < n_jobs; i++) results[i] = nullptr;
  spk_batch* b = nullptr;
  int rc = spk_batch_start(ctx, jobs, n_jobs, &b);
  if (rc) return rc;
  int status = SPK_OK;
  std::string msg;
  for (int q = 0; q < n_jobs; q++) {
    int i = -1;
    spk_result* r = nullptr;
    const int st = spk_batch_next(b, &i, &r);
    if (st && status == SPK_OK) {
      status = st;
      msg = spk_last_error();
    }
    if (i >= 0) results[i] = r;
  }
  spk_batch_end(b);
  if (status != SPK_OK) {
    for (int i = 0; i < n_jobs; i++) {
      spk_result_free(results[i]);
      results[i] = nullptr;
    }
    return fail(status, msg);
  }
  return SPK_OK;
}

}  // extern "C"
