// spk_batch.cu -- batched counting of independent samples (spk_count_batch).
//
// The samples of a batch are independent jobs (their own Bloom tiers, table
// and lists).  Measured on one B200, a sample's device work already runs at
// the rate of one large sample (64 samples of 3-150 M occurrences: 142 ms of
// device time, 144 ms counted one after another from device memory), so what
// one-at-a-time counting from host buffers loses is the copies: every
// sample's packed reads go up before its count starts and its device idles
// meanwhile.  The batch is therefore a pipeline:
//   uploader   one host thread enqueues each job's upload on one upload
//              stream (pageable memory through the context's pinned chunks),
//              up to kAhead jobs ahead of the counts;
//   lanes      kLanes host threads take the jobs in order and run each count
//              on the lane's stream once its upload has landed, so one job's
//              copies overlap the counts of the jobs before it and a lane's
//              host readbacks overlap the other lane's kernels.
// A lane starts a job only while the estimated device memory of the jobs in
// flight (spk_job_hbm_estimate) fits 90% of the free HBM, or when nothing
// else is in flight.  The batch runs on the context's own upload and lane
// streams (spk_ctx::batch_streams), and a job's result keeps its lane's
// stream for its later work.  Every result is exactly spk_count's on that
// sample alone: the jobs share nothing but the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "spk_internal.h"

namespace spk {
int run_job(spk_ctx* ctx, const spk_job& j, const std::vector<uint32_t>& ks, void** out);
int upload_reads(spk_result* res, cudaStream_t st, const uint8_t* data, size_t data_len,
                 const uint64_t* offsets, const uint32_t* lengths, size_t n_reads, ReadsView* rv,
                 bool chunked);
uint64_t job_estimate(const spk_job& j, uint64_t total_mem);
uint64_t usable_device_memory(spk_ctx* ctx);
constexpr int kLanes = 2;   // jobs counting at once
constexpr int kAhead = 4;   // uploads enqueued ahead of the first unfinished count

namespace {
struct BatchSlot {
  spk_result* res = nullptr;
  ReadsView rv{};
  cudaEvent_t uploaded = nullptr;  // the job's copies are on the device
  int status = SPK_OK;
  std::string err;
};
}  // namespace
}  // namespace spk

extern "C" int spk_count_batch(spk_ctx* ctx, const spk_job* jobs, int n_jobs, spk_result** results) {
  using namespace spk;
  if (!ctx || (n_jobs > 0 && (!jobs || !results))) return fail(SPK_E_INVALID_ARG, "null argument");
  if (n_jobs < 0) return fail(SPK_E_INVALID_ARG, "negative job count");
  for (int i = 0; i < n_jobs; i++) results[i] = nullptr;
  if (n_jobs == 0) return SPK_OK;
  for (int i = 0; i < n_jobs; i++) {
    const spk_job& j = jobs[i];
    if (!j.ks || j.n_k < 1) return fail(SPK_E_INVALID_ARG, "job has no k");
    for (int q = 0; q < j.n_k; q++)
      if (j.ks[q] < 1 || j.ks[q] > 127) return fail(SPK_E_INVALID_K, "k outside 1..=127");
    if (j.n_reads && (!j.offsets || !j.lengths)) return fail(SPK_E_INVALID_ARG, "null offsets/lengths");
    if (j.data_len && !j.data) return fail(SPK_E_INVALID_ARG, "null data");
  }
  SPK_CUDA(cudaSetDevice(ctx->device));
  std::lock_guard<std::mutex> batch_lock(ctx->batch_mu);
  for (int q = 0; q <= kLanes; q++)
    if (!ctx->batch_streams[q]) SPK_CUDA(cudaStreamCreateWithFlags(&ctx->batch_streams[q], cudaStreamNonBlocking));
  cudaStream_t up_st = ctx->batch_streams[0];
  std::vector<uint64_t> need(n_jobs);
  const uint64_t budget = (uint64_t)(usable_device_memory(ctx) * 0.9);
  for (int i = 0; i < n_jobs; i++) need[i] = job_estimate(jobs[i], ctx->total_mem);

  std::vector<BatchSlot> slot(n_jobs);
  std::mutex mu;
  std::condition_variable cv;
  int uploaded = 0;        // jobs whose upload is enqueued (or failed)
  int finished = 0;        // jobs whose count returned
  int next_start = 0;      // the job the lanes start next (in order)
  uint64_t inflight = 0;   // estimated device bytes of the counts running
  int running = 0;

  std::thread uploader([&] {
    cudaSetDevice(ctx->device);
    for (int i = 0; i < n_jobs; i++) {
      {
        std::unique_lock<std::mutex> l(mu);
        cv.wait(l, [&] { return i - finished < kAhead + kLanes; });
      }
      BatchSlot& s = slot[i];
      const spk_job& j = jobs[i];
      int rc = SPK_OK;
      std::string err;
      spk_result* res = result_new(ctx, up_st, false);
      cudaEvent_t ev = pooled_event(false);
      if (!res) {
        rc = SPK_E_OOM;
      } else if (!ev) {
        rc = fail(SPK_E_CUDA, "upload event");
      } else {
        res->opts = j.opts;
        if (!res->opts.bloom_bits) res->opts.bloom_bits = 512ULL << 20;
        if (!res->opts.list_min_count) res->opts.list_min_count = 2;
        rc = upload_reads(res, up_st, j.data, j.data_len, j.offsets, j.lengths, j.n_reads, &s.rv, false);
        if (!rc && cudaEventRecord(ev, up_st) != cudaSuccess) rc = cuda_fail(cudaGetLastError(), "upload event");
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
  });

  auto lane = [&](cudaStream_t st) {
    cudaSetDevice(ctx->device);
    for (;;) {
      int i;
      {
        std::unique_lock<std::mutex> l(mu);
        // jobs start in order; one whose memory does not fit beside the
        // running ones waits for them (alone it always starts)
        cv.wait(l, [&] {
          return next_start >= n_jobs ||
                 (uploaded > next_start && (running == 0 || inflight + need[next_start] <= budget));
        });
        if (next_start >= n_jobs) return;
        i = next_start++;
        inflight += need[i];
        running++;
      }
      cv.notify_all();
      BatchSlot& s = slot[i];
      int rc = s.status;
      std::string err = s.err;
      spk_result* res = s.res;
      if (res) res->stream = st;  // the job counts, and its result works, on this lane's stream
      if (!rc && cudaStreamWaitEvent(st, s.uploaded, 0) != cudaSuccess)
        rc = cuda_fail(cudaGetLastError(), "wait for the upload");
      if (s.uploaded) pooled_event_put(s.uploaded, false);
      if (!rc) {
        const spk_job& j = jobs[i];
        rc = count_pipeline(ctx, st, s.rv, 0, j.ks, j.n_k, res->opts, res);
        if (rc) err = spk_last_error();
      }
      if (res) {
        // the reads were allocated on the upload stream; their frees follow
        // this lane's count
        res->reads.st = res->offs.st = res->lens.st = st;
        res->reads.release();
        res->offs.release();
        res->lens.release();
        if (rc) {
          spk_result_free(res);
          res = nullptr;
        }
      }
      {
        std::lock_guard<std::mutex> l(mu);
        s.res = res;
        s.status = rc;
        s.err = err;
        inflight -= need[i];
        running--;
        finished++;
      }
      cv.notify_all();
    }
  };
  std::vector<std::thread> lanes;
  for (int q = 0; q < std::min(kLanes, n_jobs); q++) lanes.emplace_back(lane, ctx->batch_streams[1 + q]);
  for (std::thread& t : lanes) t.join();
  uploader.join();

  // A job that ran out of device memory next to the others runs again alone,
  // with the pool's cached memory given back first (fragments of the other
  // jobs' buffers may be what it could not fit).
  int status = SPK_OK;
  std::string msg;
  for (int i = 0; i < n_jobs; i++) {
    BatchSlot& s = slot[i];
    if (s.status == SPK_E_OOM) {
      cudaDeviceSynchronize();
      if (ctx->pool) cudaMemPoolTrimTo(ctx->pool, 0);
      const spk_job& j = jobs[i];
      std::vector<uint32_t> ks(j.ks, j.ks + j.n_k);
      void* r = nullptr;
      s.status = run_job(ctx, j, ks, &r);
      if (s.status) s.err = spk_last_error();
      else s.res = (spk_result*)r;
    }
    results[i] = s.res;
    if (s.status && status == SPK_OK) {
      status = s.status;
      msg = "job " + std::to_string(i) + " of the batch failed: " + s.err;
    }
  }
  if (status != SPK_OK) {
    for (int i = 0; i < n_jobs; i++) {
      spk_result_free(results[i]);
      results[i] = nullptr;
    }
    return fail(status, msg);
  }
  return SPK_OK;
}
