// spk_batch.cu -- batched counting of independent samples (spk_count_batch).
//
// The samples of a batch are independent jobs (their own Bloom tiers, table
// and lists).  They run concurrently, each on its own stream with its own
// staging block, admitted by the serving scheduler (spk_sched.h) while their
// estimated device memory fits 90% of the free HBM and at most
// kBatchInflight run at once.  A job's kernels then overlap another job's
// host decisions (table and list sizing), short kernels and copies, which
// one-at-a-time counting leaves idle.  Every result is exactly spk_count's
// on that sample alone: the jobs share nothing but the device.
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "spk_internal.h"
#include "spk_sched.h"

namespace spk {
int run_job(spk_ctx* ctx, const spk_job& j, const std::vector<uint32_t>& ks, void** out);
uint64_t job_estimate(const spk_job& j, uint64_t total_mem);
uint64_t usable_device_memory(spk_ctx* ctx);
constexpr int kBatchInflight = 8;
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
  // A job larger than the whole budget still runs, alone.
  std::vector<uint64_t> need(n_jobs);
  uint64_t budget = (uint64_t)(usable_device_memory(ctx) * 0.9);
  for (int i = 0; i < n_jobs; i++) {
    need[i] = job_estimate(jobs[i], ctx->total_mem);
    budget = std::max<uint64_t>(budget, need[i]);
  }
  int status = SPK_OK;
  std::string msg;
  std::vector<std::string> errs(n_jobs);  // the error message of a failed job
  std::vector<int> sts(n_jobs, SPK_OK);
  {
    Scheduler sched(budget, kBatchInflight);
    std::vector<uint64_t> tickets(n_jobs);
    for (int i = 0; i < n_jobs; i++) {
      spk_job j = jobs[i];
      std::vector<uint32_t> ks(j.ks, j.ks + j.n_k);
      tickets[i] = sched.submit(need[i], [ctx, j, ks](void** out, std::string* err) {
        const int rc = run_job(ctx, j, ks, out);
        if (rc) *err = spk_last_error();
        return rc;
      }, need[i] > budget / 4);  // a large job runs alone
    }
    for (int i = 0; i < n_jobs; i++) {
      int st = 0;
      void* r = nullptr;
      sched.wait(tickets[i], -1, &st, &r, nullptr, &errs[i]);
      results[i] = (spk_result*)r;
      sts[i] = st;
    }
  }
  // A job that ran out of device memory next to the others runs again alone,
  // with the pool's cached memory given back first (fragments of the other
  // jobs' buffers may be what it could not fit).
  for (int i = 0; i < n_jobs; i++) {
    if (sts[i] == SPK_E_OOM) {
      cudaDeviceSynchronize();
      if (ctx->pool) cudaMemPoolTrimTo(ctx->pool, 0);
      const spk_job& j = jobs[i];
      std::vector<uint32_t> ks(j.ks, j.ks + j.n_k);
      void* r = nullptr;
      sts[i] = run_job(ctx, j, ks, &r);
      if (sts[i]) errs[i] = spk_last_error();
      else results[i] = (spk_result*)r;
    }
    if (sts[i] && status == SPK_OK) {
      status = sts[i];
      msg = "job " + std::to_string(i) + " of the batch failed: " + errs[i];
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
