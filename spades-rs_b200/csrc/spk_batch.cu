// spk_batch.cu -- batched counting of independent samples (spk_count_batch).
#include <cuda_runtime.h>

#include "spk_internal.h"

extern "C" int spk_count_batch(spk_ctx* ctx, const spk_job* jobs, int n_jobs, spk_result** results) {
  using namespace spk;
  if (!ctx || (n_jobs > 0 && (!jobs || !results))) return fail(SPK_E_INVALID_ARG, "null argument");
  for (int i = 0; i < n_jobs; i++) results[i] = nullptr;
  for (int i = 0; i < n_jobs; i++) {
    const spk_job& j = jobs[i];
    int rc = spk_count(ctx, j.data, j.data_len, j.offsets, j.lengths, j.n_reads, j.ks, j.n_k, &j.opts,
                       &results[i]);
    if (rc) {
      for (int q = 0; q < i; q++) { spk_result_free(results[q]); results[q] = nullptr; }
      return rc;
    }
  }
  return SPK_OK;
}
