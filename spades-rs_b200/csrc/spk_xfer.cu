// spk_xfer.cu -- copies between pageable host memory and the device.
//
// cudaMemcpyAsync from or to pageable memory goes through the driver's own
// pinned buffers with one host thread (about 11 GB/s on a B200 host, against
// 55 GB/s from pinned memory).  Here host threads move pieces of the copy
// between the caller's memory and pinned chunks of the context, and the copy
// engine moves other pieces between chunks and the device meanwhile.  Memory
// that is already pinned is copied directly.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "spk_internal.h"

namespace spk {

constexpr size_t kXferChunk = 4u << 20;   // bytes per piece
constexpr size_t kXferDirect = 8u << 20;  // smaller copies go through the driver
constexpr int kXferMaxWorkers = 8;

struct XferPool {
  struct Chunk {
    uint8_t* h = nullptr;
    cudaEvent_t done = nullptr;  // the last copy that used the chunk
  };
  struct Batch {
    const std::function<void(size_t)>* fn = nullptr;
    size_t n = 0;
    std::atomic<size_t> next{0};
    size_t done = 0;  // under mu
  };

  int device = 0;
  std::vector<std::thread> workers;
  std::vector<Chunk> chunks;
  std::vector<Chunk*> free_chunks;
  std::deque<std::shared_ptr<Batch>> queue;
  std::mutex mu;
  std::condition_variable cv_work, cv_done, cv_chunk;
  bool stopping = false;
  bool ok = false;

  XferPool(int dev, int nworkers) : device(dev) {
    cudaSetDevice(device);
    chunks.resize(2 * nworkers + 2);
    for (Chunk& c : chunks) {
      if (cudaMallocHost((void**)&c.h, kXferChunk) != cudaSuccess ||
          cudaEventCreateWithFlags(&c.done, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        return;
      }
      free_chunks.push_back(&c);
    }
    for (int i = 0; i < nworkers; i++) workers.emplace_back([this] { work(); });
    ok = true;
  }
  ~XferPool() {
    {
      std::lock_guard<std::mutex> l(mu);
      stopping = true;
    }
    cv_work.notify_all();
    for (std::thread& t : workers) t.join();
    for (Chunk& c : chunks) {
      if (c.done) {
        cudaEventSynchronize(c.done);
        cudaEventDestroy(c.done);
      }
      if (c.h) cudaFreeHost(c.h);
    }
  }

  // Runs the batch's items until none is left; true if this call ran the last.
  bool run_items(Batch& b) {
    size_t ran = 0;
    for (size_t i; (i = b.next.fetch_add(1)) < b.n; ran++) (*b.fn)(i);
    if (!ran) return false;
    std::lock_guard<std::mutex> l(mu);
    b.done += ran;
    if (b.done == b.n) {
      cv_done.notify_all();
      return true;
    }
    return false;
  }
  void work() {
    cudaSetDevice(device);
    for (;;) {
      std::shared_ptr<Batch> b;
      {
        std::unique_lock<std::mutex> l(mu);
        cv_work.wait(l, [&] { return stopping || !queue.empty(); });
        if (stopping) return;
        b = queue.front();
        if (b->next.load() >= b->n) {  // every item taken: drop the batch
          queue.pop_front();
          continue;
        }
      }
      run_items(*b);
    }
  }
  // fn(i) for i in [0, n) on the workers and the calling thread.
  void parallel_for(size_t n, const std::function<void(size_t)>& fn) {
    if (n == 0) return;
    auto b = std::make_shared<Batch>();
    b->fn = &fn;
    b->n = n;
    {
      std::lock_guard<std::mutex> l(mu);
      queue.push_back(b);
    }
    cv_work.notify_all();
    run_items(*b);
    std::unique_lock<std::mutex> l(mu);
    cv_done.wait(l, [&] { return b->done == b->n; });
    auto it = std::find(queue.begin(), queue.end(), b);
    if (it != queue.end()) queue.erase(it);
  }
  Chunk* acquire() {
    std::unique_lock<std::mutex> l(mu);
    cv_chunk.wait(l, [&] { return !free_chunks.empty(); });
    Chunk* c = free_chunks.back();
    free_chunks.pop_back();
    return c;
  }
  void release(Chunk* c) {
    {
      std::lock_guard<std::mutex> l(mu);
      free_chunks.push_back(c);
    }
    cv_chunk.notify_one();
  }
};

static XferPool* xfer_pool(spk_ctx* ctx) {
  std::lock_guard<std::mutex> l(ctx->xfer_mu);
  if (!ctx->xfer) {
    const unsigned hw = std::max(2u, std::thread::hardware_concurrency());
    auto* p = new XferPool(ctx->device, (int)std::min<unsigned>(kXferMaxWorkers, hw / 2));
    if (!p->ok) {
      delete p;
      return nullptr;
    }
    ctx->xfer = p;
  }
  return ctx->xfer;
}

void xfer_shutdown(spk_ctx* ctx) {
  delete ctx->xfer;
  ctx->xfer = nullptr;
}

static bool is_pageable(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return true;
  }
  return a.type == cudaMemoryTypeUnregistered;
}

int xfer_h2d(spk_ctx* ctx, void* dst, const void* src, size_t n, cudaStream_t st) {
  if (n == 0) return SPK_OK;
  XferPool* pool = n >= kXferDirect && is_pageable(src) ? xfer_pool(ctx) : nullptr;
  if (!pool) {
    SPK_CUDA(cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, st));
    return SPK_OK;
  }
  std::atomic<int> err{0};
  const std::function<void(size_t)> piece = [&](size_t i) {
    const size_t o = i * kXferChunk, m = std::min(kXferChunk, n - o);
    XferPool::Chunk* c = pool->acquire();
    cudaError_t e = cudaEventSynchronize(c->done);  // its last copy has read it
    if (e == cudaSuccess) {
      std::memcpy(c->h, (const uint8_t*)src + o, m);
      e = cudaMemcpyAsync((uint8_t*)dst + o, c->h, m, cudaMemcpyHostToDevice, st);
    }
    if (e == cudaSuccess) e = cudaEventRecord(c->done, st);
    if (e != cudaSuccess) err.store((int)e);
    pool->release(c);
  };
  pool->parallel_for((n + kXferChunk - 1) / kXferChunk, piece);
  if (err.load()) return cuda_fail((cudaError_t)err.load(), "upload through pinned chunks");
  return SPK_OK;
}

int xfer_d2h(spk_ctx* ctx, void* dst, const void* src, size_t n, cudaStream_t st) {
  if (n == 0) return SPK_OK;
  XferPool* pool = n >= kXferDirect && is_pageable(dst) ? xfer_pool(ctx) : nullptr;
  if (!pool) {
    SPK_CUDA(cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, st));
    SPK_CUDA(cudaStreamSynchronize(st));
    return SPK_OK;
  }
  std::atomic<int> err{0};
  const std::function<void(size_t)> piece = [&](size_t i) {
    const size_t o = i * kXferChunk, m = std::min(kXferChunk, n - o);
    XferPool::Chunk* c = pool->acquire();
    cudaError_t e = cudaEventSynchronize(c->done);
    if (e == cudaSuccess) e = cudaMemcpyAsync(c->h, (const uint8_t*)src + o, m, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaEventRecord(c->done, st);
    if (e == cudaSuccess) e = cudaEventSynchronize(c->done);
    if (e == cudaSuccess) std::memcpy((uint8_t*)dst + o, c->h, m);
    if (e != cudaSuccess) err.store((int)e);
    pool->release(c);
  };
  pool->parallel_for((n + kXferChunk - 1) / kXferChunk, piece);
  if (err.load()) return cuda_fail((cudaError_t)err.load(), "download through pinned chunks");
  return SPK_OK;
}

}  // namespace spk
