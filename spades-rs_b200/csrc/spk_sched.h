// spk_sched.h -- admission scheduler of the serving loop (host-only C++).
//
// Jobs are admitted in arrival order while (a) their estimated device-memory
// need fits the remaining HBM budget and (b) fewer than max_inflight jobs
// run.  A job whose need exceeds the whole budget is rejected at once
// (SPK_E_ADMISSION) instead of blocking the queue forever.  The runner
// callback executes one job (on its own CUDA stream in libspk; a fake in the
// CPU tests) on a worker thread; when it returns, its memory and slot are
// released and the next jobs are admitted.  No CUDA here, so the policy is
// tested on machines without a GPU (tests/sched_test.cpp).
//
// Lifetime.  A caller blocked in wait() holds the scheduler through a
// shared_ptr of its own, so stop() followed by the owner dropping its pointer
// never destroys the mutex or condition variables under a waiter.  stop()
// frees (with the deleter given at construction) the results of finished jobs
// nobody waits for, so tickets never collected do not leak their results.
#pragma once
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace spk {

struct SchedJob {
  uint64_t ticket = 0;
  uint64_t need = 0;                 // estimated device bytes
  // returns status, sets an opaque result and, on failure, the error message
  std::function<int(void**, std::string*)> run;
  std::chrono::steady_clock::time_point t_submit, t_start, t_done;
  bool done = false;
  int status = 0;
  void* result = nullptr;
  std::string msg;                   // error message of a failed job
  int waiters = 0;                   // callers inside wait() for this job
  bool exclusive = false;            // runs with no other job in flight
};

class Scheduler {
 public:
  enum { kAdmissionError = 8 /* SPK_E_ADMISSION */ };

  // free_result: how to free the result of a job nobody collected (may be
  // empty).  shared_budget (0: the whole budget): jobs run side by side only
  // while their needs together stay within it; a job that needs more than it
  // runs alone (see submit).
  Scheduler(uint64_t budget, int max_inflight, std::function<void(void*)> free_result = nullptr,
            uint64_t shared_budget = 0)
      : budget_(budget), shared_budget_(shared_budget ? std::min(shared_budget, budget) : budget),
        max_inflight_(max_inflight < 1 ? 1 : max_inflight), free_result_(std::move(free_result)) {
    thread_ = std::thread([this] { loop(); });
  }
  ~Scheduler() {
    stop();
    // No waiter is left (each holds the scheduler): free what nobody took.
    std::unique_lock<std::mutex> l(mu_);
    for (auto& kv : jobs_)
      if (kv.second->result && free_result_) free_result_(kv.second->result);
    jobs_.clear();
  }

  void stop() {
    {
      std::unique_lock<std::mutex> l(mu_);
      if (stopping_) return;
      stopping_ = true;
      cv_.notify_all();
    }
    if (thread_.joinable()) thread_.join();
    std::unique_lock<std::mutex> l(mu_);
    // Queued jobs that were never admitted end as cancelled (admission error).
    for (auto& j : queue_) {
      j->done = true;
      j->status = kAdmissionError;
      j->t_start = j->t_done = std::chrono::steady_clock::now();
    }
    queue_.clear();
    done_cv_.notify_all();
    // Running jobs finish on their own worker threads.
    done_cv_.wait(l, [&] { return inflight_ == 0; });
    // Results of finished jobs that no caller is waiting for are freed; a
    // waiter already inside wait() still collects its own.
    for (auto it = jobs_.begin(); it != jobs_.end();) {
      auto& j = it->second;
      if (j->waiters == 0) {
        if (j->result && free_result_) free_result_(j->result);
        it = jobs_.erase(it);
      } else {
        ++it;
      }
    }
  }

  // exclusive: the job is admitted only when no other job runs, and no other
  // job is admitted while it runs (jobs of a large share of the budget, whose
  // neighbours would fragment the memory they need).
  // A job that needs more than the shared budget is exclusive too.
  uint64_t submit(uint64_t need, std::function<int(void**, std::string*)> run, bool exclusive = false) {
    std::unique_lock<std::mutex> l(mu_);
    auto j = std::make_shared<SchedJob>();
    j->ticket = ++next_ticket_;
    j->need = need;
    j->exclusive = exclusive || need > shared_budget_;
    j->run = std::move(run);
    j->t_submit = std::chrono::steady_clock::now();
    jobs_[j->ticket] = j;
    if (stopping_ || need > budget_) {  // stopped, or can never fit: fail now
      j->done = true;
      j->status = kAdmissionError;
      j->t_start = j->t_done = j->t_submit;
    } else {
      queue_.push_back(j);
    }
    cv_.notify_all();
    return j->ticket;
  }

  // 1 = done, 0 = running/queued, -1 = unknown ticket
  int poll(uint64_t ticket) {
    std::unique_lock<std::mutex> l(mu_);
    auto it = jobs_.find(ticket);
    if (it == jobs_.end()) return -1;
    return it->second->done ? 1 : 0;
  }

  // Waits up to timeout_ms (< 0: forever).  Returns -1 unknown ticket, 0 not
  // ready, 1 done (the job is removed and its fields copied out; msg gets the
  // error message of a failed job).
  int wait(uint64_t ticket, int timeout_ms, int* status, void** result, double* latency_ms,
           std::string* msg = nullptr) {
    std::unique_lock<std::mutex> l(mu_);
    auto it = jobs_.find(ticket);
    if (it == jobs_.end()) return -1;
    auto j = it->second;
    auto pred = [&] { return j->done; };
    j->waiters++;
    bool ready = true;
    if (timeout_ms < 0) done_cv_.wait(l, pred);
    else ready = done_cv_.wait_for(l, std::chrono::milliseconds(timeout_ms), pred);
    j->waiters--;
    if (!ready) return 0;
    if (jobs_.find(ticket) == jobs_.end()) return -1;  // another waiter took it
    if (status) *status = j->status;
    if (result) *result = j->result;
    if (msg) *msg = j->msg;
    if (latency_ms)
      *latency_ms = std::chrono::duration<double, std::milli>(j->t_done - j->t_submit).count();
    jobs_.erase(ticket);
    return 1;
  }

  uint64_t in_use() {
    std::unique_lock<std::mutex> l(mu_);
    return in_use_;
  }
  int inflight() {
    std::unique_lock<std::mutex> l(mu_);
    return inflight_;
  }
  int peak_inflight() {
    std::unique_lock<std::mutex> l(mu_);
    return peak_inflight_;
  }

 private:
  void loop() {
    std::unique_lock<std::mutex> l(mu_);
    for (;;) {
      cv_.wait(l, [&] {
        if (stopping_) return true;
        if (queue_.empty() || inflight_ >= max_inflight_ || exclusive_running_) return false;
        const auto& f = queue_.front();
        return f->exclusive ? inflight_ == 0 : (inflight_ == 0 || in_use_ + f->need <= shared_budget_);
      });
      if (stopping_) break;
      auto j = queue_.front();
      queue_.pop_front();
      in_use_ += j->need;
      inflight_++;
      if (j->exclusive) exclusive_running_ = true;
      if (inflight_ > peak_inflight_) peak_inflight_ = inflight_;
      j->t_start = std::chrono::steady_clock::now();
      std::thread([this, j] {
        void* r = nullptr;
        std::string msg;
        int st = j->run(&r, &msg);
        std::unique_lock<std::mutex> l2(mu_);
        j->status = st;
        j->result = r;
        j->msg = std::move(msg);
        j->t_done = std::chrono::steady_clock::now();
        j->done = true;
        in_use_ -= j->need;
        inflight_--;
        if (j->exclusive) exclusive_running_ = false;
        cv_.notify_all();
        done_cv_.notify_all();
      }).detach();
    }
  }

  std::mutex mu_;
  std::condition_variable cv_, done_cv_;
  std::deque<std::shared_ptr<SchedJob>> queue_;
  std::map<uint64_t, std::shared_ptr<SchedJob>> jobs_;
  std::thread thread_;
  uint64_t budget_;
  uint64_t shared_budget_;
  uint64_t in_use_ = 0;
  uint64_t next_ticket_ = 0;
  int max_inflight_;
  int inflight_ = 0;
  int peak_inflight_ = 0;
  bool stopping_ = false;
  bool exclusive_running_ = false;
  std::function<void(void*)> free_result_;
};

}  // namespace spk
