// CPU test of the admission scheduler of the serving loop and of batches
// (spades-rs_b200/csrc/spk_sched.h), built and run by tests/test_sched.py.
// Fake jobs (sleeps and heap results) stand in for counting jobs.  Exit
// status 0 when every check passes; each failure prints its line.
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../spades-rs_b200/csrc/spk_sched.h"

using spk::Scheduler;
using namespace std::chrono_literals;

static int g_fail = 0;
#define CHECK(c)                                              \
  do {                                                        \
    if (!(c)) {                                               \
      std::printf("FAIL %s:%d: %s\n", __FILE__, __LINE__, #c); \
      g_fail++;                                               \
    }                                                         \
  } while (0)

static std::atomic<int> g_freed{0};
static void free_int(void* p) {
  delete (int*)p;
  g_freed++;
}

// Jobs are admitted by budget and slot count; a job above the whole budget
// is refused at once; results and latencies come back through wait().
static void admission() {
  std::atomic<int> running{0}, peak{0};
  Scheduler s(100, 2, free_int);
  std::vector<uint64_t> t;
  for (int i = 0; i < 6; i++)
    t.push_back(s.submit(40, [&, i](void** out, std::string*) {
      int now = ++running;
      int p = peak.load();
      while (now > p && !peak.compare_exchange_weak(p, now)) {
      }
      std::this_thread::sleep_for(20ms);
      running--;
      *out = new int(i);
      return 0;
    }));
  const uint64_t big = s.submit(101, [](void**, std::string*) { return 0; });
  for (int i = 0; i < 6; i++) {
    int st = -1;
    void* r = nullptr;
    double lat = 0;
    CHECK(s.wait(t[i], -1, &st, &r, &lat) == 1);
    CHECK(st == 0 && r && *(int*)r == i && lat > 0);
    free_int(r);
  }
  CHECK(peak.load() <= 2);
  CHECK(s.peak_inflight() <= 2);
  int st = 0;
  CHECK(s.wait(big, 1000, &st, nullptr, nullptr) == 1);
  CHECK(st == Scheduler::kAdmissionError);
  CHECK(s.wait(12345, 0, &st, nullptr, nullptr) == -1);
}

// A failed job's message travels with its status from the worker thread.
static void error_message() {
  Scheduler s(100, 1);
  const uint64_t t = s.submit(1, [](void**, std::string* msg) {
    *msg = "count table overflow";
    return 5;
  });
  int st = 0;
  std::string msg;
  CHECK(s.wait(t, -1, &st, nullptr, nullptr, &msg) == 1);
  CHECK(st == 5 && msg == "count table overflow");
}

// A caller blocked in wait() while another thread stops the scheduler and
// drops its own reference: the waiter keeps the scheduler alive, gets its
// result, and the scheduler is destroyed when the waiter lets go.
static void waiter_survives_stop() {
  g_freed = 0;
  auto owner = std::make_shared<Scheduler>(100, 1, free_int);
  const uint64_t slow = owner->submit(1, [](void** out, std::string*) {
    std::this_thread::sleep_for(150ms);
    *out = new int(7);
    return 0;
  });
  const uint64_t queued = owner->submit(1, [](void** out, std::string*) {
    *out = new int(8);
    return 0;
  });
  std::atomic<int> got{-1}, got_status{-1}, queued_status{-1};
  std::weak_ptr<Scheduler> watch = owner;
  std::thread waiter([sched = owner, slow, &got, &got_status]() mutable {
    int st = -1;
    void* r = nullptr;
    if (sched->wait(slow, -1, &st, &r, nullptr) == 1 && r) {
      got = *(int*)r;
      free_int(r);
    }
    got_status = st;
    sched.reset();
  });
  std::thread waiter2([sched = owner, queued, &queued_status]() mutable {
    int st = -1;
    void* r = nullptr;
    sched->wait(queued, -1, &st, &r, nullptr);
    queued_status = st;
    if (r) free_int(r);
    sched.reset();
  });
  std::this_thread::sleep_for(30ms);
  owner->stop();   // the running job finishes, the queued one is cancelled
  owner.reset();   // the waiters still hold the scheduler
  waiter.join();
  waiter2.join();
  CHECK(got.load() == 7 && got_status.load() == 0);
  CHECK(queued_status.load() == Scheduler::kAdmissionError);
  CHECK(watch.expired());
}

// Finished jobs whose tickets are never collected have their results freed
// at stop; jobs submitted after stop are refused.
static void uncollected_results_freed() {
  g_freed = 0;
  Scheduler s(100, 4, free_int);
  std::vector<uint64_t> t;
  for (int i = 0; i < 3; i++)
    t.push_back(s.submit(1, [i](void** out, std::string*) {
      *out = new int(i);
      return 0;
    }));
  for (int i = 0; i < 200 && (s.poll(t[0]) != 1 || s.poll(t[1]) != 1 || s.poll(t[2]) != 1); i++)
    std::this_thread::sleep_for(5ms);
  s.stop();
  CHECK(g_freed.load() == 3);
  CHECK(s.poll(t[0]) == -1);
  const uint64_t late = s.submit(1, [](void**, std::string*) { return 0; });
  int st = 0;
  CHECK(s.wait(late, 1000, &st, nullptr, nullptr) == 1);
  CHECK(st == Scheduler::kAdmissionError);
}

// An exclusive job waits for the running jobs to finish and runs alone;
// nothing is admitted next to it.
static void exclusive_runs_alone() {
  std::atomic<int> running{0}, overlap_with_big{0};
  std::atomic<bool> big_running{false};
  Scheduler s(100, 8);
  std::vector<uint64_t> t;
  auto small = [&](void** out, std::string*) {
    running++;
    if (big_running) overlap_with_big++;
    std::this_thread::sleep_for(15ms);
    running--;
    *out = nullptr;
    return 0;
  };
  for (int i = 0; i < 3; i++) t.push_back(s.submit(1, small));
  t.push_back(s.submit(50, [&](void**, std::string*) {
    if (running.load() != 0) overlap_with_big++;
    big_running = true;
    std::this_thread::sleep_for(30ms);
    big_running = false;
    return 0;
  }, true));
  for (int i = 0; i < 3; i++) t.push_back(s.submit(1, small));
  for (auto x : t) {
    int st = -1;
    CHECK(s.wait(x, -1, &st, nullptr, nullptr) == 1 && st == 0);
  }
  CHECK(overlap_with_big.load() == 0);
  CHECK(s.peak_inflight() >= 2);  // the small ones did share the device
}

// With a shared budget, jobs run side by side only while their needs
// together fit it, and a job above it runs alone.
static void shared_budget_pairs() {
  std::atomic<int> running{0}, peak{0}, overlap_with_big{0};
  std::atomic<bool> big_running{false};
  Scheduler s(100, 8, nullptr, 20);
  std::vector<uint64_t> t;
  auto job = [&](void** out, std::string*) {
    const int r = ++running;
    int p = peak.load();
    while (r > p && !peak.compare_exchange_weak(p, r)) {
    }
    if (big_running) overlap_with_big++;
    std::this_thread::sleep_for(15ms);
    running--;
    *out = nullptr;
    return 0;
  };
  for (int i = 0; i < 6; i++) t.push_back(s.submit(8, job));  // two of them fit 20 at a time
  t.push_back(s.submit(30, [&](void**, std::string*) {        // above 20: alone
    if (running.load() != 0) overlap_with_big++;
    big_running = true;
    std::this_thread::sleep_for(20ms);
    big_running = false;
    return 0;
  }));
  for (int i = 0; i < 2; i++) t.push_back(s.submit(8, job));
  for (auto x : t) {
    int st = -1;
    CHECK(s.wait(x, -1, &st, nullptr, nullptr) == 1 && st == 0);
  }
  CHECK(peak.load() == 2);
  CHECK(overlap_with_big.load() == 0);
}

int main() {
  admission();
  exclusive_runs_alone();
  shared_budget_pairs();
  error_message();
  waiter_survives_stop();
  uncollected_results_freed();
  if (g_fail) return 1;
  std::printf("sched ok\n");
  return 0;
}
