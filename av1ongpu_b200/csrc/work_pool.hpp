/*
 * work_pool.hpp - a small fixed pool of host threads for the planner.
 *
 * run(n, fn) calls fn(0) .. fn(n - 1) across the workers and the calling
 * thread and returns when every call has returned. One run at a time per
 * pool. Tasks are claimed from an atomic counter, so uneven pieces balance
 * themselves.
 *
 * A plan is a burst of short runs separated by short serial steps, so a
 * worker that finished a run spins for a few tens of microseconds before it
 * sleeps: the next run of the burst finds it awake instead of paying a futex
 * wake-up per worker (tens of microseconds each). Every worker takes part in
 * every run (`active_` counts them down), so a run's arguments are never
 * replaced while a worker may still read them.
 */
#ifndef AV1B_WORK_POOL_HPP
#define AV1B_WORK_POOL_HPP

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#if defined(__x86_64__) || defined(__i386__)
#include <immintrin.h>
#define AV1B_CPU_RELAX() _mm_pause()
#else
#define AV1B_CPU_RELAX() std::this_thread::yield()
#endif

/* How long an idle worker spins before it sleeps, in microseconds. */
#ifndef AV1B_POOL_SPIN_US
#define AV1B_POOL_SPIN_US 40
#endif

namespace av1b {

class WorkPool {
 public:
  /* `threads` counts the caller: threads - 1 workers are started. */
  explicit WorkPool(int threads) {
    const int n = std::max(1, threads) - 1;
    for (int i = 0; i < n; ++i) workers_.emplace_back([this] { loop(); });
  }

  ~WorkPool() {
    stop_.store(true, std::memory_order_release);
    gen_.fetch_add(1, std::memory_order_acq_rel);
    {
      std::lock_guard<std::mutex> lk(mu_);
    }
    cv_.notify_all();
    for (std::thread& t : workers_) t.join();
  }

  WorkPool(const WorkPool&) = delete;
  WorkPool& operator=(const WorkPool&) = delete;

  int threads() const { return static_cast<int>(workers_.size()) + 1; }

  void run(int n, const std::function<void(int)>& fn) {
    if (n <= 0) return;
    if (n == 1 || workers_.empty()) {
      for (int i = 0; i < n; ++i) fn(i);
      return;
    }
    fn_ = &fn;
    n_ = n;
    next_.store(0, std::memory_order_relaxed);
    active_.store(static_cast<int>(workers_.size()), std::memory_order_relaxed);
    gen_.fetch_add(1, std::memory_order_acq_rel);
    {
      /* a worker between its last look at gen_ and its wait holds the lock */
      std::lock_guard<std::mutex> lk(mu_);
    }
    cv_.notify_all();
    drain();
    for (int spins = 0; active_.load(std::memory_order_acquire) != 0; ++spins) {
      if (spins < 4096)
        AV1B_CPU_RELAX();
      else
        std::this_thread::yield();
    }
    fn_ = nullptr;
  }

 private:
  void drain() {
    for (;;) {
      const int i = next_.fetch_add(1, std::memory_order_relaxed);
      if (i >= n_) break;
      (*fn_)(i);
    }
  }

  void loop() {
    unsigned long long seen = 0;
    for (;;) {
      if (gen_.load(std::memory_order_acquire) == seen) {
        const auto until = std::chrono::steady_clock::now() + std::chrono::microseconds(AV1B_POOL_SPIN_US);
        for (int k = 1; gen_.load(std::memory_order_acquire) == seen; ++k) {
          AV1B_CPU_RELAX();
          if ((k & 63) == 0 && std::chrono::steady_clock::now() > until) break;
        }
      }
      if (gen_.load(std::memory_order_acquire) == seen) {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return gen_.load(std::memory_order_acquire) != seen; });
      }
      seen = gen_.load(std::memory_order_acquire);
      if (stop_.load(std::memory_order_acquire)) return;
      drain();
      active_.fetch_sub(1, std::memory_order_acq_rel);
    }
  }

  std::vector<std::thread> workers_;
  std::mutex mu_;
  std::condition_variable cv_;
  const std::function<void(int)>* fn_ = nullptr;
  int n_ = 0;
  std::atomic<int> next_{0};
  std::atomic<int> active_{0};
  std::atomic<unsigned long long> gen_{0};
  std::atomic<bool> stop_{false};
};

}  // namespace av1b

#endif
