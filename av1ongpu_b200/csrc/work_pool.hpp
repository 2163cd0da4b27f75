/*
 * work_pool.hpp - a small fixed pool of host threads for the planner.
 *
 * run(n, fn) calls fn(0) .. fn(n - 1) across the workers and the calling
 * thread and returns when every call has returned. One run at a time: the
 * decoder serializes its planners. Tasks are claimed from an atomic counter,
 * so uneven pieces balance themselves.
 */
#ifndef AV1B_WORK_POOL_HPP
#define AV1B_WORK_POOL_HPP

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace av1b {

class WorkPool {
 public:
  /* `threads` counts the caller: threads - 1 workers are started. */
  explicit WorkPool(int threads) {
    const int n = std::max(1, threads) - 1;
    for (int i = 0; i < n; ++i) workers_.emplace_back([this] { loop(); });
  }

  ~WorkPool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
      ++generation_;
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
    {
      std::lock_guard<std::mutex> lk(mu_);
      fn_ = &fn;
      n_ = n;
      next_.store(0);
      active_ = static_cast<int>(workers_.size());
      ++generation_;
    }
    cv_.notify_all();
    drain();
    std::unique_lock<std::mutex> lk(mu_);
    done_cv_.wait(lk, [this] { return active_ == 0; });
    fn_ = nullptr;
  }

 private:
  void drain() {
    for (;;) {
      const int i = next_.fetch_add(1);
      if (i >= n_) break;
      (*fn_)(i);
    }
  }

  void loop() {
    unsigned long long seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return generation_ != seen; });
        seen = generation_;
        if (stop_) return;
      }
      drain();
      {
        std::lock_guard<std::mutex> lk(mu_);
        if (--active_ == 0) done_cv_.notify_one();
      }
    }
  }

  std::vector<std::thread> workers_;
  std::mutex mu_;
  std::condition_variable cv_, done_cv_;
  const std::function<void(int)>* fn_ = nullptr;
  int n_ = 0;
  std::atomic<int> next_{0};
  int active_ = 0;
  unsigned long long generation_ = 0;
  bool stop_ = false;
};

}  // namespace av1b

#endif
