// A small persistent pool of host threads for work that is latency-bound
// per item and independent across items: the framing walk of a batch of
// compressed chunks (each a chain of dependent loads through its own chunk,
// so several walk at once where one thread walks them one after another).
#pragma once

#include <atomic>
#include <condition_variable>
#include <cstddef>
#include <cstdint>
#include <exception>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace sf {

class HostPool {
public:
  explicit HostPool(int threads) {
    for (int t = 0; t < threads; t++)
      threads_.emplace_back([this] { work(); });
  }
  ~HostPool() {
    {
      std::lock_guard<std::mutex> g(m_);
      stop_ = true;
    }
    cv_.notify_all();
    for (std::thread &t : threads_)
      t.join();
  }
  HostPool(const HostPool &) = delete;
  HostPool &operator=(const HostPool &) = delete;

  // fn(i) for every i in [0, n), on the pool's threads and the caller's;
  // returns once all are done, rethrowing the first exception any raised.
  // One call at a time.
  void run(size_t n, const std::function<void(size_t)> &fn) {
    {
      std::lock_guard<std::mutex> g(m_);
      fn_ = &fn;
      n_ = n;
      next_.store(0);
      busy_ = threads_.size();
      err_ = nullptr;
      gen_++;
    }
    cv_.notify_all();
    take(fn, n);
    std::unique_lock<std::mutex> lk(m_);
    done_cv_.wait(lk, [&] { return busy_ == 0; });
    fn_ = nullptr;
    if (err_)
      std::rethrow_exception(err_);
  }

private:
  void take(const std::function<void(size_t)> &fn, size_t n) {
    for (size_t i = next_.fetch_add(1); i < n; i = next_.fetch_add(1)) {
      try {
        fn(i);
      } catch (...) {
        std::lock_guard<std::mutex> g(m_);
        if (!err_)
          err_ = std::current_exception();
      }
    }
  }

  void work() {
    uint64_t seen = 0;
    while (true) {
      const std::function<void(size_t)> *fn;
      size_t n;
      {
        std::unique_lock<std::mutex> lk(m_);
        cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
        if (stop_)
          return;
        seen = gen_;
        fn = fn_;
        n = n_;
      }
      take(*fn, n);
      {
        std::lock_guard<std::mutex> g(m_);
        busy_--;
      }
      done_cv_.notify_all();
    }
  }

  std::vector<std::thread> threads_;
  std::mutex m_;
  std::condition_variable cv_, done_cv_;
  const std::function<void(size_t)> *fn_ = nullptr;
  size_t n_ = 0;
  std::atomic<size_t> next_{0};
  size_t busy_ = 0;
  uint64_t gen_ = 0;
  bool stop_ = false;
  std::exception_ptr err_;
};

} // namespace sf
