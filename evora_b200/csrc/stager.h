// stager.h -- host copies split into chunks and run by worker threads
// (the serving loop's copies of request states; no CUDA).
#pragma once

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstddef>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

namespace evora {

// Host copies of request states (into the page-locked pool, and results
// out of it) run on worker threads in 4 MB chunks: one core moves a few
// GB/s, the host's memory system several times that.  post() queues a copy
// and returns at once; *left counts its chunks still to copy (0: complete).
// copy() posts and helps until its own copy is complete.  The workers start
// with the first posted copy; stop() lets them finish every queued chunk.
class Stager {
 public:
  ~Stager() { stop(); }

  void post(void* dst, const void* src, size_t bytes, std::atomic<int>* left) {
    const size_t nchunks = bytes == 0 ? 1 : (bytes + kChunk - 1) / kChunk;
    left->fetch_add((int)nchunks, std::memory_order_relaxed);
    start();
    {
      std::lock_guard<std::mutex> lk(m_);
      for (size_t i = 0; i < nchunks; ++i) {
        const size_t off = i * kChunk;
        q_.push_back(Task{static_cast<char*>(dst) + off, static_cast<const char*>(src) + off,
                          std::min(kChunk, bytes - std::min(bytes, off)), left});
      }
    }
    cv_.notify_all();
  }

  void copy(void* dst, const void* src, size_t bytes) {
    if (bytes < kMinSplit) {
      std::memcpy(dst, src, bytes);
      return;
    }
    std::atomic<int> left{0};
    post(dst, src, bytes, &left);
    std::unique_lock<std::mutex> lk(m_);
    while (left.load(std::memory_order_acquire) > 0) {
      if (!q_.empty()) {   // run queued chunks (FIFO) until this copy's are done
        const Task t = q_.front();
        q_.pop_front();
        lk.unlock();
        run(t);
        lk.lock();
        continue;
      }
      done_.wait(lk, [&] { return left.load(std::memory_order_acquire) == 0 || !q_.empty(); });
    }
  }

  void stop() {
    {
      std::lock_guard<std::mutex> lk(m_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : th_) t.join();
    th_.clear();
    // without workers (none could be started) the queue is run here
    while (!q_.empty()) {
      const Task t = q_.front();
      q_.pop_front();
      run(t);
    }
  }

 private:
  static constexpr size_t kMinSplit = 4u << 20;
  static constexpr size_t kChunk = 4u << 20;
  struct Task {
    char* dst;
    const char* src;
    size_t bytes;
    std::atomic<int>* left;
  };

  void start() {
    if (started_) return;
    started_ = true;
    const unsigned hw = std::thread::hardware_concurrency();
    const int n = (int)std::min(8u, hw > 1 ? hw : 2u);
    try {
      for (int i = 0; i < n; ++i) th_.emplace_back([this] { worker(); });
    } catch (...) {   // no threads: copy() and stop() run the queue themselves
    }
  }

  void run(const Task& t) {
    if (t.bytes) std::memcpy(t.dst, t.src, t.bytes);
    if (t.left->fetch_sub(1, std::memory_order_acq_rel) == 1) {
      std::lock_guard<std::mutex> lk(m_);
      done_.notify_all();
    }
  }

  void worker() {
    std::unique_lock<std::mutex> lk(m_);
    for (;;) {
      cv_.wait(lk, [&] { return stop_ || !q_.empty(); });
      if (q_.empty()) return;   // stopping, and every queued chunk is done
      const Task t = q_.front();
      q_.pop_front();
      lk.unlock();
      run(t);
      lk.lock();
    }
  }

  std::vector<std::thread> th_;
  bool started_ = false, stop_ = false;
  std::mutex m_;
  std::condition_variable cv_, done_;
  std::deque<Task> q_;
};

}  // namespace evora
