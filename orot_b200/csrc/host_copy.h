// host_copy.h -- host memory copies on several threads.
//
// One memcpy thread moves about 10 GB/s, below what a pass of the engine
// consumes or produces, so large copies between caller memory and pinned
// staging are split into 1 MiB chunks that a few threads copy at once.
#pragma once
#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

namespace orotb {

struct Copy {
  uint8_t* dst;
  const uint8_t* src;
  size_t n;
};

class CopyPool {
 public:
  explicit CopyPool(int n) {
    for (int i = 0; i < n; ++i) th_.emplace_back([this] { work(); });
  }
  ~CopyPool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : th_) t.join();
  }
  // Performs every copy in `v`; returns when all bytes are in place.
  void run(const std::vector<Copy>& v) {
    uint64_t total = 0;
    for (const Copy& c : v) total += c.n;
    if (th_.empty() || total < kParallelBytes) {
      for (const Copy& c : v) std::memcpy(c.dst, c.src, c.n);
      return;
    }
    {
      std::lock_guard<std::mutex> lk(mu_);
      chunks_.clear();
      for (const Copy& c : v)
        for (size_t o = 0; o < c.n; o += kChunk) chunks_.push_back({c.dst + o, c.src + o, std::min(kChunk, c.n - o)});
      next_.store(0);
      done_.store(0);
      open_ = true;
      ++gen_;
    }
    cv_.notify_all();
    drain();
    while (done_.load(std::memory_order_acquire) < chunks_.size()) std::this_thread::yield();
    std::unique_lock<std::mutex> lk(mu_);
    open_ = false;
    cv_idle_.wait(lk, [this] { return busy_ == 0; });
  }

 private:
  static constexpr uint64_t kParallelBytes = 4ull << 20;
  static constexpr size_t kChunk = size_t(1) << 20;
  void drain() {
    for (;;) {
      const size_t i = next_.fetch_add(1);
      if (i >= chunks_.size()) return;
      std::memcpy(chunks_[i].dst, chunks_[i].src, chunks_[i].n);
      done_.fetch_add(1, std::memory_order_release);
    }
  }
  void work() {
    uint64_t seen = 0;
    for (;;) {
      std::unique_lock<std::mutex> lk(mu_);
      cv_.wait(lk, [&] { return stop_ || (open_ && gen_ != seen); });
      if (stop_) return;
      seen = gen_;
      ++busy_;
      lk.unlock();
      drain();
      lk.lock();
      if (--busy_ == 0) cv_idle_.notify_all();
    }
  }
  std::vector<std::thread> th_;
  std::mutex mu_;
  std::condition_variable cv_, cv_idle_;
  std::vector<Copy> chunks_;
  std::atomic<size_t> next_{0}, done_{0};
  uint64_t gen_ = 0;
  int busy_ = 0;
  bool open_ = false, stop_ = false;
};

// Copies n bytes on the process-wide copy threads (created on first use);
// copies below a few MiB, and copies while another thread's large copy runs,
// are done by the calling thread.  Defined in engine.cu.
void host_copy(void* dst, const void* src, size_t n);

}  // namespace orotb
