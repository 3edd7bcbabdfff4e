// A small pool of host threads that copies pageable host memory into page-locked staging buffers
// in parallel. One thread copies at roughly the speed of one core's memory stream, well below the
// rate the device's copy engine takes page-locked memory at, so a caller's pageable witness is
// split over several threads before each staged piece goes to the device.
#pragma once
#include <condition_variable>
#include <cstddef>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

namespace lbg {

class CopyPool {
 public:
  // `workers` threads besides the caller's own (which copies one part of every request).
  explicit CopyPool(int workers) {
    for (int i = 0; i < workers; i++) threads_.emplace_back([this, i] { loop(i); });
  }
  ~CopyPool() {
    {
      std::lock_guard<std::mutex> g(mu_);
      stop_ = true;
      gen_++;
    }
    wake_.notify_all();
    for (auto& t : threads_) t.join();
  }
  CopyPool(const CopyPool&) = delete;
  CopyPool& operator=(const CopyPool&) = delete;

  // Copies `bytes` from src to dst; returns once every part has landed.
  void copy(void* dst, const void* src, size_t bytes) {
    const int parts = (int)threads_.size() + 1;
    if (bytes < ((size_t)1 << 20) || parts == 1) {
      std::memcpy(dst, src, bytes);
      return;
    }
    {
      std::lock_guard<std::mutex> g(mu_);
      dst_ = (char*)dst;
      src_ = (const char*)src;
      bytes_ = bytes;
      parts_ = parts;
      pending_ = parts - 1;
      gen_++;
    }
    wake_.notify_all();
    part(parts - 1);
    std::unique_lock<std::mutex> g(mu_);
    done_.wait(g, [this] { return pending_ == 0; });
  }

 private:
  // part p of the current request: 64-byte aligned boundaries
  void part(int p) {
    const size_t per = ((bytes_ / parts_) + 63) & ~(size_t)63;
    const size_t a = (size_t)p * per, b = a + per < bytes_ ? a + per : bytes_;
    if (a < b) std::memcpy(dst_ + a, src_ + a, b - a);
  }
  void loop(int i) {
    unsigned long long seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> g(mu_);
        wake_.wait(g, [&] { return gen_ != seen; });
        seen = gen_;
        if (stop_) return;
      }
      part(i);
      {
        std::lock_guard<std::mutex> g(mu_);
        if (--pending_ == 0) done_.notify_one();
      }
    }
  }

  std::vector<std::thread> threads_;
  std::mutex mu_;
  std::condition_variable wake_, done_;
  unsigned long long gen_ = 0;
  bool stop_ = false;
  char* dst_ = nullptr;
  const char* src_ = nullptr;
  size_t bytes_ = 0;
  int parts_ = 1, pending_ = 0;
};

}  // namespace lbg
