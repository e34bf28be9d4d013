// Copies of large host ranges on several threads.  The pipelined host advance stages a
// pageable caller buffer through pinned memory of its own (the DMA engines read and write only
// pinned memory at full speed); one thread's memcpy would be slower than the host link.
#pragma once
#include <algorithm>
#include <condition_variable>
#include <cstddef>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

class HostCopyPool {
 public:
  explicit HostCopyPool(int nthreads) : n_(nthreads < 1 ? 1 : nthreads)
  {
    for (int i = 1; i < n_; ++i) th_.emplace_back([this, i] { run(i); });
  }
  ~HostCopyPool()
  {
    {
      std::lock_guard<std::mutex> l(m_);
      quit_ = true;
    }
    cv_.notify_all();
    for (auto &t : th_) t.join();
  }
  HostCopyPool(const HostCopyPool &) = delete;
  HostCopyPool &operator=(const HostCopyPool &) = delete;

  // dst <- src (bytes), split into one part per thread, the calling thread copying part 0;
  // returns when every part is copied.  Not reentrant: one copy at a time.
  void copy(void *dst, const void *src, size_t bytes)
  {
    if (n_ == 1 || bytes < (size_t(8) << 20)) {
      memcpy(dst, src, bytes);
      return;
    }
    {
      std::lock_guard<std::mutex> l(m_);
      dst_ = static_cast<char *>(dst);
      src_ = static_cast<const char *>(src);
      bytes_ = bytes;
      left_ = n_ - 1;
      ++gen_;
    }
    cv_.notify_all();
    part(0);
    std::unique_lock<std::mutex> l(m_);
    done_.wait(l, [this] { return left_ == 0; });
  }

 private:
  void part(int i)
  {
    const size_t chunk = ((bytes_ + n_ - 1) / n_ + 4095) / 4096 * 4096;   // n_ parts cover every byte
    const size_t b = std::min(bytes_, chunk * (size_t) i), e = std::min(bytes_, b + chunk);
    if (e > b) memcpy(dst_ + b, src_ + b, e - b);
  }

  void run(int i)
  {
    unsigned seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> l(m_);
        cv_.wait(l, [&] { return quit_ || gen_ != seen; });
        if (quit_) return;
        seen = gen_;
      }
      part(i);
      std::lock_guard<std::mutex> l(m_);
      if (--left_ == 0) done_.notify_one();
    }
  }

  int n_;
  std::vector<std::thread> th_;
  std::mutex m_;
  std::condition_variable cv_, done_;
  char *dst_ = nullptr;
  const char *src_ = nullptr;
  size_t bytes_ = 0;
  int left_ = 0;
  unsigned gen_ = 0;
  bool quit_ = false;
};
