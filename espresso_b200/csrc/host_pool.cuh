// Persistent host worker pool for the host-pointer staging path: parallel
// copies between user buffers and pinned staging, chunked so that each chunk's
// DMA overlaps the host copy of the next one.
#pragma once

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstdint>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>
#if defined(__x86_64__) || defined(_M_X64)
#include <emmintrin.h>
#endif

namespace p3mx {

// memcpy with non-temporal (streaming) stores: the destination lines are
// not read first, so a large copy moves 2 bytes of memory traffic per byte
// instead of 3.  The stores are fenced before return.
inline void copy_stream(void *dst, const void *src, size_t bytes) {
#if defined(__x86_64__) || defined(_M_X64)
  char *d = static_cast<char *>(dst);
  const char *s = static_cast<const char *>(src);
  size_t const head = std::min(bytes, (16 - (reinterpret_cast<uintptr_t>(d) & 15)) & 15);
  std::memcpy(d, s, head);
  d += head;
  s += head;
  bytes -= head;
  size_t const n16 = bytes / 16;
  for (size_t i = 0; i < n16; ++i)
    _mm_stream_si128(reinterpret_cast<__m128i *>(d) + i,
                     _mm_loadu_si128(reinterpret_cast<const __m128i *>(s) + i));
  std::memcpy(d + 16 * n16, s + 16 * n16, bytes - 16 * n16);
  _mm_sfence();
#else
  std::memcpy(dst, src, bytes);
#endif
}

class HostPool {
public:
  // Threads: P3MX_HOST_THREADS if set, else min(hardware threads, 16).
  HostPool() {
    int n = static_cast<int>(std::thread::hardware_concurrency());
    if (const char *s = std::getenv("P3MX_HOST_THREADS"))
      n = std::atoi(s);
    n = std::clamp(n, 1, 16);
    for (int i = 1; i < n; ++i) // the caller is the n-th worker
      m_workers.emplace_back([this] { loop(); });
  }
  ~HostPool() {
    {
      std::lock_guard<std::mutex> lk(m_mu);
      m_stop = true;
      m_stop_pub.store(true);
    }
    m_cv.notify_all();
    for (auto &t : m_workers)
      t.join();
  }
  HostPool(HostPool const &) = delete;
  HostPool &operator=(HostPool const &) = delete;

  int size() const { return static_cast<int>(m_workers.size()) + 1; }

  // Run fn(i) for i in [0, n_tasks) on the pool and the caller; returns when
  // every task has finished.
  void run(int n_tasks, std::function<void(int)> const &fn) {
    if (n_tasks <= 0)
      return;
    if (m_workers.empty() || n_tasks == 1) {
      for (int i = 0; i < n_tasks; ++i)
        fn(i);
      return;
    }
    unsigned gen;
    {
      std::lock_guard<std::mutex> lk(m_mu);
      m_fn = &fn;
      m_n = n_tasks;
      m_done_pub.store(0);
      gen = ++m_gen;
      m_next.store(static_cast<unsigned long long>(gen) << 32);
      m_gen_pub.store(gen, std::memory_order_release);
    }
    m_cv.notify_all();
    int const mine = work(gen, n_tasks, &fn);
    // tasks finish within microseconds of each other: spin on the count
    int done = m_done_pub.fetch_add(mine, std::memory_order_acq_rel) + mine;
    while (done < n_tasks)
      done = m_done_pub.load(std::memory_order_acquire);
    std::lock_guard<std::mutex> lk(m_mu);
    m_fn = nullptr;
  }

  // Parallel copy with streaming stores, split into pieces of at least 64 KB.
  void copy(void *dst, const void *src, size_t bytes) {
    size_t const piece = std::max<size_t>(64 << 10, (bytes + size() - 1) / size());
    int const n = static_cast<int>((bytes + piece - 1) / piece);
    run(n, [&](int i) {
      size_t const b0 = i * piece, b1 = std::min(bytes, b0 + piece);
      copy_stream(static_cast<char *>(dst) + b0, static_cast<const char *>(src) + b0, b1 - b0);
    });
  }

  // Parallel memcmp: true when the two byte ranges are equal.
  bool equal(const void *a, const void *b, size_t bytes) {
    size_t const piece = std::max<size_t>(64 << 10, (bytes + size() - 1) / size());
    int const n = static_cast<int>((bytes + piece - 1) / piece);
    std::atomic<bool> same{true};
    run(n, [&](int i) {
      size_t const b0 = i * piece, b1 = std::min(bytes, b0 + piece);
      if (std::memcmp(static_cast<const char *>(a) + b0, static_cast<const char *>(b) + b0,
                      b1 - b0) != 0)
        same.store(false, std::memory_order_relaxed);
    });
    return same.load();
  }

private:
  // Claim tasks of generation gen: the counter holds (generation << 32 |
  // next index), so a worker holding a stale generation claims nothing.
  int work(unsigned gen, int n, std::function<void(int)> const *fn) {
    int count = 0;
    for (;;) {
      unsigned long long v = m_next.load();
      for (;;) {
        if ((v >> 32) != gen || static_cast<int>(v & 0xffffffffull) >= n)
          return count;
        if (m_next.compare_exchange_weak(v, v + 1))
          break;
      }
      (*fn)(static_cast<int>(v & 0xffffffffull));
      ++count;
    }
  }
  void loop() {
    unsigned seen = 0;
    for (;;) {
      unsigned gen;
      int n;
      std::function<void(int)> const *fn;
      // chunks of one staging call follow each other within microseconds:
      // spin on the generation counter for a while before sleeping, so a
      // hot pool picks up the next chunk without a wake-up
      auto const t_spin = std::chrono::steady_clock::now() + std::chrono::microseconds(300);
      while (m_gen_pub.load(std::memory_order_acquire) == seen && !m_stop_pub.load() &&
             std::chrono::steady_clock::now() < t_spin) {
      }
      {
        std::unique_lock<std::mutex> lk(m_mu);
        m_cv.wait(lk, [&] { return m_stop || m_gen != seen; });
        if (m_stop)
          return;
        seen = gen = m_gen;
        n = m_n;
        fn = m_fn;
      }
      int const mine = work(gen, n, fn);
      // a stale generation claimed no task (mine == 0): nothing to report
      if (mine > 0)
        m_done_pub.fetch_add(mine, std::memory_order_acq_rel);
    }
  }

  std::vector<std::thread> m_workers;
  std::mutex m_mu;
  std::condition_variable m_cv;
  std::function<void(int)> const *m_fn = nullptr;
  int m_n = 0;
  std::atomic<int> m_done_pub{0}; // finished tasks of the current generation
  std::atomic<unsigned long long> m_next{0};
  unsigned m_gen = 0;
  bool m_stop = false;
  std::atomic<unsigned> m_gen_pub{0}; // m_gen, readable without the lock
  std::atomic<bool> m_stop_pub{false};
};

} // namespace p3mx
