// Shim for building the reference CPU MPT without oneTBB (test checker only).
// blocked_range + parallel_for over std::thread; the thread count is set by
// the driver (1 = serial).
#pragma once
#include <atomic>
#include <thread>
#include <vector>
#include "oneapi/tbb/scalable_allocator.h"
namespace tbb {
inline int g_shim_threads = 1;
template <typename T>
class blocked_range {
 public:
  blocked_range(T b, T e) : b_(b), e_(e) {}
  T begin() const { return b_; }
  T end() const { return e_; }
 private:
  T b_, e_;
};
template <typename T, typename F>
void parallel_for(const blocked_range<T> &r, const F &f) {
  T n = r.end() - r.begin();
  int nt = g_shim_threads;
  if (nt <= 1 || n < 2 * nt) {
    f(r);
    return;
  }
  // interleaved small chunks so threads share hot and cold keys evenly
  const T chunk = 1024;
  std::atomic<long long> next{(long long)r.begin()};
  std::vector<std::thread> ts;
  for (int t = 0; t < nt; ++t)
    ts.emplace_back([&]() {
      for (;;) {
        long long b = next.fetch_add(chunk);
        if (b >= (long long)r.end()) break;
        T e = (T)((b + chunk) < (long long)r.end() ? (b + chunk) : (long long)r.end());
        f(blocked_range<T>((T)b, e));
      }
    });
  for (auto &th : ts) th.join();
}
}  // namespace tbb
