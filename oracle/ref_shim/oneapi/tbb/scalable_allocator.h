// Shim for building the reference CPU MPT without oneTBB (test checker only).
// scalable_allocator -> malloc/free.
#pragma once
#include <cstddef>
#include <cstdlib>
namespace tbb {
template <typename T>
struct scalable_allocator {
  T *allocate(std::size_t n) { return static_cast<T *>(std::malloc(n * sizeof(T))); }
  void deallocate(T *p, std::size_t) { std::free(p); }
};
}  // namespace tbb
