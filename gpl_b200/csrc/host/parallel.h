// Host threads for the construction's loops over instances, nets and pins. The reference is
// single-threaded; every loop run through parallel_for here writes each output slot from
// exactly one iteration and reads nothing another iteration writes, so its results do not
// depend on the number of threads or their timing.
#pragma once
#include <sys/mman.h>

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <thread>
#include <vector>

namespace gpl {

// The construction's large host arrays (pins, cells and their copies, some 4 to 200 MB each):
// the storage is reserved, the kernel asked for transparent huge pages on it (one fault per
// 2 MB instead of per 4 KB where THP is in madvise mode; ignored elsewhere), and only then
// sized and filled. Only the page size changes, never a value.
inline void advise_huge(const void *p, size_t bytes) {
  const uintptr_t a = ((uintptr_t)p + 4095) & ~(uintptr_t)4095, e = ((uintptr_t)p + bytes) & ~(uintptr_t)4095;
  if (e > a) madvise((void *)a, e - a, MADV_HUGEPAGE);
}
template <class V>
void reserve_huge(V &v, size_t n) {
  if (v.capacity() >= n || n * sizeof(typename V::value_type) < ((size_t)4 << 20)) return;
  v.reserve(n);
  advise_huge(v.data(), n * sizeof(typename V::value_type));
}
template <class V>
void big_resize(V &v, size_t n) {
  reserve_huge(v, n);
  v.resize(n);
}
template <class V, class T>
void big_assign(V &v, size_t n, const T &x) {
  reserve_huge(v, n);
  v.assign(n, x);
}

// The host threads the construction uses: the machine's, at most 16.
inline unsigned host_threads() {
  static unsigned n = [] {
    unsigned h = std::thread::hardware_concurrency();
    return std::max(1u, std::min(16u, h));
  }();
  return n;
}

// f(begin, end) over [0, n) in contiguous chunks, one per thread (the calling thread takes
// the first); ranges shorter than `grain` per thread run on fewer threads.
template <class F>
void parallel_for(size_t n, F &&f, size_t grain = 16384) {
  size_t t = std::min<size_t>(host_threads(), (n + grain - 1) / std::max<size_t>(grain, 1));
  if (t <= 1) {
    if (n) f((size_t)0, n);
    return;
  }
  const size_t chunk = (n + t - 1) / t;
  std::vector<std::thread> pool;
  pool.reserve(t - 1);
  for (size_t i = 1; i < t; i++) {
    size_t a = i * chunk, b = std::min(n, a + chunk);
    if (a < b) pool.emplace_back([&f, a, b] { f(a, b); });
  }
  f((size_t)0, std::min(n, chunk));
  for (auto &th : pool) th.join();
}

}  // namespace gpl
