// Host threads for the construction's loops over instances, nets and pins. The reference is
// single-threaded; every loop run through parallel_for here writes each output slot from
// exactly one iteration and reads nothing another iteration writes, so its results do not
// depend on the number of threads or their timing.
#pragma once
#include <algorithm>
#include <cstddef>
#include <thread>
#include <vector>

namespace gpl {

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
