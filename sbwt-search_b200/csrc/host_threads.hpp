// Host threads of the library's file readers and host-side layouts: a count
// of threads for a job and a fork-join over them.  Work functions report
// failures through flags, never by throwing.
#pragma once

#include <algorithm>
#include <cstdint>
#include <thread>
#include <vector>

namespace sbwt {

// Threads for `items` items of at least `grain` items each: at least 1, at
// most `cap` and the host's hardware threads.
inline size_t host_threads(uint64_t items, uint64_t grain, size_t cap) {
  const size_t hw = std::max(1u, std::thread::hardware_concurrency());
  const uint64_t by_items = items / std::max<uint64_t>(grain, 1);
  return (size_t)std::max<uint64_t>(1, std::min<uint64_t>(std::min(hw, cap), by_items));
}

// Runs work(t) for t = 0 .. n - 1 (t = 0 on the calling thread) and joins.
template <class F>
void run_threads(size_t n, F &&work) {
  std::vector<std::thread> th;
  th.reserve(n > 1 ? n - 1 : 0);
  for (size_t t = 1; t < n; ++t) th.emplace_back([&work, t] { work(t); });
  if (n) work(size_t{0});
  for (auto &x : th) x.join();
}

// Runs f(lo, hi) over [0, n) in `parts` contiguous parts, one per thread.
template <class F>
void run_parts(uint64_t n, size_t parts, F &&f) {
  run_threads(parts, [&](size_t p) { f(n * p / parts, n * (p + 1) / parts); });
}

}  // namespace sbwt
