// Stand-in for tbb::parallel_for used by the reference's ParallelFor over image
// tiles: a dynamic std::thread pool that hands out one index at a time.
// GYREF_THREADS (environment) overrides the thread count.
#pragma once
#include <atomic>
#include <cstdlib>
#include <thread>
#include <vector>

namespace tbb {
namespace detail_shim {
inline int& tls_index() { static thread_local int idx = 0; return idx; }
inline int thread_count() {
  const char* e = std::getenv("GYREF_THREADS");
  int n = e ? std::atoi(e) : 0;
  if (n <= 0) n = (int)std::thread::hardware_concurrency();
  return n > 0 ? n : 1;
}
}  // namespace detail_shim

struct task_arena {
  explicit task_arena(int = 0) {}
  template <typename F> void execute(const F& f) { f(); }
  static int current_thread_index() { return detail_shim::tls_index(); }
};

template <typename Index, typename Body>
void parallel_for(Index begin, Index end, const Body& body) {
  std::atomic<long long> next((long long)begin);
  int n = detail_shim::thread_count();
  std::vector<std::thread> pool;
  for (int t = 0; t < n; ++t) {
    pool.emplace_back([&, t]() {
      detail_shim::tls_index() = t;
      for (;;) {
        long long i = next.fetch_add(1);
        if (i >= (long long)end) break;
        body((Index)i);
      }
    });
  }
  for (auto& th : pool) th.join();
}
}  // namespace tbb
