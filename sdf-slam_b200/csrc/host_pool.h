// Persistent host worker pool for the symbolic analysis.
//
// The analysis runs a handful of parallel phases of a few hundred
// microseconds each per problem; creating and joining threads for every
// phase costs about as much as the work. The pool's workers start once per
// process and park on a condition variable between jobs.
#pragma once

#include <cstdint>
#include <functional>

namespace sdfgpu {

/// Threads a job runs on: the pool's workers plus the calling thread.
int PoolThreads();

/// Runs fn(p) for every p in [0, parts) on the pool's workers and the calling
/// thread and returns once all parts finished, rethrowing the first failure.
/// A call made from inside a part, or while another thread's job holds the
/// pool, runs its parts inline in ascending order.
void PoolRun(int parts, const std::function<void(int)>& fn);

/// Splits [0, n) into at most `threads` contiguous ranges of at least
/// `min_per_thread` items (capped by PoolThreads()) and runs fn(begin, end)
/// on each through PoolRun; inline when one range suffices.
template <typename Fn>
void ParallelRanges(int threads, int64_t n, int64_t min_per_thread, Fn fn) {
  int64_t parts = n / (min_per_thread > 0 ? min_per_thread : 1);
  if (parts > threads) {
    parts = threads;
  }
  if (parts > PoolThreads()) {
    parts = PoolThreads();
  }
  if (parts <= 1) {
    fn(int64_t{0}, n);
    return;
  }
  PoolRun(static_cast<int>(parts), [&](int p) { fn(n * p / parts, n * (p + 1) / parts); });
}

}  // namespace sdfgpu
