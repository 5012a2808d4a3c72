#include "host_pool.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <exception>
#include <mutex>
#include <thread>

namespace sdfgpu {

namespace {

// Upper bound on the threads: the analysis phases of one problem split into
// tens of ranges at most, so more threads only add wake-up cost.
constexpr int kMaxPoolThreads = 16;
// A worker that finished a job keeps polling for the next one this long
// before it parks: the phases of one analysis follow each other within
// microseconds, and waking a parked thread costs tens of them.
constexpr auto kSpinTime = std::chrono::microseconds(300);

thread_local bool t_in_part = false;

inline void Relax() {
#if defined(__x86_64__) || defined(__i386__)
  __builtin_ia32_pause();
#else
  std::this_thread::yield();
#endif
}

/// One PoolRun call. Lives on the caller's stack; the caller returns only
/// after every part finished and no worker can still reach the job.
struct Job {
  const std::function<void(int)>* fn = nullptr;
  int parts = 0;
  std::atomic<int> next{0};
  std::atomic<int> pending{0};  // parts not finished
  std::mutex error_mu;
  std::exception_ptr error;
};

class Pool {
 public:
  Pool() {
    const int hw = static_cast<int>(std::thread::hardware_concurrency());
    threads_ = std::clamp(hw, 1, kMaxPoolThreads);
    for (int w = 1; w < threads_; ++w) {
      // parked for the life of the process; never joined
      std::thread(&Pool::Worker, this).detach();
    }
  }

  int threads() const { return threads_; }

  void Run(int parts, const std::function<void(int)>& fn) {
    std::unique_lock<std::mutex> own(run_mu_, std::try_to_lock);
    if (t_in_part || !own.owns_lock() || threads_ <= 1) {
      RunInline(parts, fn);
      return;
    }
    Job job;
    job.fn = &fn;
    job.parts = parts;
    job.pending.store(parts);
    job_.store(&job);
    generation_.fetch_add(1);
    if (parked_.load() > 0) {
      const std::lock_guard<std::mutex> lock(park_mu_);
      park_cv_.notify_all();
    }
    Work(job);
    while (job.pending.load(std::memory_order_acquire) != 0) {
      Relax();
    }
    // no worker may pick the job up from here on; wait for those that did
    job_.store(nullptr);
    while (visiting_.load() != 0) {
      Relax();
    }
    if (job.error) {
      std::rethrow_exception(job.error);
    }
  }

 private:
  static void RunInline(int parts, const std::function<void(int)>& fn) {
    const bool outer = t_in_part;
    t_in_part = true;
    try {
      for (int p = 0; p < parts; ++p) {
        fn(p);
      }
    } catch (...) {
      t_in_part = outer;
      throw;
    }
    t_in_part = outer;
  }

  // Takes parts of `job` until none is left; records the first failure.
  static void Work(Job& job) {
    t_in_part = true;
    for (;;) {
      const int p = job.next.fetch_add(1);
      if (p >= job.parts) {
        break;
      }
      try {
        (*job.fn)(p);
      } catch (...) {
        const std::lock_guard<std::mutex> lock(job.error_mu);
        if (!job.error) {
          job.error = std::current_exception();
        }
      }
      job.pending.fetch_sub(1, std::memory_order_release);
    }
    t_in_part = false;
  }

  void Worker() {
    uint64_t seen = generation_.load();
    for (;;) {
      // poll, then park until the generation moves
      auto idle_since = std::chrono::steady_clock::now();
      int polls = 0;
      while (generation_.load() == seen) {
        Relax();
        if (++polls == 256) {
          polls = 0;
          if (std::chrono::steady_clock::now() - idle_since > kSpinTime) {
            std::unique_lock<std::mutex> lock(park_mu_);
            parked_.fetch_add(1);
            park_cv_.wait(lock, [&] { return generation_.load() != seen; });
            parked_.fetch_sub(1);
          }
        }
      }
      seen = generation_.load();
      // visiting_ is raised before job_ is read (both sequentially
      // consistent), so the owner either sees the visit or this thread sees
      // the job withdrawn
      visiting_.fetch_add(1);
      Job* job = job_.load();
      if (job != nullptr) {
        Work(*job);
      }
      visiting_.fetch_sub(1);
    }
  }

  int threads_ = 1;
  std::mutex run_mu_;  // one job at a time
  std::atomic<Job*> job_{nullptr};
  std::atomic<uint64_t> generation_{0};
  std::atomic<int> visiting_{0};
  std::atomic<int> parked_{0};
  std::mutex park_mu_;
  std::condition_variable park_cv_;
};

Pool& GetPool() {
  // created on first use and kept for the life of the process
  static Pool* pool = new Pool();
  return *pool;
}

}  // namespace

int PoolThreads() { return GetPool().threads(); }

void PoolRun(int parts, const std::function<void(int)>& fn) {
  if (parts <= 0) {
    return;
  }
  if (parts == 1) {
    const bool outer = t_in_part;
    t_in_part = true;
    try {
      fn(0);
    } catch (...) {
      t_in_part = outer;
      throw;
    }
    t_in_part = outer;
    return;
  }
  GetPool().Run(parts, fn);
}

}  // namespace sdfgpu
