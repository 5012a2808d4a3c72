// Serving loop with continuous batching. Requests that are waiting when the
// loop has room are merged into one batched engine (a cohort): every kernel
// of an LM iteration covers all of its members, whatever their sizes, and
// the cohort keeps their states, symbolic structure and factors resident on
// the device. Several cohorts run at once on their own CUDA streams, so
// requests that arrive while others are on the GPU are admitted as soon as a
// cohort slot and memory are free and their work overlaps with the running
// ones. The loop keeps one iteration of every cohort in flight, finishes it
// when its stream's event reports it done and enqueues the next; a member
// whose solve has ended is answered at once (its latency stops there) while
// the others keep iterating. Admission is by device footprint (state,
// specs, symbolic structure and factors) against the budget, computed from
// the symbolic analysis that Submit runs and the cohort's engine then reuses.
// Host work of a cohort (building its engine, re-analysing a member whose
// state left its pattern) runs on a helper thread while the other cohorts
// keep iterating. A member's iterations are bitwise those of its solve alone.
#pragma once

#include <condition_variable>
#include <cstdint>
#include <deque>
#include <future>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "engine.h"

namespace sdfgpu {

/// Device bytes an engine for `hp` will hold (state, specs, symbolic
/// structure, fronts; the mixed-precision copies when `mixed`), from its
/// host-side symbolic analysis `piece`.
int64_t EstimateDeviceBytes(const HostProblem& hp, const SymPiece& piece, bool mixed);

class Server {
 public:
  Server(int64_t budget_bytes, int max_batch);
  ~Server();
  Server(const Server&) = delete;
  Server& operator=(const Server&) = delete;

  int64_t Submit(HostProblem hp, const sdfgpu_solver_options& options);
  void Poll(int64_t id, sdfgpu_solve_result* result, double* map_values, double* poses);
  void Cancel(int64_t id);
  void Stats(double* stats);
  void Drain(int64_t timeout_ms);

 private:
  enum class State { kQueued, kRunning, kDone, kCancelled };
  struct Request {
    int64_t id{0};
    HostProblem hp;
    SymPiece piece;  // its symbolic analysis (handed to the cohort's engine)
    sdfgpu_solve_result result{};
    sdfgpu_solver_options options{};
    int64_t bytes{0};
    State state{State::kQueued};
    bool answered{false};  // result and state copied out
    std::chrono::steady_clock::time_point submitted;
    std::vector<double> map_values;
    std::vector<double> poses;
  };
  /// Requests solved together in one batched engine.
  struct Cohort {
    std::vector<Request*> members;  // instance i of the engine is members[i]
    std::unique_ptr<Engine> engine;
    std::future<void> job;  // host work in flight (engine setup, re-analysis)
    bool in_flight{false};  // an LM iteration is enqueued on the device
    bool failed{false};
    int status{SDFGPU_OK};
    int64_t bytes{0};
  };
  void Loop();
  /// True while the cohort's host job runs; collects a finished job (a
  /// failure marks the cohort failed).
  bool Busy(Cohort& c);
  /// Copies out the result and state of every member whose solve has ended.
  void Answer(Cohort& c);

  int64_t budget_;
  int max_batch_;
  int device_{0};
  std::mutex mu_;
  std::condition_variable cv_;
  std::condition_variable done_cv_;
  bool stop_{false};
  std::deque<int64_t> queue_;
  std::map<int64_t, std::unique_ptr<Request>> requests_;
  std::vector<std::unique_ptr<Cohort>> cohorts_;
  int64_t running_{0};  // requests in cohorts that have not been answered
  int64_t used_bytes_{0};
  int64_t next_id_{1};
  int64_t submitted_{0};
  int64_t completed_{0};
  int64_t iterations_{0};
  std::vector<double> latencies_ms_;
  std::chrono::steady_clock::time_point created_;
  std::thread worker_;
};

}  // namespace sdfgpu
