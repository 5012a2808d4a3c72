// Serving loop with continuous batching. Each admitted request keeps its
// state, symbolic analysis and factors resident on the device in its own
// engine (own CUDA stream). The loop keeps one LM iteration of every running
// request in flight: it finishes an iteration as soon as its stream's event
// reports it done and enqueues that request's next one, so requests of very
// different sizes overlap on the GPU without waiting for one another. Requests are admitted while their estimated device footprint
// fits the budget and retire as soon as their solve ends. Host work of a
// request (building its engine, re-analysing a pattern its state left) runs
// on a helper thread while the other requests keep iterating.
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
/// structure, fronts; the mixed-precision copies when `mixed`), from a
/// host-side symbolic analysis.
int64_t EstimateDeviceBytes(const HostProblem& hp, bool mixed);

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
    sdfgpu_solver_options options{};
    int64_t bytes{0};
    State state{State::kQueued};
    std::chrono::steady_clock::time_point submitted;
    std::unique_ptr<Engine> engine;
    std::future<void> job;  // host work in flight (engine setup, re-analysis)
    bool in_flight{false};  // an LM iteration is enqueued on the device
    sdfgpu_solve_result result{};
    std::vector<double> map_values;
    std::vector<double> poses;
  };
  void Loop();
  void Retire(Request& r);
  /// True while the request's host job runs; collects a finished job (a
  /// failure marks the request failed).
  bool Busy(Request& r);

  int64_t budget_;
  int max_batch_;
  int device_{0};
  std::mutex mu_;
  std::condition_variable cv_;
  std::condition_variable done_cv_;
  bool stop_{false};
  std::deque<int64_t> queue_;
  std::map<int64_t, std::unique_ptr<Request>> requests_;
  std::vector<Request*> running_;
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
