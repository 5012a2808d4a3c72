// Serving loop (see server.h).
#include "server.h"

#include <algorithm>
#include <cmath>

namespace sdfgpu {

int64_t EstimateDeviceBytes(const HostProblem& hp, bool mixed) {
  std::vector<HostProblem> v{hp};
  InstanceLayout L{};
  L.col_off = 0;
  const Symbolic S = Analyze(v, {L}, 32, 64);
  const int64_t P = hp.num_points();
  const int64_t nodes = static_cast<int64_t>(hp.nx) * hp.ny;
  // fronts grow when a re-analysis widens the coupling margin; a mixed solve
  // adds the FP64 assembled copy and the FP32 work copy
  int64_t bytes = S.front_doubles * (mixed ? 20 : 8) * 2;
  bytes += P * (8 * 8 + 4 * 8 + 4 * 8 + 48);       // row records, pose offsets, cells, sort buffers, specs
  bytes += nodes * (8 * 3 + 4 * 4);                 // map, backup, index maps
  bytes += static_cast<int64_t>(S.mm_off.size()) * 8 + static_cast<int64_t>(S.mp_off.size()) * 12;
  bytes += static_cast<int64_t>(S.sn_rows.size()) * 8 + static_cast<int64_t>(S.update_tasks.size()) * 4;
  bytes += static_cast<int64_t>(hp.num_params()) * 8 * 8;
  return bytes;
}

Server::Server(int64_t budget_bytes, int max_batch)
    : budget_(budget_bytes), max_batch_(max_batch), created_(std::chrono::steady_clock::now()) {
  CudaCheck(cudaGetDevice(&device_), "cudaGetDevice");
  worker_ = std::thread([this] {
    cudaSetDevice(device_);
    Loop();
  });
}

bool Server::Busy(Request& r) {
  if (!r.job.valid()) {
    return false;
  }
  if (r.job.wait_for(std::chrono::seconds(0)) != std::future_status::ready) {
    return true;
  }
  try {
    r.job.get();
  } catch (const Error& e) {
    r.engine.reset();
    r.result.status = e.code();
  } catch (...) {
    r.engine.reset();
    r.result.status = SDFGPU_ERR_CUDA;
  }
  return false;
}

Server::~Server() {
  {
    std::lock_guard<std::mutex> lk(mu_);
    stop_ = true;
  }
  cv_.notify_all();
  if (worker_.joinable()) {
    worker_.join();
  }
}

int64_t Server::Submit(HostProblem hp, const sdfgpu_solver_options& options) {
  if (options.max_iterations < 0 || !(options.lambda_init >= 0.0) || !(options.lambda_factor > 0.0) ||
      (options.precision != SDFGPU_PRECISION_FP64 && options.precision != SDFGPU_PRECISION_MIXED) ||
      options.refine_steps < 0 || options.refine_steps > 16) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT, "invalid solver options");
  }
  const int64_t bytes = EstimateDeviceBytes(hp, options.precision == SDFGPU_PRECISION_MIXED);
  if (bytes > budget_) {
    Fail(SDFGPU_ERR_OUT_OF_MEMORY, "request footprint " + std::to_string(bytes) + " bytes exceeds the budget");
  }
  auto r = std::make_unique<Request>();
  r->hp = std::move(hp);
  r->options = options;
  r->bytes = bytes;
  r->submitted = std::chrono::steady_clock::now();
  int64_t id = 0;
  {
    std::lock_guard<std::mutex> lk(mu_);
    id = next_id_++;
    r->id = id;
    requests_[id] = std::move(r);
    queue_.push_back(id);
    ++submitted_;
  }
  cv_.notify_all();
  return id;
}

void Server::Poll(int64_t id, sdfgpu_solve_result* result, double* map_values, double* poses) {
  std::lock_guard<std::mutex> lk(mu_);
  auto it = requests_.find(id);
  if (it == requests_.end()) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT, "unknown request id");
  }
  Request& r = *it->second;
  if (r.state == State::kQueued || r.state == State::kRunning) {
    Fail(SDFGPU_ERR_NOT_READY, "request not finished");
  }
  if (result != nullptr) {
    *result = r.result;
  }
  if (map_values != nullptr && !r.map_values.empty()) {
    std::copy(r.map_values.begin(), r.map_values.end(), map_values);
  }
  if (poses != nullptr && !r.poses.empty()) {
    std::copy(r.poses.begin(), r.poses.end(), poses);
  }
  requests_.erase(it);
}

void Server::Cancel(int64_t id) {
  std::lock_guard<std::mutex> lk(mu_);
  auto it = requests_.find(id);
  if (it == requests_.end()) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT, "unknown request id");
  }
  Request& r = *it->second;
  if (r.state == State::kQueued) {
    queue_.erase(std::remove(queue_.begin(), queue_.end(), id), queue_.end());
    r.state = State::kCancelled;
    r.result.status = SDFGPU_ERR_INVALID_ARGUMENT;
    done_cv_.notify_all();
  } else if (r.state == State::kRunning) {
    r.state = State::kCancelled;  // the worker frees it after the current round
  }
}

void Server::Stats(double* stats) {
  std::lock_guard<std::mutex> lk(mu_);
  std::vector<double> lat = latencies_ms_;
  std::sort(lat.begin(), lat.end());
  auto pct = [&lat](double p) {
    if (lat.empty()) {
      return 0.0;
    }
    const size_t idx = std::min(lat.size() - 1, static_cast<size_t>(std::ceil(p * lat.size())) - 1);
    return lat[idx];
  };
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - created_).count();
  stats[0] = static_cast<double>(submitted_);
  stats[1] = static_cast<double>(completed_);
  stats[2] = static_cast<double>(queue_.size());
  stats[3] = static_cast<double>(running_.size());
  stats[4] = pct(0.50);
  stats[5] = pct(0.99);
  stats[6] = secs > 0 ? completed_ / secs : 0.0;
  stats[7] = secs > 0 ? iterations_ / secs : 0.0;
}

void Server::Drain(int64_t timeout_ms) {
  std::unique_lock<std::mutex> lk(mu_);
  const bool ok = done_cv_.wait_for(lk, std::chrono::milliseconds(timeout_ms),
                                    [this] { return queue_.empty() && running_.empty(); });
  if (!ok) {
    Fail(SDFGPU_ERR_TIMEOUT, "requests still pending after the drain timeout");
  }
}

void Server::Retire(Request& r) {
  // caller holds no lock; engine work happens outside the mutex
  r.result.status = r.result.status;
  r.engine.reset();
}

void Server::Loop() {
  for (;;) {
    std::vector<Request*> admitted;
    {
      std::unique_lock<std::mutex> lk(mu_);
      cv_.wait_for(lk, std::chrono::milliseconds(50),
                   [this] { return stop_ || !queue_.empty() || !running_.empty(); });
      if (stop_) {
        break;
      }
      while (!queue_.empty() && static_cast<int>(running_.size() + admitted.size()) < max_batch_) {
        Request& r = *requests_[queue_.front()];
        if (used_bytes_ + r.bytes > budget_ && !(running_.empty() && admitted.empty())) {
          break;  // wait for memory to free up
        }
        queue_.pop_front();
        used_bytes_ += r.bytes;
        r.state = State::kRunning;
        admitted.push_back(&r);
      }
    }
    for (Request* r : admitted) {
      // engine setup (upload, symbolic analysis, initial cost) off this thread
      r->job = std::async(std::launch::async, [this, r] {
        cudaSetDevice(device_);
        std::vector<HostProblem> v{r->hp};
        r->engine = std::make_unique<Engine>(std::move(v));
        r->engine->BeginSolve({r->options});
      });
      std::lock_guard<std::mutex> lk(mu_);
      running_.push_back(r);
    }
    // one pass: finish every iteration whose device work is done, enqueue
    // the next iteration of every idle request; a request whose state left
    // its pattern is re-analysed off this thread
    bool progressed = false;
    for (Request* r : running_) {
      if (Busy(*r)) {
        continue;
      }
      if (!r->engine) {
        continue;
      }
      try {
        if (r->in_flight) {
          if (!r->engine->IterationReady()) {
            continue;
          }
          r->in_flight = false;
          r->engine->FinishIteration();
          progressed = true;
          std::lock_guard<std::mutex> lk(mu_);
          ++iterations_;
        }
        if (r->state != State::kRunning || r->engine->SolveDone()) {
          continue;
        }
        if (r->engine->NeedsReanalysis()) {
          Engine* e = r->engine.get();
          r->job = std::async(std::launch::async, [this, e] {
            cudaSetDevice(device_);
            e->ReanalyzeNow();
          });
          continue;
        }
        r->engine->LaunchIteration();
        r->in_flight = true;
        progressed = true;
      } catch (const Error& e) {
        r->in_flight = false;
        r->result.status = e.code();
        r->engine.reset();
      }
    }
    if (!progressed) {
      // nothing finished and nothing new to enqueue: yield briefly
      std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
    // retire finished, failed and cancelled requests
    std::vector<Request*> still;
    for (Request* r : running_) {
      if (r->job.valid() || r->in_flight) {
        still.push_back(r);  // its host job or device iteration must end first
        continue;
      }
      const bool cancelled = r->state == State::kCancelled;
      const bool failed = !r->engine;
      const bool done = !failed && r->engine->SolveDone();
      if (!(cancelled || failed || done)) {
        still.push_back(r);
        continue;
      }
      if (done && !cancelled) {
        try {
          r->engine->EndSolve(&r->result, nullptr, 0);
          r->map_values.resize(static_cast<size_t>(r->hp.nx) * r->hp.ny);
          r->poses.resize(3 * static_cast<size_t>(r->hp.num_frames()));
          r->engine->GetState(0, r->map_values.data(), r->poses.data());
        } catch (const Error& e) {
          r->result.status = e.code();
        }
      }
      Retire(*r);
      std::lock_guard<std::mutex> lk(mu_);
      used_bytes_ -= r->bytes;
      if (!cancelled) {
        r->state = State::kDone;
        ++completed_;
        latencies_ms_.push_back(
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - r->submitted).count());
      } else {
        r->result.status = SDFGPU_ERR_INVALID_ARGUMENT;
      }
    }
    {
      std::lock_guard<std::mutex> lk(mu_);
      running_.swap(still);
      if (queue_.empty() && running_.empty()) {
        done_cv_.notify_all();
      }
    }
  }
  for (Request* r : running_) {
    if (r->job.valid()) {
      r->job.wait();
    }
    if (r->engine && r->in_flight) {
      cudaStreamSynchronize(r->engine->stream());
    }
    r->engine.reset();
  }
}

}  // namespace sdfgpu
