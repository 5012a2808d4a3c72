// Serving loop (see server.h).
#include "server.h"

#include <algorithm>
#include <cmath>

namespace sdfgpu {

int64_t EstimateDeviceBytes(const HostProblem& hp, const SymPiece& piece, bool mixed) {
  const Symbolic& S = piece.s;
  const int64_t P = hp.num_points();
  const int64_t nodes = static_cast<int64_t>(hp.nx) * hp.ny;
  // fronts grow when a re-analysis widens the coupling margin; a mixed solve
  // adds the FP64 assembled copy and the FP32 work copy
  int64_t bytes = S.front_doubles * (mixed ? 20 : 8) * 2;
  bytes += P * (8 * 8 + 4 * 8 + 4 * 8 + 48);       // row records, pose offsets, cells, sort buffers, specs
  bytes += nodes * (8 * 3 + 4 * 4);                 // map, backup, index maps
  bytes += static_cast<int64_t>(S.mm_off.size()) * 8 + static_cast<int64_t>(S.mp_off.size()) * 12;
  bytes += static_cast<int64_t>(S.sn_rows.size()) * 8 + static_cast<int64_t>(S.sn.size()) * 256;
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

bool Server::Busy(Cohort& c) {
  if (!c.job.valid()) {
    return false;
  }
  if (c.job.wait_for(std::chrono::seconds(0)) != std::future_status::ready) {
    return true;
  }
  try {
    c.job.get();
  } catch (const Error& e) {
    c.failed = true;
    c.status = e.code();
  } catch (...) {
    c.failed = true;
    c.status = SDFGPU_ERR_CUDA;
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
      options.refine_steps < 0 || options.refine_steps > 16 ||
      !(options.refine_tolerance >= 0.0 && options.refine_tolerance < 1.0)) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT, "invalid solver options");
  }
  // the analysis that sizes the request is the one its engine will use
  SymPiece piece = AnalyzeInstance(hp, kDefaultMargin);
  const int64_t bytes = EstimateDeviceBytes(hp, piece, options.precision == SDFGPU_PRECISION_MIXED);
  if (bytes > budget_) {
    Fail(SDFGPU_ERR_OUT_OF_MEMORY, "request footprint " + std::to_string(bytes) + " bytes exceeds the budget");
  }
  auto r = std::make_unique<Request>();
  r->hp = std::move(hp);
  r->piece = std::move(piece);
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
    // its cohort keeps iterating it; the result is dropped
    r.state = State::kCancelled;
    r.result.status = SDFGPU_ERR_INVALID_ARGUMENT;
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
  stats[3] = static_cast<double>(running_);
  stats[4] = pct(0.50);
  stats[5] = pct(0.99);
  stats[6] = secs > 0 ? completed_ / secs : 0.0;
  stats[7] = secs > 0 ? iterations_ / secs : 0.0;
}

void Server::Drain(int64_t timeout_ms) {
  std::unique_lock<std::mutex> lk(mu_);
  const bool ok = done_cv_.wait_for(lk, std::chrono::milliseconds(timeout_ms),
                                    [this] { return queue_.empty() && running_ == 0; });
  if (!ok) {
    Fail(SDFGPU_ERR_TIMEOUT, "requests still pending after the drain timeout");
  }
}

void Server::Answer(Cohort& c) {
  for (size_t i = 0; i < c.members.size(); ++i) {
    Request& r = *c.members[i];
    if (r.answered || (!c.failed && !c.engine->InstanceDone(static_cast<int>(i)))) {
      continue;
    }
    sdfgpu_solve_result res{};
    if (c.failed) {
      res.status = c.status;
    } else {
      try {
        res = c.engine->InstanceResult(static_cast<int>(i));
        r.map_values.resize(static_cast<size_t>(r.hp.nx) * r.hp.ny);
        r.poses.resize(3 * static_cast<size_t>(r.hp.num_frames()));
        c.engine->GetState(static_cast<int>(i), r.map_values.data(), r.poses.data());
      } catch (const Error& e) {
        res.status = e.code();
      }
    }
    r.answered = true;
    std::lock_guard<std::mutex> lk(mu_);
    --running_;
    if (r.state == State::kCancelled) {
      continue;
    }
    r.result = res;
    r.state = State::kDone;
    ++completed_;
    latencies_ms_.push_back(
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - r.submitted).count());
  }
}

void Server::Loop() {
  // Cohorts running at once: a request that arrives while this many are on
  // the GPU waits for the next cohort, which takes every request then
  // waiting (up to max_batch running requests in all).
  constexpr size_t kMaxCohorts = 4;
  for (;;) {
    std::unique_ptr<Cohort> fresh;
    {
      std::unique_lock<std::mutex> lk(mu_);
      cv_.wait_for(lk, std::chrono::milliseconds(50), [this] { return stop_ || !queue_.empty() || running_ > 0; });
      if (stop_) {
        break;
      }
      if (!queue_.empty() && cohorts_.size() < kMaxCohorts && running_ < max_batch_) {
        auto c = std::make_unique<Cohort>();
        while (!queue_.empty() && running_ + static_cast<int64_t>(c->members.size()) < max_batch_) {
          Request& r = *requests_[queue_.front()];
          if (used_bytes_ + c->bytes + r.bytes > budget_ && !(cohorts_.empty() && c->members.empty())) {
            break;  // wait for memory to free up
          }
          queue_.pop_front();
          c->bytes += r.bytes;
          r.state = State::kRunning;
          c->members.push_back(&r);
        }
        if (!c->members.empty()) {
          used_bytes_ += c->bytes;
          running_ += static_cast<int64_t>(c->members.size());
          fresh = std::move(c);
        }
      }
    }
    if (fresh) {
      // engine setup (concatenation of the members' analyses, upload,
      // initial cost) off this thread
      Cohort* c = fresh.get();
      c->job = std::async(std::launch::async, [this, c] {
        cudaSetDevice(device_);
        std::vector<HostProblem> problems;
        std::vector<SymPiece> pieces;
        std::vector<sdfgpu_solver_options> options;
        for (Request* r : c->members) {
          problems.push_back(r->hp);
          pieces.push_back(std::move(r->piece));
          options.push_back(r->options);
        }
        c->engine = std::make_unique<Engine>(std::move(problems), std::move(pieces));
        c->engine->BeginSolve(options);
      });
      cohorts_.push_back(std::move(fresh));
    }
    // one pass: finish every iteration whose device work is done, answer the
    // members whose solves ended, enqueue the next iteration of every idle
    // cohort; a cohort with a member whose state left its pattern is
    // re-analysed off this thread
    bool progressed = false;
    for (auto& cp : cohorts_) {
      Cohort& c = *cp;
      if (Busy(c) || c.failed || !c.engine) {
        continue;
      }
      try {
        if (c.in_flight) {
          if (!c.engine->IterationReady()) {
            continue;
          }
          c.in_flight = false;
          c.engine->FinishIteration();
          progressed = true;
          int running = 0;
          for (size_t i = 0; i < c.members.size(); ++i) {
            running += c.engine->InstanceDone(static_cast<int>(i)) ? 0 : 1;
          }
          std::lock_guard<std::mutex> lk(mu_);
          iterations_ += running;
        }
        Answer(c);
        if (c.engine->SolveDone()) {
          continue;
        }
        if (c.engine->NeedsReanalysis()) {
          Engine* e = c.engine.get();
          c.job = std::async(std::launch::async, [this, e] {
            cudaSetDevice(device_);
            e->ReanalyzeNow();
          });
          continue;
        }
        c.engine->LaunchIteration();
        c.in_flight = true;
        progressed = true;
      } catch (const Error& e) {
        c.in_flight = false;
        c.failed = true;
        c.status = e.code();
      }
    }
    if (!progressed) {
      // nothing finished and nothing new to enqueue: yield briefly
      std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
    // retire cohorts whose members are all answered (or that failed)
    std::vector<std::unique_ptr<Cohort>> still;
    for (auto& cp : cohorts_) {
      Cohort& c = *cp;
      if (c.job.valid() || c.in_flight) {
        still.push_back(std::move(cp));  // its host job or device iteration must end first
        continue;
      }
      if (!c.failed && c.engine && !c.engine->SolveDone()) {
        still.push_back(std::move(cp));
        continue;
      }
      Answer(c);
      c.engine.reset();
      std::lock_guard<std::mutex> lk(mu_);
      used_bytes_ -= c.bytes;
    }
    {
      std::lock_guard<std::mutex> lk(mu_);
      cohorts_.swap(still);
      if (queue_.empty() && running_ == 0) {
        done_cv_.notify_all();
      }
    }
  }
  for (auto& cp : cohorts_) {
    if (cp->job.valid()) {
      cp->job.wait();
    }
    if (cp->engine && cp->in_flight) {
      cudaStreamSynchronize(cp->engine->stream());
    }
    cp->engine.reset();
  }
}

}  // namespace sdfgpu
