// The incremental driver of run_slam (Run in incremental mode,
// src/pipeline/runner.cpp:226-285; the dissertation's algorithm 2): frames
// are appended `increment_size` at a time, each new pose composed from the
// last optimized pose and the dataset's odometry, then the problem over all
// frames so far is rebuilt (map and poses carried over) and solved for
// `iterations_per_increment` LM iterations on the GPU engine.
//
// Per increment the problem is built (optionally by the device builder) and
// replaces the previous one in the same GPU engine: the point rows of the
// frames already there stay on the device and only the new frames' rows go
// up. The state comes back to the host for the next build. The next
// increment's symbolic analysis does not wait for the solve: it runs on a
// host thread while the GPU iterates, on the problem the next increment
// would have if the solve left the poses where they are (whose point rows
// the next build takes over), and the engine checks every iteration that the
// solved state still lies in that pattern (re-analysing when a point left
// it).
#include <chrono>
#include <cmath>
#include <future>
#include <memory>
#include <utility>
#include <vector>

#include "engine.h"
#include "incremental.h"
#include "internal.h"

namespace sdfgpu {

namespace {

struct Pose {
  double x;
  double y;
  double theta;
};

/// WrapAngle (src/core/pose.hpp:9): atan2(sin a, cos a).
inline double Wrap(double a) { return std::atan2(std::sin(a), std::cos(a)); }

/// Pose2::Compose (pose.hpp:33-36): (R(theta) t_rel + t, wrap(theta + theta_rel)).
inline Pose Compose(const Pose& a, const Pose& rel) {
  const double c = std::cos(a.theta);
  const double s = std::sin(a.theta);
  return {(c * rel.x + (-s) * rel.y) + a.x, (s * rel.x + c * rel.y) + a.y, Wrap(a.theta + rel.theta)};
}

/// Pose2::RelativeTo (pose.hpp:38-43): (R(theta)^T (t_o - t), wrap(theta_o - theta)).
inline Pose RelativeTo(const Pose& a, const Pose& o) {
  const double c = std::cos(a.theta);
  const double s = std::sin(a.theta);
  const double dx = o.x - a.x;
  const double dy = o.y - a.y;
  return {c * dx + s * dy, (-s) * dx + c * dy, Wrap(o.theta - a.theta)};
}

double Seconds(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

void RunIncremental(const IncrementalInput& in, const sdfgpu_problem_options& po, const sdfgpu_solver_options& so,
                    IncrementalOutput* out) {
  const int F = in.num_frames;
  if (F < 2) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT, "dataset needs at least two scans");
  }
  if (in.increment_size < 1) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT, "increment_size must be >= 1");
  }
  if (in.iterations_per_increment < 0) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT, "iterations_per_increment must be >= 0");
  }
  if (in.poses == nullptr || in.scan_offsets == nullptr || (in.scan_offsets[F] > 0 && in.scan_xy == nullptr)) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT, "poses and scans are required");
  }
  if (in.num_relations > 0 && (in.relation_ij == nullptr || in.relation_meas == nullptr)) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT, "relation arrays missing");
  }
  const auto start = std::chrono::steady_clock::now();
  // odometry between consecutive dataset poses (runner.cpp:52-59)
  std::vector<Pose> dataset(static_cast<size_t>(F));
  for (int i = 0; i < F; ++i) {
    dataset[static_cast<size_t>(i)] = {in.poses[3 * i], in.poses[3 * i + 1], in.poses[3 * i + 2]};
  }
  std::vector<double> odometry(3 * static_cast<size_t>(F - 1));
  for (int i = 0; i + 1 < F; ++i) {
    const Pose r = RelativeTo(dataset[static_cast<size_t>(i)], dataset[static_cast<size_t>(i) + 1]);
    odometry[3 * static_cast<size_t>(i)] = r.x;
    odometry[3 * static_cast<size_t>(i) + 1] = r.y;
    odometry[3 * static_cast<size_t>(i) + 2] = r.theta;
  }
  const size_t nodes = static_cast<size_t>(in.nx) * static_cast<size_t>(in.ny);
  std::vector<double> map(nodes, 0.0);
  if (in.map_values != nullptr) {
    std::copy(in.map_values, in.map_values + nodes, map.begin());
  }
  std::vector<double> est{dataset[0].x, dataset[0].y, dataset[0].theta};
  auto append = [&](std::vector<double>& poses, int from, int to) {
    for (int i = from; i < to; ++i) {
      const size_t b = poses.size() - 3;
      const Pose p = Compose({poses[b], poses[b + 1], poses[b + 2]},
                             {odometry[3 * static_cast<size_t>(i - 1)], odometry[3 * static_cast<size_t>(i - 1) + 1],
                              odometry[3 * static_cast<size_t>(i - 1) + 2]});
      poses.push_back(p.x);
      poses.push_back(p.y);
      poses.push_back(p.theta);
    }
  };
  auto build = [&](const std::vector<double>& m, const std::vector<double>& poses, int frames, bool rows) {
    return BuildProblem(in.nx, in.ny, in.min_x, in.min_y, in.max_x, in.max_y, m.data(), frames, poses.data(),
                        in.scan_offsets, in.scan_xy, odometry.data(), frames - 1, in.num_relations, in.relation_ij,
                        in.relation_meas, in.relation_sqrt_weight, po, BuildMode{in.build_on_device != 0, false, rows});
  };
  sdfgpu_solver_options step_options = so;
  step_options.max_iterations = in.iterations_per_increment;
  sdfgpu_solve_result& total = out->total;
  total = sdfgpu_solve_result{};
  total.initial_cost = -1.0;
  out->cost_history.clear();
  out->phases = IncrementalPhases{};
  std::vector<double> hist(static_cast<size_t>(in.iterations_per_increment) + 2);
  int next_frame = 1;
  int increment = 0;
  // The engine stays across steps: each step's problem replaces the last
  // one's, whose point rows (a prefix of the new rows: rows depend on the
  // scans alone and come frame by frame) stay on the device.
  std::unique_ptr<Engine> engine;
  int64_t engine_rows = 0;
  // The coming step's pattern-only problem (point rows, active map and pose
  // pairs at the poses the current step started from) and its analysis,
  // made on a host thread while the GPU iterates.
  struct Speculative {
    HostProblem problem;
    SymPiece piece;
  };
  std::future<Speculative> speculative;
  int speculative_frames = 0;
  while (next_frame < F) {
    const int last = std::min(F, next_frame + in.increment_size);
    append(est, next_frame, last);
    next_frame = last;
    auto t0 = std::chrono::steady_clock::now();
    Speculative spec;
    bool have_spec = false;
    if (speculative.valid()) {
      spec = speculative.get();
      have_spec = speculative_frames == next_frame;
    }
    out->phases.wait_analysis += Seconds(t0);
    t0 = std::chrono::steady_clock::now();
    // the device builder leaves out the point rows when the speculative
    // problem has them (the same rows)
    const bool rows_given = have_spec && in.build_on_device != 0;
    HostProblem hp = build(map, est, next_frame, !rows_given);
    if (rows_given) {
      hp.pt_frame = std::move(spec.problem.pt_frame);
      hp.pt_xy = std::move(spec.problem.pt_xy);
      hp.pt_expected = std::move(spec.problem.pt_expected);
      hp.pt_sqrtw = std::move(spec.problem.pt_sqrtw);
    }
    out->phases.build += Seconds(t0);
    // the analysis is usable when it analysed the same columns (the active
    // set can move with the poses when the active region is on)
    const bool have_piece = have_spec && spec.problem.node_to_active == hp.node_to_active;
    if (have_piece) {
      ++out->phases.warm_analyses;
    }
    t0 = std::chrono::steady_clock::now();
    if (engine != nullptr && engine->CanReplace(hp)) {
      engine->Replace(std::move(hp), have_piece ? &spec.piece : nullptr, engine_rows);
    } else if (have_piece) {
      engine.reset();
      engine = std::make_unique<Engine>(std::move(hp), std::move(spec.piece));
    } else {
      engine.reset();
      std::vector<HostProblem> v;
      v.push_back(std::move(hp));
      engine = std::make_unique<Engine>(std::move(v));
    }
    engine_rows = engine->host(0).num_points();
    out->phases.setup += Seconds(t0);
    if (in.warm_analysis != 0 && next_frame < F) {
      const int frames = std::min(F, next_frame + in.increment_size);
      std::vector<double> guess = est;
      append(guess, next_frame, frames);
      speculative_frames = frames;
      speculative = std::async(std::launch::async, [&, guess = std::move(guess), frames] {
        Speculative next;
        next.problem = BuildProblem(in.nx, in.ny, in.min_x, in.min_y, in.max_x, in.max_y, nullptr, frames,
                                    guess.data(), in.scan_offsets, in.scan_xy, odometry.data(), frames - 1,
                                    in.num_relations, in.relation_ij, in.relation_meas, in.relation_sqrt_weight, po,
                                    BuildMode{false, true, true});
        next.piece = AnalyzeInstance(next.problem, kDefaultMargin);
        return next;
      });
    }
    t0 = std::chrono::steady_clock::now();
    sdfgpu_solve_result step{};
    engine->Solve({step_options}, &step, hist.data(), static_cast<int>(hist.size()));
    out->phases.solve += Seconds(t0);
    out->phases.reanalyses += engine->times().reanalyses;
    out->phases.reanalysis += engine->times().reanalysis_host;
    out->phases.capture += engine->times().capture_host;
    if (step.status != SDFGPU_OK) {
      if (speculative.valid()) {
        speculative.wait();
      }
      Fail(step.status, step.status == SDFGPU_ERR_NUMERICAL ? "sparse Cholesky factorization failed"
                                                           : "increment solve failed");
    }
    t0 = std::chrono::steady_clock::now();
    engine->GetState(0, map.data(), est.data());
    out->phases.readback += Seconds(t0);
    if (total.initial_cost < 0.0) {
      total.initial_cost = step.initial_cost;
    }
    total.iterations += step.iterations;
    total.final_cost = step.final_cost;
    total.duration_seconds += step.duration_seconds;
    total.converged = step.converged;
    out->cost_history.insert(out->cost_history.end(), hist.begin(), hist.begin() + step.cost_history_length);
    ++increment;
    if (in.snapshot != nullptr && in.snapshot_every > 0 &&
        (increment % in.snapshot_every == 0 || next_frame == F)) {
      in.snapshot(in.snapshot_user, next_frame, map.data(), est.data());
    }
  }
  const auto t0 = std::chrono::steady_clock::now();
  engine.reset();
  out->phases.teardown += Seconds(t0);
  out->map = std::move(map);
  out->poses = std::move(est);
  out->phases.increments = increment;
  out->phases.wall = Seconds(start);
}

}  // namespace sdfgpu
