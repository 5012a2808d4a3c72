// The incremental run_slam driver on the GPU engine (Run in incremental mode,
// src/pipeline/runner.cpp:226-285).
#pragma once

#include <vector>

#include "sdfgpu.h"

namespace sdfgpu {

struct IncrementalInput {
  int nx{2};
  int ny{2};
  double min_x{0.0};
  double min_y{0.0};
  double max_x{1.0};
  double max_y{1.0};
  const double* map_values{nullptr};  // nx * ny initial values (null: zeros)
  int num_frames{0};
  const double* poses{nullptr};  // dataset poses, 3 per frame
  const int32_t* scan_offsets{nullptr};
  const double* scan_xy{nullptr};
  int num_relations{0};
  const int32_t* relation_ij{nullptr};
  const double* relation_meas{nullptr};
  const double* relation_sqrt_weight{nullptr};
  int increment_size{1};
  int iterations_per_increment{10};
  int snapshot_every{0};
  sdfgpu_snapshot_fn snapshot{nullptr};
  void* snapshot_user{nullptr};
  int build_on_device{1};
  int warm_analysis{1};
};

/// Host seconds per part of the run, summed over its increments.
struct IncrementalPhases {
  double build{0};          // problem construction
  double wait_analysis{0};  // waiting for the overlapped analysis
  double setup{0};          // engine set-up: upload, analysis (when not overlapped), structure
  double solve{0};          // the LM iterations
  double readback{0};       // state back to the host
  double teardown{0};       // releasing the step's engine
  double wall{0};           // the whole run
  int increments{0};
  int warm_analyses{0};     // increments whose analysis overlapped the previous solve
  int reanalyses{0};        // pattern re-analyses inside the steps' iterations
  double reanalysis{0};     // host seconds of those re-analyses (part of solve)
  double capture{0};        // host seconds capturing iteration graphs (part of solve)
};

struct IncrementalOutput {
  std::vector<double> map;    // nx * ny
  std::vector<double> poses;  // 3 per frame
  sdfgpu_solve_result total{};
  std::vector<double> cost_history;  // every increment's history, concatenated
  IncrementalPhases phases;
};

void RunIncremental(const IncrementalInput& in, const sdfgpu_problem_options& problem_options,
                    const sdfgpu_solver_options& solver_options, IncrementalOutput* out);

}  // namespace sdfgpu
