// C ABI of the sdfgpu library (declared in include/sdfgpu.h). Every entry
// point converts exceptions into status codes and records the message for
// sdfgpu_last_error_message().
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "engine.h"
#include "incremental.h"
#include "internal.h"
#include "ldlt.h"
#include "server.h"

namespace sdfgpu {
void DenseLdltSolveNoAlloc(int n, const double* a, const double* b, double* x);
}  // namespace sdfgpu

struct sdfgpu_problem {
  std::vector<sdfgpu::HostProblem> host;  // specs as given (state lives on the device once uploaded)
  std::unique_ptr<sdfgpu::Engine> engine;
  sdfgpu::Engine& Device() {
    if (!engine) {
      engine = std::make_unique<sdfgpu::Engine>(host);
    }
    return *engine;
  }
};

struct sdfgpu_ldlt {
  std::unique_ptr<sdfgpu::LdltEngine> engine;
};

struct sdfgpu_server {
  std::unique_ptr<sdfgpu::Server> server;
};

namespace {

thread_local std::string g_last_error;

template <typename Fn>
int Guard(Fn&& fn) {
  try {
    g_last_error.clear();
    fn();
    return SDFGPU_OK;
  } catch (const sdfgpu::Error& e) {
    g_last_error = e.what();
    return e.code();
  } catch (const std::bad_alloc&) {
    g_last_error = "host allocation failed";
    return SDFGPU_ERR_OUT_OF_MEMORY;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return SDFGPU_ERR_CUDA;
  } catch (...) {
    g_last_error = "unknown error";
    return SDFGPU_ERR_CUDA;
  }
}

void NeedHandle(const void* p, const char* what) {
  if (p == nullptr) {
    sdfgpu::Fail(SDFGPU_ERR_INVALID_ARGUMENT, std::string(what) + " is NULL");
  }
}

sdfgpu::Engine& Eng(sdfgpu_problem* p) {
  NeedHandle(p, "problem");
  return p->Device();
}

void CheckIndex(const sdfgpu_problem* p, int32_t index) {
  NeedHandle(p, "problem");
  if (index < 0 || index >= static_cast<int32_t>(p->host.size())) {
    sdfgpu::Fail(SDFGPU_ERR_INVALID_ARGUMENT, "instance index out of range");
  }
}

}  // namespace

extern "C" {

const char* sdfgpu_last_error_message(void) { return g_last_error.c_str(); }

const char* sdfgpu_version(void) { return "sdfgpu 0.1 (sm_100a)"; }

int32_t sdfgpu_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

void sdfgpu_problem_options_default(sdfgpu_problem_options* o) {
  if (o == nullptr) {
    return;
  }
  *o = sdfgpu_problem_options{};
  o->weight_scan = 1.0;
  o->weight_hallucination = 1.0;
  o->weight_eikonal = 1.0;
  o->weight_odometry = 1.0;
  o->weight_relation = 1.0;
  o->hallucination_points_per_scan_point = 6;
  o->hallucination_step_size = 0.1;
  o->hallucination_both_directions = 1;
  o->normals_method = 2;
  o->normals_k_neighbors = 10;
  o->normals_per_scan = 0;
  o->normals_corner_threshold = 0.2;
  o->huber_delta = 0.0;
  o->smooth_gradient = 1;
  o->smooth_gradient_step = 0.0;
  o->active_region = 0;
  o->active_margin = 2;
}

void sdfgpu_solver_options_default(sdfgpu_solver_options* o) {
  if (o == nullptr) {
    return;
  }
  *o = sdfgpu_solver_options{};
  o->max_iterations = 100;
  o->step_tolerance = 1e-6;
  o->lambda_init = 1.0;
  o->lambda_factor = 1.0;
  o->reject_worse_steps = 0;
  o->marquardt_scaling = 0;
  o->trust_region = 0;
  o->num_threads = 0;
  o->precision = SDFGPU_PRECISION_FP64;
  o->refine_steps = 3;
  o->refine_tolerance = sdfgpu::kDefaultRefineTol;
}

// sdfgpu_problem_build and sdfgpu_problem_build_device (on_device: the point
// specs, active maps and Eikonal spec list by CUDA kernels).
static int BuildProblemHandle(bool on_device, int32_t nx, int32_t ny, double min_x, double min_y, double max_x,
                              double max_y, const double* map_values, int32_t num_frames, const double* poses,
                              const int32_t* scan_offsets, const double* scan_xy, const double* odometry,
                              int32_t num_odometry, int32_t num_relations, const int32_t* relation_ij,
                              const double* relation_meas, const double* relation_sqrt_weight,
                              const sdfgpu_problem_options* options, sdfgpu_problem** out) {
  return Guard([&] {
    NeedHandle(out, "out");
    *out = nullptr;
    sdfgpu_problem_options o;
    if (options != nullptr) {
      o = *options;
    } else {
      sdfgpu_problem_options_default(&o);
    }
    if (num_relations > 0 && (relation_ij == nullptr || relation_meas == nullptr)) {
      sdfgpu::Fail(SDFGPU_ERR_INVALID_ARGUMENT, "relation arrays missing");
    }
    if (num_odometry > 0 && odometry == nullptr) {
      sdfgpu::Fail(SDFGPU_ERR_INVALID_ARGUMENT, "odometry array missing");
    }
    std::vector<sdfgpu::HostProblem> v;
    v.push_back(sdfgpu::BuildProblem(nx, ny, min_x, min_y, max_x, max_y, map_values, num_frames, poses,
                                     scan_offsets, scan_xy, odometry, num_odometry, num_relations, relation_ij,
                                     relation_meas, relation_sqrt_weight, o,
                                     sdfgpu::BuildMode{on_device, false, true}));
    auto h = std::make_unique<sdfgpu_problem>();
    h->host = std::move(v);
    *out = h.release();
  });
}

int sdfgpu_problem_build(int32_t nx, int32_t ny, double min_x, double min_y, double max_x, double max_y,
                         const double* map_values, int32_t num_frames, const double* poses,
                         const int32_t* scan_offsets, const double* scan_xy, const double* odometry,
                         int32_t num_odometry, int32_t num_relations, const int32_t* relation_ij,
                         const double* relation_meas, const double* relation_sqrt_weight,
                         const sdfgpu_problem_options* options, sdfgpu_problem** out) {
  return BuildProblemHandle(false, nx, ny, min_x, min_y, max_x, max_y, map_values, num_frames, poses, scan_offsets,
                            scan_xy, odometry, num_odometry, num_relations, relation_ij, relation_meas,
                            relation_sqrt_weight, options, out);
}

int sdfgpu_problem_build_device(int32_t nx, int32_t ny, double min_x, double min_y, double max_x, double max_y,
                                const double* map_values, int32_t num_frames, const double* poses,
                                const int32_t* scan_offsets, const double* scan_xy, const double* odometry,
                                int32_t num_odometry, int32_t num_relations, const int32_t* relation_ij,
                                const double* relation_meas, const double* relation_sqrt_weight,
                                const sdfgpu_problem_options* options, sdfgpu_problem** out) {
  return BuildProblemHandle(true, nx, ny, min_x, min_y, max_x, max_y, map_values, num_frames, poses, scan_offsets,
                            scan_xy, odometry, num_odometry, num_relations, relation_ij, relation_meas,
                            relation_sqrt_weight, options, out);
}

int sdfgpu_problem_create(const sdfgpu_problem_desc* desc, sdfgpu_problem** out) {
  return sdfgpu_problem_create_batch(desc, 1, out);
}

int sdfgpu_problem_create_batch(const sdfgpu_problem_desc* descs, int32_t count, sdfgpu_problem** out) {
  return Guard([&] {
    NeedHandle(out, "out");
    *out = nullptr;
    NeedHandle(descs, "desc");
    if (count < 1) {
      sdfgpu::Fail(SDFGPU_ERR_INVALID_ARGUMENT, "batch count must be >= 1");
    }
    std::vector<sdfgpu::HostProblem> v;
    v.reserve(static_cast<size_t>(count));
    for (int32_t i = 0; i < count; ++i) {
      v.push_back(sdfgpu::FromDesc(descs[i]));
    }
    auto h = std::make_unique<sdfgpu_problem>();
    h->host = std::move(v);
    *out = h.release();
  });
}

int sdfgpu_problem_destroy(sdfgpu_problem* problem) {
  return Guard([&] { delete problem; });
}

int sdfgpu_release_cached_memory(void) {
  return Guard([&] { sdfgpu::ReleaseCachedDeviceMemory(); });
}

int sdfgpu_measure_fp64_peak(double* tflops) {
  return Guard([&] {
    NeedHandle(tflops, "tflops");
    *tflops = sdfgpu::MeasureFp64PeakTflops();
  });
}

int sdfgpu_debug_solve_fault(sdfgpu_problem* problem, int32_t withhold_front, uint32_t wait_polls) {
  return Guard([&] { Eng(problem).SetSolveFault(withhold_front, wait_polls); });
}

int32_t sdfgpu_debug_supernode_count(sdfgpu_problem* problem) {
  if (problem == nullptr || !problem->engine) {
    return 0;
  }
  return static_cast<int32_t>(problem->engine->symbolic().sn.size());
}

static_assert(sdfgpu::KernelTimer::kClasses == SDFGPU_KERNEL_CLASSES, "kernel class count");

int sdfgpu_kernel_timing(sdfgpu_problem* problem, uint32_t class_mask) {
  return Guard([&] { Eng(problem).SetKernelTiming(class_mask); });
}

int sdfgpu_kernel_times(sdfgpu_problem* problem, double* ms, int64_t* launches, double* work, int32_t count) {
  return Guard([&] {
    if (count < 0 || count > sdfgpu::KernelTimer::kClasses) {
      sdfgpu::Fail(SDFGPU_ERR_INVALID_ARGUMENT, "count is outside 0..SDFGPU_KERNEL_CLASSES");
    }
    const sdfgpu::KernelTimer& t = Eng(problem).kernel_timer();
    for (int c = 0; c < count; ++c) {
      if (ms != nullptr) {
        ms[c] = t.Ms(c);
      }
      if (launches != nullptr) {
        launches[c] = t.Launches(c);
      }
      if (work != nullptr) {
        work[c] = t.Work(c);
      }
    }
  });
}

const char* sdfgpu_kernel_class_name(int32_t kernel_class) { return sdfgpu::KernelTimer::Name(kernel_class); }

int32_t sdfgpu_kernel_class_is_memory_bound(int32_t kernel_class) {
  return sdfgpu::KernelTimer::ByteBound(kernel_class) ? 1 : 0;
}

int32_t sdfgpu_problem_count(const sdfgpu_problem* problem) {
  return problem == nullptr ? 0 : static_cast<int32_t>(problem->host.size());
}

int sdfgpu_problem_sizes(const sdfgpu_problem* problem, int32_t index, int32_t* sizes) {
  return Guard([&] {
    CheckIndex(problem, index);
    NeedHandle(sizes, "sizes");
    const sdfgpu::HostProblem& hp = problem->host[static_cast<size_t>(index)];
    sizes[0] = hp.num_points();
    sizes[1] = hp.num_eikonal();
    sizes[2] = hp.num_odom();
    sizes[3] = hp.num_active();
    sizes[4] = hp.num_params();
    sizes[5] = hp.num_rows();
    sizes[6] = hp.num_frames();
    sizes[7] = hp.nx;
    sizes[8] = hp.ny;
  });
}

int sdfgpu_problem_get_specs(const sdfgpu_problem* problem, int32_t index, int32_t* point_frame,
                             double* point_xy, double* point_expected, double* point_sqrt_weight,
                             int32_t* eikonal_wh, double* eikonal_normal, double* eikonal_sqrt_weight,
                             int32_t* odom_ij, double* odom_meas, double* odom_sqrt_weight,
                             int32_t* node_to_active) {
  return Guard([&] {
    CheckIndex(problem, index);
    const sdfgpu::HostProblem& hp = problem->host[static_cast<size_t>(index)];
    auto cp = [](auto* dst, const auto& v) {
      if (dst != nullptr && !v.empty()) {
        std::memcpy(dst, v.data(), v.size() * sizeof(v[0]));
      }
    };
    cp(point_frame, hp.pt_frame);
    cp(point_xy, hp.pt_xy);
    cp(point_expected, hp.pt_expected);
    cp(point_sqrt_weight, hp.pt_sqrtw);
    cp(eikonal_wh, hp.eik_wh);
    cp(eikonal_normal, hp.eik_n);
    cp(eikonal_sqrt_weight, hp.eik_sqrtw);
    cp(odom_ij, hp.odom_ij);
    cp(odom_meas, hp.odom_meas);
    cp(odom_sqrt_weight, hp.odom_sqrtw);
    cp(node_to_active, hp.node_to_active);
  });
}

int sdfgpu_get_state(sdfgpu_problem* problem, int32_t index, double* map_values, double* poses) {
  return Guard([&] {
    CheckIndex(problem, index);
    if (!problem->engine) {
      // not uploaded yet: the state is the host copy
      const sdfgpu::HostProblem& hp = problem->host[static_cast<size_t>(index)];
      if (map_values != nullptr) {
        std::memcpy(map_values, hp.map_values.data(), hp.map_values.size() * sizeof(double));
      }
      if (poses != nullptr) {
        std::memcpy(poses, hp.poses.data(), hp.poses.size() * sizeof(double));
      }
      return;
    }
    Eng(problem).GetState(index, map_values, poses);
  });
}

int sdfgpu_set_state(sdfgpu_problem* problem, int32_t index, const double* map_values, const double* poses) {
  return Guard([&] {
    CheckIndex(problem, index);
    if (!problem->engine) {
      sdfgpu::HostProblem& hp = problem->host[static_cast<size_t>(index)];
      if (map_values != nullptr) {
        std::memcpy(hp.map_values.data(), map_values, hp.map_values.size() * sizeof(double));
      }
      if (poses != nullptr) {
        std::memcpy(hp.poses.data(), poses, hp.poses.size() * sizeof(double));
      }
      return;
    }
    Eng(problem).SetState(index, map_values, poses);
  });
}

int sdfgpu_cost(sdfgpu_problem* problem, int32_t index, double* cost) {
  return Guard([&] {
    CheckIndex(problem, index);
    NeedHandle(cost, "cost");
    *cost = Eng(problem).Cost(index);
  });
}

int sdfgpu_apply_step(sdfgpu_problem* problem, int32_t index, const double* step) {
  return Guard([&] {
    CheckIndex(problem, index);
    NeedHandle(step, "step");
    Eng(problem).ApplyStep(index, step);
  });
}

static void CheckSolverOptions(const sdfgpu_solver_options& o) {
  if (o.max_iterations < 0 || !(o.lambda_init >= 0.0) || !(o.lambda_factor > 0.0)) {
    sdfgpu::Fail(SDFGPU_ERR_INVALID_ARGUMENT, "invalid solver options");
  }
  if (o.precision != SDFGPU_PRECISION_FP64 && o.precision != SDFGPU_PRECISION_MIXED) {
    sdfgpu::Fail(SDFGPU_ERR_INVALID_ARGUMENT, "unknown precision");
  }
  if (o.refine_steps < 0 || o.refine_steps > 16) {
    sdfgpu::Fail(SDFGPU_ERR_INVALID_ARGUMENT, "refine_steps must lie in [0, 16]");
  }
  if (!(o.refine_tolerance >= 0.0 && o.refine_tolerance < 1.0)) {
    sdfgpu::Fail(SDFGPU_ERR_INVALID_ARGUMENT, "refine_tolerance must lie in [0, 1)");
  }
}

int sdfgpu_solve(sdfgpu_problem* problem, const sdfgpu_solver_options* options, sdfgpu_solve_result* results,
                 double* cost_history, int32_t capacity) {
  int first_status = SDFGPU_OK;
  const int rc = Guard([&] {
    sdfgpu::Engine& e = Eng(problem);
    NeedHandle(results, "results");
    sdfgpu_solver_options def;
    sdfgpu_solver_options_default(&def);
    std::vector<sdfgpu_solver_options> opts(static_cast<size_t>(e.count()), def);
    if (options != nullptr) {
      opts.assign(options, options + e.count());
    }
    for (const auto& o : opts) {
      CheckSolverOptions(o);
    }
    e.Solve(opts, results, cost_history, capacity > 0 ? capacity : 0);
    for (int i = 0; i < e.count(); ++i) {
      if (results[i].status != SDFGPU_OK && first_status == SDFGPU_OK) {
        first_status = results[i].status;
      }
    }
  });
  if (rc != SDFGPU_OK) {
    return rc;
  }
  if (first_status == SDFGPU_ERR_NUMERICAL) {
    g_last_error = "sparse Cholesky factorization failed";
  }
  return first_status;
}

int sdfgpu_run_incremental(const sdfgpu_incremental_desc* desc, const sdfgpu_problem_options* problem_options,
                           const sdfgpu_solver_options* solver_options, double* map_out, double* poses_out,
                           sdfgpu_solve_result* total, double* cost_history, int32_t capacity, double* phases) {
  return Guard([&] {
    NeedHandle(desc, "desc");
    NeedHandle(map_out, "map_out");
    NeedHandle(poses_out, "poses_out");
    NeedHandle(total, "total");
    sdfgpu_problem_options po;
    if (problem_options != nullptr) {
      po = *problem_options;
    } else {
      sdfgpu_problem_options_default(&po);
    }
    sdfgpu_solver_options so;
    if (solver_options != nullptr) {
      so = *solver_options;
    } else {
      sdfgpu_solver_options_default(&so);
    }
    CheckSolverOptions(so);
    sdfgpu::IncrementalInput in;
    in.nx = desc->nx;
    in.ny = desc->ny;
    in.min_x = desc->min_x;
    in.min_y = desc->min_y;
    in.max_x = desc->max_x;
    in.max_y = desc->max_y;
    in.map_values = desc->map_values;
    in.num_frames = desc->num_frames;
    in.poses = desc->poses;
    in.scan_offsets = desc->scan_offsets;
    in.scan_xy = desc->scan_xy;
    in.num_relations = desc->num_relations;
    in.relation_ij = desc->relation_ij;
    in.relation_meas = desc->relation_meas;
    in.relation_sqrt_weight = desc->relation_sqrt_weight;
    in.increment_size = desc->increment_size;
    in.iterations_per_increment = desc->iterations_per_increment;
    in.snapshot_every = desc->snapshot_every;
    in.snapshot = desc->snapshot;
    in.snapshot_user = desc->snapshot_user;
    in.build_on_device = desc->build_on_device;
    in.warm_analysis = desc->warm_analysis;
    if (in.nx < 2 || in.ny < 2) {
      sdfgpu::Fail(SDFGPU_ERR_INVALID_ARGUMENT, "GridMap needs nx, ny >= 2 and max > min");
    }
    sdfgpu::IncrementalOutput out;
    sdfgpu::RunIncremental(in, po, so, &out);
    std::copy(out.map.begin(), out.map.end(), map_out);
    std::copy(out.poses.begin(), out.poses.end(), poses_out);
    *total = out.total;
    const size_t n = std::min(out.cost_history.size(), static_cast<size_t>(std::max(0, capacity)));
    if (cost_history != nullptr) {
      std::copy(out.cost_history.begin(), out.cost_history.begin() + static_cast<std::ptrdiff_t>(n), cost_history);
      total->cost_history_length = static_cast<int32_t>(n);
    } else {
      total->cost_history_length = 0;
    }
    total->status = SDFGPU_OK;
    if (phases != nullptr) {
      const sdfgpu::IncrementalPhases& p = out.phases;
      const double v[12] = {p.build,    p.wait_analysis, p.setup, p.solve, p.readback, p.teardown, p.wall,
                            static_cast<double>(p.increments), static_cast<double>(p.warm_analyses),
                            static_cast<double>(p.reanalyses), p.reanalysis, p.capture};
      std::copy(v, v + 12, phases);
    }
  });
}

static void CheckGrid(int32_t nx, int32_t ny, double min_x, double min_y, double max_x, double max_y) {
  if (nx < 2 || ny < 2 || !(max_x > min_x) || !(max_y > min_y)) {
    sdfgpu::Fail(SDFGPU_ERR_INVALID_ARGUMENT, "GridMap needs nx, ny >= 2 and max > min");
  }
}

static void CheckScans(int32_t num_frames, const double* poses, const int32_t* scan_offsets,
                       const double* scan_xy) {
  if (num_frames < 0 || (num_frames > 0 && (poses == nullptr || scan_offsets == nullptr))) {
    sdfgpu::Fail(SDFGPU_ERR_INVALID_ARGUMENT, "poses and scans are required");
  }
  for (int32_t f = 0; f < num_frames; ++f) {
    if (scan_offsets[f + 1] < scan_offsets[f]) {
      sdfgpu::Fail(SDFGPU_ERR_INVALID_ARGUMENT, "scan offsets must not decrease");
    }
  }
  if (num_frames > 0 && scan_offsets[0] != 0) {
    sdfgpu::Fail(SDFGPU_ERR_INVALID_ARGUMENT, "scan offsets must start at 0");
  }
  if (num_frames > 0 && scan_offsets[num_frames] > 0 && scan_xy == nullptr) {
    sdfgpu::Fail(SDFGPU_ERR_INVALID_ARGUMENT, "scan points missing");
  }
}

int sdfgpu_write_poses(const char* path, const double* poses, int32_t num_frames) {
  return Guard([&] {
    if (num_frames < 0 || (num_frames > 0 && poses == nullptr)) {
      sdfgpu::Fail(SDFGPU_ERR_INVALID_ARGUMENT, "poses missing");
    }
    sdfgpu::WritePoses(path, poses, num_frames);
  });
}

int sdfgpu_write_map(const char* path, int32_t nx, int32_t ny, double min_x, double min_y, double max_x,
                     double max_y, const double* map_values) {
  return Guard([&] {
    CheckGrid(nx, ny, min_x, min_y, max_x, max_y);
    NeedHandle(map_values, "map_values");
    sdfgpu::WriteMap(path, nx, ny, min_x, min_y, max_x, max_y, map_values);
  });
}

int sdfgpu_write_scan_points(const char* path, int32_t num_frames, const double* poses,
                             const int32_t* scan_offsets, const double* scan_xy) {
  return Guard([&] {
    CheckScans(num_frames, poses, scan_offsets, scan_xy);
    sdfgpu::WriteScanPoints(path, num_frames, poses, scan_offsets, scan_xy);
  });
}

int sdfgpu_write_metrics(const char* path, const sdfgpu_solve_result* result, const double* metrics) {
  return Guard([&] {
    NeedHandle(result, "result");
    sdfgpu::WriteMetrics(path, *result, metrics);
  });
}

int sdfgpu_evaluate_trajectory(const double* estimated, const double* ground_truth, int32_t num_frames,
                               double* metrics) {
  return Guard([&] {
    NeedHandle(estimated, "estimated");
    NeedHandle(ground_truth, "ground_truth");
    NeedHandle(metrics, "metrics");
    sdfgpu::EvaluateTrajectory(estimated, ground_truth, num_frames, metrics);
  });
}

int sdfgpu_points_outside_map(int32_t nx, int32_t ny, double min_x, double min_y, double max_x, double max_y,
                              int32_t num_frames, const double* poses, const int32_t* scan_offsets,
                              const double* scan_xy, int64_t* outside, int64_t* total) {
  return Guard([&] {
    CheckGrid(nx, ny, min_x, min_y, max_x, max_y);
    CheckScans(num_frames, poses, scan_offsets, scan_xy);
    NeedHandle(outside, "outside");
    NeedHandle(total, "total");
    sdfgpu::PointsOutsideMap(nx, ny, min_x, min_y, max_x, max_y, num_frames, poses, scan_offsets, scan_xy,
                             outside, total);
  });
}

int sdfgpu_linearize(sdfgpu_problem* problem, int32_t index, double lambda, int32_t marquardt,
                     int32_t compute_step) {
  return Guard([&] {
    CheckIndex(problem, index);
    Eng(problem).Linearize(index, lambda, marquardt != 0, compute_step != 0);
  });
}

int sdfgpu_linearization_sizes(sdfgpu_problem* problem, int64_t* sizes) {
  return Guard([&] {
    NeedHandle(sizes, "sizes");
    Eng(problem).LinearizationSizes(sizes);
  });
}

int sdfgpu_linearization_get(sdfgpu_problem* problem, double* residuals, int32_t* point_cell, int32_t* j_outer,
                             int32_t* j_inner, double* j_values, int32_t* n_outer, int32_t* n_inner,
                             double* n_values, double* rhs, double* step) {
  return Guard([&] {
    Eng(problem).LinearizationGet(residuals, point_cell, j_outer, j_inner, j_values, n_outer, n_inner, n_values,
                                  rhs, step);
  });
}

int sdfgpu_last_profile(sdfgpu_problem* problem, double* phases) {
  return Guard([&] {
    NeedHandle(phases, "phases");
    const sdfgpu::IterTimes& t = Eng(problem).times();
    phases[0] = t.assemble;
    phases[1] = t.normal;
    phases[2] = t.factor;
    phases[3] = t.solve;
    phases[4] = t.update;
    phases[5] = t.iterations;
    phases[6] = t.span;
    phases[7] = static_cast<double>(t.launches);
    phases[8] = static_cast<double>(Eng(problem).factor_flops()) * 2.0;
    phases[9] = static_cast<double>(t.reanalyses);
    phases[10] = t.reanalysis_host;
    phases[11] = t.capture_host;
  });
}

int sdfgpu_autotune(sdfgpu_problem* problem, int32_t* schedule, double* factor_ms, double* trials,
                    int32_t max_trials, int32_t* num_trials) {
  return Guard([&] {
    std::vector<std::pair<sdfgpu::Schedule, double>> t;
    const double best = Eng(problem).Autotune(&t);
    const sdfgpu::Schedule& s = Eng(problem).schedule();
    if (schedule != nullptr) {
      schedule[0] = s.small_pivots;
      schedule[1] = s.front_rows;
      schedule[2] = s.panel_rows;
    }
    if (factor_ms != nullptr) {
      *factor_ms = best;
    }
    if (trials != nullptr) {
      for (size_t q = 0; q < t.size() && static_cast<int32_t>(q) < max_trials; ++q) {
        trials[4 * q] = t[q].first.small_pivots;
        trials[4 * q + 1] = t[q].first.front_rows;
        trials[4 * q + 2] = t[q].first.panel_rows;
        trials[4 * q + 3] = t[q].second;
      }
    }
    if (num_trials != nullptr) {
      *num_trials = static_cast<int32_t>(t.size());
    }
  });
}

int sdfgpu_set_schedule(sdfgpu_problem* problem, const int32_t* schedule) {
  return Guard([&] {
    if (schedule == nullptr) {
      sdfgpu::Fail(SDFGPU_ERR_INVALID_ARGUMENT, "schedule is NULL");
    }
    // the tensor-core choice of mixed solves stays as it is
    sdfgpu::Schedule s = Eng(problem).schedule();
    s.small_pivots = schedule[0];
    s.front_rows = schedule[1];
    s.panel_rows = schedule[2];
    Eng(problem).SetSchedule(s);
  });
}

int sdfgpu_tensor_core_choice(sdfgpu_problem* problem, int32_t* min_rows, double* ms_with, double* ms_without) {
  return Guard([&] {
    NeedHandle(min_rows, "min_rows");
    *min_rows = Eng(problem).schedule().tc_min_rows;
    if (ms_with != nullptr) {
      *ms_with = Eng(problem).tc_trial_ms(true);
    }
    if (ms_without != nullptr) {
      *ms_without = Eng(problem).tc_trial_ms(false);
    }
  });
}

int sdfgpu_set_tensor_core_choice(sdfgpu_problem* problem, int32_t min_rows) {
  return Guard([&] {
    if (min_rows != 0 && (min_rows < 128 || min_rows > 65536)) {
      sdfgpu::Fail(SDFGPU_ERR_INVALID_ARGUMENT, "min_rows must be 0 or lie in [128, 65536]");
    }
    sdfgpu::Schedule s = Eng(problem).schedule();
    s.tc_min_rows = min_rows;
    Eng(problem).SetSchedule(s);
  });
}

int sdfgpu_ldlt_create(int32_t n, const int32_t* outer, const int32_t* inner, const int32_t* perm,
                       sdfgpu_ldlt** out) {
  return Guard([&] {
    NeedHandle(out, "out");
    *out = nullptr;
    if (n < 1 || outer == nullptr || inner == nullptr) {
      sdfgpu::Fail(SDFGPU_ERR_INVALID_ARGUMENT, "ldlt needs n >= 1 and a CSC pattern");
    }
    auto h = std::make_unique<sdfgpu_ldlt>();
    h->engine = std::make_unique<sdfgpu::LdltEngine>(n, outer, inner, perm);
    *out = h.release();
  });
}

int sdfgpu_ldlt_factorize(sdfgpu_ldlt* ldlt, const double* values) {
  return Guard([&] {
    NeedHandle(ldlt, "ldlt");
    NeedHandle(values, "values");
    ldlt->engine->Factorize(values);
  });
}

int sdfgpu_ldlt_solve(sdfgpu_ldlt* ldlt, const double* b, double* x) {
  return Guard([&] {
    NeedHandle(ldlt, "ldlt");
    NeedHandle(b, "b");
    NeedHandle(x, "x");
    ldlt->engine->Solve(b, x);
  });
}

int sdfgpu_ldlt_destroy(sdfgpu_ldlt* ldlt) {
  return Guard([&] { delete ldlt; });
}

int sdfgpu_server_create(int64_t memory_budget_bytes, int32_t max_batch, sdfgpu_server** out) {
  return Guard([&] {
    NeedHandle(out, "out");
    *out = nullptr;
    if (memory_budget_bytes <= 0 || max_batch < 1) {
      sdfgpu::Fail(SDFGPU_ERR_INVALID_ARGUMENT, "server needs a positive budget and batch size");
    }
    auto h = std::make_unique<sdfgpu_server>();
    h->server = std::make_unique<sdfgpu::Server>(memory_budget_bytes, max_batch);
    *out = h.release();
  });
}

int sdfgpu_server_submit(sdfgpu_server* server, const sdfgpu_problem_desc* desc,
                         const sdfgpu_solver_options* options, int64_t* request_id) {
  return Guard([&] {
    NeedHandle(server, "server");
    NeedHandle(desc, "desc");
    NeedHandle(request_id, "request_id");
    sdfgpu_solver_options o;
    sdfgpu_solver_options_default(&o);
    if (options != nullptr) {
      o = *options;
    }
    *request_id = server->server->Submit(sdfgpu::FromDesc(*desc), o);
  });
}

int sdfgpu_server_poll(sdfgpu_server* server, int64_t request_id, sdfgpu_solve_result* result,
                       double* map_values, double* poses) {
  return Guard([&] {
    NeedHandle(server, "server");
    server->server->Poll(request_id, result, map_values, poses);
  });
}

int sdfgpu_server_cancel(sdfgpu_server* server, int64_t request_id) {
  return Guard([&] {
    NeedHandle(server, "server");
    server->server->Cancel(request_id);
  });
}

int sdfgpu_server_stats(sdfgpu_server* server, double* stats) {
  return Guard([&] {
    NeedHandle(server, "server");
    NeedHandle(stats, "stats");
    server->server->Stats(stats);
  });
}

int sdfgpu_server_drain(sdfgpu_server* server, int64_t timeout_ms) {
  return Guard([&] {
    NeedHandle(server, "server");
    server->server->Drain(timeout_ms);
  });
}

int sdfgpu_server_destroy(sdfgpu_server* server) {
  return Guard([&] { delete server; });
}

int sdfgpu_dense_ldlt_solve_noalloc(int32_t n, const double* a, const double* b, double* x) {
  return Guard([&] { sdfgpu::DenseLdltSolveNoAlloc(n, a, b, x); });
}

}  // extern "C"
