// C entry points of the CPU oracle, loaded by oracle/oracle.py through ctypes.
// TEST INFRASTRUCTURE ONLY (see oracle.hpp).
#include <cstdint>
#include <cstring>
#include <exception>
#include <random>
#include <string>

#include "oracle.hpp"

using namespace oracle;

namespace {

void SetError(char* err, int len, const char* msg) {
  if (err != nullptr && len > 0) {
    std::strncpy(err, msg, static_cast<size_t>(len) - 1);
    err[len - 1] = '\0';
  }
}

GridMap MakeMap(int nx, int ny, double min_x, double min_y, double max_x, double max_y,
                const double* values) {
  GridMap map(nx, ny, {min_x, min_y}, {max_x, max_y}, 0.0);
  if (values != nullptr) {
    for (int i = 0; i < nx * ny; ++i) {
      map.values()[static_cast<size_t>(i)] = values[i];
    }
  }
  return map;
}

std::vector<Pose2> MakePoses(int n, const double* p) {
  std::vector<Pose2> poses(static_cast<size_t>(n));
  for (int i = 0; i < n; ++i) {
    poses[static_cast<size_t>(i)] = {p[3 * i], p[3 * i + 1], p[3 * i + 2]};
  }
  return poses;
}

struct LinHandle {
  Linearization lin;
};

}  // namespace

extern "C" {

// opts_d: weights scan, hallucination, eikonal, odometry, relation;
//         hallucination step_size; huber_delta; smooth_gradient_step;
//         normals corner_threshold.
// opts_i: points_per_scan_point, both_directions, normals method, k_neighbors,
//         per_scan, smooth_gradient, active_region, active_margin.
void* oracle_problem_build(int nx, int ny, double min_x, double min_y, double max_x, double max_y,
                           const double* map_values, int num_frames, const double* poses,
                           const int* scan_offsets, const double* scan_xy,
                           const double* odometry, int num_odometry, int num_relations,
                           const int* rel_ij, const double* rel_meas, const double* rel_w,
                           const double* opts_d, const int* opts_i, char* err, int errlen) {
  try {
    ProblemOptions o;
    o.weights = {opts_d[0], opts_d[1], opts_d[2], opts_d[3], opts_d[4]};
    o.hallucination.step_size = opts_d[5];
    o.huber_delta = opts_d[6];
    o.smooth_gradient_step = opts_d[7];
    o.normals.corner_threshold = opts_d[8];
    o.hallucination.points_per_scan_point = opts_i[0];
    o.hallucination.both_directions = opts_i[1] != 0;
    o.normals.method = static_cast<NormalMethod>(opts_i[2]);
    o.normals.k_neighbors = opts_i[3];
    o.normals.per_scan = opts_i[4] != 0;
    o.smooth_gradient = opts_i[5] != 0;
    o.active_region = opts_i[6] != 0;
    o.active_margin = opts_i[7];
    std::vector<std::vector<Vec2>> scans(static_cast<size_t>(num_frames));
    for (int f = 0; f < num_frames; ++f) {
      for (int q = scan_offsets[f]; q < scan_offsets[f + 1]; ++q) {
        scans[static_cast<size_t>(f)].push_back({scan_xy[2 * q], scan_xy[2 * q + 1]});
      }
    }
    std::vector<Pose2> odo = MakePoses(num_odometry, odometry);
    std::vector<RelationMeasurement> rels(static_cast<size_t>(num_relations));
    for (int r = 0; r < num_relations; ++r) {
      rels[static_cast<size_t>(r)] = {rel_ij[2 * r], rel_ij[2 * r + 1],
                                      {rel_meas[3 * r], rel_meas[3 * r + 1], rel_meas[3 * r + 2]},
                                      rel_w[r]};
    }
    return new Problem(MakeMap(nx, ny, min_x, min_y, max_x, max_y, map_values),
                       MakePoses(num_frames, poses), scans, odo, o, rels);
  } catch (const std::exception& e) {
    SetError(err, errlen, e.what());
    return nullptr;
  }
}

void* oracle_problem_from_specs(int nx, int ny, double min_x, double min_y, double max_x,
                                double max_y, const double* map_values, int num_frames,
                                const double* poses, int num_points, const int* pt_frame,
                                const double* pt_xy, const double* pt_expected,
                                const double* pt_sqrtw, int num_eik, const int* eik_wh,
                                const double* eik_n, const double* eik_sqrtw, int num_odom,
                                const int* odom_ij, const double* odom_meas,
                                const double* odom_sqrtw, const int* node_to_active,
                                double huber_delta, int smooth_gradient,
                                double smooth_gradient_step, char* err, int errlen) {
  try {
    std::vector<PointSpec> pts(static_cast<size_t>(num_points));
    for (int i = 0; i < num_points; ++i) {
      pts[static_cast<size_t>(i)] = {pt_frame[i], {pt_xy[2 * i], pt_xy[2 * i + 1]}, pt_expected[i], pt_sqrtw[i]};
    }
    std::vector<EikonalSpec> eik(static_cast<size_t>(num_eik));
    for (int i = 0; i < num_eik; ++i) {
      eik[static_cast<size_t>(i)] = {eik_wh[2 * i], eik_wh[2 * i + 1], {eik_n[2 * i], eik_n[2 * i + 1]}, eik_sqrtw[i]};
    }
    std::vector<OdomSpec> odo(static_cast<size_t>(num_odom));
    for (int i = 0; i < num_odom; ++i) {
      odo[static_cast<size_t>(i)] = {odom_ij[2 * i], odom_ij[2 * i + 1],
                                     {odom_meas[3 * i], odom_meas[3 * i + 1], odom_meas[3 * i + 2]},
                                     odom_sqrtw[i]};
    }
    std::vector<int> n2a(node_to_active, node_to_active + static_cast<size_t>(nx) * static_cast<size_t>(ny));
    return new Problem(Problem::FromSpecs(MakeMap(nx, ny, min_x, min_y, max_x, max_y, map_values),
                                          MakePoses(num_frames, poses), std::move(pts), std::move(eik),
                                          std::move(odo), std::move(n2a), huber_delta,
                                          smooth_gradient != 0, smooth_gradient_step));
  } catch (const std::exception& e) {
    SetError(err, errlen, e.what());
    return nullptr;
  }
}

void oracle_problem_free(void* p) { delete static_cast<Problem*>(p); }

// out: num_points, num_eik, num_odom, num_active, num_params, num_residuals,
//      num_frames, nx, ny
void oracle_problem_sizes(void* h, int* out) {
  const Problem& p = *static_cast<Problem*>(h);
  out[0] = static_cast<int>(p.point_specs().size());
  out[1] = static_cast<int>(p.eikonal_specs().size());
  out[2] = static_cast<int>(p.odom_specs().size());
  out[3] = p.num_active_nodes();
  out[4] = p.num_parameters();
  out[5] = p.num_residuals();
  out[6] = static_cast<int>(p.poses().size());
  out[7] = p.map().nx();
  out[8] = p.map().ny();
}

void oracle_problem_get_specs(void* h, int* pt_frame, double* pt_xy, double* pt_expected,
                              double* pt_sqrtw, int* eik_wh, double* eik_n, double* eik_sqrtw,
                              int* odom_ij, double* odom_meas, double* odom_sqrtw,
                              int* node_to_active) {
  const Problem& p = *static_cast<Problem*>(h);
  for (size_t i = 0; i < p.point_specs().size(); ++i) {
    const PointSpec& s = p.point_specs()[i];
    pt_frame[i] = s.frame;
    pt_xy[2 * i] = s.point_sensor.x;
    pt_xy[2 * i + 1] = s.point_sensor.y;
    pt_expected[i] = s.expected_sdf;
    pt_sqrtw[i] = s.sqrt_weight;
  }
  for (size_t i = 0; i < p.eikonal_specs().size(); ++i) {
    const EikonalSpec& s = p.eikonal_specs()[i];
    eik_wh[2 * i] = s.w;
    eik_wh[2 * i + 1] = s.h;
    eik_n[2 * i] = s.normal.x;
    eik_n[2 * i + 1] = s.normal.y;
    eik_sqrtw[i] = s.sqrt_weight;
  }
  for (size_t i = 0; i < p.odom_specs().size(); ++i) {
    const OdomSpec& s = p.odom_specs()[i];
    odom_ij[2 * i] = s.frame_i;
    odom_ij[2 * i + 1] = s.frame_j;
    odom_meas[3 * i] = s.measurement.x;
    odom_meas[3 * i + 1] = s.measurement.y;
    odom_meas[3 * i + 2] = s.measurement.theta;
    odom_sqrtw[i] = s.sqrt_weight;
  }
  for (size_t i = 0; i < p.node_to_active().size(); ++i) {
    node_to_active[i] = p.node_to_active()[i];
  }
}

void oracle_problem_get_state(void* h, double* map_values, double* poses) {
  const Problem& p = *static_cast<Problem*>(h);
  std::memcpy(map_values, p.map().values().data(), p.map().values().size() * sizeof(double));
  for (size_t i = 0; i < p.poses().size(); ++i) {
    poses[3 * i] = p.poses()[i].x;
    poses[3 * i + 1] = p.poses()[i].y;
    poses[3 * i + 2] = p.poses()[i].theta;
  }
}

void oracle_problem_set_state(void* h, const double* map_values, const double* poses) {
  Problem& p = *static_cast<Problem*>(h);
  std::memcpy(p.map().values().data(), map_values, p.map().values().size() * sizeof(double));
  for (size_t i = 0; i < p.poses().size(); ++i) {
    p.poses()[i] = {poses[3 * i], poses[3 * i + 1], poses[3 * i + 2]};
  }
}

double oracle_problem_cost(void* h) { return static_cast<Problem*>(h)->Cost(); }

int oracle_problem_apply_step(void* h, const double* step) {
  Problem& p = *static_cast<Problem*>(h);
  p.ApplyStep(std::vector<double>(step, step + p.num_parameters()));
  return 0;
}

int oracle_nd_ordering(void* h, int* perm) {
  const std::vector<int> order = GridNestedDissection(*static_cast<Problem*>(h));
  std::memcpy(perm, order.data(), order.size() * sizeof(int));
  return static_cast<int>(order.size());
}

void* oracle_linearize(void* h, double lambda, int marquardt, int num_threads, int compute_step) {
  auto* out = new LinHandle;
  out->lin = Linearize(*static_cast<Problem*>(h), lambda, marquardt != 0, num_threads, compute_step != 0);
  return out;
}

// out: num_rows, num_params, nnz(J), nnz(normal), factor_ok, nnz(L), has_step
void oracle_lin_sizes(void* h, int64_t* out) {
  const Linearization& l = static_cast<LinHandle*>(h)->lin;
  out[0] = l.jacobian.rows;
  out[1] = l.jacobian.cols;
  out[2] = static_cast<int64_t>(l.jacobian.inner.size());
  out[3] = static_cast<int64_t>(l.normal.inner.size());
  out[4] = l.factor_ok ? 1 : 0;
  out[5] = l.nnz_l;
  out[6] = l.step.empty() ? 0 : 1;
}

void oracle_lin_get(void* h, double* residuals, int* point_cell, int* j_outer, int* j_inner,
                    double* j_values, int* n_outer, int* n_inner, double* n_values, double* rhs,
                    double* step) {
  const Linearization& l = static_cast<LinHandle*>(h)->lin;
  std::memcpy(residuals, l.residuals.data(), l.residuals.size() * sizeof(double));
  std::memcpy(point_cell, l.point_cell.data(), l.point_cell.size() * sizeof(int));
  std::memcpy(j_outer, l.jacobian.outer.data(), l.jacobian.outer.size() * sizeof(int));
  std::memcpy(j_inner, l.jacobian.inner.data(), l.jacobian.inner.size() * sizeof(int));
  std::memcpy(j_values, l.jacobian.values.data(), l.jacobian.values.size() * sizeof(double));
  std::memcpy(n_outer, l.normal.outer.data(), l.normal.outer.size() * sizeof(int));
  std::memcpy(n_inner, l.normal.inner.data(), l.normal.inner.size() * sizeof(int));
  std::memcpy(n_values, l.normal.values.data(), l.normal.values.size() * sizeof(double));
  std::memcpy(rhs, l.rhs.data(), l.rhs.size() * sizeof(double));
  if (!l.step.empty() && step != nullptr) {
    std::memcpy(step, l.step.data(), l.step.size() * sizeof(double));
  }
}

void oracle_lin_free(void* h) { delete static_cast<LinHandle*>(h); }

// opts_d: step_tolerance, lambda_init, lambda_factor
// opts_i: max_iterations, reject_worse_steps, marquardt_scaling, trust_region,
//         num_threads
// result_d: initial_cost, final_cost, duration_seconds, phase seconds x5
// result_i: converged, iterations, cost_history length
int oracle_solve(void* h, const double* opts_d, const int* opts_i, double* result_d, int* result_i,
                 double* cost_history, int cap, char* err, int errlen) {
  try {
    SolverOptions o;
    o.step_tolerance = opts_d[0];
    o.lambda_init = opts_d[1];
    o.lambda_factor = opts_d[2];
    o.max_iterations = opts_i[0];
    o.reject_worse_steps = opts_i[1] != 0;
    o.marquardt_scaling = opts_i[2] != 0;
    o.trust_region = opts_i[3] != 0;
    o.num_threads = opts_i[4];
    const SolveResult r = SolveLm(*static_cast<Problem*>(h), o);
    result_d[0] = r.initial_cost;
    result_d[1] = r.final_cost;
    result_d[2] = r.duration_seconds;
    for (int i = 0; i < 5; ++i) {
      result_d[3 + i] = r.phase_seconds[static_cast<size_t>(i)];
    }
    result_i[0] = r.converged ? 1 : 0;
    result_i[1] = r.iterations;
    result_i[2] = static_cast<int>(r.cost_history.size());
    for (int i = 0; i < cap && i < static_cast<int>(r.cost_history.size()); ++i) {
      cost_history[i] = r.cost_history[static_cast<size_t>(i)];
    }
    return 0;
  } catch (const std::exception& e) {
    SetError(err, errlen, e.what());
    return 1;
  }
}

// Factor-only path (parallel_ldlt.hpp:38-51 + Eigen solve). Returns 0 on
// success, 1 on a zero pivot (Eigen::NumericalIssue).
int oracle_ldlt_solve(int n, const int* outer, const int* inner, const double* values,
                      const int* perm, int num_threads, const double* b, double* x,
                      double* diag_out) {
  Csc a;
  a.rows = a.cols = n;
  a.outer.assign(outer, outer + n + 1);
  a.inner.assign(inner, inner + outer[n]);
  a.values.assign(values, values + outer[n]);
  std::vector<int> p;
  if (perm != nullptr) {
    p.assign(perm, perm + n);
  }
  Ldlt ldlt;
  ldlt.Analyze(a, p, num_threads);
  if (!ldlt.Factorize(a)) {
    return 1;
  }
  const std::vector<double> sol = ldlt.Solve(std::vector<double>(b, b + n));
  std::memcpy(x, sol.data(), sol.size() * sizeof(double));
  if (diag_out != nullptr) {
    std::memcpy(diag_out, ldlt.diag().data(), ldlt.diag().size() * sizeof(double));
  }
  return 0;
}

// ---------------------------------------------------- known-answer probes --

// Returns 1 when p lies in the domain. cell_wh[2], ab[2], value, grad[2].
int oracle_locate(int nx, int ny, double min_x, double min_y, double max_x, double max_y,
                  const double* values, double px, double py, int* cell_wh, double* ab,
                  double* value, double* grad) {
  const GridMap map = MakeMap(nx, ny, min_x, min_y, max_x, max_y, values);
  GridMap::CellRef cell;
  if (!map.Locate({px, py}, cell)) {
    return 0;
  }
  cell_wh[0] = cell.w;
  cell_wh[1] = cell.h;
  ab[0] = cell.alpha;
  ab[1] = cell.beta;
  *value = map.Interpolate(cell);
  const Vec2 g = map.Gradient(cell);
  grad[0] = g.x;
  grad[1] = g.y;
  return 1;
}

// out_d: residual, d_nodes[4], d_pose[3]; out_i: valid, node ids[4]
void oracle_eval_point(int nx, int ny, double min_x, double min_y, double max_x, double max_y,
                       const double* values, const double* pose, double px, double py, double delta,
                       int smooth, double smooth_step, double* out_d, int* out_i) {
  const GridMap map = MakeMap(nx, ny, min_x, min_y, max_x, max_y, values);
  const PointResidualJacobian r =
      EvalPointResidual(map, {pose[0], pose[1], pose[2]}, {px, py}, delta, smooth != 0, smooth_step);
  out_d[0] = r.residual;
  for (int i = 0; i < 4; ++i) {
    out_d[1 + i] = r.d_nodes[static_cast<size_t>(i)];
    out_i[1 + i] = r.node_ids[static_cast<size_t>(i)];
  }
  for (int i = 0; i < 3; ++i) {
    out_d[5 + i] = r.d_pose[static_cast<size_t>(i)];
  }
  out_i[0] = r.valid ? 1 : 0;
}

// out: residual[3], d_pose_i[9], d_pose_j[9] (row-major)
void oracle_eval_odom(const double* pi, const double* pj, const double* meas, double* out) {
  const OdomResidualJacobian r = EvalOdomResidual({pi[0], pi[1], pi[2]}, {pj[0], pj[1], pj[2]},
                                                  {meas[0], meas[1], meas[2]});
  for (int i = 0; i < 3; ++i) {
    out[i] = r.residual[static_cast<size_t>(i)];
    for (int c = 0; c < 3; ++c) {
      out[3 + 3 * i + c] = r.d_pose_i[static_cast<size_t>(i)][static_cast<size_t>(c)];
      out[12 + 3 * i + c] = r.d_pose_j[static_cast<size_t>(i)][static_cast<size_t>(c)];
    }
  }
}

// out: residual, d_nodes[3]; ids[3]
void oracle_eval_eikonal(int nx, int ny, double min_x, double min_y, double max_x, double max_y,
                         const double* values, int w, int h, double nxv, double nyv, double* out,
                         int* ids) {
  const GridMap map = MakeMap(nx, ny, min_x, min_y, max_x, max_y, values);
  const EikonalResidualJacobian r = EvalEikonalResidual(map, w, h, {nxv, nyv});
  out[0] = r.residual;
  for (int i = 0; i < 3; ++i) {
    out[1 + i] = r.d_nodes[static_cast<size_t>(i)];
    ids[i] = r.node_ids[static_cast<size_t>(i)];
  }
}

int oracle_hallucinate(const double* pts, int n, int per_point, double step, int both,
                       double* out_xy, double* out_expected) {
  std::vector<Vec2> scan(static_cast<size_t>(n));
  for (int i = 0; i < n; ++i) {
    scan[static_cast<size_t>(i)] = {pts[2 * i], pts[2 * i + 1]};
  }
  HallucinationOptions o;
  o.points_per_scan_point = per_point;
  o.step_size = step;
  o.both_directions = both != 0;
  const auto out = GenerateHallucinatedPoints(scan, o);
  for (size_t i = 0; i < out.size(); ++i) {
    if (out_xy != nullptr) {
      out_xy[2 * i] = out[i].point_sensor.x;
      out_xy[2 * i + 1] = out[i].point_sensor.y;
      out_expected[i] = out[i].expected_sdf;
    }
  }
  return static_cast<int>(out.size());
}

// mode 0: apply(p) -> out[0..1]; 1: compose(b) -> out[0..2];
// 2: relative_to(b) -> out[0..2]; 3: wrap(a[0]) -> out[0]
void oracle_pose_op(int mode, const double* a, const double* b, double* out) {
  const Pose2 pa{a[0], a[1], a[2]};
  if (mode == 0) {
    const Vec2 r = pa.Apply({b[0], b[1]});
    out[0] = r.x;
    out[1] = r.y;
  } else if (mode == 1 || mode == 2) {
    const Pose2 pb{b[0], b[1], b[2]};
    const Pose2 r = mode == 1 ? pa.Compose(pb) : pa.RelativeTo(pb);
    out[0] = r.x;
    out[1] = r.y;
    out[2] = r.theta;
  } else {
    out[0] = WrapAngle(a[0]);
  }
}

// out per scan point: normal x, y, cornerness. Node normals: nx*ny x
// (normal x, normal y, eikonal_scale).
void oracle_normals(int num_frames, const double* poses, const int* scan_offsets,
                    const double* scan_xy, int k, int per_scan, double* out_points,
                    int nx, int ny, double min_x, double min_y, double max_x, double max_y,
                    int method, double corner_threshold, double* out_nodes) {
  std::vector<std::vector<Vec2>> scans(static_cast<size_t>(num_frames));
  for (int f = 0; f < num_frames; ++f) {
    for (int q = scan_offsets[f]; q < scan_offsets[f + 1]; ++q) {
      scans[static_cast<size_t>(f)].push_back({scan_xy[2 * q], scan_xy[2 * q + 1]});
    }
  }
  const ScanNormals sn = ComputeScanNormals(scans, MakePoses(num_frames, poses), k, per_scan != 0);
  for (size_t i = 0; i < sn.points.size(); ++i) {
    out_points[3 * i] = sn.normals[i].x;
    out_points[3 * i + 1] = sn.normals[i].y;
    out_points[3 * i + 2] = sn.cornerness[i];
  }
  if (out_nodes != nullptr) {
    const GridMap map = MakeMap(nx, ny, min_x, min_y, max_x, max_y, nullptr);
    NormalOptions o;
    o.method = static_cast<NormalMethod>(method);
    o.k_neighbors = k;
    o.corner_threshold = corner_threshold;
    const auto nodes = AssignNodeNormals(map, sn, o);
    for (size_t i = 0; i < nodes.size(); ++i) {
      out_nodes[3 * i] = nodes[i].normal.x;
      out_nodes[3 * i + 1] = nodes[i].normal.y;
      out_nodes[3 * i + 2] = nodes[i].eikonal_scale;
    }
  }
}

// RandomMap of tests/test_jacobians.cpp:13-20: a 6 x 5 grid over
// [-3, 3] x [-2, 2] with node values uniform in [-2, 2] drawn from
// std::mt19937(seed), in node order. values receives 30 doubles.
void oracle_random_map(uint32_t seed, double* values) {
  std::mt19937 rng(seed);
  std::uniform_real_distribution<double> dist(-2.0, 2.0);
  for (int i = 0; i < 30; ++i) {
    values[i] = dist(rng);
  }
}

// Port of tests/test_jacobians.cpp:33-153 (mt19937 seeds 42, 7, 43; central
// differences with eps 1e-6, tolerance 1e-5; frozen-cell check omitted as it
// is Ceres-only). Returns the number of failed comparisons; `checked` gets the
// number of comparisons made.
int oracle_selftest_jacobians(int* checked) {
  constexpr double kEps = 1e-6;
  constexpr double kTol = 1e-5;
  int failures = 0;
  int count = 0;
  auto random_map = [](std::mt19937& rng) {
    GridMap map(6, 5, {-3.0, -2.0}, {3.0, 2.0});
    std::uniform_real_distribution<double> dist(-2.0, 2.0);
    for (int i = 0; i < map.num_nodes(); ++i) {
      map.values()[static_cast<size_t>(i)] = dist(rng);
    }
    return map;
  };
  {
    std::mt19937 rng(42);
    std::uniform_real_distribution<double> point_dist(-1.0, 1.0);
    std::uniform_real_distribution<double> pose_dist(-0.5, 0.5);
    for (int trial = 0; trial < 20; ++trial) {
      GridMap map = random_map(rng);
      const double px_ = pose_dist(rng);
      const double py_ = pose_dist(rng);
      const double pt_ = pose_dist(rng) * 3.0;
      const Pose2 pose{px_, py_, pt_};
      const double qx = point_dist(rng);
      const double qy = point_dist(rng);
      const Vec2 p{qx, qy};
      const double delta = point_dist(rng);
      const PointResidualJacobian eval = EvalPointResidual(map, pose, p, delta);
      if (!eval.valid) {
        continue;
      }
      for (size_t k = 0; k < 4; ++k) {
        GridMap m2 = map;
        m2.values()[static_cast<size_t>(eval.node_ids[k])] += kEps;
        const double plus = EvalPointResidual(m2, pose, p, delta).residual;
        m2.values()[static_cast<size_t>(eval.node_ids[k])] -= 2 * kEps;
        const double minus = EvalPointResidual(m2, pose, p, delta).residual;
        ++count;
        if (std::abs(eval.d_nodes[k] - (plus - minus) / (2 * kEps)) > kTol) {
          ++failures;
        }
      }
      const Pose2 plus[3] = {{pose.x + kEps, pose.y, pose.theta},
                             {pose.x, pose.y + kEps, pose.theta},
                             {pose.x, pose.y, pose.theta + kEps}};
      const Pose2 minus[3] = {{pose.x - kEps, pose.y, pose.theta},
                              {pose.x, pose.y - kEps, pose.theta},
                              {pose.x, pose.y, pose.theta - kEps}};
      for (int k = 0; k < 3; ++k) {
        const PointResidualJacobian ep = EvalPointResidual(map, plus[k], p, delta);
        const PointResidualJacobian em = EvalPointResidual(map, minus[k], p, delta);
        if (!ep.valid || !em.valid || ep.node_ids != eval.node_ids || em.node_ids != eval.node_ids) {
          continue;
        }
        ++count;
        if (std::abs(eval.d_pose[static_cast<size_t>(k)] - (ep.residual - em.residual) / (2 * kEps)) > kTol) {
          ++failures;
        }
      }
    }
  }
  {
    std::mt19937 rng(43);
    GridMap map = random_map(rng);
    const Vec2 normal{0.6, 0.8};
    const EikonalResidualJacobian eval = EvalEikonalResidual(map, 2, 1, normal);
    for (size_t k = 0; k < 3; ++k) {
      map.values()[static_cast<size_t>(eval.node_ids[k])] += kEps;
      const double plus = EvalEikonalResidual(map, 2, 1, normal).residual;
      map.values()[static_cast<size_t>(eval.node_ids[k])] -= 2 * kEps;
      const double minus = EvalEikonalResidual(map, 2, 1, normal).residual;
      map.values()[static_cast<size_t>(eval.node_ids[k])] += kEps;
      ++count;
      if (std::abs(eval.d_nodes[k] - (plus - minus) / (2 * kEps)) > kTol) {
        ++failures;
      }
    }
  }
  {
    const Pose2 pose_i{0.5, -1.0, 0.9};
    const Pose2 pose_j{1.5, 0.25, 1.4};
    const Pose2 meas{0.9, 1.1, 0.45};
    const OdomResidualJacobian eval = EvalOdomResidual(pose_i, pose_j, meas);
    auto perturb = [](const Pose2& p, int param, double amount) {
      Pose2 o = p;
      if (param == 0) {
        o.x += amount;
      } else if (param == 1) {
        o.y += amount;
      } else {
        o.theta += amount;
      }
      return o;
    };
    for (int param = 0; param < 3; ++param) {
      const auto ri_p = EvalOdomResidual(perturb(pose_i, param, kEps), pose_j, meas).residual;
      const auto ri_m = EvalOdomResidual(perturb(pose_i, param, -kEps), pose_j, meas).residual;
      const auto rj_p = EvalOdomResidual(pose_i, perturb(pose_j, param, kEps), meas).residual;
      const auto rj_m = EvalOdomResidual(pose_i, perturb(pose_j, param, -kEps), meas).residual;
      for (int r = 0; r < 3; ++r) {
        const double fd_i = (ri_p[static_cast<size_t>(r)] - ri_m[static_cast<size_t>(r)]) / (2 * kEps);
        const double fd_j = (rj_p[static_cast<size_t>(r)] - rj_m[static_cast<size_t>(r)]) / (2 * kEps);
        count += 2;
        if (std::abs(eval.d_pose_i[static_cast<size_t>(r)][static_cast<size_t>(param)] - fd_i) > kTol) {
          ++failures;
        }
        if (std::abs(eval.d_pose_j[static_cast<size_t>(r)][static_cast<size_t>(param)] - fd_j) > kTol) {
          ++failures;
        }
      }
    }
  }
  *checked = count;
  return failures;
}

}  // extern "C"
