// CPU oracle for the joint Levenberg-Marquardt path of sdf-slam.
//
// TEST INFRASTRUCTURE ONLY. This is a dependency-free restatement of the
// reference's FP64 arithmetic, used as the checker by tests/, by
// __graft_entry__.smoke() and by bench.py's CPU baseline leg. Nothing in the
// product library links, loads or calls it.
//
// Every function cites the reference file:line whose arithmetic it follows
// (paths relative to the RobinJehn/sdf-slam repository). Floating-point
// contraction is disabled for the whole translation unit
// (-ffp-contract=off); std::fma appears exactly where the reference's LDLT
// row kernel pins it (src/solvers/parallel_ldlt.hpp:186,196).
//
// Pinning: the grid, pose, hallucination and Jacobian functions are pinned by
// the reference's own known-answer and finite-difference tests (ported in
// tests/test_oracle_known_answers.py and oracle_selftest_*). The elimination
// ordering differs from Eigen's AMD (a third-party routine absent here), so the
// oracle's LM step delta is a restatement whose bitwise agreement with Eigen is
// unpinned; it agrees with any exact solve to cond(A) * eps.
#pragma once

#include <array>
#include <cmath>
#include <cstdint>
#include <vector>

namespace oracle {

struct Vec2 {
  double x{0.0};
  double y{0.0};
};

/// src/core/pose.hpp:9
inline double WrapAngle(double angle) { return std::atan2(std::sin(angle), std::cos(angle)); }

/// src/core/pose.hpp:12-44
struct Pose2 {
  double x{0.0};
  double y{0.0};
  double theta{0.0};

  /// Rotation() * p + Translation(), pose.hpp:19-30. Eigen's 2x2 * 2x1 product
  /// sums r(i,0)*p0 + r(i,1)*p1 per row with r = [c -s; s c].
  [[nodiscard]] Vec2 Apply(const Vec2& p) const {
    const double c = std::cos(theta);
    const double s = std::sin(theta);
    return {(c * p.x + (-s) * p.y) + x, (s * p.x + c * p.y) + y};
  }
  /// pose.hpp:33-36
  [[nodiscard]] Pose2 Compose(const Pose2& rel) const {
    const Vec2 t = Apply({rel.x, rel.y});
    return {t.x, t.y, WrapAngle(theta + rel.theta)};
  }
  /// pose.hpp:40-43: R^T (t_other - t).
  [[nodiscard]] Pose2 RelativeTo(const Pose2& other) const {
    const double c = std::cos(theta);
    const double s = std::sin(theta);
    const double dx = other.x - x;
    const double dy = other.y - y;
    return {c * dx + s * dy, (-s) * dx + c * dy, WrapAngle(other.theta - theta)};
  }
};

/// src/core/grid_map.hpp:11-123
class GridMap {
 public:
  GridMap() = default;
  GridMap(int nx, int ny, Vec2 min_corner, Vec2 max_corner, double initial_value = 0.0);

  struct CellRef {
    int w{0};
    int h{0};
    double alpha{0.0};
    double beta{0.0};
    std::array<int, 4> node_ids{};
    std::array<double, 4> weights{};
  };

  [[nodiscard]] int nx() const { return nx_; }
  [[nodiscard]] int ny() const { return ny_; }
  [[nodiscard]] double dx() const { return dx_; }
  [[nodiscard]] double dy() const { return dy_; }
  [[nodiscard]] Vec2 min_corner() const { return min_; }
  [[nodiscard]] Vec2 max_corner() const { return max_; }
  [[nodiscard]] int num_nodes() const { return nx_ * ny_; }
  [[nodiscard]] int NodeId(int w, int h) const { return h * nx_ + w; }
  [[nodiscard]] Vec2 NodePosition(int w, int h) const {
    return {min_.x + w * dx_, min_.y + h * dy_};
  }
  [[nodiscard]] double Value(int w, int h) const { return values_[static_cast<size_t>(NodeId(w, h))]; }
  std::vector<double>& values() { return values_; }
  [[nodiscard]] const std::vector<double>& values() const { return values_; }

  bool Locate(const Vec2& p, CellRef& cell) const;
  void LocateClamped(const Vec2& p, CellRef& cell) const;
  [[nodiscard]] double Interpolate(const CellRef& cell) const;
  [[nodiscard]] Vec2 Gradient(const CellRef& cell) const;

 private:
  void FillCell(CellRef& cell) const;
  int nx_{2};
  int ny_{2};
  Vec2 min_{};
  Vec2 max_{};
  double dx_{1.0};
  double dy_{1.0};
  std::vector<double> values_;
};

/// src/problem/residual_math.hpp:27-33
struct PointResidualJacobian {
  bool valid{false};
  double residual{0.0};
  std::array<int, 4> node_ids{};
  std::array<double, 4> d_nodes{};
  std::array<double, 3> d_pose{};
  int cell_w{-1};
  int cell_h{-1};
};

Vec2 SmoothGradient(const GridMap& map, const GridMap::CellRef& cell);
Vec2 SmoothGradientMeters(const GridMap& map, const Vec2& p, double step);
PointResidualJacobian EvalPointResidual(const GridMap& map, const Pose2& pose, const Vec2& p,
                                        double delta, bool smooth_gradient = false,
                                        double smooth_gradient_step = 0.0);

struct EikonalResidualJacobian {
  double residual{0.0};
  std::array<int, 3> node_ids{};
  std::array<double, 3> d_nodes{};
};
EikonalResidualJacobian EvalEikonalResidual(const GridMap& map, int w, int h, const Vec2& normal);

struct OdomResidualJacobian {
  std::array<double, 3> residual{};
  std::array<std::array<double, 3>, 3> d_pose_i{};
  std::array<std::array<double, 3>, 3> d_pose_j{};
};
OdomResidualJacobian EvalOdomResidual(const Pose2& pose_i, const Pose2& pose_j, const Pose2& meas);

// ---------------------------------------------------------------- problem --

struct PointSpec {
  int frame{0};
  Vec2 point_sensor{};
  double expected_sdf{0.0};
  double sqrt_weight{1.0};
};
struct EikonalSpec {
  int w{0};
  int h{0};
  Vec2 normal{};
  double sqrt_weight{1.0};
};
struct OdomSpec {
  int frame_i{0};
  int frame_j{0};
  Pose2 measurement{};
  double sqrt_weight{1.0};
};
struct RelationMeasurement {
  int frame_i{0};
  int frame_j{0};
  Pose2 measurement{};
  double sqrt_weight{1.0};
};

struct Weights {
  double scan{1.0};
  double hallucination{1.0};
  double eikonal{1.0};
  double odometry{1.0};
  double relation{1.0};
};
struct HallucinationOptions {
  int points_per_scan_point{6};
  double step_size{0.1};
  bool both_directions{true};
};
enum class NormalMethod : int { kPca = 0, kHybrid = 1, kWeighted = 2 };
struct NormalOptions {
  NormalMethod method{NormalMethod::kWeighted};
  int k_neighbors{10};
  bool per_scan{false};
  double corner_threshold{0.2};
};
struct ProblemOptions {
  Weights weights;
  HallucinationOptions hallucination;
  NormalOptions normals;
  double huber_delta{0.0};
  bool smooth_gradient{true};
  double smooth_gradient_step{0.0};
  bool active_region{false};
  int active_margin{2};
};

struct HallucinatedPoint {
  Vec2 point_sensor;
  double expected_sdf{0.0};
};
/// src/core/hallucination.cpp:5-28
std::vector<HallucinatedPoint> GenerateHallucinatedPoints(const std::vector<Vec2>& scan,
                                                          const HallucinationOptions& options);

struct ScanNormals {
  std::vector<Vec2> points;
  std::vector<Vec2> normals;
  std::vector<double> cornerness;
};
struct NodeNormal {
  Vec2 normal{};
  double eikonal_scale{1.0};
};
/// src/core/normals.cpp:127-160 (exact kNN, neighbours ordered by (d^2, index))
ScanNormals ComputeScanNormals(const std::vector<std::vector<Vec2>>& scans,
                               const std::vector<Pose2>& poses, int k_neighbors, bool per_scan);
/// src/core/normals.cpp:162-220
std::vector<NodeNormal> AssignNodeNormals(const GridMap& map, const ScanNormals& scan_normals,
                                          const NormalOptions& options);

/// src/problem/problem.hpp:92-161 / problem.cpp:11-156
class Problem {
 public:
  Problem() = default;
  Problem(GridMap map, std::vector<Pose2> poses, const std::vector<std::vector<Vec2>>& scans,
          const std::vector<Pose2>& odometry, const ProblemOptions& options,
          const std::vector<RelationMeasurement>& relations);
  /// Identical input state: specs and index maps given directly.
  static Problem FromSpecs(GridMap map, std::vector<Pose2> poses, std::vector<PointSpec> points,
                           std::vector<EikonalSpec> eik, std::vector<OdomSpec> odom,
                           std::vector<int> node_to_active, double huber_delta,
                           bool smooth_gradient, double smooth_gradient_step);

  GridMap& map() { return map_; }
  [[nodiscard]] const GridMap& map() const { return map_; }
  std::vector<Pose2>& poses() { return poses_; }
  [[nodiscard]] const std::vector<Pose2>& poses() const { return poses_; }
  [[nodiscard]] const std::vector<PointSpec>& point_specs() const { return point_specs_; }
  [[nodiscard]] const std::vector<EikonalSpec>& eikonal_specs() const { return eikonal_specs_; }
  [[nodiscard]] const std::vector<OdomSpec>& odom_specs() const { return odom_specs_; }
  [[nodiscard]] const std::vector<int>& node_to_active() const { return node_to_active_; }
  [[nodiscard]] const std::vector<int>& active_to_node() const { return active_to_node_; }
  [[nodiscard]] double huber_delta() const { return huber_delta_; }
  [[nodiscard]] bool smooth_gradient() const { return smooth_gradient_; }
  [[nodiscard]] double smooth_gradient_step() const { return smooth_gradient_step_; }

  /// problem.hpp:115-121
  [[nodiscard]] double HuberWeight(double weighted_residual) const {
    if (huber_delta_ <= 0.0) {
      return 1.0;
    }
    const double abs_r = std::abs(weighted_residual);
    return abs_r <= huber_delta_ ? 1.0 : huber_delta_ / abs_r;
  }
  [[nodiscard]] int num_active_nodes() const { return static_cast<int>(active_to_node_.size()); }
  [[nodiscard]] int num_parameters() const {
    return num_active_nodes() + 3 * (static_cast<int>(poses_.size()) - 1);
  }
  [[nodiscard]] int num_residuals() const {
    return static_cast<int>(point_specs_.size() + eikonal_specs_.size() + 3 * odom_specs_.size());
  }
  [[nodiscard]] int NodeColumn(int node_id) const {
    return node_to_active_[static_cast<size_t>(node_id)];
  }
  [[nodiscard]] int PoseColumn(int frame) const { return num_active_nodes() + 3 * (frame - 1); }

  /// problem.cpp:117-130
  void ApplyStep(const std::vector<double>& step);
  /// problem.cpp:132-156
  [[nodiscard]] double Cost() const;

 private:
  GridMap map_;
  std::vector<Pose2> poses_;
  double huber_delta_{0.0};
  bool smooth_gradient_{false};
  double smooth_gradient_step_{0.0};
  std::vector<PointSpec> point_specs_;
  std::vector<EikonalSpec> eikonal_specs_;
  std::vector<OdomSpec> odom_specs_;
  std::vector<int> node_to_active_;
  std::vector<int> active_to_node_;
};

// ----------------------------------------------------------------- sparse --

/// Compressed sparse column matrix (Eigen::SparseMatrix<double> column-major
/// layout after makeCompressed: sorted inner indices).
struct Csc {
  int rows{0};
  int cols{0};
  std::vector<int> outer;  // cols + 1
  std::vector<int> inner;
  std::vector<double> values;
};

/// Simplicial LDL^T with the reference's up-looking row kernel
/// (src/solvers/parallel_ldlt.hpp:150-244) over a caller-supplied symmetric
/// permutation. `perm[new] = old`.
class Ldlt {
 public:
  /// Symbolic analysis (elimination tree and column counts of L).
  void Analyze(const Csc& a, const std::vector<int>& perm, int num_threads);
  /// Numeric factorization; false on a zero pivot (NumericalIssue).
  bool Factorize(const Csc& a);
  /// x = P^T L^-T D^-1 L^-1 P b (Eigen SimplicialLDLT::_solve_impl order).
  [[nodiscard]] std::vector<double> Solve(const std::vector<double>& b) const;
  [[nodiscard]] int64_t nnz_l() const { return static_cast<int64_t>(lp_.back()); }
  [[nodiscard]] const std::vector<double>& diag() const { return d_; }

 private:
  void BuildSchedule(int num_threads);
  int n_{0};
  std::vector<int> perm_;  // new -> old
  std::vector<int> pinv_;  // old -> new
  std::vector<int> parent_;
  std::vector<int> lp_;
  std::vector<int> li_;
  std::vector<double> lx_;
  std::vector<double> d_;
  std::vector<std::vector<int>> thread_rows_;
  std::vector<int> trunk_rows_;
  Csc upper_;  // permuted upper triangle (PAP^T)
};

// -------------------------------------------------------------------- LM ---

/// src/solvers/solver.hpp:29-55
struct SolverOptions {
  int max_iterations{100};
  double step_tolerance{1e-6};
  double lambda_init{1.0};
  double lambda_factor{1.0};
  bool reject_worse_steps{false};
  bool marquardt_scaling{false};
  bool trust_region{false};
  int num_threads{0};
};
/// src/solvers/solver.hpp:57-64
struct SolveResult {
  bool converged{false};
  int iterations{0};
  double initial_cost{0.0};
  double final_cost{0.0};
  double duration_seconds{0.0};
  std::vector<double> cost_history;
  /// Seconds spent per phase (assembly, J^T J + J^T r, factor, solve, cost).
  std::array<double, 5> phase_seconds{};
};

/// Everything one LM iteration computes before it moves the state.
struct Linearization {
  std::vector<double> residuals;    // num_rows
  std::vector<int> point_cell;      // per point row: h*nx+w, or -1 outside
  Csc jacobian;                     // num_rows x num_params
  Csc normal;                       // J^T J + damping, full symmetric
  std::vector<double> rhs;          // -J^T r
  std::vector<double> step;         // delta
  bool factor_ok{true};
  int64_t nnz_l{0};
};

/// Elimination ordering used by the oracle: geometric nested dissection of the
/// active grid nodes with every pose column ordered last. perm[new] = old.
std::vector<int> GridNestedDissection(const Problem& problem);

/// One iteration's assembly, normal equations, damping and step
/// (src/solvers/lm_solver.cpp:304-436) without touching the state.
Linearization Linearize(const Problem& problem, double lambda, bool marquardt, int num_threads,
                        bool compute_step);

/// src/solvers/lm_solver.cpp:201-434
SolveResult SolveLm(Problem& problem, const SolverOptions& options);

}  // namespace oracle
