// CPU oracle (test infrastructure only; see oracle.hpp for the scope and the
// pinning notes). Compiled with -O2 -ffp-contract=off.
#include "oracle.hpp"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <functional>
#include <limits>
#include <numeric>
#include <queue>
#include <stdexcept>
#include <thread>
#include <tuple>

namespace oracle {

// ---------------------------------------------------------------- GridMap --

GridMap::GridMap(int nx, int ny, Vec2 min_corner, Vec2 max_corner, double initial_value)
    : nx_(nx),
      ny_(ny),
      min_(min_corner),
      max_(max_corner),
      dx_((max_corner.x - min_corner.x) / (nx - 1)),
      dy_((max_corner.y - min_corner.y) / (ny - 1)),
      values_(static_cast<size_t>(nx) * static_cast<size_t>(ny), initial_value) {
  if (nx < 2 || ny < 2 || !(dx_ > 0.0) || !(dy_ > 0.0)) {
    throw std::invalid_argument("GridMap needs nx, ny >= 2 and max > min");
  }
}

// grid_map.hpp:109-115
void GridMap::FillCell(CellRef& cell) const {
  cell.node_ids = {NodeId(cell.w, cell.h), NodeId(cell.w + 1, cell.h), NodeId(cell.w, cell.h + 1),
                   NodeId(cell.w + 1, cell.h + 1)};
  const double a = cell.alpha;
  const double b = cell.beta;
  cell.weights = {(1.0 - a) * (1.0 - b), a * (1.0 - b), (1.0 - a) * b, a * b};
}

// grid_map.hpp:58-70
bool GridMap::Locate(const Vec2& p, CellRef& cell) const {
  const double fx = (p.x - min_.x) / dx_;
  const double fy = (p.y - min_.y) / dy_;
  if (fx < 0.0 || fy < 0.0 || fx > nx_ - 1 || fy > ny_ - 1) {
    return false;
  }
  cell.w = std::min(static_cast<int>(fx), nx_ - 2);
  cell.h = std::min(static_cast<int>(fy), ny_ - 2);
  cell.alpha = fx - cell.w;
  cell.beta = fy - cell.h;
  FillCell(cell);
  return true;
}

// grid_map.hpp:75-83
void GridMap::LocateClamped(const Vec2& p, CellRef& cell) const {
  const double fx = (p.x - min_.x) / dx_;
  const double fy = (p.y - min_.y) / dy_;
  cell.w = std::clamp(static_cast<int>(fx), 0, nx_ - 2);
  cell.h = std::clamp(static_cast<int>(fy), 0, ny_ - 2);
  cell.alpha = fx - cell.w;
  cell.beta = fy - cell.h;
  FillCell(cell);
}

// grid_map.hpp:86-93: sequential sum starting from 0.0.
double GridMap::Interpolate(const CellRef& cell) const {
  double value = 0.0;
  for (int i = 0; i < 4; ++i) {
    value += cell.weights[static_cast<size_t>(i)] *
             values_[static_cast<size_t>(cell.node_ids[static_cast<size_t>(i)])];
  }
  return value;
}

// grid_map.hpp:98-106
Vec2 GridMap::Gradient(const CellRef& cell) const {
  const double d00 = values_[static_cast<size_t>(cell.node_ids[0])];
  const double d10 = values_[static_cast<size_t>(cell.node_ids[1])];
  const double d01 = values_[static_cast<size_t>(cell.node_ids[2])];
  const double d11 = values_[static_cast<size_t>(cell.node_ids[3])];
  const double gx = ((1.0 - cell.beta) * (d10 - d00) + cell.beta * (d11 - d01)) / dx_;
  const double gy = ((1.0 - cell.alpha) * (d01 - d00) + cell.alpha * (d11 - d10)) / dy_;
  return {gx, gy};
}

// ---------------------------------------------------------- residual math --

// residual_math.hpp:40-57
Vec2 SmoothGradient(const GridMap& map, const GridMap::CellRef& cell) {
  const auto node_gradient = [&map](int w, int h) -> Vec2 {
    const int w_lo = std::max(w - 1, 0);
    const int w_hi = std::min(w + 1, map.nx() - 1);
    const int h_lo = std::max(h - 1, 0);
    const int h_hi = std::min(h + 1, map.ny() - 1);
    const double gx = (map.Value(w_hi, h) - map.Value(w_lo, h)) / ((w_hi - w_lo) * map.dx());
    const double gy = (map.Value(w, h_hi) - map.Value(w, h_lo)) / ((h_hi - h_lo) * map.dy());
    return {gx, gy};
  };
  const Vec2 g00 = node_gradient(cell.w, cell.h);
  const Vec2 g10 = node_gradient(cell.w + 1, cell.h);
  const Vec2 g01 = node_gradient(cell.w, cell.h + 1);
  const Vec2 g11 = node_gradient(cell.w + 1, cell.h + 1);
  const double a = cell.alpha;
  const double b = cell.beta;
  const double s00 = (1.0 - a) * (1.0 - b);
  const double s10 = a * (1.0 - b);
  const double s01 = (1.0 - a) * b;
  const double s11 = a * b;
  return {((s00 * g00.x + s10 * g10.x) + s01 * g01.x) + s11 * g11.x,
          ((s00 * g00.y + s10 * g10.y) + s01 * g01.y) + s11 * g11.y};
}

// residual_math.hpp:63-73
Vec2 SmoothGradientMeters(const GridMap& map, const Vec2& p, double step) {
  GridMap::CellRef cell;
  const auto value = [&map, &cell](double x, double y) {
    map.LocateClamped({x, y}, cell);
    return map.Interpolate(cell);
  };
  const double gx = (value(p.x + step, p.y) - value(p.x - step, p.y)) / (2.0 * step);
  const double gy = (value(p.x, p.y + step) - value(p.x, p.y - step)) / (2.0 * step);
  return {gx, gy};
}

// residual_math.hpp:75-106
PointResidualJacobian EvalPointResidual(const GridMap& map, const Pose2& pose, const Vec2& p,
                                        double delta, bool smooth_gradient,
                                        double smooth_gradient_step) {
  PointResidualJacobian out;
  const Vec2 g = pose.Apply(p);
  GridMap::CellRef cell;
  if (!map.Locate(g, cell)) {
    out.residual = -delta;
    return out;
  }
  out.valid = true;
  out.cell_w = cell.w;
  out.cell_h = cell.h;
  out.residual = map.Interpolate(cell) - delta;
  out.node_ids = cell.node_ids;
  out.d_nodes = cell.weights;
  Vec2 grad;
  if (smooth_gradient && smooth_gradient_step > 0.0) {
    grad = SmoothGradientMeters(map, g, smooth_gradient_step);
  } else if (smooth_gradient) {
    grad = SmoothGradient(map, cell);
  } else {
    grad = map.Gradient(cell);
  }
  const double c = std::cos(pose.theta);
  const double s = std::sin(pose.theta);
  const double dx_dtheta = (-s) * p.x - c * p.y;
  const double dy_dtheta = c * p.x - s * p.y;
  out.d_pose = {grad.x, grad.y, grad.x * dx_dtheta + grad.y * dy_dtheta};
  return out;
}

// residual_math.hpp:158-171
EikonalResidualJacobian EvalEikonalResidual(const GridMap& map, int w, int h, const Vec2& normal) {
  EikonalResidualJacobian out;
  const double d00 = map.Value(w, h);
  const double d10 = map.Value(w + 1, h);
  const double d01 = map.Value(w, h + 1);
  const double gx = (d10 - d00) / map.dx();
  const double gy = (d01 - d00) / map.dy();
  out.residual = 1.0 - (normal.x * gx + normal.y * gy);
  out.node_ids = {map.NodeId(w, h), map.NodeId(w + 1, h), map.NodeId(w, h + 1)};
  out.d_nodes = {normal.x / map.dx() + normal.y / map.dy(), -normal.x / map.dx(),
                 -normal.y / map.dy()};
  return out;
}

// residual_math.hpp:182-205. R(-theta_i) = [c s; -s c]; the theta column of
// d_pose_i is (-R(-theta_i) J) dt with J = [0 -1; 1 0], i.e. rows
// (-s dtx + c dty, -c dtx - s dty).
OdomResidualJacobian EvalOdomResidual(const Pose2& pose_i, const Pose2& pose_j, const Pose2& meas) {
  OdomResidualJacobian out;
  const double c = std::cos(pose_i.theta);
  const double s = std::sin(pose_i.theta);
  const double dtx = pose_j.x - pose_i.x;
  const double dty = pose_j.y - pose_i.y;
  const double rx = c * dtx + s * dty;
  const double ry = (-s) * dtx + c * dty;
  out.residual = {rx - meas.x, ry - meas.y, WrapAngle(pose_j.theta - pose_i.theta - meas.theta)};
  out.d_pose_i[0] = {-c, -s, (-s) * dtx + c * dty};
  out.d_pose_i[1] = {s, -c, (-c) * dtx + (-s) * dty};
  out.d_pose_i[2] = {0.0, 0.0, -1.0};
  out.d_pose_j[0] = {c, s, 0.0};
  out.d_pose_j[1] = {-s, c, 0.0};
  out.d_pose_j[2] = {0.0, 0.0, 1.0};
  return out;
}

// ---------------------------------------------------------- hallucination --

// hallucination.cpp:5-28. Eigen evaluates `point + toward_origin * j` as
// p + (t * j) per component, with t = (-p / norm) * step.
std::vector<HallucinatedPoint> GenerateHallucinatedPoints(const std::vector<Vec2>& scan,
                                                          const HallucinationOptions& options) {
  std::vector<HallucinatedPoint> result;
  if (options.points_per_scan_point <= 0) {
    return result;
  }
  const int per_side = options.points_per_scan_point / (options.both_directions ? 2 : 1);
  for (const Vec2& p : scan) {
    const double norm = std::sqrt(p.x * p.x + p.y * p.y);
    if (norm < 1e-9) {
      continue;
    }
    const Vec2 t = {(-p.x) / norm * options.step_size, (-p.y) / norm * options.step_size};
    for (int j = 1; j <= per_side; ++j) {
      const double jd = static_cast<double>(j);
      result.push_back({{p.x + t.x * jd, p.y + t.y * jd}, options.step_size * jd});
      if (options.both_directions) {
        result.push_back({{p.x - t.x * jd, p.y - t.y * jd}, -options.step_size * jd});
      }
    }
  }
  return result;
}

// ---------------------------------------------------------------- normals --

namespace {

/// Exact k-nearest-neighbour search on a uniform bucket grid. Neighbours are
/// returned ordered by (squared distance, index).
class Knn {
 public:
  explicit Knn(const std::vector<Vec2>& pts) : pts_(pts) {
    double min_x = std::numeric_limits<double>::max();
    double min_y = min_x;
    double max_x = -min_x;
    double max_y = -min_x;
    for (const Vec2& p : pts) {
      min_x = std::min(min_x, p.x);
      min_y = std::min(min_y, p.y);
      max_x = std::max(max_x, p.x);
      max_y = std::max(max_y, p.y);
    }
    if (pts.empty()) {
      min_x = min_y = 0.0;
      max_x = max_y = 1.0;
    }
    ox_ = min_x;
    oy_ = min_y;
    const double ex = std::max(max_x - min_x, 1e-9);
    const double ey = std::max(max_y - min_y, 1e-9);
    const double n = std::max<double>(1.0, static_cast<double>(pts.size()));
    cell_ = std::max({std::sqrt(ex * ey / n) * 1.5, ex / 2048.0, ey / 2048.0, 1e-9});
    gx_ = std::min(2048, static_cast<int>(ex / cell_) + 1);
    gy_ = std::min(2048, static_cast<int>(ey / cell_) + 1);
    start_.assign(static_cast<size_t>(gx_) * gy_ + 1, 0);
    for (const Vec2& p : pts) {
      ++start_[static_cast<size_t>(Bucket(p)) + 1];
    }
    for (size_t b = 1; b < start_.size(); ++b) {
      start_[b] += start_[b - 1];
    }
    items_.resize(pts.size());
    std::vector<int> fill(start_.begin(), start_.end() - 1);
    for (int i = 0; i < static_cast<int>(pts.size()); ++i) {
      items_[static_cast<size_t>(fill[static_cast<size_t>(Bucket(pts[static_cast<size_t>(i)]))]++)] = i;
    }
  }

  /// Returns up to k neighbours of q ordered by (d^2, index).
  void Query(const Vec2& q, size_t k, std::vector<std::pair<double, int>>& out) const {
    out.clear();
    if (pts_.empty() || k == 0) {
      return;
    }
    const int cx = std::clamp(static_cast<int>((q.x - ox_) / cell_), 0, gx_ - 1);
    const int cy = std::clamp(static_cast<int>((q.y - oy_) / cell_), 0, gy_ - 1);
    // Distance from q to the boundary of its own (clamped) bucket, used as a
    // conservative lower bound for points in farther rings.
    const double bx0 = ox_ + cx * cell_;
    const double by0 = oy_ + cy * cell_;
    const double inner = std::max(0.0, std::min({q.x - bx0, bx0 + cell_ - q.x, q.y - by0,
                                                  by0 + cell_ - q.y}));
    const int max_ring = std::max(gx_, gy_);
    auto cmp = [](const std::pair<double, int>& a, const std::pair<double, int>& b) { return a < b; };
    std::priority_queue<std::pair<double, int>, std::vector<std::pair<double, int>>, decltype(cmp)> heap(cmp);
    for (int r = 0; r <= max_ring; ++r) {
      for (int y = cy - r; y <= cy + r; ++y) {
        if (y < 0 || y >= gy_) {
          continue;
        }
        const bool edge_row = (y == cy - r || y == cy + r);
        for (int x = cx - r; x <= cx + r; ++x) {
          if (x < 0 || x >= gx_) {
            continue;
          }
          if (!edge_row && x != cx - r && x != cx + r) {
            continue;
          }
          const size_t b = static_cast<size_t>(y) * gx_ + x;
          for (int s = start_[b]; s < start_[b + 1]; ++s) {
            const int idx = items_[static_cast<size_t>(s)];
            const double ddx = pts_[static_cast<size_t>(idx)].x - q.x;
            const double ddy = pts_[static_cast<size_t>(idx)].y - q.y;
            const std::pair<double, int> cand{ddx * ddx + ddy * ddy, idx};
            if (heap.size() < k) {
              heap.push(cand);
            } else if (cand < heap.top()) {
              heap.pop();
              heap.push(cand);
            }
          }
        }
      }
      if (heap.size() == std::min(k, pts_.size())) {
        const double bound = inner + r * cell_;
        if (heap.top().first < bound * bound) {
          break;
        }
      }
    }
    while (!heap.empty()) {
      out.push_back(heap.top());
      heap.pop();
    }
    std::reverse(out.begin(), out.end());
  }

 private:
  int Bucket(const Vec2& p) const {
    const int x = std::clamp(static_cast<int>((p.x - ox_) / cell_), 0, gx_ - 1);
    const int y = std::clamp(static_cast<int>((p.y - oy_) / cell_), 0, gy_ - 1);
    return y * gx_ + x;
  }
  const std::vector<Vec2>& pts_;
  double ox_{0.0};
  double oy_{0.0};
  double cell_{1.0};
  int gx_{1};
  int gy_{1};
  std::vector<int> start_;
  std::vector<int> items_;
};

/// normals.cpp:70-101 with a closed-form 2x2 symmetric eigen-decomposition in
/// place of Eigen's SelfAdjointEigenSolver.
void PcaNormal(const std::vector<Vec2>& points, const Knn& knn, size_t i, size_t k,
               const Vec2& origin, Vec2& normal_out, double& cornerness_out,
               std::vector<std::pair<double, int>>& scratch) {
  knn.Query(points[i], k, scratch);
  const size_t found = scratch.size();
  double mx = 0.0;
  double my = 0.0;
  for (size_t j = 0; j < found; ++j) {
    mx += points[static_cast<size_t>(scratch[j].second)].x;
    my += points[static_cast<size_t>(scratch[j].second)].y;
  }
  mx /= static_cast<double>(found);
  my /= static_cast<double>(found);
  double a = 0.0;
  double b = 0.0;
  double c = 0.0;
  for (size_t j = 0; j < found; ++j) {
    const double dx = points[static_cast<size_t>(scratch[j].second)].x - mx;
    const double dy = points[static_cast<size_t>(scratch[j].second)].y - my;
    a += dx * dx;
    b += dx * dy;
    c += dy * dy;
  }
  const double half_tr = 0.5 * (a + c);
  const double half_diff = 0.5 * (a - c);
  const double disc = std::sqrt(half_diff * half_diff + b * b);
  const double ev_min = half_tr - disc;
  const double ev_max = half_tr + disc;
  double vx;
  double vy;
  if (half_diff >= 0.0) {
    vx = b;
    vy = ev_min - a;
  } else {
    vx = ev_min - c;
    vy = b;
  }
  double vn = std::sqrt(vx * vx + vy * vy);
  if (!(vn > 0.0)) {
    vx = 1.0;
    vy = 0.0;
    vn = 1.0;
  }
  Vec2 normal{vx / vn, vy / vn};
  const double lambda_min = std::max(ev_min, 0.0);
  const double lambda_max = std::max(ev_max, 1e-12);
  if (normal.x * (origin.x - points[i].x) + normal.y * (origin.y - points[i].y) < 0.0) {
    normal = {-normal.x, -normal.y};
  }
  normal_out = normal;
  cornerness_out = lambda_min / lambda_max;
}

}  // namespace

ScanNormals ComputeScanNormals(const std::vector<std::vector<Vec2>>& scans,
                               const std::vector<Pose2>& poses, int k_neighbors, bool per_scan) {
  if (scans.size() != poses.size()) {
    throw std::invalid_argument("scan count != pose count");
  }
  const size_t k = static_cast<size_t>(std::max(2, k_neighbors));
  ScanNormals result;
  std::vector<std::pair<double, int>> scratch;
  if (per_scan) {
    // normals.cpp:102-125
    for (size_t s = 0; s < scans.size(); ++s) {
      const std::vector<Vec2>& local = scans[s];
      const Knn knn(local);
      const double c = std::cos(poses[s].theta);
      const double sn = std::sin(poses[s].theta);
      for (size_t i = 0; i < local.size(); ++i) {
        Vec2 normal;
        double corner = 0.0;
        PcaNormal(local, knn, i, std::min(k, local.size()), {0.0, 0.0}, normal, corner, scratch);
        result.points.push_back(poses[s].Apply(local[i]));
        result.normals.push_back({c * normal.x + (-sn) * normal.y, sn * normal.x + c * normal.y});
        result.cornerness.push_back(corner);
      }
    }
    return result;
  }
  std::vector<Vec2> origins;
  for (size_t i = 0; i < scans.size(); ++i) {
    for (const Vec2& p : scans[i]) {
      result.points.push_back(poses[i].Apply(p));
      origins.push_back({poses[i].x, poses[i].y});
    }
  }
  const size_t n = result.points.size();
  result.normals.resize(n);
  result.cornerness.resize(n);
  if (n == 0) {
    return result;
  }
  const Knn knn(result.points);
  for (size_t i = 0; i < n; ++i) {
    PcaNormal(result.points, knn, i, std::min(k, n), origins[i], result.normals[i],
              result.cornerness[i], scratch);
  }
  return result;
}

std::vector<NodeNormal> AssignNodeNormals(const GridMap& map, const ScanNormals& scan_normals,
                                          const NormalOptions& options) {
  std::vector<NodeNormal> node_normals(static_cast<size_t>(map.num_nodes()));
  if (scan_normals.points.empty()) {
    return node_normals;
  }
  const Knn knn(scan_normals.points);
  std::vector<std::pair<double, int>> scratch;
  for (int h = 0; h < map.ny(); ++h) {
    for (int w = 0; w < map.nx(); ++w) {
      const Vec2 node = map.NodePosition(w, h);
      knn.Query(node, 1, scratch);
      const size_t nearest = static_cast<size_t>(scratch[0].second);
      const Vec2 n_pca = scan_normals.normals[nearest];
      const double corner =
          std::clamp(scan_normals.cornerness[nearest] / options.corner_threshold, 0.0, 1.0);
      NodeNormal out;
      switch (options.method) {
        case NormalMethod::kPca:
          out.normal = n_pca;
          break;
        case NormalMethod::kHybrid: {
          const Vec2 to_surface = {scan_normals.points[nearest].x - node.x,
                                   scan_normals.points[nearest].y - node.y};
          const double norm = std::sqrt(to_surface.x * to_surface.x + to_surface.y * to_surface.y);
          if (norm < 1e-9) {
            out.normal = n_pca;
            break;
          }
          Vec2 cue = {to_surface.x / norm, to_surface.y / norm};
          if (cue.x * n_pca.x + cue.y * n_pca.y < 0.0) {
            cue = {-cue.x, -cue.y};
          }
          const Vec2 blended = {(1.0 - corner) * n_pca.x + corner * cue.x,
                                (1.0 - corner) * n_pca.y + corner * cue.y};
          const double bn = std::sqrt(blended.x * blended.x + blended.y * blended.y);
          out.normal = bn > 1e-9 ? Vec2{blended.x / bn, blended.y / bn} : n_pca;
          break;
        }
        case NormalMethod::kWeighted:
          out.normal = n_pca;
          out.eikonal_scale = 1.0 - corner;
          break;
      }
      node_normals[static_cast<size_t>(map.NodeId(w, h))] = out;
    }
  }
  return node_normals;
}

// ---------------------------------------------------------------- Problem --

// problem.cpp:11-115
Problem::Problem(GridMap map, std::vector<Pose2> poses, const std::vector<std::vector<Vec2>>& scans,
                 const std::vector<Pose2>& odometry, const ProblemOptions& options,
                 const std::vector<RelationMeasurement>& relations)
    : map_(std::move(map)),
      poses_(std::move(poses)),
      huber_delta_(options.huber_delta),
      smooth_gradient_(options.smooth_gradient),
      smooth_gradient_step_(options.smooth_gradient_step) {
  if (scans.size() != poses_.size()) {
    throw std::invalid_argument("scan count != pose count");
  }
  if (!odometry.empty() && odometry.size() != scans.size() - 1) {
    throw std::invalid_argument("odometry count must be frames - 1");
  }
  const double sqrt_ws = std::sqrt(options.weights.scan);
  const double sqrt_wh = std::sqrt(options.weights.hallucination);
  for (size_t i = 0; i < scans.size(); ++i) {
    const int frame = static_cast<int>(i);
    for (const Vec2& p : scans[i]) {
      point_specs_.push_back({frame, p, 0.0, sqrt_ws});
    }
    for (const auto& hall : GenerateHallucinatedPoints(scans[i], options.hallucination)) {
      point_specs_.push_back({frame, hall.point_sensor, hall.expected_sdf, sqrt_wh});
    }
  }
  node_to_active_.assign(static_cast<size_t>(map_.num_nodes()), -1);
  std::vector<char> active(static_cast<size_t>(map_.num_nodes()), 0);
  if (options.active_region) {
    const int margin = options.active_margin;
    for (const auto& spec : point_specs_) {
      const Vec2 global = poses_[static_cast<size_t>(spec.frame)].Apply(spec.point_sensor);
      GridMap::CellRef cell;
      if (!map_.Locate(global, cell)) {
        continue;
      }
      for (int h = std::max(0, cell.h - margin); h <= std::min(map_.ny() - 1, cell.h + 1 + margin); ++h) {
        for (int w = std::max(0, cell.w - margin); w <= std::min(map_.nx() - 1, cell.w + 1 + margin); ++w) {
          active[static_cast<size_t>(map_.NodeId(w, h))] = 1;
        }
      }
    }
  } else {
    std::fill(active.begin(), active.end(), 1);
  }
  for (int node = 0; node < map_.num_nodes(); ++node) {
    if (active[static_cast<size_t>(node)] != 0) {
      node_to_active_[static_cast<size_t>(node)] = static_cast<int>(active_to_node_.size());
      active_to_node_.push_back(node);
    }
  }
  const ScanNormals scan_normals =
      ComputeScanNormals(scans, poses_, options.normals.k_neighbors, options.normals.per_scan);
  const std::vector<NodeNormal> node_normals = AssignNodeNormals(map_, scan_normals, options.normals);
  const double sqrt_we = std::sqrt(options.weights.eikonal);
  for (int h = 0; h + 1 < map_.ny(); ++h) {
    for (int w = 0; w + 1 < map_.nx(); ++w) {
      const int node = map_.NodeId(w, h);
      if (node_to_active_[static_cast<size_t>(node)] < 0 ||
          node_to_active_[static_cast<size_t>(map_.NodeId(w + 1, h))] < 0 ||
          node_to_active_[static_cast<size_t>(map_.NodeId(w, h + 1))] < 0) {
        continue;
      }
      const NodeNormal& nn = node_normals[static_cast<size_t>(node)];
      const double scale = nn.eikonal_scale;
      if (scale <= 0.0) {
        continue;
      }
      eikonal_specs_.push_back({w, h, nn.normal, sqrt_we * std::sqrt(scale)});
    }
  }
  const double sqrt_wo = std::sqrt(options.weights.odometry);
  for (size_t i = 0; i + 1 < scans.size() && i < odometry.size(); ++i) {
    odom_specs_.push_back({static_cast<int>(i), static_cast<int>(i) + 1, odometry[i], sqrt_wo});
  }
  const double sqrt_wr = std::sqrt(options.weights.relation);
  const int frames = static_cast<int>(scans.size());
  for (const RelationMeasurement& rel : relations) {
    if (rel.frame_i < 0 || rel.frame_j <= rel.frame_i) {
      throw std::invalid_argument("relation frames must satisfy 0 <= i < j");
    }
    if (rel.frame_j < frames) {
      odom_specs_.push_back({rel.frame_i, rel.frame_j, rel.measurement, sqrt_wr * rel.sqrt_weight});
    }
  }
}

Problem Problem::FromSpecs(GridMap map, std::vector<Pose2> poses, std::vector<PointSpec> points,
                           std::vector<EikonalSpec> eik, std::vector<OdomSpec> odom,
                           std::vector<int> node_to_active, double huber_delta,
                           bool smooth_gradient, double smooth_gradient_step) {
  Problem p;
  p.map_ = std::move(map);
  p.poses_ = std::move(poses);
  p.point_specs_ = std::move(points);
  p.eikonal_specs_ = std::move(eik);
  p.odom_specs_ = std::move(odom);
  p.node_to_active_ = std::move(node_to_active);
  p.huber_delta_ = huber_delta;
  p.smooth_gradient_ = smooth_gradient;
  p.smooth_gradient_step_ = smooth_gradient_step;
  for (int node = 0; node < static_cast<int>(p.node_to_active_.size()); ++node) {
    if (p.node_to_active_[static_cast<size_t>(node)] >= 0) {
      p.active_to_node_.push_back(node);
    }
  }
  return p;
}

// problem.cpp:117-130
void Problem::ApplyStep(const std::vector<double>& step) {
  if (static_cast<int>(step.size()) != num_parameters()) {
    throw std::invalid_argument("step size != parameter count");
  }
  for (int a = 0; a < num_active_nodes(); ++a) {
    map_.values()[static_cast<size_t>(active_to_node_[static_cast<size_t>(a)])] += step[static_cast<size_t>(a)];
  }
  for (size_t i = 1; i < poses_.size(); ++i) {
    const size_t col = static_cast<size_t>(PoseColumn(static_cast<int>(i)));
    poses_[i].x += step[col];
    poses_[i].y += step[col + 1];
    poses_[i].theta = WrapAngle(poses_[i].theta + step[col + 2]);
  }
}

// problem.cpp:132-156
double Problem::Cost() const {
  double cost = 0.0;
  for (const auto& spec : point_specs_) {
    const PointResidualJacobian eval = EvalPointResidual(
        map_, poses_[static_cast<size_t>(spec.frame)], spec.point_sensor, spec.expected_sdf);
    const double r = spec.sqrt_weight * eval.residual;
    if (huber_delta_ > 0.0 && std::abs(r) > huber_delta_) {
      cost += huber_delta_ * (2.0 * std::abs(r) - huber_delta_);
    } else {
      cost += r * r;
    }
  }
  for (const auto& spec : eikonal_specs_) {
    const EikonalResidualJacobian eval = EvalEikonalResidual(map_, spec.w, spec.h, spec.normal);
    const double r = spec.sqrt_weight * eval.residual;
    cost += r * r;
  }
  for (const auto& spec : odom_specs_) {
    const OdomResidualJacobian eval = EvalOdomResidual(
        poses_[static_cast<size_t>(spec.frame_i)], poses_[static_cast<size_t>(spec.frame_j)],
        spec.measurement);
    const double e0 = spec.sqrt_weight * eval.residual[0];
    const double e1 = spec.sqrt_weight * eval.residual[1];
    const double e2 = spec.sqrt_weight * eval.residual[2];
    cost += (e0 * e0 + e1 * e1) + e2 * e2;
  }
  return cost;
}

// ---------------------------------------------------------------- threads --

namespace {

// lm_solver.cpp:85-105
void ParallelRanges(size_t n, size_t num_threads, const std::function<void(size_t, size_t)>& fn) {
  const size_t threads = std::min(n, std::max<size_t>(1, num_threads));
  if (threads <= 1) {
    fn(0, n);
    return;
  }
  const size_t chunk = (n + threads - 1) / threads;
  std::vector<std::thread> workers;
  for (size_t t = 0; t < threads; ++t) {
    const size_t begin = t * chunk;
    const size_t end = std::min(n, begin + chunk);
    if (begin >= end) {
      break;
    }
    workers.emplace_back([begin, end, &fn] { fn(begin, end); });
  }
  for (auto& w : workers) {
    w.join();
  }
}

size_t ResolveThreads(int requested) {
  if (requested > 0) {
    return static_cast<size_t>(requested);
  }
  return std::max(1U, std::thread::hardware_concurrency());
}

}  // namespace

// ------------------------------------------------------------------- LDLT --

void Ldlt::Analyze(const Csc& a, const std::vector<int>& perm, int num_threads) {
  n_ = a.cols;
  perm_ = perm;
  if (perm_.empty()) {
    perm_.resize(static_cast<size_t>(n_));
    std::iota(perm_.begin(), perm_.end(), 0);
  }
  pinv_.assign(static_cast<size_t>(n_), 0);
  for (int i = 0; i < n_; ++i) {
    pinv_[static_cast<size_t>(perm_[static_cast<size_t>(i)])] = i;
  }
  // Upper triangle of P A P^T from the lower triangle of A
  // (Eigen::internal::permute_symm_to_symm<Lower, Upper>), rows sorted.
  upper_.rows = upper_.cols = n_;
  std::vector<int> count(static_cast<size_t>(n_) + 1, 0);
  for (int j = 0; j < n_; ++j) {
    for (int p = a.outer[static_cast<size_t>(j)]; p < a.outer[static_cast<size_t>(j) + 1]; ++p) {
      const int i = a.inner[static_cast<size_t>(p)];
      if (i < j) {
        continue;
      }
      const int ip = pinv_[static_cast<size_t>(i)];
      const int jp = pinv_[static_cast<size_t>(j)];
      ++count[static_cast<size_t>(std::max(ip, jp)) + 1];
    }
  }
  for (int k = 0; k < n_; ++k) {
    count[static_cast<size_t>(k) + 1] += count[static_cast<size_t>(k)];
  }
  upper_.outer = count;
  upper_.inner.assign(static_cast<size_t>(count.back()), 0);
  upper_.values.assign(static_cast<size_t>(count.back()), 0.0);
  std::vector<int> fill(count.begin(), count.end() - 1);
  for (int j = 0; j < n_; ++j) {
    for (int p = a.outer[static_cast<size_t>(j)]; p < a.outer[static_cast<size_t>(j) + 1]; ++p) {
      const int i = a.inner[static_cast<size_t>(p)];
      if (i < j) {
        continue;
      }
      const int ip = pinv_[static_cast<size_t>(i)];
      const int jp = pinv_[static_cast<size_t>(j)];
      const int col = std::max(ip, jp);
      upper_.inner[static_cast<size_t>(fill[static_cast<size_t>(col)]++)] = std::min(ip, jp);
    }
  }
  for (int k = 0; k < n_; ++k) {
    std::sort(upper_.inner.begin() + upper_.outer[static_cast<size_t>(k)],
              upper_.inner.begin() + upper_.outer[static_cast<size_t>(k) + 1]);
  }
  // Elimination tree and column counts (Eigen SimplicialCholeskyBase::
  // analyzePattern_preordered, after T. A. Davis' LDL).
  parent_.assign(static_cast<size_t>(n_), -1);
  std::vector<int> tags(static_cast<size_t>(n_), -1);
  std::vector<int> nz(static_cast<size_t>(n_), 0);
  for (int k = 0; k < n_; ++k) {
    tags[static_cast<size_t>(k)] = k;
    for (int p = upper_.outer[static_cast<size_t>(k)]; p < upper_.outer[static_cast<size_t>(k) + 1]; ++p) {
      int i = upper_.inner[static_cast<size_t>(p)];
      if (i < k) {
        for (; tags[static_cast<size_t>(i)] != k; i = parent_[static_cast<size_t>(i)]) {
          if (parent_[static_cast<size_t>(i)] == -1) {
            parent_[static_cast<size_t>(i)] = k;
          }
          ++nz[static_cast<size_t>(i)];
          tags[static_cast<size_t>(i)] = k;
        }
      }
    }
  }
  lp_.assign(static_cast<size_t>(n_) + 1, 0);
  for (int k = 0; k < n_; ++k) {
    lp_[static_cast<size_t>(k) + 1] = lp_[static_cast<size_t>(k)] + nz[static_cast<size_t>(k)];
  }
  li_.assign(static_cast<size_t>(lp_.back()), 0);
  lx_.assign(static_cast<size_t>(lp_.back()), 0.0);
  d_.assign(static_cast<size_t>(n_), 0.0);
  BuildSchedule(num_threads);
}

// parallel_ldlt.hpp:59-148: subtree split until pieces balance, serial trunk,
// longest-processing-time assignment of subtrees to workers.
void Ldlt::BuildSchedule(int num_threads_in) {
  const size_t num_threads = static_cast<size_t>(std::max(1, num_threads_in));
  const int n = n_;
  thread_rows_.assign(num_threads, {});
  trunk_rows_.clear();
  if (num_threads <= 1 || n < 256) {
    thread_rows_.resize(1);
    thread_rows_[0].resize(static_cast<size_t>(n));
    std::iota(thread_rows_[0].begin(), thread_rows_[0].end(), 0);
    return;
  }
  std::vector<std::vector<int>> children(static_cast<size_t>(n));
  std::vector<int> subtree(static_cast<size_t>(n), 1);
  std::vector<int> roots;
  for (int i = 0; i < n; ++i) {
    const int p = parent_[static_cast<size_t>(i)];
    if (p >= 0) {
      children[static_cast<size_t>(p)].push_back(i);
    } else {
      roots.push_back(i);
    }
  }
  for (int i = 0; i < n; ++i) {
    const int p = parent_[static_cast<size_t>(i)];
    if (p >= 0) {
      subtree[static_cast<size_t>(p)] += subtree[static_cast<size_t>(i)];
    }
  }
  auto by_size = [&subtree](int a, int b) { return subtree[static_cast<size_t>(a)] < subtree[static_cast<size_t>(b)]; };
  std::priority_queue<int, std::vector<int>, decltype(by_size)> heap(by_size);
  for (const int r : roots) {
    heap.push(r);
  }
  std::vector<int> subtree_roots;
  const int target = std::max(1, n / static_cast<int>(num_threads * 8));
  while (!heap.empty()) {
    const int top = heap.top();
    const bool splittable = !children[static_cast<size_t>(top)].empty();
    if (subtree[static_cast<size_t>(top)] <= target || subtree_roots.size() + heap.size() >= num_threads * 16 ||
        !splittable) {
      break;
    }
    heap.pop();
    trunk_rows_.push_back(top);
    for (const int c : children[static_cast<size_t>(top)]) {
      heap.push(c);
    }
  }
  while (!heap.empty()) {
    subtree_roots.push_back(heap.top());
    heap.pop();
  }
  std::sort(subtree_roots.begin(), subtree_roots.end(),
            [&](int a, int b) { return subtree[static_cast<size_t>(a)] > subtree[static_cast<size_t>(b)]; });
  std::vector<long> load(num_threads, 0);
  std::vector<int> stack;
  for (const int r : subtree_roots) {
    const size_t t = static_cast<size_t>(std::min_element(load.begin(), load.end()) - load.begin());
    load[t] += subtree[static_cast<size_t>(r)];
    stack.push_back(r);
    while (!stack.empty()) {
      const int v = stack.back();
      stack.pop_back();
      thread_rows_[t].push_back(v);
      for (const int c : children[static_cast<size_t>(v)]) {
        stack.push_back(c);
      }
    }
  }
  for (auto& rows : thread_rows_) {
    std::sort(rows.begin(), rows.end());
  }
  std::sort(trunk_rows_.begin(), trunk_rows_.end());
}

// parallel_ldlt.hpp:150-244 (row kernel :165-206).
bool Ldlt::Factorize(const Csc& a) {
  // Refill the permuted upper triangle with the current values.
  for (int j = 0; j < n_; ++j) {
    for (int p = a.outer[static_cast<size_t>(j)]; p < a.outer[static_cast<size_t>(j) + 1]; ++p) {
      const int i = a.inner[static_cast<size_t>(p)];
      if (i < j) {
        continue;
      }
      const int ip = pinv_[static_cast<size_t>(i)];
      const int jp = pinv_[static_cast<size_t>(j)];
      const int col = std::max(ip, jp);
      const int row = std::min(ip, jp);
      // Locate row in the sorted column.
      const auto begin = upper_.inner.begin() + upper_.outer[static_cast<size_t>(col)];
      const auto end = upper_.inner.begin() + upper_.outer[static_cast<size_t>(col) + 1];
      const auto it = std::lower_bound(begin, end, row);
      upper_.values[static_cast<size_t>(it - upper_.inner.begin())] = a.values[static_cast<size_t>(p)];
    }
  }
  const int size = n_;
  std::vector<int> nonzeros_per_col(static_cast<size_t>(n_), 0);
  const double shift_scale = 1.0;
  const double shift_offset = 0.0;
  std::atomic<bool> ok{true};
  const auto process_row = [&](int k, double* y, int* pattern, int* tags) {
    y[k] = 0.0;
    int top = size;
    tags[k] = k;
    nonzeros_per_col[static_cast<size_t>(k)] = 0;
    for (int p = upper_.outer[static_cast<size_t>(k)]; p < upper_.outer[static_cast<size_t>(k) + 1]; ++p) {
      int i = upper_.inner[static_cast<size_t>(p)];
      if (i <= k) {
        y[i] += upper_.values[static_cast<size_t>(p)];
        int len = 0;
        for (; tags[i] != k; i = parent_[static_cast<size_t>(i)]) {
          pattern[len++] = i;
          tags[i] = k;
        }
        while (len > 0) {
          pattern[--top] = pattern[--len];
        }
      }
    }
    double d = std::fma(y[k], shift_scale, shift_offset);
    y[k] = 0.0;
    for (; top < size; ++top) {
      const int i = pattern[top];
      const double yi = y[i];
      y[i] = 0.0;
      const double l_ki = yi / d_[static_cast<size_t>(i)];
      const int p2 = lp_[static_cast<size_t>(i)] + nonzeros_per_col[static_cast<size_t>(i)];
      int p = lp_[static_cast<size_t>(i)];
      for (; p < p2; ++p) {
        y[li_[static_cast<size_t>(p)]] = std::fma(-lx_[static_cast<size_t>(p)], yi, y[li_[static_cast<size_t>(p)]]);
      }
      const double diag_update = l_ki * yi;
      d -= diag_update;
      li_[static_cast<size_t>(p)] = k;
      lx_[static_cast<size_t>(p)] = l_ki;
      ++nonzeros_per_col[static_cast<size_t>(i)];
    }
    d_[static_cast<size_t>(k)] = d;
    return d != 0.0;
  };
  const auto process_rows = [&](const std::vector<int>& rows) {
    std::vector<double> y(static_cast<size_t>(size), 0.0);
    std::vector<int> pattern(static_cast<size_t>(size), 0);
    std::vector<int> tags(static_cast<size_t>(size), -1);
    for (const int k : rows) {
      if (!ok.load(std::memory_order_relaxed)) {
        return;
      }
      if (!process_row(k, y.data(), pattern.data(), tags.data())) {
        ok.store(false, std::memory_order_relaxed);
        return;
      }
    }
  };
  if (thread_rows_.size() <= 1) {
    if (!thread_rows_.empty()) {
      process_rows(thread_rows_[0]);
    }
  } else {
    std::vector<std::thread> workers;
    for (const auto& rows : thread_rows_) {
      workers.emplace_back(process_rows, std::cref(rows));
    }
    for (auto& w : workers) {
      w.join();
    }
  }
  if (ok.load()) {
    process_rows(trunk_rows_);
  }
  return ok.load();
}

// Eigen SimplicialLDLT::_solve_impl: permute, unit-lower solve (column
// oriented, skipping zero pivots of the right-hand side), diagonal inverse
// times vector, unit-upper solve (row oriented), inverse permute.
std::vector<double> Ldlt::Solve(const std::vector<double>& b) const {
  std::vector<double> x(static_cast<size_t>(n_));
  for (int i = 0; i < n_; ++i) {
    x[static_cast<size_t>(i)] = b[static_cast<size_t>(perm_[static_cast<size_t>(i)])];
  }
  for (int j = 0; j < n_; ++j) {
    const double tmp = x[static_cast<size_t>(j)];
    if (tmp != 0.0) {
      for (int p = lp_[static_cast<size_t>(j)]; p < lp_[static_cast<size_t>(j) + 1]; ++p) {
        x[static_cast<size_t>(li_[static_cast<size_t>(p)])] -= tmp * lx_[static_cast<size_t>(p)];
      }
    }
  }
  for (int i = 0; i < n_; ++i) {
    x[static_cast<size_t>(i)] = (1.0 / d_[static_cast<size_t>(i)]) * x[static_cast<size_t>(i)];
  }
  for (int j = n_ - 1; j >= 0; --j) {
    double tmp = x[static_cast<size_t>(j)];
    for (int p = lp_[static_cast<size_t>(j)]; p < lp_[static_cast<size_t>(j) + 1]; ++p) {
      tmp -= lx_[static_cast<size_t>(p)] * x[static_cast<size_t>(li_[static_cast<size_t>(p)])];
    }
    x[static_cast<size_t>(j)] = tmp;
  }
  std::vector<double> out(static_cast<size_t>(n_));
  for (int i = 0; i < n_; ++i) {
    out[static_cast<size_t>(perm_[static_cast<size_t>(i)])] = x[static_cast<size_t>(i)];
  }
  return out;
}

// ----------------------------------------------------------- ND ordering --

std::vector<int> GridNestedDissection(const Problem& problem) {
  const GridMap& map = problem.map();
  std::vector<int> order;
  order.reserve(static_cast<size_t>(problem.num_parameters()));
  // Recursive bisection of [w0,w1) x [h0,h1): halves first, then the
  // separating grid line (one node wide separates the 9-point stencil).
  std::function<void(int, int, int, int)> dissect = [&](int w0, int w1, int h0, int h1) {
    const int width = w1 - w0;
    const int height = h1 - h0;
    if (width <= 0 || height <= 0) {
      return;
    }
    if (width * height <= 36 || (width < 3 && height < 3)) {
      for (int h = h0; h < h1; ++h) {
        for (int w = w0; w < w1; ++w) {
          const int col = problem.NodeColumn(map.NodeId(w, h));
          if (col >= 0) {
            order.push_back(col);
          }
        }
      }
      return;
    }
    if (width >= height) {
      const int mid = w0 + width / 2;
      dissect(w0, mid, h0, h1);
      dissect(mid + 1, w1, h0, h1);
      for (int h = h0; h < h1; ++h) {
        const int col = problem.NodeColumn(map.NodeId(mid, h));
        if (col >= 0) {
          order.push_back(col);
        }
      }
    } else {
      const int mid = h0 + height / 2;
      dissect(w0, w1, h0, mid);
      dissect(w0, w1, mid + 1, h1);
      for (int w = w0; w < w1; ++w) {
        const int col = problem.NodeColumn(map.NodeId(w, mid));
        if (col >= 0) {
          order.push_back(col);
        }
      }
    }
  };
  dissect(0, map.nx(), 0, map.ny());
  for (int c = problem.num_active_nodes(); c < problem.num_parameters(); ++c) {
    order.push_back(c);
  }
  return order;
}

// ----------------------------------------------------------- LM assembly --

namespace {

struct RowEntries {
  int count{0};
  std::array<int, 7> col{};
  std::array<double, 7> val{};
};

/// Rows as CSR (row order = spec order), plus the residual vector
/// (lm_solver.cpp:30-82 and the odometry tail :275-296).
void AssembleRows(const Problem& problem, size_t num_threads, std::vector<double>& residuals,
                  std::vector<int>& row_ptr, std::vector<int>& cols, std::vector<double>& vals,
                  std::vector<int>& point_cell) {
  const auto& points = problem.point_specs();
  const auto& eik = problem.eikonal_specs();
  const auto& odom = problem.odom_specs();
  const int np = static_cast<int>(points.size());
  const int ne = static_cast<int>(eik.size());
  const int num_rows = problem.num_residuals();
  residuals.assign(static_cast<size_t>(num_rows), 0.0);
  point_cell.assign(static_cast<size_t>(np), -1);
  std::vector<RowEntries> rows(static_cast<size_t>(num_rows));
  const GridMap& map = problem.map();
  ParallelRanges(static_cast<size_t>(np), num_threads, [&](size_t begin, size_t end) {
    for (size_t s = begin; s < end; ++s) {
      const PointSpec& spec = points[s];
      const PointResidualJacobian eval = EvalPointResidual(
          map, problem.poses()[static_cast<size_t>(spec.frame)], spec.point_sensor, spec.expected_sdf,
          problem.smooth_gradient(), problem.smooth_gradient_step());
      const double weighted = spec.sqrt_weight * eval.residual;
      const double sw = std::sqrt(problem.HuberWeight(weighted));
      residuals[s] = sw * weighted;
      if (!eval.valid) {
        continue;
      }
      point_cell[s] = eval.cell_h * map.nx() + eval.cell_w;
      const double scale = sw * spec.sqrt_weight;
      RowEntries& row = rows[s];
      for (size_t k = 0; k < 4; ++k) {
        const int col = problem.NodeColumn(eval.node_ids[k]);
        if (col >= 0) {
          row.col[static_cast<size_t>(row.count)] = col;
          row.val[static_cast<size_t>(row.count)] = scale * eval.d_nodes[k];
          ++row.count;
        }
      }
      if (spec.frame >= 1) {
        const int pose_col = problem.PoseColumn(spec.frame);
        for (int k = 0; k < 3; ++k) {
          row.col[static_cast<size_t>(row.count)] = pose_col + k;
          row.val[static_cast<size_t>(row.count)] = scale * eval.d_pose[static_cast<size_t>(k)];
          ++row.count;
        }
      }
    }
  });
  ParallelRanges(static_cast<size_t>(ne), num_threads, [&](size_t begin, size_t end) {
    for (size_t e = begin; e < end; ++e) {
      const EikonalSpec& spec = eik[e];
      const EikonalResidualJacobian eval = EvalEikonalResidual(map, spec.w, spec.h, spec.normal);
      const size_t row_idx = static_cast<size_t>(np) + e;
      residuals[row_idx] = spec.sqrt_weight * eval.residual;
      RowEntries& row = rows[row_idx];
      for (size_t k = 0; k < 3; ++k) {
        const int col = problem.NodeColumn(eval.node_ids[k]);
        if (col >= 0) {
          row.col[static_cast<size_t>(row.count)] = col;
          row.val[static_cast<size_t>(row.count)] = spec.sqrt_weight * eval.d_nodes[k];
          ++row.count;
        }
      }
    }
  });
  for (size_t o = 0; o < odom.size(); ++o) {
    const OdomSpec& spec = odom[o];
    const OdomResidualJacobian eval = EvalOdomResidual(
        problem.poses()[static_cast<size_t>(spec.frame_i)], problem.poses()[static_cast<size_t>(spec.frame_j)],
        spec.measurement);
    const size_t row0 = static_cast<size_t>(np + ne) + 3 * o;
    for (int r = 0; r < 3; ++r) {
      residuals[row0 + static_cast<size_t>(r)] = spec.sqrt_weight * eval.residual[static_cast<size_t>(r)];
      RowEntries& row = rows[row0 + static_cast<size_t>(r)];
      // Triplets are (row, col) pairs; setFromTriplets sorts them, so the
      // i block and the j block land in column order whatever i, j are.
      std::array<std::pair<int, double>, 6> tmp{};
      int cnt = 0;
      if (spec.frame_i >= 1) {
        const int col_i = problem.PoseColumn(spec.frame_i);
        for (int c = 0; c < 3; ++c) {
          tmp[static_cast<size_t>(cnt++)] = {col_i + c, spec.sqrt_weight * eval.d_pose_i[static_cast<size_t>(r)][static_cast<size_t>(c)]};
        }
      }
      const int col_j = problem.PoseColumn(spec.frame_j);
      for (int c = 0; c < 3; ++c) {
        tmp[static_cast<size_t>(cnt++)] = {col_j + c, spec.sqrt_weight * eval.d_pose_j[static_cast<size_t>(r)][static_cast<size_t>(c)]};
      }
      for (int a = 1; a < cnt; ++a) {
        for (int b = a; b > 0 && tmp[static_cast<size_t>(b)].first < tmp[static_cast<size_t>(b - 1)].first; --b) {
          std::swap(tmp[static_cast<size_t>(b)], tmp[static_cast<size_t>(b - 1)]);
        }
      }
      for (int q = 0; q < cnt; ++q) {
        row.col[static_cast<size_t>(q)] = tmp[static_cast<size_t>(q)].first;
        row.val[static_cast<size_t>(q)] = tmp[static_cast<size_t>(q)].second;
      }
      row.count = cnt;
    }
  }
  row_ptr.assign(static_cast<size_t>(num_rows) + 1, 0);
  for (int r = 0; r < num_rows; ++r) {
    row_ptr[static_cast<size_t>(r) + 1] = row_ptr[static_cast<size_t>(r)] + rows[static_cast<size_t>(r)].count;
  }
  cols.resize(static_cast<size_t>(row_ptr.back()));
  vals.resize(static_cast<size_t>(row_ptr.back()));
  for (int r = 0; r < num_rows; ++r) {
    const RowEntries& row = rows[static_cast<size_t>(r)];
    for (int q = 0; q < row.count; ++q) {
      cols[static_cast<size_t>(row_ptr[static_cast<size_t>(r)] + q)] = row.col[static_cast<size_t>(q)];
      vals[static_cast<size_t>(row_ptr[static_cast<size_t>(r)] + q)] = row.val[static_cast<size_t>(q)];
    }
  }
}

/// setFromTriplets: CSC with rows ascending within each column.
Csc RowsToCsc(int num_rows, int num_cols, const std::vector<int>& row_ptr, const std::vector<int>& cols,
              const std::vector<double>& vals) {
  Csc m;
  m.rows = num_rows;
  m.cols = num_cols;
  m.outer.assign(static_cast<size_t>(num_cols) + 1, 0);
  for (const int c : cols) {
    ++m.outer[static_cast<size_t>(c) + 1];
  }
  for (int c = 0; c < num_cols; ++c) {
    m.outer[static_cast<size_t>(c) + 1] += m.outer[static_cast<size_t>(c)];
  }
  m.inner.resize(cols.size());
  m.values.resize(cols.size());
  std::vector<int> fill(m.outer.begin(), m.outer.end() - 1);
  for (int r = 0; r < num_rows; ++r) {
    for (int p = row_ptr[static_cast<size_t>(r)]; p < row_ptr[static_cast<size_t>(r) + 1]; ++p) {
      const int c = cols[static_cast<size_t>(p)];
      const int dst = fill[static_cast<size_t>(c)]++;
      m.inner[static_cast<size_t>(dst)] = r;
      m.values[static_cast<size_t>(dst)] = vals[static_cast<size_t>(p)];
    }
  }
  return m;
}

/// lm_solver.cpp:113-172 (per-column accumulation in ascending k, first touch
/// assigns) followed by the damping of :321-330, which inserts missing
/// diagonal entries.
Csc NormalMatrix(const Csc& jac, const std::vector<int>& row_ptr, const std::vector<int>& rcols,
                 const std::vector<double>& rvals, double lambda, bool marquardt, size_t num_threads) {
  const int n = jac.cols;
  std::vector<std::vector<int>> col_idx(static_cast<size_t>(n));
  std::vector<std::vector<double>> col_val(static_cast<size_t>(n));
  ParallelRanges(static_cast<size_t>(n), num_threads, [&](size_t begin, size_t end) {
    std::vector<char> mask(static_cast<size_t>(n), 0);
    std::vector<double> values(static_cast<size_t>(n), 0.0);
    std::vector<int> indices;
    for (size_t j = begin; j < end; ++j) {
      indices.clear();
      for (int q = jac.outer[j]; q < jac.outer[j + 1]; ++q) {
        const double y = jac.values[static_cast<size_t>(q)];
        const int k = jac.inner[static_cast<size_t>(q)];
        for (int p = row_ptr[static_cast<size_t>(k)]; p < row_ptr[static_cast<size_t>(k) + 1]; ++p) {
          const size_t i = static_cast<size_t>(rcols[static_cast<size_t>(p)]);
          const double x = rvals[static_cast<size_t>(p)];
          if (mask[i] == 0) {
            mask[i] = 1;
            values[i] = x * y;
            indices.push_back(static_cast<int>(i));
          } else {
            values[i] += x * y;
          }
        }
      }
      std::sort(indices.begin(), indices.end());
      auto& oi = col_idx[j];
      auto& ov = col_val[j];
      for (const int i : indices) {
        oi.push_back(i);
        ov.push_back(values[static_cast<size_t>(i)]);
        mask[static_cast<size_t>(i)] = 0;
      }
      // coeffRef(d, d) inserts a missing diagonal as an explicit 0.
      const auto pos = std::lower_bound(oi.begin(), oi.end(), static_cast<int>(j));
      if (pos == oi.end() || *pos != static_cast<int>(j)) {
        const auto off = pos - oi.begin();
        oi.insert(pos, static_cast<int>(j));
        ov.insert(ov.begin() + off, 0.0);
      }
      for (size_t e = 0; e < oi.size(); ++e) {
        if (oi[e] == static_cast<int>(j)) {
          if (marquardt) {
            const double diag = std::max(ov[e], 1e-12);
            ov[e] += lambda * diag;
          } else {
            ov[e] += lambda;
          }
        }
      }
    }
  });
  Csc out;
  out.rows = out.cols = n;
  out.outer.assign(static_cast<size_t>(n) + 1, 0);
  for (int j = 0; j < n; ++j) {
    out.outer[static_cast<size_t>(j) + 1] = out.outer[static_cast<size_t>(j)] + static_cast<int>(col_idx[static_cast<size_t>(j)].size());
  }
  out.inner.reserve(static_cast<size_t>(out.outer.back()));
  out.values.reserve(static_cast<size_t>(out.outer.back()));
  for (int j = 0; j < n; ++j) {
    out.inner.insert(out.inner.end(), col_idx[static_cast<size_t>(j)].begin(), col_idx[static_cast<size_t>(j)].end());
    out.values.insert(out.values.end(), col_val[static_cast<size_t>(j)].begin(), col_val[static_cast<size_t>(j)].end());
  }
  return out;
}

/// lm_solver.cpp:178-197: two accumulators alternating over the column.
std::vector<double> NegAtb(const Csc& jac, const std::vector<double>& r, size_t num_threads) {
  std::vector<double> rhs(static_cast<size_t>(jac.cols));
  ParallelRanges(static_cast<size_t>(jac.cols), num_threads, [&](size_t begin, size_t end) {
    for (size_t j = begin; j < end; ++j) {
      double tmp_a = 0.0;
      double tmp_b = 0.0;
      int q = jac.outer[j];
      const int qe = jac.outer[j + 1];
      while (q < qe) {
        tmp_a += jac.values[static_cast<size_t>(q)] * r[static_cast<size_t>(jac.inner[static_cast<size_t>(q)])];
        ++q;
        if (q < qe) {
          tmp_b += jac.values[static_cast<size_t>(q)] * r[static_cast<size_t>(jac.inner[static_cast<size_t>(q)])];
          ++q;
        }
      }
      rhs[j] = -(tmp_a + tmp_b);
    }
  });
  return rhs;
}

double Seconds(std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
  return std::chrono::duration<double>(b - a).count();
}

double Norm(const std::vector<double>& v) {
  double s = 0.0;
  for (const double x : v) {
    s += x * x;
  }
  return std::sqrt(s);
}

double Dot(const std::vector<double>& a, const std::vector<double>& b) {
  double s = 0.0;
  for (size_t i = 0; i < a.size(); ++i) {
    s += a[i] * b[i];
  }
  return s;
}

}  // namespace

Linearization Linearize(const Problem& problem, double lambda, bool marquardt, int num_threads,
                        bool compute_step) {
  const size_t threads = ResolveThreads(num_threads);
  Linearization lin;
  std::vector<int> row_ptr;
  std::vector<int> rcols;
  std::vector<double> rvals;
  AssembleRows(problem, threads, lin.residuals, row_ptr, rcols, rvals, lin.point_cell);
  lin.jacobian = RowsToCsc(problem.num_residuals(), problem.num_parameters(), row_ptr, rcols, rvals);
  lin.normal = NormalMatrix(lin.jacobian, row_ptr, rcols, rvals, lambda, marquardt, threads);
  lin.rhs = NegAtb(lin.jacobian, lin.residuals, threads);
  if (compute_step) {
    Ldlt ldlt;
    ldlt.Analyze(lin.normal, GridNestedDissection(problem), static_cast<int>(threads));
    lin.factor_ok = ldlt.Factorize(lin.normal);
    lin.nnz_l = ldlt.nnz_l();
    if (lin.factor_ok) {
      lin.step = ldlt.Solve(lin.rhs);
    }
  }
  return lin;
}

// lm_solver.cpp:201-434
SolveResult SolveLm(Problem& problem, const SolverOptions& options) {
  using Clock = std::chrono::steady_clock;
  const auto start_time = Clock::now();
  SolveResult result;
  const size_t threads = ResolveThreads(options.num_threads);
  auto t0 = Clock::now();
  result.initial_cost = problem.Cost();
  result.phase_seconds[4] += Seconds(t0, Clock::now());
  result.cost_history.push_back(result.initial_cost);
  double lambda = options.lambda_init;
  double previous_cost = result.initial_cost;
  double nielsen_nu = 2.0;
  Ldlt ldlt;
  std::vector<int> pattern_outer;
  std::vector<int> pattern_inner;
  const std::vector<int> perm = GridNestedDissection(problem);
  for (int iter = 0; iter < options.max_iterations; ++iter) {
    t0 = Clock::now();
    std::vector<double> residuals;
    std::vector<int> row_ptr;
    std::vector<int> rcols;
    std::vector<double> rvals;
    std::vector<int> cells;
    AssembleRows(problem, threads, residuals, row_ptr, rcols, rvals, cells);
    const Csc jac = RowsToCsc(problem.num_residuals(), problem.num_parameters(), row_ptr, rcols, rvals);
    auto t1 = Clock::now();
    result.phase_seconds[0] += Seconds(t0, t1);
    const Csc normal = NormalMatrix(jac, row_ptr, rcols, rvals, lambda, options.marquardt_scaling, threads);
    const std::vector<double> rhs = NegAtb(jac, residuals, threads);
    auto t2 = Clock::now();
    result.phase_seconds[1] += Seconds(t1, t2);
    const bool same_pattern = pattern_outer == normal.outer && pattern_inner == normal.inner;
    if (!same_pattern) {
      ldlt.Analyze(normal, perm, static_cast<int>(threads));
      pattern_outer = normal.outer;
      pattern_inner = normal.inner;
    }
    if (!ldlt.Factorize(normal)) {
      throw std::runtime_error("sparse Cholesky factorization failed");
    }
    auto t3 = Clock::now();
    result.phase_seconds[2] += Seconds(t2, t3);
    const std::vector<double> step = ldlt.Solve(rhs);
    auto t4 = Clock::now();
    result.phase_seconds[3] += Seconds(t3, t4);
    std::vector<double> map_backup;
    std::vector<Pose2> pose_backup;
    if (options.reject_worse_steps || options.trust_region) {
      map_backup = problem.map().values();
      pose_backup = problem.poses();
    }
    problem.ApplyStep(step);
    const double cost = problem.Cost();
    result.phase_seconds[4] += Seconds(t4, Clock::now());
    result.iterations = iter + 1;
    if (Norm(step) < options.step_tolerance) {
      result.cost_history.push_back(cost);
      result.final_cost = cost;
      result.converged = true;
      break;
    }
    double current_cost = cost;
    if (options.trust_region) {
      std::vector<double> tmp(step.size());
      for (size_t i = 0; i < step.size(); ++i) {
        tmp[i] = lambda * step[i] + rhs[i];
      }
      const double predicted = Dot(step, tmp);
      const double rho = predicted > 0.0 ? (previous_cost - cost) / predicted : -1.0;
      if (rho > 0.0) {
        previous_cost = cost;
        const double shrink = 1.0 - std::pow(2.0 * rho - 1.0, 3);
        lambda = std::max(lambda * std::max(1.0 / 3.0, shrink), 1e-7);
        nielsen_nu = 2.0;
      } else {
        problem.map().values() = map_backup;
        problem.poses() = pose_backup;
        current_cost = previous_cost;
        lambda *= nielsen_nu;
        nielsen_nu *= 2.0;
      }
    } else if (cost < previous_cost) {
      lambda /= options.lambda_factor;
      previous_cost = cost;
    } else {
      lambda *= options.lambda_factor;
      if (options.reject_worse_steps) {
        problem.map().values() = map_backup;
        problem.poses() = pose_backup;
        current_cost = previous_cost;
      } else {
        previous_cost = cost;
      }
    }
    result.cost_history.push_back(current_cost);
    result.final_cost = current_cost;
  }
  if (result.iterations == 0) {
    result.final_cost = result.initial_cost;
  }
  result.duration_seconds = Seconds(start_time, Clock::now());
  return result;
}

}  // namespace oracle
