// Host-side construction and validation of LM problems.
//
// BuildProblem follows Problem::Problem (src/problem/problem.cpp:11-115):
// point specs frame by frame (scan points, then hallucinated points,
// src/core/hallucination.cpp:5-28), the active-region index maps
// (problem.cpp:39-70), Eikonal specs from k-NN PCA normals
// (src/core/normals.cpp:70-220; exact k-NN with neighbours ordered by squared
// distance then index, and a closed-form 2x2 eigen-decomposition), then the
// odometry and relation specs (problem.cpp:96-114). Setup work, run once per
// problem on the host.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <queue>
#include <utility>

#include "internal.h"

namespace sdfgpu {

namespace {

struct P2 {
  double x;
  double y;
};

/// Pose2::Apply (src/core/pose.hpp:28-30): (c px - s py) + tx, (s px + c py) + ty.
inline P2 ApplyPose(const double* pose, P2 p) {
  const double c = std::cos(pose[2]);
  const double s = std::sin(pose[2]);
  return {(c * p.x + (-s) * p.y) + pose[0], (s * p.x + c * p.y) + pose[1]};
}

/// GridMap::Locate (src/core/grid_map.hpp:58-70): cell (w, h) or false.
inline bool LocateCell(const HostProblem& hp, P2 g, int* w, int* h) {
  const double fx = (g.x - hp.min_x) / hp.dx();
  const double fy = (g.y - hp.min_y) / hp.dy();
  // NaN coordinates count as outside (never converted to a cell)
  if (!(fx >= 0.0) || !(fy >= 0.0) || !(fx <= hp.nx - 1) || !(fy <= hp.ny - 1)) {
    return false;
  }
  *w = std::min(static_cast<int>(fx), hp.nx - 2);
  *h = std::min(static_cast<int>(fy), hp.ny - 2);
  return true;
}

/// Exact k nearest neighbours on a bucket grid; ties broken by index.
class BucketKnn {
 public:
  explicit BucketKnn(const std::vector<P2>& pts) : pts_(pts) {
    double lo_x = std::numeric_limits<double>::max();
    double lo_y = lo_x;
    double hi_x = -lo_x;
    double hi_y = -lo_x;
    for (const P2& p : pts) {
      lo_x = std::min(lo_x, p.x);
      lo_y = std::min(lo_y, p.y);
      hi_x = std::max(hi_x, p.x);
      hi_y = std::max(hi_y, p.y);
    }
    if (pts.empty()) {
      lo_x = lo_y = 0.0;
      hi_x = hi_y = 1.0;
    }
    ox_ = lo_x;
    oy_ = lo_y;
    const double ex = std::max(hi_x - lo_x, 1e-9);
    const double ey = std::max(hi_y - lo_y, 1e-9);
    const double n = std::max<double>(1.0, static_cast<double>(pts.size()));
    cell_ = std::max({std::sqrt(ex * ey / n) * 1.5, ex / 2048.0, ey / 2048.0, 1e-9});
    gx_ = std::min(2048, static_cast<int>(ex / cell_) + 1);
    gy_ = std::min(2048, static_cast<int>(ey / cell_) + 1);
    start_.assign(static_cast<size_t>(gx_) * gy_ + 1, 0);
    for (const P2& p : pts) {
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

  /// The grid's parameters and arrays (for the device search).
  void Export(KnnBuckets* b) const {
    b->ox = ox_;
    b->oy = oy_;
    b->cell = cell_;
    b->gx = gx_;
    b->gy = gy_;
    b->start = start_;
    b->items = items_;
  }

  void Query(P2 q, size_t k, std::vector<std::pair<double, int>>& out) const {
    out.clear();
    if (pts_.empty() || k == 0) {
      return;
    }
    const size_t want = std::min(k, pts_.size());
    const int cx = CellOf((q.x - ox_) / cell_, gx_);
    const int cy = CellOf((q.y - oy_) / cell_, gy_);
    const double bx0 = ox_ + cx * cell_;
    const double by0 = oy_ + cy * cell_;
    const double inner = std::max(0.0, std::min({q.x - bx0, bx0 + cell_ - q.x, q.y - by0, by0 + cell_ - q.y}));
    std::priority_queue<std::pair<double, int>> heap;  // max-heap on (d2, idx)
    const int max_ring = std::max(gx_, gy_);
    for (int r = 0; r <= max_ring; ++r) {
      const int y0 = cy - r;
      const int y1 = cy + r;
      for (int y = std::max(0, y0); y <= std::min(gy_ - 1, y1); ++y) {
        const bool full = (y == y0 || y == y1);
        const int step = full ? 1 : 2 * r;
        for (int x = cx - r; x <= cx + r; x += (step > 0 ? step : 1)) {
          if (x < 0 || x >= gx_) {
            continue;
          }
          const size_t b = static_cast<size_t>(y) * gx_ + x;
          for (int s = start_[b]; s < start_[b + 1]; ++s) {
            const int idx = items_[static_cast<size_t>(s)];
            const double ddx = pts_[static_cast<size_t>(idx)].x - q.x;
            const double ddy = pts_[static_cast<size_t>(idx)].y - q.y;
            const std::pair<double, int> cand{ddx * ddx + ddy * ddy, idx};
            if (heap.size() < want) {
              heap.push(cand);
            } else if (cand < heap.top()) {
              heap.pop();
              heap.push(cand);
            }
          }
        }
      }
      if (heap.size() == want) {
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
  /// floor(f) clamped to [0, g - 1]; NaN goes to 0. (The comparisons come
  /// first so that no out-of-range value is converted.)
  static int CellOf(double f, int g) {
    if (!(f > 0.0)) {
      return 0;
    }
    if (f >= static_cast<double>(g - 1)) {
      return g - 1;
    }
    return static_cast<int>(f);
  }
  int Bucket(P2 p) const { return CellOf((p.y - oy_) / cell_, gy_) * gx_ + CellOf((p.x - ox_) / cell_, gx_); }
  const std::vector<P2>& pts_;
  double ox_{0.0};
  double oy_{0.0};
  double cell_{1.0};
  int gx_{1};
  int gy_{1};
  std::vector<int> start_;
  std::vector<int> items_;
};

/// PCA normal and cornerness of the k neighbours of points[i]
/// (src/core/normals.cpp:70-101), oriented toward `origin`.
void PcaNormal(const std::vector<P2>& points, const BucketKnn& knn, size_t i, size_t k, P2 origin,
               P2* normal_out, double* corner_out, std::vector<std::pair<double, int>>& nb) {
  knn.Query(points[i], k, nb);
  const size_t found = nb.size();
  double mx = 0.0;
  double my = 0.0;
  for (size_t j = 0; j < found; ++j) {
    mx += points[static_cast<size_t>(nb[j].second)].x;
    my += points[static_cast<size_t>(nb[j].second)].y;
  }
  mx /= static_cast<double>(found);
  my /= static_cast<double>(found);
  double sxx = 0.0;
  double sxy = 0.0;
  double syy = 0.0;
  for (size_t j = 0; j < found; ++j) {
    const double dx = points[static_cast<size_t>(nb[j].second)].x - mx;
    const double dy = points[static_cast<size_t>(nb[j].second)].y - my;
    sxx += dx * dx;
    sxy += dx * dy;
    syy += dy * dy;
  }
  // Eigenvalues (sxx+syy)/2 -+ sqrt(((sxx-syy)/2)^2 + sxy^2); the eigenvector
  // of the smaller one from whichever row of (C - lambda I) avoids
  // cancellation.
  const double half_tr = 0.5 * (sxx + syy);
  const double half_diff = 0.5 * (sxx - syy);
  const double disc = std::sqrt(half_diff * half_diff + sxy * sxy);
  const double ev_min = half_tr - disc;
  const double ev_max = half_tr + disc;
  double vx;
  double vy;
  if (half_diff >= 0.0) {
    vx = sxy;
    vy = ev_min - sxx;
  } else {
    vx = ev_min - syy;
    vy = sxy;
  }
  double vn = std::sqrt(vx * vx + vy * vy);
  if (!(vn > 0.0)) {
    vx = 1.0;
    vy = 0.0;
    vn = 1.0;
  }
  P2 n{vx / vn, vy / vn};
  const double lmin = std::max(ev_min, 0.0);
  const double lmax = std::max(ev_max, 1e-12);
  if (n.x * (origin.x - points[i].x) + n.y * (origin.y - points[i].y) < 0.0) {
    n = {-n.x, -n.y};
  }
  *normal_out = n;
  *corner_out = lmin / lmax;
}

}  // namespace

HostProblem FromDesc(const sdfgpu_problem_desc& d) {
  auto bad = [](const std::string& m) { Fail(SDFGPU_ERR_INVALID_ARGUMENT, m); };
  if (d.nx < 2 || d.ny < 2) {
    bad("grid needs nx >= 2 and ny >= 2");
  }
  if (static_cast<int64_t>(d.nx) * d.ny > (int64_t{1} << 30)) {
    bad("grid too large");
  }
  if (!(d.max_x > d.min_x) || !(d.max_y > d.min_y)) {
    bad("grid max corner must exceed min corner");
  }
  if (d.num_frames < 1 || d.poses == nullptr) {
    bad("problem needs at least one pose");
  }
  if (d.num_points < 0 || d.num_eikonal < 0 || d.num_odom < 0) {
    bad("negative spec count");
  }
  if (d.map_values == nullptr || d.node_to_active == nullptr) {
    bad("map_values and node_to_active are required");
  }
  if (d.num_points > 0 && (d.point_frame == nullptr || d.point_xy == nullptr ||
                           d.point_expected == nullptr || d.point_sqrt_weight == nullptr)) {
    bad("point spec arrays missing");
  }
  if (d.num_eikonal > 0 && (d.eikonal_wh == nullptr || d.eikonal_normal == nullptr ||
                            d.eikonal_sqrt_weight == nullptr)) {
    bad("eikonal spec arrays missing");
  }
  if (d.num_odom > 0 && (d.odom_ij == nullptr || d.odom_meas == nullptr || d.odom_sqrt_weight == nullptr)) {
    bad("odometry spec arrays missing");
  }
  HostProblem hp;
  hp.nx = d.nx;
  hp.ny = d.ny;
  hp.min_x = d.min_x;
  hp.min_y = d.min_y;
  hp.max_x = d.max_x;
  hp.max_y = d.max_y;
  const size_t nodes = static_cast<size_t>(d.nx) * static_cast<size_t>(d.ny);
  hp.map_values.assign(d.map_values, d.map_values + nodes);
  hp.poses.assign(d.poses, d.poses + 3 * static_cast<size_t>(d.num_frames));
  const size_t P = static_cast<size_t>(d.num_points);
  if (P > 0) {
    hp.pt_frame.assign(d.point_frame, d.point_frame + P);
    hp.pt_xy.assign(d.point_xy, d.point_xy + 2 * P);
    hp.pt_expected.assign(d.point_expected, d.point_expected + P);
    hp.pt_sqrtw.assign(d.point_sqrt_weight, d.point_sqrt_weight + P);
  }
  for (const int32_t f : hp.pt_frame) {
    if (f < 0 || f >= d.num_frames) {
      bad("point spec frame out of range");
    }
  }
  const size_t E = static_cast<size_t>(d.num_eikonal);
  if (E > 0) {
    hp.eik_wh.assign(d.eikonal_wh, d.eikonal_wh + 2 * E);
    hp.eik_n.assign(d.eikonal_normal, d.eikonal_normal + 2 * E);
    hp.eik_sqrtw.assign(d.eikonal_sqrt_weight, d.eikonal_sqrt_weight + E);
  }
  const size_t O = static_cast<size_t>(d.num_odom);
  if (O > 0) {
    hp.odom_ij.assign(d.odom_ij, d.odom_ij + 2 * O);
    hp.odom_meas.assign(d.odom_meas, d.odom_meas + 3 * O);
    hp.odom_sqrtw.assign(d.odom_sqrt_weight, d.odom_sqrt_weight + O);
  }
  for (size_t o = 0; o < O; ++o) {
    const int fi = hp.odom_ij[2 * o];
    const int fj = hp.odom_ij[2 * o + 1];
    if (fi < 0 || fj < 0 || fi >= d.num_frames || fj >= d.num_frames || fi == fj) {
      bad("odometry spec frames out of range");
    }
  }
  hp.node_to_active.assign(d.node_to_active, d.node_to_active + nodes);
  for (size_t node = 0; node < nodes; ++node) {
    const int a = hp.node_to_active[node];
    if (a >= 0) {
      if (a != static_cast<int>(hp.active_to_node.size())) {
        bad("node_to_active must number active nodes 0, 1, 2, ... in node order");
      }
      hp.active_to_node.push_back(static_cast<int32_t>(node));
    } else if (a != -1) {
      bad("node_to_active entries must be -1 or a column index");
    }
  }
  // Eikonal specs need their three nodes inside the grid and active
  // (problem.cpp:79-94).
  std::vector<int32_t> eik_seen(nodes, 0);
  for (size_t e = 0; e < E; ++e) {
    const int w = hp.eik_wh[2 * e];
    const int h = hp.eik_wh[2 * e + 1];
    if (w < 0 || h < 0 || w + 1 >= d.nx || h + 1 >= d.ny) {
      bad("eikonal spec node out of range");
    }
    const size_t n0 = static_cast<size_t>(h) * d.nx + w;
    if (hp.node_to_active[n0] < 0 || hp.node_to_active[n0 + 1] < 0 || hp.node_to_active[n0 + d.nx] < 0) {
      bad("eikonal spec touches a constant node");
    }
    if (eik_seen[n0] != 0) {
      bad("duplicate eikonal spec at one node");
    }
    eik_seen[n0] = 1;
    if (e > 0) {
      const int pw = hp.eik_wh[2 * e - 2];
      const int ph = hp.eik_wh[2 * e - 1];
      if (ph > h || (ph == h && pw >= w)) {
        bad("eikonal specs must be ordered by h, then w (problem.cpp:79-94)");
      }
    }
  }
  hp.huber_delta = d.huber_delta;
  hp.smooth_gradient = d.smooth_gradient != 0;
  hp.smooth_gradient_step = d.smooth_gradient_step;
  return hp;
}

namespace {

/// Scan-point normals and per-node normals and Eikonal scales (two values
/// and one per node, row-major) on the host.
void HostNodeNormals(const HostProblem& hp, int num_frames, const int32_t* scan_offsets, const double* scan_xy,
                     const sdfgpu_problem_options& o, std::vector<double>& node_normal_out,
                     std::vector<double>& node_scale_out) {
  auto bad = [](const std::string& m) { Fail(SDFGPU_ERR_INVALID_ARGUMENT, m); };
  const int nx = hp.nx;
  const int ny = hp.ny;
  const double min_x = hp.min_x;
  const double min_y = hp.min_y;
  const size_t nodes = static_cast<size_t>(nx) * static_cast<size_t>(ny);
  // Scan normals over the union of all scans at the current poses, or per
  // scan in the sensor frame (normals.cpp:102-160).
  const size_t k = static_cast<size_t>(std::max(2, o.normals_k_neighbors));
  std::vector<P2> spts;
  std::vector<P2> snorm;
  std::vector<double> scorner;
  std::vector<std::pair<double, int>> nb;
  if (o.normals_per_scan != 0) {
    for (int f = 0; f < num_frames; ++f) {
      std::vector<P2> local;
      for (int q = scan_offsets[f]; q < scan_offsets[f + 1]; ++q) {
        local.push_back({scan_xy[2 * q], scan_xy[2 * q + 1]});
      }
      const BucketKnn knn(local);
      const double* pose = &hp.poses[3 * static_cast<size_t>(f)];
      const double c = std::cos(pose[2]);
      const double s = std::sin(pose[2]);
      for (size_t i = 0; i < local.size(); ++i) {
        P2 n{};
        double corner = 0.0;
        PcaNormal(local, knn, i, std::min(k, local.size()), {0.0, 0.0}, &n, &corner, nb);
        spts.push_back(ApplyPose(pose, local[i]));
        snorm.push_back({c * n.x + (-s) * n.y, s * n.x + c * n.y});
        scorner.push_back(corner);
      }
    }
  } else {
    std::vector<P2> origins;
    for (int f = 0; f < num_frames; ++f) {
      const double* pose = &hp.poses[3 * static_cast<size_t>(f)];
      for (int q = scan_offsets[f]; q < scan_offsets[f + 1]; ++q) {
        spts.push_back(ApplyPose(pose, {scan_xy[2 * q], scan_xy[2 * q + 1]}));
        origins.push_back({pose[0], pose[1]});
      }
    }
    snorm.resize(spts.size());
    scorner.resize(spts.size());
    if (!spts.empty()) {
      const BucketKnn knn(spts);
      for (size_t i = 0; i < spts.size(); ++i) {
        PcaNormal(spts, knn, i, std::min(k, spts.size()), origins[i], &snorm[i], &scorner[i], nb);
      }
    }
  }

  // Node normals (normals.cpp:162-220).
  std::vector<P2> node_normal(nodes, P2{0.0, 0.0});
  std::vector<double> node_scale(nodes, 1.0);
  if (!spts.empty()) {
    const BucketKnn knn(spts);
    const double dxg = hp.dx();
    const double dyg = hp.dy();
    for (int h = 0; h < ny; ++h) {
      for (int w = 0; w < nx; ++w) {
        const P2 node{min_x + w * dxg, min_y + h * dyg};
        knn.Query(node, 1, nb);
        const size_t nearest = static_cast<size_t>(nb[0].second);
        const P2 npca = snorm[nearest];
        const double corner = std::clamp(scorner[nearest] / o.normals_corner_threshold, 0.0, 1.0);
        const size_t id = static_cast<size_t>(h) * nx + w;
        if (o.normals_method == 0) {
          node_normal[id] = npca;
        } else if (o.normals_method == 1) {
          const P2 ts{spts[nearest].x - node.x, spts[nearest].y - node.y};
          const double tn = std::sqrt(ts.x * ts.x + ts.y * ts.y);
          if (tn < 1e-9) {
            node_normal[id] = npca;
          } else {
            P2 cue{ts.x / tn, ts.y / tn};
            if (cue.x * npca.x + cue.y * npca.y < 0.0) {
              cue = {-cue.x, -cue.y};
            }
            const P2 bl{(1.0 - corner) * npca.x + corner * cue.x, (1.0 - corner) * npca.y + corner * cue.y};
            const double bn = std::sqrt(bl.x * bl.x + bl.y * bl.y);
            node_normal[id] = bn > 1e-9 ? P2{bl.x / bn, bl.y / bn} : npca;
          }
        } else if (o.normals_method == 2) {
          node_normal[id] = npca;
          node_scale[id] = 1.0 - corner;
        } else {
          bad("unknown normals.method");
        }
      }
    }
  }
  node_normal_out.resize(2 * nodes);
  for (size_t q = 0; q < nodes; ++q) {
    node_normal_out[2 * q] = node_normal[q].x;
    node_normal_out[2 * q + 1] = node_normal[q].y;
  }
  node_scale_out = std::move(node_scale);
}

}  // namespace

void PrepareNormalGrids(const HostProblem& hp, int num_frames, const int32_t* scan_offsets, const double* scan_xy,
                        bool per_scan, NormalGrids* out) {
  std::vector<P2> world;
  world.reserve(static_cast<size_t>(scan_offsets[num_frames]));
  out->frame_grids.clear();
  std::vector<P2> local;
  for (int f = 0; f < num_frames; ++f) {
    const double* pose = &hp.poses[3 * static_cast<size_t>(f)];
    const double c = std::cos(pose[2]);  // ApplyPose with the frame's cos and sin taken once
    const double sn = std::sin(pose[2]);
    local.clear();
    for (int q = scan_offsets[f]; q < scan_offsets[f + 1]; ++q) {
      const P2 p{scan_xy[2 * q], scan_xy[2 * q + 1]};
      local.push_back(p);
      world.push_back({(c * p.x + (-sn) * p.y) + pose[0], (sn * p.x + c * p.y) + pose[1]});
    }
    if (per_scan) {
      out->frame_grids.emplace_back();
      BucketKnn(local).Export(&out->frame_grids.back());
    }
  }
  BucketKnn(world).Export(&out->world_grid);
  out->world.resize(2 * world.size());
  static_assert(sizeof(P2) == 2 * sizeof(double));
  std::memcpy(out->world.data(), world.data(), world.size() * sizeof(P2));
}

HostProblem BuildProblem(int nx, int ny, double min_x, double min_y, double max_x, double max_y,
                         const double* map_values, int num_frames, const double* poses,
                         const int32_t* scan_offsets, const double* scan_xy,
                         const double* odometry, int num_odometry, int num_relations,
                         const int32_t* relation_ij, const double* relation_meas,
                         const double* relation_sqrt_weight, const sdfgpu_problem_options& o,
                         const BuildMode& mode) {
  const bool device_stages = mode.device_stages;
  const bool pattern_only = mode.pattern_only;
  auto bad = [](const std::string& m) { Fail(SDFGPU_ERR_INVALID_ARGUMENT, m); };
  if (device_stages && pattern_only) {
    bad("a pattern-only build runs on the host");
  }
  if (!mode.rows && !device_stages) {
    bad("the host stages always build the point rows");
  }
  if (nx < 2 || ny < 2 || !(max_x > min_x) || !(max_y > min_y)) {
    bad("GridMap needs nx, ny >= 2 and max > min");
  }
  if (num_frames < 1 || poses == nullptr || scan_offsets == nullptr) {
    bad("scan count != pose count");
  }
  if (num_odometry != 0 && num_odometry != num_frames - 1) {
    bad("odometry count must be frames - 1");
  }
  HostProblem hp;
  hp.nx = nx;
  hp.ny = ny;
  hp.min_x = min_x;
  hp.min_y = min_y;
  hp.max_x = max_x;
  hp.max_y = max_y;
  const size_t nodes = static_cast<size_t>(nx) * static_cast<size_t>(ny);
  hp.map_values.assign(nodes, 0.0);
  if (map_values != nullptr) {
    std::memcpy(hp.map_values.data(), map_values, nodes * sizeof(double));
  }
  hp.poses.assign(poses, poses + 3 * static_cast<size_t>(num_frames));
  hp.huber_delta = o.huber_delta;
  hp.smooth_gradient = o.smooth_gradient != 0;
  hp.smooth_gradient_step = o.smooth_gradient_step;

  for (int f = 0; f < num_frames; ++f) {
    if (scan_offsets[f + 1] < scan_offsets[f]) {
      bad("scan offsets must not decrease");
    }
  }
  if (!device_stages) {
  // Point specs (problem.cpp:26-37) with hallucinated points
  // (hallucination.cpp:5-28): toward = (-p / |p|) * step; interleaved
  // p + toward*j (expected +step*j) and p - toward*j (expected -step*j).
  const double sqrt_ws = std::sqrt(o.weight_scan);
  const double sqrt_wh = std::sqrt(o.weight_hallucination);
  const int per_side = o.hallucination_points_per_scan_point > 0
                           ? o.hallucination_points_per_scan_point / (o.hallucination_both_directions ? 2 : 1)
                           : 0;
  for (int f = 0; f < num_frames; ++f) {
    const int b = scan_offsets[f];
    const int e = scan_offsets[f + 1];
    for (int q = b; q < e; ++q) {
      hp.pt_frame.push_back(f);
      hp.pt_xy.push_back(scan_xy[2 * q]);
      hp.pt_xy.push_back(scan_xy[2 * q + 1]);
      hp.pt_expected.push_back(0.0);
      hp.pt_sqrtw.push_back(sqrt_ws);
    }
    for (int q = b; q < e && per_side > 0; ++q) {
      const double px = scan_xy[2 * q];
      const double py = scan_xy[2 * q + 1];
      const double norm = std::sqrt(px * px + py * py);
      if (norm < 1e-9) {
        continue;
      }
      const double tx = (-px) / norm * o.hallucination_step_size;
      const double ty = (-py) / norm * o.hallucination_step_size;
      for (int j = 1; j <= per_side; ++j) {
        const double jd = static_cast<double>(j);
        hp.pt_frame.push_back(f);
        hp.pt_xy.push_back(px + tx * jd);
        hp.pt_xy.push_back(py + ty * jd);
        hp.pt_expected.push_back(o.hallucination_step_size * jd);
        hp.pt_sqrtw.push_back(sqrt_wh);
        if (o.hallucination_both_directions != 0) {
          hp.pt_frame.push_back(f);
          hp.pt_xy.push_back(px - tx * jd);
          hp.pt_xy.push_back(py - ty * jd);
          hp.pt_expected.push_back(-o.hallucination_step_size * jd);
          hp.pt_sqrtw.push_back(sqrt_wh);
        }
      }
    }
  }

  // Active-region maps (problem.cpp:39-70).
  hp.node_to_active.assign(nodes, -1);
  std::vector<char> active(nodes, 0);
  if (o.active_region != 0) {
    const int margin = o.active_margin;
    for (size_t s = 0; s < hp.pt_frame.size(); ++s) {
      const P2 g = ApplyPose(&hp.poses[3 * static_cast<size_t>(hp.pt_frame[s])], {hp.pt_xy[2 * s], hp.pt_xy[2 * s + 1]});
      int w = 0;
      int h = 0;
      if (!LocateCell(hp, g, &w, &h)) {
        continue;
      }
      for (int hh = std::max(0, h - margin); hh <= std::min(ny - 1, h + 1 + margin); ++hh) {
        for (int ww = std::max(0, w - margin); ww <= std::min(nx - 1, w + 1 + margin); ++ww) {
          active[static_cast<size_t>(hh) * nx + ww] = 1;
        }
      }
    }
  } else {
    std::fill(active.begin(), active.end(), 1);
  }
  for (size_t node = 0; node < nodes; ++node) {
    if (active[node] != 0) {
      hp.node_to_active[node] = static_cast<int32_t>(hp.active_to_node.size());
      hp.active_to_node.push_back(static_cast<int32_t>(node));
    }
  }
  }  // host point specs and active maps

  std::vector<double> node_normal;
  std::vector<double> node_scale;
  if (!device_stages && !pattern_only) {
    HostNodeNormals(hp, num_frames, scan_offsets, scan_xy, o, node_normal, node_scale);
  }
  if (pattern_only) {
    // no Eikonal specs
  } else if (device_stages) {
    // point specs, active maps, node normals and the Eikonal spec list by
    // CUDA kernels
    DeviceBuildSpecs(hp, num_frames, scan_offsets, scan_xy, o, mode.rows);
  } else {
  const double sqrt_we = std::sqrt(o.weight_eikonal);
  for (int h = 0; h + 1 < ny; ++h) {
    for (int w = 0; w + 1 < nx; ++w) {
      const size_t id = static_cast<size_t>(h) * nx + w;
      if (hp.node_to_active[id] < 0 || hp.node_to_active[id + 1] < 0 || hp.node_to_active[id + nx] < 0) {
        continue;
      }
      const double scale = node_scale[id];
      if (scale <= 0.0) {
        continue;
      }
      hp.eik_wh.push_back(w);
      hp.eik_wh.push_back(h);
      hp.eik_n.push_back(node_normal[2 * id]);
      hp.eik_n.push_back(node_normal[2 * id + 1]);
      hp.eik_sqrtw.push_back(sqrt_we * std::sqrt(scale));
    }
  }
  }  // host Eikonal specs

  // Odometry and relation specs (problem.cpp:96-114).
  const double sqrt_wo = std::sqrt(o.weight_odometry);
  for (int i = 0; i + 1 < num_frames && i < num_odometry; ++i) {
    hp.odom_ij.push_back(i);
    hp.odom_ij.push_back(i + 1);
    hp.odom_meas.insert(hp.odom_meas.end(), odometry + 3 * i, odometry + 3 * i + 3);
    hp.odom_sqrtw.push_back(sqrt_wo);
  }
  const double sqrt_wr = std::sqrt(o.weight_relation);
  for (int r = 0; r < num_relations; ++r) {
    const int fi = relation_ij[2 * r];
    const int fj = relation_ij[2 * r + 1];
    if (fi < 0 || fj <= fi) {
      bad("relation frames must satisfy 0 <= i < j");
    }
    if (fj < num_frames) {
      hp.odom_ij.push_back(fi);
      hp.odom_ij.push_back(fj);
      hp.odom_meas.insert(hp.odom_meas.end(), relation_meas + 3 * r, relation_meas + 3 * r + 3);
      hp.odom_sqrtw.push_back(sqrt_wr * (relation_sqrt_weight != nullptr ? relation_sqrt_weight[r] : 1.0));
    }
  }
  return hp;
}

}  // namespace sdfgpu
