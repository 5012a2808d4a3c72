// run_slam's output files and trajectory metrics (src/pipeline/runner.cpp:
// 82-192), in the same formats, so that the reference's plotting and
// evaluation scripts read this library's runs unchanged:
//   poses CSV   "x,y,theta" header, one pose per line, 17 significant digits
//   map.txt     "nx ny min_x min_y dx dy", then ny lines of nx values
//   scan points "x,y" header, every scan point at its frame's pose, 9 digits
//   metrics     a flat JSON object: converged, iterations, costs, duration,
//               and the four mean trajectory errors when ground truth exists
#include <cmath>
#include <fstream>
#include <iomanip>
#include <string>

#include "internal.h"
#include "sdfgpu.h"

namespace sdfgpu {

namespace {

/// WrapAngle (src/core/pose.hpp:9).
inline double Wrap(double a) { return std::atan2(std::sin(a), std::cos(a)); }

std::ofstream Open(const char* path) {
  if (path == nullptr) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT, "path is null");
  }
  std::ofstream file(path);
  if (!file.is_open()) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT, std::string("cannot open output file: ") + path);
  }
  return file;
}

void Close(std::ofstream& file, const char* path) {
  file.close();
  if (file.fail()) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT, std::string("cannot write output file: ") + path);
  }
}

/// Pose2::RelativeTo (pose.hpp:38-43).
inline void Relative(const double* a, const double* o, double* out) {
  const double c = std::cos(a[2]);
  const double s = std::sin(a[2]);
  const double dx = o[0] - a[0];
  const double dy = o[1] - a[1];
  out[0] = c * dx + s * dy;
  out[1] = (-s) * dx + c * dy;
  out[2] = Wrap(o[2] - a[2]);
}

}  // namespace

/// WritePoses (runner.cpp:82-88).
void WritePoses(const char* path, const double* poses, int num_frames) {
  std::ofstream file = Open(path);
  file << std::setprecision(17) << "x,y,theta\n";
  for (int i = 0; i < num_frames; ++i) {
    file << poses[3 * i] << "," << poses[3 * i + 1] << "," << poses[3 * i + 2] << "\n";
  }
  Close(file, path);
}

/// WriteMap (runner.cpp:90-99); dx, dy as GridMap computes them
/// (grid_map.hpp:13-20).
void WriteMap(const char* path, int nx, int ny, double min_x, double min_y, double max_x, double max_y,
              const double* values) {
  const double dx = (max_x - min_x) / (nx - 1);
  const double dy = (max_y - min_y) / (ny - 1);
  std::ofstream file = Open(path);
  file << std::setprecision(17) << nx << " " << ny << " " << min_x << " " << min_y << " " << dx << " " << dy
       << "\n";
  for (int h = 0; h < ny; ++h) {
    for (int w = 0; w < nx; ++w) {
      file << values[static_cast<size_t>(h) * nx + w] << (w + 1 < nx ? " " : "\n");
    }
  }
  Close(file, path);
}

/// WriteGlobalScanPoints (runner.cpp:101-114): Pose2::Apply of every point.
void WriteScanPoints(const char* path, int num_frames, const double* poses, const int32_t* offsets,
                     const double* xy) {
  std::ofstream file = Open(path);
  file << std::setprecision(9) << "x,y\n";
  for (int f = 0; f < num_frames; ++f) {
    const double c = std::cos(poses[3 * f + 2]);
    const double s = std::sin(poses[3 * f + 2]);
    for (int q = offsets[f]; q < offsets[f + 1]; ++q) {
      const double px = xy[2 * q];
      const double py = xy[2 * q + 1];
      file << (c * px + (-s) * py) + poses[3 * f] << "," << (s * px + c * py) + poses[3 * f + 1] << "\n";
    }
  }
  Close(file, path);
}

/// The count WarnIfPointsOutsideMap (runner.cpp:116-137) reports: scan points
/// whose global position GridMap::Locate rejects (grid_map.hpp:58-63).
void PointsOutsideMap(int nx, int ny, double min_x, double min_y, double max_x, double max_y, int num_frames,
                      const double* poses, const int32_t* offsets, const double* xy, int64_t* outside,
                      int64_t* total) {
  const double dx = (max_x - min_x) / (nx - 1);
  const double dy = (max_y - min_y) / (ny - 1);
  *outside = 0;
  *total = 0;
  for (int f = 0; f < num_frames; ++f) {
    const double c = std::cos(poses[3 * f + 2]);
    const double s = std::sin(poses[3 * f + 2]);
    for (int q = offsets[f]; q < offsets[f + 1]; ++q) {
      const double gx = (c * xy[2 * q] + (-s) * xy[2 * q + 1]) + poses[3 * f];
      const double gy = (s * xy[2 * q] + c * xy[2 * q + 1]) + poses[3 * f + 1];
      const double fx = (gx - min_x) / dx;
      const double fy = (gy - min_y) / dy;
      if (!(fx >= 0.0) || !(fy >= 0.0) || !(fx <= nx - 1) || !(fy <= ny - 1)) {
        ++*outside;
      }
      ++*total;
    }
  }
}

/// Evaluate (runner.cpp:145-170): mean translation and |wrapped rotation|
/// errors of the poses, then of consecutive relative poses.
void EvaluateTrajectory(const double* est, const double* gt, int num_frames, double* metrics) {
  if (num_frames < 2) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT, "pose count mismatch between estimate and ground truth");
  }
  double t = 0.0;
  double r = 0.0;
  for (int i = 0; i < num_frames; ++i) {
    const double dx = est[3 * i] - gt[3 * i];
    const double dy = est[3 * i + 1] - gt[3 * i + 1];
    t += std::sqrt(dx * dx + dy * dy);
    r += std::abs(Wrap(est[3 * i + 2] - gt[3 * i + 2]));
  }
  metrics[0] = t / static_cast<double>(num_frames);
  metrics[1] = r / static_cast<double>(num_frames);
  const int pairs = num_frames - 1;
  double rt = 0.0;
  double rr = 0.0;
  for (int i = 0; i < pairs; ++i) {
    double re[3];
    double rg[3];
    Relative(est + 3 * i, est + 3 * (i + 1), re);
    Relative(gt + 3 * i, gt + 3 * (i + 1), rg);
    const double dx = re[0] - rg[0];
    const double dy = re[1] - rg[1];
    rt += std::sqrt(dx * dx + dy * dy);
    rr += std::abs(Wrap(re[2] - rg[2]));
  }
  metrics[2] = rt / static_cast<double>(pairs);
  metrics[3] = rr / static_cast<double>(pairs);
}

/// WriteJson (runner.cpp:172-192).
void WriteMetrics(const char* path, const sdfgpu_solve_result& result, const double* metrics) {
  std::ofstream file = Open(path);
  file << std::setprecision(17) << "{\n";
  file << "  \"converged\": " << (result.converged != 0 ? "true" : "false") << ",\n";
  file << "  \"iterations\": " << result.iterations << ",\n";
  file << "  \"initial_cost\": " << result.initial_cost << ",\n";
  file << "  \"final_cost\": " << result.final_cost << ",\n";
  file << "  \"duration_seconds\": " << result.duration_seconds;
  if (metrics != nullptr) {
    file << ",\n";
    file << "  \"mean_translation_error\": " << metrics[0] << ",\n";
    file << "  \"mean_rotation_error\": " << metrics[1] << ",\n";
    file << "  \"mean_relative_translation_error\": " << metrics[2] << ",\n";
    file << "  \"mean_relative_rotation_error\": " << metrics[3] << "\n";
  } else {
    file << "\n";
  }
  file << "}\n";
  Close(file, path);
}

}  // namespace sdfgpu
