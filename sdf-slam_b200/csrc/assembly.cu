// Residual / Jacobian assembly, J^T J and -J^T r accumulation, step and cost
// kernels of the FP64 LM path.
//
// This translation unit is compiled with --fmad=false: every product and sum
// is rounded separately, in the association order of the reference's C++
// (src/core/pose.hpp, src/core/grid_map.hpp, src/problem/residual_math.hpp,
// src/solvers/lm_solver.cpp), so cells are assigned bit-exactly and the
// Jacobian entries, J^T J and -J^T r agree with a plain FP64 evaluation of the
// reference's expressions. J^T J entries are accumulated per entry in
// ascending row order with the first product assigned (ParallelAtA,
// lm_solver.cpp:113-172); -J^T r alternates two accumulators over each
// column's entries (ParallelNegAtb, lm_solver.cpp:178-197).
#include <cuda_runtime.h>

#include <climits>

#include "device.cuh"

namespace sdfgpu {

namespace {

struct PointEval {
  bool valid;
  int w, h;
  double residual;
  double wts[4];
  double d_pose[3];
};

__device__ __forceinline__ double MapValue(const DeviceView& V, const InstDev& I, int w, int h) {
  return V.map[I.node_off + static_cast<int64_t>(h) * I.nx + w];
}

/// GridMap::Interpolate for cell (w, h) with bilinear weights
/// (grid_map.hpp:86-93, FillCell :109-115).
__device__ __forceinline__ double Interp(const DeviceView& V, const InstDev& I, int w, int h, double a,
                                         double b, double* wts) {
  wts[0] = (1.0 - a) * (1.0 - b);
  wts[1] = a * (1.0 - b);
  wts[2] = (1.0 - a) * b;
  wts[3] = a * b;
  const int64_t n0 = I.node_off + static_cast<int64_t>(h) * I.nx + w;
  double value = 0.0;
  value += wts[0] * V.map[n0];
  value += wts[1] * V.map[n0 + 1];
  value += wts[2] * V.map[n0 + I.nx];
  value += wts[3] * V.map[n0 + I.nx + 1];
  return value;
}

/// LocateClamped + Interpolate (grid_map.hpp:75-93).
__device__ double ClampedValue(const DeviceView& V, const InstDev& I, double x, double y) {
  const double fx = (x - I.min_x) / I.dx;
  const double fy = (y - I.min_y) / I.dy;
  const int w = min(max(static_cast<int>(fx), 0), I.nx - 2);
  const int h = min(max(static_cast<int>(fy), 0), I.ny - 2);
  double wts[4];
  return Interp(V, I, w, h, fx - w, fy - h, wts);
}

/// EvalPointResidual (residual_math.hpp:75-106); gradient mode 0 exact
/// patch gradient (grid_map.hpp:98-106), 1 node central differences
/// (SmoothGradient :40-57), 2 metric finite differences (:63-73).
__device__ void EvalPoint(const DeviceView& V, const InstDev& I, double c, double s, const double* pose,
                          double px, double py, double delta, int mode, bool jac, PointEval& out) {
  const double gx = (c * px + (-s) * py) + pose[0];
  const double gy = (s * px + c * py) + pose[1];
  const double fx = (gx - I.min_x) / I.dx;
  const double fy = (gy - I.min_y) / I.dy;
  if (fx < 0.0 || fy < 0.0 || fx > I.nx - 1 || fy > I.ny - 1) {
    out.valid = false;
    out.residual = -delta;
    return;
  }
  out.valid = true;
  const int w = min(static_cast<int>(fx), I.nx - 2);
  const int h = min(static_cast<int>(fy), I.ny - 2);
  out.w = w;
  out.h = h;
  const double a = fx - w;
  const double b = fy - h;
  out.residual = Interp(V, I, w, h, a, b, out.wts) - delta;
  if (!jac) {
    return;
  }
  double grx;
  double gry;
  if (mode == 2) {
    const double st = I.smooth_gradient_step;
    grx = (ClampedValue(V, I, gx + st, gy) - ClampedValue(V, I, gx - st, gy)) / (2.0 * st);
    gry = (ClampedValue(V, I, gx, gy + st) - ClampedValue(V, I, gx, gy - st)) / (2.0 * st);
  } else if (mode == 1) {
    double g[4][2];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int ww = w + (q & 1);
      const int hh = h + (q >> 1);
      const int w_lo = max(ww - 1, 0);
      const int w_hi = min(ww + 1, I.nx - 1);
      const int h_lo = max(hh - 1, 0);
      const int h_hi = min(hh + 1, I.ny - 1);
      g[q][0] = (MapValue(V, I, w_hi, hh) - MapValue(V, I, w_lo, hh)) / (static_cast<double>(w_hi - w_lo) * I.dx);
      g[q][1] = (MapValue(V, I, ww, h_hi) - MapValue(V, I, ww, h_lo)) / (static_cast<double>(h_hi - h_lo) * I.dy);
    }
    const double s00 = (1.0 - a) * (1.0 - b);
    const double s10 = a * (1.0 - b);
    const double s01 = (1.0 - a) * b;
    const double s11 = a * b;
    grx = ((s00 * g[0][0] + s10 * g[1][0]) + s01 * g[2][0]) + s11 * g[3][0];
    gry = ((s00 * g[0][1] + s10 * g[1][1]) + s01 * g[2][1]) + s11 * g[3][1];
  } else {
    const int64_t n0 = I.node_off + static_cast<int64_t>(h) * I.nx + w;
    const double d00 = V.map[n0];
    const double d10 = V.map[n0 + 1];
    const double d01 = V.map[n0 + I.nx];
    const double d11 = V.map[n0 + I.nx + 1];
    grx = ((1.0 - b) * (d10 - d00) + b * (d11 - d01)) / I.dx;
    gry = ((1.0 - a) * (d01 - d00) + a * (d11 - d10)) / I.dy;
  }
  const double dx_dtheta = (-s) * px - c * py;
  const double dy_dtheta = c * px - s * py;
  out.d_pose[0] = grx;
  out.d_pose[1] = gry;
  out.d_pose[2] = grx * dx_dtheta + gry * dy_dtheta;
}

__device__ __forceinline__ int GradientMode(const InstDev& I) {
  if (I.smooth_gradient != 0 && I.smooth_gradient_step > 0.0) {
    return 2;
  }
  return I.smooth_gradient != 0 ? 1 : 0;
}

__device__ __forceinline__ double WrapAngle(double a) {
  double s;
  double c;
  sincos(a, &s, &c);
  return atan2(s, c);
}

}  // namespace

/// Point rows: AssemblePointRows (lm_solver.cpp:30-61) with HuberWeight
/// (problem.hpp:115-121). Writes the row record and the row's cell, and flags
/// a point whose cell lies outside its pose's analysed coupling set.
__global__ void KPointRows(DeviceView V) {
  const int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k >= V.total_points) {
    return;
  }
  const int f = V.pt_frame[k];
  const int i = V.frame_inst[f];
  const InstDev& I = V.inst[i];
  if (V.active[i] == 0) {
    return;
  }
  const double* pose = V.poses + 3 * static_cast<int64_t>(f);
  double s;
  double c;
  sincos(pose[2], &s, &c);
  const double2 p = V.pt_xy[k];
  const double delta = V.pt_exp[k];
  const double sqrt_w = V.pt_sw[k];
  PointEval ev;
  EvalPoint(V, I, c, s, pose, p.x, p.y, delta, GradientMode(I), true, ev);
  const double weighted = sqrt_w * ev.residual;
  double hw = 1.0;
  if (I.huber_delta > 0.0) {
    const double ar = fabs(weighted);
    hw = ar <= I.huber_delta ? 1.0 : I.huber_delta / ar;
  }
  const double sw = sqrt(hw);
  double* rec = V.pt_rec + k * kPointRec;
  rec[7] = sw * weighted;
  if (!ev.valid) {
    V.pt_cell[k] = -1;
    return;
  }
  const double scale = sw * sqrt_w;
  double2* r2 = reinterpret_cast<double2*>(rec);
  r2[0] = make_double2(scale * ev.wts[0], scale * ev.wts[1]);
  r2[1] = make_double2(scale * ev.wts[2], scale * ev.wts[3]);
  r2[2] = make_double2(scale * ev.d_pose[0], scale * ev.d_pose[1]);
  rec[6] = scale * ev.d_pose[2];
  const int cell = ev.h * (I.nx - 1) + ev.w;
  V.pt_cell[k] = static_cast<int32_t>(I.cell_off + cell);
  const int local = f - I.frame_off;
  if (local >= 1) {
    const uint32_t word = V.allow_bits[I.allow_off + static_cast<int64_t>(local) * I.allow_words + (cell >> 5)];
    if (((word >> (cell & 31)) & 1u) == 0u) {
      atomicOr(V.status + i, kStatusPatternOverflow);
    }
  }
}

/// Eikonal rows: EvalEikonalResidual (residual_math.hpp:158-171) scaled as in
/// AssembleEikonalRows (lm_solver.cpp:67-82).
__global__ void KEikonalRows(DeviceView V) {
  const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= V.total_eik) {
    return;
  }
  const int64_t node = V.eik_node[e];
  const int i = V.col_inst[V.node_col[node]];
  const InstDev& I = V.inst[i];
  if (V.active[i] == 0) {
    return;
  }
  const double d00 = V.map[node];
  const double d10 = V.map[node + 1];
  const double d01 = V.map[node + I.nx];
  const double gx = (d10 - d00) / I.dx;
  const double gy = (d01 - d00) / I.dy;
  const double2 n = V.eik_n[e];
  const double r = 1.0 - (n.x * gx + n.y * gy);
  const double sw = V.eik_sw[e];
  double* rec = V.eik_rec + e * kEikRec;
  rec[0] = sw * (n.x / I.dx + n.y / I.dy);
  rec[1] = sw * (-n.x / I.dx);
  rec[2] = sw * (-n.y / I.dy);
  rec[3] = sw * r;
}

/// Odometry / relation rows: EvalOdomResidual (residual_math.hpp:182-205)
/// scaled by sqrt_weight (lm_solver.cpp:275-296).
__global__ void KOdomRows(DeviceView V) {
  const int64_t o = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (o >= V.total_odom) {
    return;
  }
  const int fi = V.odom_fi[o];
  const int fj = V.odom_fj[o];
  if (V.active[V.frame_inst[fi]] == 0) {
    return;
  }
  const double* pi = V.poses + 3 * static_cast<int64_t>(fi);
  const double* pj = V.poses + 3 * static_cast<int64_t>(fj);
  const double* m = V.odom_meas + 3 * o;
  const double sw = V.odom_sw[o];
  double s;
  double c;
  sincos(pi[2], &s, &c);
  const double dtx = pj[0] - pi[0];
  const double dty = pj[1] - pi[1];
  const double rx = c * dtx + s * dty;
  const double ry = (-s) * dtx + c * dty;
  double* rec = V.odom_rec + o * kOdomRec;
  rec[0] = sw * (rx - m[0]);
  rec[1] = sw * (ry - m[1]);
  rec[2] = sw * WrapAngle(pj[2] - pi[2] - m[2]);
  // d_pose_i rows: [-c, -s, -s dtx + c dty], [s, -c, -c dtx - s dty], [0, 0, -1]
  rec[3] = sw * (-c);
  rec[4] = sw * (-s);
  rec[5] = sw * ((-s) * dtx + c * dty);
  rec[6] = sw * s;
  rec[7] = sw * (-c);
  rec[8] = sw * ((-c) * dtx + (-s) * dty);
  rec[9] = sw * 0.0;
  rec[10] = sw * 0.0;
  rec[11] = sw * -1.0;
  // d_pose_j rows: [c, s, 0], [-s, c, 0], [0, 0, 1]
  rec[12] = sw * c;
  rec[13] = sw * s;
  rec[14] = sw * 0.0;
  rec[15] = sw * (-s);
  rec[16] = sw * c;
  rec[17] = sw * 0.0;
  rec[18] = sw * 0.0;
  rec[19] = sw * 0.0;
  rec[20] = sw * 1.0;
}

/// cell_start[c] = first position of cell c in the sorted keys.
__global__ void KCellStart(const int32_t* keys, int64_t n, int64_t num_cells, int32_t* cell_start) {
  const int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (c > num_cells) {
    return;
  }
  int64_t lo = 0;
  int64_t hi = n;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (keys[mid] < c) {
      lo = mid + 1;
    } else {
      hi = mid;
    }
  }
  cell_start[c] = static_cast<int32_t>(lo);
}

namespace {

/// Adds rec[q'] * x into the stencil accumulators for the three other
/// corners (and the node itself) of a point row whose cell sits at offset C
/// (0: cell (w-1,h-1), 1: (w,h-1), 2: (w-1,h), 3: (w,h)) from node (w, h).
template <int C>
__device__ __forceinline__ void AccumulateCell(double* acc, const double* rec, double x, unsigned act) {
  constexpr int q = 3 - C;
  constexpr int jx = q & 1;
  constexpr int jy = q >> 1;
#pragma unroll
  for (int qq = 0; qq < 4; ++qq) {
    const int dw = (qq & 1) - jx;
    const int dh = (qq >> 1) - jy;
    const int slot = (dh + 1) * 3 + (dw + 1);
    if (act & (1u << slot)) {
      acc[slot] = acc[slot] + rec[qq] * x;
    }
  }
}

}  // namespace

/// Column gather for every active map node j: J^T J entries (i, j) of the 9
/// stencil neighbours and of the pose parameters of every frame whose points
/// touch j, plus -J^T r at j, all summed in ascending row order. Point rows
/// of the 4 cells around j are merged by row index; Eikonal rows follow
/// (specs at (w,h-1), (w-1,h), (w,h) in spec order). Damping
/// (lm_solver.cpp:321-330) is applied to the diagonal entry.
__global__ void KNodeColumns(DeviceView V) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= V.n) {
    return;
  }
  const int node = V.col_node[col];
  if (node < 0) {
    return;
  }
  const int i = V.col_inst[col];
  if (V.active[i] == 0) {
    return;
  }
  const InstDev& I = V.inst[i];
  const int local = node - static_cast<int>(I.node_off);
  const int w = local % I.nx;
  const int h = local / I.nx;
  unsigned act = 0;
#pragma unroll
  for (int slot = 0; slot < 9; ++slot) {
    const int ww = w + slot % 3 - 1;
    const int hh = h + slot / 3 - 1;
    if (ww >= 0 && hh >= 0 && ww < I.nx && hh < I.ny && V.node_col[node + (slot / 3 - 1) * I.nx + (slot % 3 - 1)] >= 0) {
      act |= 1u << slot;
    }
  }
  const int cw = I.nx - 1;
  const int ch = I.ny - 1;
  int pos[4];
  int end[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const int cx = w - 1 + (c & 1);
    const int cy = h - 1 + (c >> 1);
    if (cx >= 0 && cy >= 0 && cx < cw && cy < ch) {
      const int64_t cell = I.cell_off + static_cast<int64_t>(cy) * cw + cx;
      pos[c] = V.cell_start[cell];
      end[c] = V.cell_start[cell + 1];
    } else {
      pos[c] = 0;
      end[c] = 0;
    }
  }
  double acc[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) {
    acc[q] = -0.0;
  }
  double pacc[3] = {-0.0, -0.0, -0.0};
  int cur_f = -1;
  double tmp_a = 0.0;
  double tmp_b = 0.0;
  int parity = 0;
  int64_t mpc = V.mp_ptr[col];
  const int64_t mpe = V.mp_ptr[col + 1];
  bool overflow = false;
  auto flush = [&]() {
    if (cur_f < 0) {
      return;
    }
    const int fl = cur_f - I.frame_off;
    while (mpc < mpe && V.mp_frame[mpc] < fl) {
      ++mpc;
    }
    if (mpc < mpe && V.mp_frame[mpc] == fl) {
      double* dst = V.fronts + V.mp_off[mpc];
      dst[0] = pacc[0];
      dst[1] = pacc[1];
      dst[2] = pacc[2];
    } else {
      overflow = true;
    }
  };
  int head[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    head[c] = pos[c] < end[c] ? V.cell_rows[pos[c]] : INT_MAX;
  }
  while (true) {
    int best = 0;
#pragma unroll
    for (int c = 1; c < 4; ++c) {
      if (head[c] < head[best]) {
        best = c;
      }
    }
    const int k = head[best];
    if (k == INT_MAX) {
      break;
    }
    ++pos[best];
    head[best] = pos[best] < end[best] ? V.cell_rows[pos[best]] : INT_MAX;
    const double* rec = V.pt_rec + static_cast<int64_t>(k) * kPointRec;
    double rv[8];
    const double2* r2 = reinterpret_cast<const double2*>(rec);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const double2 t = r2[q];
      rv[2 * q] = t.x;
      rv[2 * q + 1] = t.y;
    }
    const double x = rv[3 - best];
    switch (best) {
      case 0:
        AccumulateCell<0>(acc, rv, x, act);
        break;
      case 1:
        AccumulateCell<1>(acc, rv, x, act);
        break;
      case 2:
        AccumulateCell<2>(acc, rv, x, act);
        break;
      default:
        AccumulateCell<3>(acc, rv, x, act);
        break;
    }
    if (parity == 0) {
      tmp_a += x * rv[7];
    } else {
      tmp_b += x * rv[7];
    }
    parity ^= 1;
    const int f = V.pt_frame[k];
    if (f - I.frame_off >= 1) {
      if (f != cur_f) {
        flush();
        cur_f = f;
        pacc[0] = -0.0;
        pacc[1] = -0.0;
        pacc[2] = -0.0;
      }
      pacc[0] = pacc[0] + rv[4] * x;
      pacc[1] = pacc[1] + rv[5] * x;
      pacc[2] = pacc[2] + rv[6] * x;
    }
  }
  flush();
  // Eikonal rows touching j: spec at (w,h-1) [j is its node 2], (w-1,h)
  // [node 1], (w,h) [node 0]; slots of the spec's other nodes relative to j.
  {
    const int e0 = h >= 1 ? V.eik_index[node - I.nx] : -1;
    const int e1 = w >= 1 ? V.eik_index[node - 1] : -1;
    const int e2 = V.eik_index[node];
    if (e0 >= 0) {
      const double* r = V.eik_rec + static_cast<int64_t>(e0) * kEikRec;
      const double x = r[2];
      acc[1] = acc[1] + r[0] * x;
      acc[2] = acc[2] + r[1] * x;
      acc[4] = acc[4] + r[2] * x;
      if (parity == 0) { tmp_a += x * r[3]; } else { tmp_b += x * r[3]; }
      parity ^= 1;
    }
    if (e1 >= 0) {
      const double* r = V.eik_rec + static_cast<int64_t>(e1) * kEikRec;
      const double x = r[1];
      acc[3] = acc[3] + r[0] * x;
      acc[4] = acc[4] + r[1] * x;
      acc[6] = acc[6] + r[2] * x;
      if (parity == 0) { tmp_a += x * r[3]; } else { tmp_b += x * r[3]; }
      parity ^= 1;
    }
    if (e2 >= 0) {
      const double* r = V.eik_rec + static_cast<int64_t>(e2) * kEikRec;
      const double x = r[0];
      acc[4] = acc[4] + r[0] * x;
      acc[5] = acc[5] + r[1] * x;
      acc[7] = acc[7] + r[2] * x;
      if (parity == 0) { tmp_a += x * r[3]; } else { tmp_b += x * r[3]; }
      parity ^= 1;
    }
  }
  const double lam = V.lam[i];
  {
    const double v = acc[4];
    acc[4] = V.marquardt[i] != 0 ? v + lam * fmax(v, 1e-12) : v + lam;
  }
  const int64_t* mo = V.mm_off + static_cast<int64_t>(col) * 9;
#pragma unroll
  for (int slot = 0; slot < 9; ++slot) {
    const int64_t off = mo[slot];
    if (off >= 0) {
      V.fronts[off] = acc[slot];
    }
  }
  V.rhs[col] = -(tmp_a + tmp_b);
  if (overflow) {
    atomicOr(V.status + i, kStatusPatternOverflow);
  }
}

/// Same-frame pose blocks (6 entries per frame) and -J^T r of the pose
/// columns: point rows of the frame in ascending order, then its odometry /
/// relation rows.
__global__ void KPoseBlocks(DeviceView V) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int f = static_cast<int>(t / 9);
  const int e = static_cast<int>(t % 9);
  if (f >= V.total_frames) {
    return;
  }
  const int i = V.frame_inst[f];
  const InstDev& I = V.inst[i];
  const int fl = f - I.frame_off;
  if (fl < 1 || V.active[i] == 0) {
    return;
  }
  const int64_t rb = V.frame_rows_ptr[f];
  const int64_t re = V.frame_rows_ptr[f + 1];
  const int64_t ob = V.frame_odom_ptr[f];
  const int64_t oe = V.frame_odom_ptr[f + 1];
  if (e < 6) {
    const int aa[6] = {0, 1, 2, 1, 2, 2};
    const int bb[6] = {0, 0, 0, 1, 1, 2};
    const int a = aa[e];
    const int b = bb[e];
    double acc = -0.0;
    for (int64_t q = rb; q < re; ++q) {
      const int k = V.frame_rows[q];
      if (V.pt_cell[k] < 0) {
        continue;
      }
      const double* rec = V.pt_rec + static_cast<int64_t>(k) * kPointRec;
      acc = acc + rec[4 + a] * rec[4 + b];
    }
    for (int64_t q = ob; q < oe; ++q) {
      const int code = V.frame_odom[q];
      const double* rec = V.odom_rec + static_cast<int64_t>(code >> 1) * kOdomRec;
      const double* blk = rec + ((code & 1) ? 12 : 3);
      for (int r = 0; r < 3; ++r) {
        acc = acc + blk[3 * r + a] * blk[3 * r + b];
      }
    }
    if (a == b) {
      const double lam = V.lam[i];
      acc = V.marquardt[i] != 0 ? acc + lam * fmax(acc, 1e-12) : acc + lam;
    }
    const int base = I.pp_first + 3 * (fl - 1);
    V.fronts[I.pp_base + static_cast<int64_t>(base + b) * I.pp_ld + (base + a)] = acc;
  } else {
    const int a = e - 6;
    double tmp_a = 0.0;
    double tmp_b = 0.0;
    int parity = 0;
    for (int64_t q = rb; q < re; ++q) {
      const int k = V.frame_rows[q];
      if (V.pt_cell[k] < 0) {
        continue;
      }
      const double* rec = V.pt_rec + static_cast<int64_t>(k) * kPointRec;
      if (parity == 0) { tmp_a += rec[4 + a] * rec[7]; } else { tmp_b += rec[4 + a] * rec[7]; }
      parity ^= 1;
    }
    for (int64_t q = ob; q < oe; ++q) {
      const int code = V.frame_odom[q];
      const double* rec = V.odom_rec + static_cast<int64_t>(code >> 1) * kOdomRec;
      const double* blk = rec + ((code & 1) ? 12 : 3);
      for (int r = 0; r < 3; ++r) {
        if (parity == 0) { tmp_a += blk[3 * r + a] * rec[r]; } else { tmp_b += blk[3 * r + a] * rec[r]; }
        parity ^= 1;
      }
    }
    V.rhs[V.frame_col[f] + a] = -(tmp_a + tmp_b);
  }
}

/// Cross-frame pose blocks of frame pairs linked by odometry / relation rows.
__global__ void KPosePairs(DeviceView V) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int p = static_cast<int>(t / 9);
  if (p >= V.num_pairs) {
    return;
  }
  const int a = static_cast<int>(t % 9) / 3;  // row var of the larger frame g
  const int b = static_cast<int>(t % 9) % 3;  // column var of the smaller frame f
  const int f = V.pair_f[p];
  const int g = V.pair_g[p];
  const int i = V.frame_inst[f];
  if (V.active[i] == 0) {
    return;
  }
  const InstDev& I = V.inst[i];
  double acc = -0.0;
  for (int64_t q = V.pair_ptr[p]; q < V.pair_ptr[p + 1]; ++q) {
    const int code = V.pair_spec[q];
    const double* rec = V.odom_rec + static_cast<int64_t>(code >> 1) * kOdomRec;
    // code bit 0 set: the spec's frame_i is the larger frame g
    const double* bg = rec + ((code & 1) ? 3 : 12);
    const double* bf = rec + ((code & 1) ? 12 : 3);
    for (int r = 0; r < 3; ++r) {
      acc = acc + bg[3 * r + a] * bf[3 * r + b];
    }
  }
  const int fl = f - I.frame_off;
  const int gl = g - I.frame_off;
  const int colf = I.pp_first + 3 * (fl - 1) + b;
  const int rowg = I.pp_first + 3 * (gl - 1) + a;
  V.fronts[I.pp_base + static_cast<int64_t>(colf) * I.pp_ld + rowg] = acc;
}

/// Saves or restores the state of active instances (backup for revert,
/// lm_solver.cpp:366-372, 405-423). dir 0: save, 1: restore where
/// revert_mask[i] != 0.
__global__ void KBackup(DeviceView V, int dir, const int32_t* revert_mask) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t < V.total_nodes) {
    const int col = V.node_col[t];
    // nodes of an instance: find instance through the column when active,
    // otherwise leave untouched (constant nodes never change)
    if (col >= 0) {
      const int i = V.col_inst[col];
      if (dir == 0 ? V.active[i] != 0 : revert_mask[i] != 0) {
        if (dir == 0) {
          V.map_backup[t] = V.map[t];
        } else {
          V.map[t] = V.map_backup[t];
        }
      }
    }
  }
  if (t < 3 * static_cast<int64_t>(V.total_frames)) {
    const int i = V.frame_inst[t / 3];
    if (dir == 0 ? V.active[i] != 0 : revert_mask[i] != 0) {
      if (dir == 0) {
        V.poses_backup[t] = V.poses[t];
      } else {
        V.poses[t] = V.poses_backup[t];
      }
    }
  }
}

/// Problem::ApplyStep (problem.cpp:117-130).
__global__ void KApplyStep(DeviceView V) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= V.n) {
    return;
  }
  const int i = V.col_inst[col];
  // a failed factorization or a stale pattern leaves the state untouched
  if (V.active[i] == 0 || (V.status[i] & (kStatusPatternOverflow | kStatusZeroPivot)) != 0) {
    return;
  }
  const int node = V.col_node[col];
  if (node >= 0) {
    V.map[node] += V.step[col];
    return;
  }
  const InstDev& I = V.inst[i];
  const int rel = col - I.col_off - I.num_active;
  if (rel % 3 != 0) {
    return;
  }
  const int f = I.frame_off + 1 + rel / 3;
  double* p = V.poses + 3 * static_cast<int64_t>(f);
  p[0] += V.step[col];
  p[1] += V.step[col + 1];
  p[2] = WrapAngle(p[2] + V.step[col + 2]);
}

/// Per-row cost terms of Problem::Cost (problem.cpp:132-156): point rows with
/// the exact (non-smooth) evaluation and the Huber loss, Eikonal rows,
/// odometry rows. Terms are laid out points, then Eikonal, then odometry.
__global__ void KCostTerms(DeviceView V, double* terms) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t < V.total_points) {
    const int f = V.pt_frame[t];
    const int i = V.frame_inst[f];
    const InstDev& I = V.inst[i];
    const double* pose = V.poses + 3 * static_cast<int64_t>(f);
    double s;
    double c;
    sincos(pose[2], &s, &c);
    const double2 p = V.pt_xy[t];
    PointEval ev;
    EvalPoint(V, I, c, s, pose, p.x, p.y, V.pt_exp[t], 0, false, ev);
    const double r = V.pt_sw[t] * ev.residual;
    double term;
    if (I.huber_delta > 0.0 && fabs(r) > I.huber_delta) {
      term = I.huber_delta * (2.0 * fabs(r) - I.huber_delta);
    } else {
      term = r * r;
    }
    terms[t] = term;
    return;
  }
  const int64_t e = t - V.total_points;
  if (e < V.total_eik) {
    const int64_t node = V.eik_node[e];
    const int i = V.col_inst[V.node_col[node]];
    const InstDev& I = V.inst[i];
    const double d00 = V.map[node];
    const double d10 = V.map[node + 1];
    const double d01 = V.map[node + I.nx];
    const double gx = (d10 - d00) / I.dx;
    const double gy = (d01 - d00) / I.dy;
    const double2 n = V.eik_n[e];
    const double r = V.eik_sw[e] * (1.0 - (n.x * gx + n.y * gy));
    terms[t] = r * r;
    return;
  }
  const int64_t o = e - V.total_eik;
  if (o < V.total_odom) {
    const double* pi = V.poses + 3 * static_cast<int64_t>(V.odom_fi[o]);
    const double* pj = V.poses + 3 * static_cast<int64_t>(V.odom_fj[o]);
    const double* m = V.odom_meas + 3 * o;
    const double sw = V.odom_sw[o];
    double s;
    double c;
    sincos(pi[2], &s, &c);
    const double dtx = pj[0] - pi[0];
    const double dty = pj[1] - pi[1];
    const double e0 = sw * ((c * dtx + s * dty) - m[0]);
    const double e1 = sw * (((-s) * dtx + c * dty) - m[1]);
    const double e2 = sw * WrapAngle(pj[2] - pi[2] - m[2]);
    terms[t] = (e0 * e0 + e1 * e1) + e2 * e2;
  }
}

/// Per-column terms for the step norm and the trust-region prediction
/// (lm_solver.cpp:378, 389-391): delta^2 and delta * (lambda delta + rhs).
__global__ void KStepTerms(DeviceView V, double* sq, double* pred) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= V.n) {
    return;
  }
  const double d = V.step[col];
  sq[col] = d * d;
  pred[col] = d * (V.lam[V.col_inst[col]] * d + V.rhs[col]);
}

/// Deterministic segmented sum: block b sums seg_begin[b]..seg_end[b] with a
/// fixed per-thread stride and a fixed tree.
__global__ void KSegmentSum(const double* x, const int64_t* seg_begin, const int64_t* seg_end, double* out) {
  __shared__ double red[256];
  const int64_t b = seg_begin[blockIdx.x];
  const int64_t e = seg_end[blockIdx.x];
  double s = 0.0;
  for (int64_t q = b + threadIdx.x; q < e; q += blockDim.x) {
    s += x[q];
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      red[threadIdx.x] += red[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[blockIdx.x] = red[0];
  }
}

}  // namespace sdfgpu
