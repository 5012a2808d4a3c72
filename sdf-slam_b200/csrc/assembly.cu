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
#include "trig.cuh"

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
  // the reference's bounds test, written so that a NaN coordinate (a pose
  // driven to NaN by a failed step) is outside too instead of reaching the
  // integer conversion
  if (!(fx >= 0.0) || !(fy >= 0.0) || !(fx <= I.nx - 1) || !(fy <= I.ny - 1)) {
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

/// WrapAngle (src/core/pose.hpp:9) of the odometry residual's angle:
/// atan2(sin a, cos a) with correctly rounded sin and cos.
__device__ __forceinline__ double WrapAngle(double a) {
  double s;
  double c;
  SinCosRn(a, &s, &c);
  return atan2(s, c);
}

}  // namespace

/// Offsets of the (pose var (frame, 0), node column) entries in the front for
/// the four corner nodes of a cell (lower-left node n0, row length nx), -1
/// where the frame is not in the node's analysed coupling set. The four
/// lower-bound searches over the nodes' ascending frames advance in lock
/// step, so every step's four loads are in flight together.
__device__ __forceinline__ void PoseOffsets4(const DeviceView& V, int64_t n0, int nx, int frame_local,
                                             int64_t off[4]) {
  int col[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    col[q] = V.node_col[n0 + (q >> 1) * nx + (q & 1)];
  }
  int64_t base[4];
  int64_t end[4];
  int64_t len[4];
  int64_t longest = 0;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    base[q] = col[q] >= 0 ? V.mp_ptr[col[q]] : 0;
    end[q] = col[q] >= 0 ? V.mp_ptr[col[q] + 1] : 0;
    len[q] = end[q] - base[q];
    longest = max(longest, len[q]);
  }
  // lower bound of frame_local in mp_frame[base, end)
  while (longest > 0) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (len[q] > 0) {
        const int64_t half = len[q] >> 1;
        if (V.mp_frame[base[q] + half] < frame_local) {
          base[q] += half + 1;
          len[q] -= half + 1;
        } else {
          len[q] = half;
        }
      }
    }
    longest >>= 1;
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const bool hit = col[q] >= 0 && base[q] < end[q] && V.mp_frame[base[q]] == frame_local;
    off[q] = hit ? V.mp_off[base[q]] : -1;
  }
}

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
  const double2 cs = V.pose_cs[f];
  const double c = cs.x;
  const double s = cs.y;
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
    // front offsets of the (pose, corner node) blocks this row adds to; the
    // lookups run here, one thread per row, so that the cell passes read them
    // instead of searching
    const int64_t n0 = I.node_off + static_cast<int64_t>(ev.h) * I.nx + ev.w;
    int64_t off[4];
    PoseOffsets4(V, n0, I.nx, local, off);
    longlong2* po = reinterpret_cast<longlong2*>(V.pt_poff + 4 * k);
    po[0] = make_longlong2(off[0], off[1]);
    po[1] = make_longlong2(off[2], off[3]);
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
  const double2 cs = V.pose_cs[fi];
  const double c = cs.x;
  const double s = cs.y;
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

__device__ __forceinline__ double WarpSum(double v) {
  // xor butterfly: every lane ends with the same, fixed-order sum
#pragma unroll
  for (int m = 16; m > 0; m >>= 1) {
    v += __shfl_xor_sync(0xffffffffu, v, m);
  }
  return v;
}

/// Front offset of the J^T J entry between the cell corners a and b of a cell
/// whose corner columns are col[], or -1 when one corner is constant.
__device__ __forceinline__ int64_t PairOffset(const DeviceView& V, const int* col, int a, int b) {
  if (col[a] < 0 || col[b] < 0) {
    return -1;
  }
  const int dw = (b & 1) - (a & 1);
  const int dh = (b >> 1) - (a >> 1);
  const int64_t off = V.mm_off[static_cast<int64_t>(col[a]) * 9 + (dh + 1) * 3 + (dw + 1)];
  if (off >= 0) {
    return off;
  }
  return V.mm_off[static_cast<int64_t>(col[b]) * 9 + (1 - dh) * 3 + (1 - dw)];
}

__device__ __forceinline__ int FindInstanceByCell(const DeviceView& V, int64_t cell) {
  int lo = 0;
  int hi = V.num_inst - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (V.inst[mid].cell_off <= cell) {
      lo = mid;
    } else {
      hi = mid - 1;
    }
  }
  return lo;
}

}  // namespace

/// One cell of a colour class (cx % 2, cy % 2) = (pass & 1, pass >> 1): cells
/// of one class share no node, so each adds its contributions to J^T J and
/// J^T r with plain read-modify-writes. One warp per cell: the 4x4 map block
/// and the corner gradients are lane-strided sums over the cell's point rows
/// reduced by a fixed butterfly; the map-pose blocks are segmented sums over
/// runs of rows of one frame (rows of a cell are sorted, so frames are
/// contiguous); the cell's Eikonal row (spec at its lower-left node) follows.
/// Passes run in a fixed order, so every entry is a deterministic sum.
__device__ __forceinline__ void CellPassOne(const DeviceView& V, int64_t cell, int lane) {
  const int i = FindInstanceByCell(V, cell);
  const InstDev& I = V.inst[i];
  if (V.active[i] == 0) {
    return;
  }
  const int cw = I.nx - 1;
  const int local = static_cast<int>(cell - I.cell_off);
  const int cx = local % cw;
  const int cy = local / cw;
  const int64_t n0 = I.node_off + static_cast<int64_t>(cy) * I.nx + cx;
  int col[4];
  col[0] = V.node_col[n0];
  col[1] = V.node_col[n0 + 1];
  col[2] = V.node_col[n0 + I.nx];
  col[3] = V.node_col[n0 + I.nx + 1];
  const int rb = V.cell_start[cell];
  const int re = V.cell_start[cell + 1];
  const int eik = V.eik_index[n0];
  if (rb == re && eik < 0) {
    return;
  }
  // One pass over the cell's rows in chunks of 32 (lane l takes rows
  // rb + l + 32 t): the 4x4 map block and corner gradients accumulate per
  // lane and are reduced by a fixed butterfly at the end; the map-pose
  // blocks are segmented sums over runs of one frame inside each chunk. A
  // chunk's records, frames and front offsets are loaded while the previous
  // chunk is scanned and written (the row indices one chunk further ahead).
  double mm[10];
  double g[4];
#pragma unroll
  for (int q = 0; q < 10; ++q) {
    mm[q] = 0.0;
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    g[q] = 0.0;
  }
  bool overflow = false;
  struct ChunkRow {
    double2 a01, a23, p01, p2r;
    longlong2 o01, o23;
    int f;
  };
  auto fetch = [&](int kk, ChunkRow& R) {
    if (kk >= 0) {
      const double2* r2 = reinterpret_cast<const double2*>(V.pt_rec + static_cast<int64_t>(kk) * kPointRec);
      const longlong2* po = reinterpret_cast<const longlong2*>(V.pt_poff + 4 * static_cast<int64_t>(kk));
      R.a01 = r2[0];
      R.a23 = r2[1];
      R.p01 = r2[2];
      R.p2r = r2[3];
      R.o01 = po[0];
      R.o23 = po[1];
      R.f = V.pt_frame[kk];
    } else {
      R.a01 = R.a23 = R.p01 = R.p2r = make_double2(0.0, 0.0);
      R.o01 = R.o23 = make_longlong2(-1, -1);
      R.f = -1;
    }
  };
  int k = (rb + lane < re) ? V.cell_rows[rb + lane] : -1;
  ChunkRow cur;
  fetch(k, cur);
  int k_next = (rb + 32 + lane < re) ? V.cell_rows[rb + 32 + lane] : -1;
  for (int base = rb; base < re; base += 32) {
    ChunkRow nxt;
    int k_after = -1;
    if (base + 32 < re) {
      fetch(k_next, nxt);
      k_after = (base + 64 + lane < re) ? V.cell_rows[base + 64 + lane] : -1;
    } else {
      fetch(-1, nxt);
    }
    const bool in = k >= 0;
    const int f = in ? cur.f : -1;
    double J[4] = {cur.a01.x, cur.a01.y, cur.a23.x, cur.a23.y};
    const double jp[3] = {cur.p01.x, cur.p01.y, cur.p2r.x};
    const double r = cur.p2r.y;
    if (in) {
      int q = 0;
#pragma unroll
      for (int aa = 0; aa < 4; ++aa) {
#pragma unroll
        for (int bb = aa; bb < 4; ++bb) {
          mm[q] = mm[q] + J[aa] * J[bb];
          ++q;
        }
        g[aa] = g[aa] + J[aa] * r;
      }
    }
    double v[12];
    const bool posed = in && (f - I.frame_off >= 1);
#pragma unroll
    for (int aa = 0; aa < 4; ++aa) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        v[3 * aa + c] = posed ? J[aa] * jp[c] : 0.0;
      }
    }
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int fu = __shfl_up_sync(0xffffffffu, f, d);
#pragma unroll
      for (int q = 0; q < 12; ++q) {
        const double vu = __shfl_up_sync(0xffffffffu, v[q], d);
        if (lane >= d && fu == f) {
          v[q] = vu + v[q];
        }
      }
    }
    const int fn = __shfl_down_sync(0xffffffffu, f, 1);
    const int p = base + lane;
    const bool tail = in && (lane == 31 || p + 1 >= re || fn != f);
    const int fl = f - I.frame_off;
    if (tail && fl >= 1) {
      // the (up to 12) entries are distinct: all loads first, then the
      // stores, so their latencies overlap
      const int64_t offs[4] = {cur.o01.x, cur.o01.y, cur.o23.x, cur.o23.y};
      double old[12];
#pragma unroll
      for (int aa = 0; aa < 4; ++aa) {
        if (col[aa] >= 0 && offs[aa] >= 0) {
          old[3 * aa] = V.asm_fronts[offs[aa]];
          old[3 * aa + 1] = V.asm_fronts[offs[aa] + 1];
          old[3 * aa + 2] = V.asm_fronts[offs[aa] + 2];
        } else {
          old[3 * aa] = old[3 * aa + 1] = old[3 * aa + 2] = 0.0;
        }
      }
#pragma unroll
      for (int aa = 0; aa < 4; ++aa) {
        if (col[aa] >= 0) {
          const int64_t off = offs[aa];
          if (off >= 0) {
            V.asm_fronts[off] = old[3 * aa] + v[3 * aa];
            V.asm_fronts[off + 1] = old[3 * aa + 1] + v[3 * aa + 1];
            V.asm_fronts[off + 2] = old[3 * aa + 2] + v[3 * aa + 2];
          } else {
            overflow = true;
          }
        }
      }
    }
    __syncwarp();
    cur = nxt;
    k = k_next;
    k_next = k_after;
  }
#pragma unroll
  for (int q = 0; q < 10; ++q) {
    mm[q] = WarpSum(mm[q]);
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    g[q] = WarpSum(g[q]);
  }
  if (rb < re) {
    // lanes 0..9 write the pairs, 10..13 the gradients
    int q = 0;
#pragma unroll
    for (int aa = 0; aa < 4; ++aa) {
#pragma unroll
      for (int bb = aa; bb < 4; ++bb) {
        if (lane == q) {
          const int64_t off = PairOffset(V, col, aa, bb);
          if (off >= 0) {
            V.asm_fronts[off] += mm[q];
          }
        }
        ++q;
      }
    }
#pragma unroll
    for (int aa = 0; aa < 4; ++aa) {
      if (lane == 10 + aa && col[aa] >= 0) {
        V.rhs[col[aa]] += g[aa];
      }
    }
  }
  __syncwarp();
  // the cell's Eikonal row: nodes (cx,cy), (cx+1,cy), (cx,cy+1) = corners
  // 0, 1, 2; lanes 0..5 add the six pairs, lanes 6..8 the three gradient
  // entries (distinct entries, one per lane)
  if (eik >= 0 && lane < 9) {
    const double* r = V.eik_rec + static_cast<int64_t>(eik) * kEikRec;
    if (lane < 6) {
      const int a = lane < 3 ? 0 : (lane < 5 ? 1 : 2);
      const int b = lane < 3 ? lane : (lane < 5 ? lane - 2 : 2);
      const int64_t off = PairOffset(V, col, a, b);
      if (off >= 0) {
        V.asm_fronts[off] += r[a] * r[b];
      }
    } else {
      const int a = lane - 6;
      V.rhs[col[a]] += r[a] * r[3];
    }
  }
  if (overflow) {
    atomicOr(V.status + i, kStatusPatternOverflow);
  }
}

/// Warps walk the pass's cell list with a grid stride (the launch holds as
/// many blocks as are resident, so no cell waits for a second wave behind a
/// busy one).
__global__ void __launch_bounds__(256, 2) KCellPass(DeviceView V, const int64_t* cells, int64_t count) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t w = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; w < count; w += warps) {
    CellPassOne(V, cells[w], lane);
  }
}

/// Same-frame pose blocks and the pose columns of J^T r: one block of 256
/// threads per frame, thread-strided over the frame's point rows, a fixed
/// butterfly per warp and a fixed order over warps, then the frame's odometry
/// / relation rows in spec order.
__global__ void __launch_bounds__(256) KPoseFrames(DeviceView V) {
  __shared__ double part[8][9];
  const int64_t f = blockIdx.x;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int i = V.frame_inst[f];
  const InstDev& I = V.inst[i];
  const int fl = static_cast<int>(f) - I.frame_off;
  if (fl < 1 || V.active[i] == 0) {
    return;
  }
  double acc[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) {
    acc[q] = 0.0;
  }
  const int64_t rb = V.frame_rows_ptr[f];
  const int64_t re = V.frame_rows_ptr[f + 1];
  // four rows per thread per pass, their loads issued together; a thread's
  // rows are still added in ascending order
  const int64_t stride = blockDim.x;
  for (int64_t q0 = rb + threadIdx.x; q0 < re; q0 += 4 * stride) {
    int kk[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int64_t q = q0 + u * stride;
      kk[u] = q < re ? V.frame_rows[q] : -1;
    }
    int cellv[4];
    double2 j01[4];
    double2 j2r[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if (kk[u] >= 0) {
        const double2* r2 = reinterpret_cast<const double2*>(V.pt_rec + static_cast<int64_t>(kk[u]) * kPointRec);
        cellv[u] = V.pt_cell[kk[u]];
        j01[u] = r2[2];
        j2r[u] = r2[3];
      } else {
        cellv[u] = -1;
        j01[u] = make_double2(0.0, 0.0);
        j2r[u] = make_double2(0.0, 0.0);
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if (cellv[u] < 0) {
        continue;
      }
      const double j0 = j01[u].x;
      const double j1 = j01[u].y;
      const double j2 = j2r[u].x;
      const double r = j2r[u].y;
      acc[0] = acc[0] + j0 * j0;
      acc[1] = acc[1] + j1 * j0;
      acc[2] = acc[2] + j2 * j0;
      acc[3] = acc[3] + j1 * j1;
      acc[4] = acc[4] + j2 * j1;
      acc[5] = acc[5] + j2 * j2;
      acc[6] = acc[6] + j0 * r;
      acc[7] = acc[7] + j1 * r;
      acc[8] = acc[8] + j2 * r;
    }
  }
#pragma unroll
  for (int q = 0; q < 9; ++q) {
    acc[q] = WarpSum(acc[q]);
  }
  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < 9; ++q) {
      part[warp][q] = acc[q];
    }
  }
  __syncthreads();
  if (threadIdx.x != 0) {
    return;
  }
  for (int q = 0; q < 9; ++q) {
    double v = part[0][q];
    for (int w = 1; w < 8; ++w) {
      v = v + part[w][q];
    }
    acc[q] = v;
  }
  const int aa[6] = {0, 1, 2, 1, 2, 2};
  const int bb[6] = {0, 0, 0, 1, 1, 2};
  for (int64_t q = V.frame_odom_ptr[f]; q < V.frame_odom_ptr[f + 1]; ++q) {
    const int code = V.frame_odom[q];
    const double* rec = V.odom_rec + static_cast<int64_t>(code >> 1) * kOdomRec;
    const double* blk = rec + ((code & 1) ? 12 : 3);
    for (int r = 0; r < 3; ++r) {
      for (int e = 0; e < 6; ++e) {
        acc[e] = acc[e] + blk[3 * r + aa[e]] * blk[3 * r + bb[e]];
      }
      for (int a = 0; a < 3; ++a) {
        acc[6 + a] = acc[6 + a] + blk[3 * r + a] * rec[r];
      }
    }
  }
  const int base = I.pp_first + 3 * (fl - 1);
  for (int e = 0; e < 6; ++e) {
    V.asm_fronts[I.pp_base + static_cast<int64_t>(base + bb[e]) * I.pp_ld + (base + aa[e])] = acc[e];
  }
  const int c0 = V.frame_col[f];
  V.rhs[c0] = acc[6];
  V.rhs[c0 + 1] = acc[7];
  V.rhs[c0 + 2] = acc[8];
}

/// Turns the accumulated J^T r into -J^T r and applies the damping of
/// lm_solver.cpp:321-330 to every diagonal entry (lambda, or lambda times
/// max(diag, 1e-12) under Marquardt scaling).
/// Zeroes the lower triangle of the assembly fronts before the row kernels
/// add into them: one warp per column c, rows c..F-1 (coalesced); task (sn,
/// first of kZeroCols columns). The upper triangles are never read before
/// the factorization writes them, so they are left as they are (half the
/// bytes of clearing the whole buffer).
__global__ void KZeroFronts(DeviceView V, const int32_t* tasks) {
  const int32_t* t = tasks + 2 * static_cast<int64_t>(blockIdx.x);
  const SupernodeRec S = V.sn[t[0]];
  const int c = t[1] + static_cast<int>(threadIdx.x >> 5);
  const int lane = static_cast<int>(threadIdx.x & 31);
  if (c >= S.F) {
    return;
  }
  double* col = V.asm_fronts + S.front_off + static_cast<int64_t>(c) * S.F;
  for (int r = c + lane; r < S.F; r += 32) {
    col[r] = 0.0;
  }
}

__global__ void KFinalizeNormal(DeviceView V) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= V.n) {
    return;
  }
  const int i = V.col_inst[col];
  if (V.active[i] == 0) {
    return;
  }
  V.rhs[col] = -V.rhs[col];
  int64_t off;
  if (V.col_node[col] >= 0) {
    off = V.mm_off[static_cast<int64_t>(col) * 9 + 4];
  } else {
    const InstDev& I = V.inst[i];
    const int rel = I.pp_first + (col - I.col_off - I.num_active);
    off = I.pp_base + static_cast<int64_t>(rel) * I.pp_ld + rel;
  }
  const double d = V.asm_fronts[off];
  const double lam = V.lam[i];
  V.asm_fronts[off] = V.marquardt[i] != 0 ? d + lam * fmax(d, 1e-12) : d + lam;
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
  V.asm_fronts[I.pp_base + static_cast<int64_t>(colf) * I.pp_ld + rowg] = acc;
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
  if (t < V.total_frames) {
    const int i = V.frame_inst[t];
    if (dir == 0 ? V.active[i] != 0 : revert_mask[i] != 0) {
      if (dir == 0) {
        V.pose_cs_backup[t] = V.pose_cs[t];
      } else {
        V.pose_cs[t] = V.pose_cs_backup[t];
      }
    }
  }
}

/// Problem::ApplyStep (problem.cpp:117-130): map values and positions; each
/// moved frame's angle theta + delta goes to theta_pre, and the pose gets a
/// provisional wrapped angle with correctly rounded cos and sin, which the
/// cost of the candidate state uses. Once the LM step is decided, the host
/// replaces the accepted angles and their cos / sin by the platform libm's
/// (KCommitPoses), so that the next linearization rotates with the
/// reference's bits.
__global__ void KApplyStep(DeviceView V) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= V.n) {
    return;
  }
  const int i = V.col_inst[col];
  // a failed factorization, a solve whose wait ran out or a stale pattern
  // leaves the state untouched
  if (V.active[i] == 0 ||
      (V.status[i] & (kStatusPatternOverflow | kStatusZeroPivot | kStatusWaitTimeout)) != 0) {
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
  const double t = p[2] + V.step[col + 2];
  V.theta_pre[f] = t;
  V.theta_upd[f] = 1;
  const double th = WrapAngle(t);
  p[2] = th;
  double sn;
  double cs;
  SinCosRn(th, &sn, &cs);
  V.pose_cs[f] = make_double2(cs, sn);
}

/// The accepted angles of the moved frames and their cos and sin, as the
/// host computed them with the platform's libm (WrapAngle, pose.hpp:9):
/// theta_out holds (theta, cos, sin, flag) per frame, flag 1 to commit.
__global__ void KCommitPoses(DeviceView V) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= V.total_frames || V.theta_out[4 * f + 3] == 0.0) {
    return;
  }
  V.poses[3 * static_cast<int64_t>(f) + 2] = V.theta_out[4 * f];
  V.pose_cs[f] = make_double2(V.theta_out[4 * f + 1], V.theta_out[4 * f + 2]);
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
    const double2 cs = V.pose_cs[f];
    const double c = cs.x;
    const double s = cs.y;
    const double2 p = V.pt_xy[t];
    PointEval ev;
    EvalPoint(V, I, c, s, pose, p.x, p.y, V.pt_exp[t], 0, false, ev);
    const int local = f - I.frame_off;
    if (ev.valid && local >= 1) {
      const uint32_t* allow = V.allow_bits + I.allow_off + static_cast<int64_t>(local) * I.allow_words;
      const int cw = I.nx - 1;
      const int cell = ev.h * cw + ev.w;
      if (((allow[cell >> 5] >> (cell & 31)) & 1u) == 0u) {
        atomicOr(V.status + i, kStatusNextOverflow);
      } else if (I.near_cells > 0 && (V.status[i] & kStatusNearEdge) == 0) {
        // the eight cells near_cells away (along the axes and the diagonals,
        // those inside the grid): one outside the set marks the instance
        const int g = I.near_cells;
        bool near = false;
#pragma unroll
        for (int q = 0; q < 9; ++q) {
          const int w = ev.w + g * (q % 3 - 1);
          const int h = ev.h + g * (q / 3 - 1);
          if (q != 4 && w >= 0 && w < cw && h >= 0 && h < I.ny - 1) {
            const int c = h * cw + w;
            near = near || ((allow[c >> 5] >> (c & 31)) & 1u) == 0u;
          }
        }
        if (near) {
          atomicOr(V.status + i, kStatusNearEdge);
        }
      }
    }
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
    const double2 cs = V.pose_cs[V.odom_fi[o]];
    const double c = cs.x;
    const double s = cs.y;
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

/// Deterministic segmented sum, first level: block (seg, part) sums the
/// part-th of kSegParts equal slices of segment seg with a fixed per-thread
/// stride and a fixed tree.
constexpr int kSegParts = 32;

__global__ void __launch_bounds__(256) KSegmentPartial(const double* x, const int64_t* seg_begin,
                                                       const int64_t* seg_end, double* partial) {
  __shared__ double red[256];
  const int seg = blockIdx.x / kSegParts;
  const int part = blockIdx.x % kSegParts;
  const int64_t b = seg_begin[seg];
  const int64_t e = seg_end[seg];
  const int64_t len = (e - b + kSegParts - 1) / kSegParts;
  const int64_t pb = b + part * len;
  const int64_t pe = min(e, pb + len);
  double s = 0.0;
  for (int64_t q = pb + threadIdx.x; q < pe; q += blockDim.x) {
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
    partial[blockIdx.x] = red[0];
  }
}

/// Second level: one warp per segment adds its kSegParts partials with a
/// fixed butterfly.
__global__ void KSegmentFinal(const double* partial, int num_segments, double* out) {
  const int seg = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (seg >= num_segments) {
    return;
  }
  const double v = WarpSum(partial[static_cast<int64_t>(seg) * kSegParts + lane]);
  if (lane == 0) {
    out[seg] = v;
  }
}

}  // namespace sdfgpu
