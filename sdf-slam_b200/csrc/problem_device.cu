// Device stages of the problem construction (Problem::Problem,
// src/problem/problem.cpp:11-115): the point specs (per frame its scan rows,
// then the hallucinated rows of its points, src/core/hallucination.cpp:5-28),
// the active-region index maps (problem.cpp:39-70) and the Eikonal spec list
// (problem.cpp:79-94), with the scan-point PCA normals and the per-node
// normals (src/core/normals.cpp:70-220) found by exact k-NN searches on the
// host builder's bucket grids.
//
// Every value is computed with the host builder's operations in its order
// (explicitly rounded intrinsics, no contraction; the pose cosines and sines
// are the host's), so the specs equal the host's bit for bit. Positions of
// the rows follow from exclusive scans: a frame's rows start at its first
// scan point plus rows_per times the hallucinating points before it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "engine.h"

namespace sdfgpu {

namespace {

constexpr int kScanThreads = 1024;
constexpr int kMaxNeighbors = 64;  // normals.k_neighbors the device search holds
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

/// Exclusive scan of each tile of kScanTile values (four per thread, loaded
/// together); the tile's total goes to sums[tile].
__global__ void __launch_bounds__(kScanThreads) KTileScan(const int32_t* in, int64_t n, int32_t* out,
                                                          int32_t* sums) {
  __shared__ int32_t warp_total[32];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kScanTile + static_cast<int64_t>(threadIdx.x) * kScanItems;
  int32_t v[kScanItems];
  int32_t local = 0;
#pragma unroll
  for (int u = 0; u < kScanItems; ++u) {
    v[u] = base + u < n ? in[base + u] : 0;
    local += v[u];
  }
  int32_t x = local;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int32_t y = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= d) {
      x += y;
    }
  }
  if (lane == 31) {
    warp_total[warp] = x;
  }
  __syncthreads();
  if (warp == 0) {
    int32_t t = warp_total[lane];
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int32_t y = __shfl_up_sync(0xffffffffu, t, d);
      if (lane >= d) {
        t += y;
      }
    }
    warp_total[lane] = t;
  }
  __syncthreads();
  int32_t run = (warp > 0 ? warp_total[warp - 1] : 0) + x - local;
#pragma unroll
  for (int u = 0; u < kScanItems; ++u) {
    if (base + u < n) {
      out[base + u] = run;
    }
    run += v[u];
  }
  if (threadIdx.x == kScanThreads - 1) {
    sums[blockIdx.x] = warp_total[31];
  }
}

/// Exclusive scan of the nb tile totals in place (one block, chunks of 1024
/// with a carry); the grand total goes to sums[nb].
__global__ void __launch_bounds__(kScanThreads) KSumScan(int32_t* sums, int nb) {
  __shared__ int32_t warp_total[32];
  __shared__ int32_t carry;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) {
    carry = 0;
  }
  __syncthreads();
  for (int c0 = 0; c0 < nb; c0 += kScanThreads) {
    const int i = c0 + static_cast<int>(threadIdx.x);
    const int32_t v = i < nb ? sums[i] : 0;
    int32_t x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int32_t y = __shfl_up_sync(0xffffffffu, x, d);
      if (lane >= d) {
        x += y;
      }
    }
    if (lane == 31) {
      warp_total[warp] = x;
    }
    __syncthreads();
    if (warp == 0) {
      int32_t t = warp_total[lane];
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const int32_t y = __shfl_up_sync(0xffffffffu, t, d);
        if (lane >= d) {
          t += y;
        }
      }
      warp_total[lane] = t;
    }
    __syncthreads();
    const int32_t before = carry + (warp > 0 ? warp_total[warp - 1] : 0) + x - v;
    if (i < nb) {
      sums[i] = before;
    }
    __syncthreads();
    if (threadIdx.x == kScanThreads - 1) {
      carry = before + v;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    sums[nb] = carry;
  }
}

__global__ void KTileAdd(int32_t* out, int64_t n, const int32_t* sums) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) {
    out[i] += sums[i / kScanTile];
  }
}

inline unsigned Grid(int64_t n, int threads) { return static_cast<unsigned>((n + threads - 1) / threads); }

/// out = exclusive scan of in[0, n); returns the total (synchronizes).
int64_t ExclusiveScan(const int32_t* in, int64_t n, int32_t* out, DevBuf<int32_t>& sums, cudaStream_t s) {
  if (n == 0) {
    return 0;
  }
  const int64_t tiles = (n + kScanTile - 1) / kScanTile;
  if (tiles >= (int64_t{1} << 31)) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT, "problem too large for the device builder");
  }
  sums.Alloc(static_cast<size_t>(tiles) + 1);
  KTileScan<<<static_cast<unsigned>(tiles), kScanThreads, 0, s>>>(in, n, out, sums.get());
  KSumScan<<<1, kScanThreads, 0, s>>>(sums.get(), static_cast<int>(tiles));
  KTileAdd<<<Grid(n, 256), 256, 0, s>>>(out, n, sums.get());
  int32_t total = 0;
  CudaCheck(cudaMemcpyAsync(&total, sums.get() + tiles, sizeof(int32_t), cudaMemcpyDeviceToHost, s), "scan total");
  CudaCheck(cudaStreamSynchronize(s), "scan");
  return total;
}

/// 1 where the scan point is hallucinated (|p| >= 1e-9, hallucination.cpp).
__global__ void KHallucinating(const double2* xy, int64_t n, int32_t* flag) {
  const int64_t q = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (q >= n) {
    return;
  }
  const double px = xy[q].x;
  const double py = xy[q].y;
  const double norm = __dsqrt_rn(__dadd_rn(__dmul_rn(px, px), __dmul_rn(py, py)));
  flag[q] = norm < 1e-9 ? 0 : 1;
}

struct ExpandArgs {
  int per_side;
  int both;
  int rows_per;  // hallucinated rows per point
  double step;
  double sqrt_ws;
  double sqrt_wh;
};

/// Writes the rows of scan point q: its scan row at the frame's start plus
/// its index in the frame, and its hallucinated rows (+j, then -j when both
/// directions) after the frame's scan rows, in point order.
__global__ void KExpandPoints(const double2* xy, const int32_t* frame_of, const int32_t* offsets,
                              const int32_t* hal_before, const int32_t* hal, int64_t n, ExpandArgs a,
                              int32_t* pt_frame, double2* pt_xy, double* pt_exp, double* pt_sw) {
  const int64_t q = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (q >= n) {
    return;
  }
  const int f = frame_of[q];
  const int b = offsets[f];
  const int e = offsets[f + 1];
  const int64_t start = static_cast<int64_t>(b) + static_cast<int64_t>(a.rows_per) * hal_before[b];
  const double px = xy[q].x;
  const double py = xy[q].y;
  const int64_t r = start + (q - b);
  pt_frame[r] = f;
  pt_xy[r] = make_double2(px, py);
  pt_exp[r] = 0.0;
  pt_sw[r] = a.sqrt_ws;
  if (a.per_side <= 0 || hal[q] == 0) {
    return;
  }
  const double norm = __dsqrt_rn(__dadd_rn(__dmul_rn(px, px), __dmul_rn(py, py)));
  const double tx = __dmul_rn(__ddiv_rn(-px, norm), a.step);
  const double ty = __dmul_rn(__ddiv_rn(-py, norm), a.step);
  int64_t h = start + (e - b) + static_cast<int64_t>(a.rows_per) * (hal_before[q] - hal_before[b]);
  for (int j = 1; j <= a.per_side; ++j) {
    const double jd = static_cast<double>(j);
    pt_frame[h] = f;
    pt_xy[h] = make_double2(__dadd_rn(px, __dmul_rn(tx, jd)), __dadd_rn(py, __dmul_rn(ty, jd)));
    pt_exp[h] = __dmul_rn(a.step, jd);
    pt_sw[h] = a.sqrt_wh;
    ++h;
    if (a.both != 0) {
      pt_frame[h] = f;
      pt_xy[h] = make_double2(__dsub_rn(px, __dmul_rn(tx, jd)), __dsub_rn(py, __dmul_rn(ty, jd)));
      pt_exp[h] = __dmul_rn(-a.step, jd);
      pt_sw[h] = a.sqrt_wh;
      ++h;
    }
  }
}

struct GridArgs {
  int nx;
  int ny;
  double min_x;
  double min_y;
  double dx;
  double dy;
};

/// Marks the nodes of the cell every row falls in at its frame's pose,
/// dilated by `margin` and clipped to the grid (problem.cpp:45-60). Rows
/// outside the grid mark nothing. frame_trig: per frame cos, sin, x, y.
__global__ void KActiveMark(const int32_t* pt_frame, const double2* pt_xy, int64_t rows, const double* frame_trig,
                            GridArgs g, int margin, int32_t* active) {
  const int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (s >= rows) {
    return;
  }
  const double* t = frame_trig + 4 * static_cast<int64_t>(pt_frame[s]);
  const double c = t[0];
  const double sn = t[1];
  const double2 p = pt_xy[s];
  const double gx = __dadd_rn(__dadd_rn(__dmul_rn(c, p.x), __dmul_rn(-sn, p.y)), t[2]);
  const double gy = __dadd_rn(__dadd_rn(__dmul_rn(sn, p.x), __dmul_rn(c, p.y)), t[3]);
  const double fx = __ddiv_rn(__dsub_rn(gx, g.min_x), g.dx);
  const double fy = __ddiv_rn(__dsub_rn(gy, g.min_y), g.dy);
  // NaN coordinates count as outside (never converted to a cell)
  if (!(fx >= 0.0) || !(fy >= 0.0) || !(fx <= static_cast<double>(g.nx - 1)) ||
      !(fy <= static_cast<double>(g.ny - 1))) {
    return;
  }
  const int w = min(static_cast<int>(fx), g.nx - 2);
  const int h = min(static_cast<int>(fy), g.ny - 2);
  for (int hh = max(0, h - margin); hh <= min(g.ny - 1, h + 1 + margin); ++hh) {
    for (int ww = max(0, w - margin); ww <= min(g.nx - 1, w + 1 + margin); ++ww) {
      active[static_cast<int64_t>(hh) * g.nx + ww] = 1;
    }
  }
}

/// node_to_active / active_to_node from the active flags and their scan.
__global__ void KNodeMaps(const int32_t* active, const int32_t* prefix, int64_t nodes, int32_t* node_to_active,
                          int32_t* active_to_node) {
  const int64_t node = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (node >= nodes) {
    return;
  }
  if (active[node] != 0) {
    node_to_active[node] = prefix[node];
    active_to_node[prefix[node]] = static_cast<int32_t>(node);
  } else {
    node_to_active[node] = -1;
  }
}

/// 1 where lower-left node (w, h) has an Eikonal spec: (w, h), (w + 1, h)
/// and (w, h + 1) active and a positive scale; t = h * (nx - 1) + w.
__global__ void KEikonalFlags(const int32_t* node_to_active, const double* scale, int nx, int ny, int32_t* flag) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t cells = static_cast<int64_t>(nx - 1) * (ny - 1);
  if (t >= cells) {
    return;
  }
  const int w = static_cast<int>(t % (nx - 1));
  const int h = static_cast<int>(t / (nx - 1));
  const int64_t id = static_cast<int64_t>(h) * nx + w;
  flag[t] = (node_to_active[id] >= 0 && node_to_active[id + 1] >= 0 && node_to_active[id + nx] >= 0 &&
             scale[id] > 0.0)
                ? 1
                : 0;
}

__global__ void KEikonalSpecs(const int32_t* flag, const int32_t* prefix, const double* node_normal,
                              const double* scale, int nx, int ny, double sqrt_we, int32_t* eik_wh, double* eik_n,
                              double* eik_sw) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t cells = static_cast<int64_t>(nx - 1) * (ny - 1);
  if (t >= cells || flag[t] == 0) {
    return;
  }
  const int w = static_cast<int>(t % (nx - 1));
  const int h = static_cast<int>(t / (nx - 1));
  const int64_t id = static_cast<int64_t>(h) * nx + w;
  const int64_t k = prefix[t];
  eik_wh[2 * k] = w;
  eik_wh[2 * k + 1] = h;
  eik_n[2 * k] = node_normal[2 * id];
  eik_n[2 * k + 1] = node_normal[2 * id + 1];
  eik_sw[k] = __dmul_rn(sqrt_we, __dsqrt_rn(scale[id]));
}

/// One bucket grid in the concatenated device arrays: its start offsets begin
/// at start_off, its items (indices into the grid's own points) at pt_off,
/// and its points are the pt_off-th onward of the point array it serves.
struct KnnGridDev {
  double ox;
  double oy;
  double cell;
  int gx;
  int gy;
  int64_t start_off;
  int64_t pt_off;
  int count;
};

/// floor(f) clamped to [0, g - 1], NaN to 0 (the host grid's cell index).
__device__ __forceinline__ int CellOf(double f, int g) {
  if (!(f > 0.0)) {
    return 0;
  }
  if (f >= static_cast<double>(g - 1)) {
    return g - 1;
  }
  return static_cast<int>(f);
}

/// (d2, idx) lexicographic order, as std::pair's operator<.
__device__ __forceinline__ bool PairLess(double a, int ia, double b, int ib) {
  return a < b || (!(b < a) && ia < ib);
}

/// The want (1 <= want <= min(KMAX, count)) nearest points of grid G to q,
/// ascending by (squared distance, index) into bd / bi: the host grid's ring
/// search (rings of cells around q's clamped cell, stopping once the
/// want-th best is closer than the ring's inner bound) with its rounding,
/// keeping a sorted list where the host keeps a max-heap; both hold the
/// want smallest pairs seen, so the results agree.
template <int KMAX>
__device__ __forceinline__ void KnnSearch(const KnnGridDev& G, const int32_t* __restrict__ start,
                                          const int32_t* __restrict__ items, const double2* __restrict__ pts,
                                          double qx, double qy, int want, double* bd, int* bi) {
  const int32_t* st = start + G.start_off;
  const int32_t* it = items + G.pt_off;
  const int cx = CellOf(__ddiv_rn(__dsub_rn(qx, G.ox), G.cell), G.gx);
  const int cy = CellOf(__ddiv_rn(__dsub_rn(qy, G.oy), G.cell), G.gy);
  const double bx0 = __dadd_rn(G.ox, __dmul_rn(static_cast<double>(cx), G.cell));
  const double by0 = __dadd_rn(G.oy, __dmul_rn(static_cast<double>(cy), G.cell));
  // max(0, min(qx - bx0, bx0 + cell - qx, qy - by0, by0 + cell - qy)),
  // first minimum kept as std::min over a list does
  double m = __dsub_rn(qx, bx0);
  double t = __dsub_rn(__dadd_rn(bx0, G.cell), qx);
  m = t < m ? t : m;
  t = __dsub_rn(qy, by0);
  m = t < m ? t : m;
  t = __dsub_rn(__dadd_rn(by0, G.cell), qy);
  m = t < m ? t : m;
  const double inner = 0.0 < m ? m : 0.0;
  int size = 0;
  const int max_ring = max(G.gx, G.gy);
  for (int r = 0; r <= max_ring; ++r) {
    const int y0 = cy - r;
    const int y1 = cy + r;
    for (int y = max(0, y0); y <= min(G.gy - 1, y1); ++y) {
      // ring r's cells in row y: the whole span on its first and last row,
      // else the two ends
      const bool full = (y == y0 || y == y1);
      const int xa = full ? max(0, cx - r) : cx - r;
      const int xb = full ? min(G.gx - 1, cx + r) : cx + r;
      const int step = full || r == 0 ? 1 : 2 * r;
      for (int x = xa; x <= xb; x += step) {
        if (x < 0 || x >= G.gx) {
          continue;
        }
        const int64_t b = static_cast<int64_t>(y) * G.gx + x;
        const int e = st[b + 1];
        for (int s = st[b]; s < e; ++s) {
          const int idx = it[s];
          const double2 p = pts[idx];
          const double ddx = __dsub_rn(p.x, qx);
          const double ddy = __dsub_rn(p.y, qy);
          const double d2 = __dadd_rn(__dmul_rn(ddx, ddx), __dmul_rn(ddy, ddy));
          int pos;
          if (size < want) {
            pos = size++;
          } else if (PairLess(d2, idx, bd[want - 1], bi[want - 1])) {
            pos = want - 1;
          } else {
            continue;
          }
          while (pos > 0 && PairLess(d2, idx, bd[pos - 1], bi[pos - 1])) {
            bd[pos] = bd[pos - 1];
            bi[pos] = bi[pos - 1];
            --pos;
          }
          bd[pos] = d2;
          bi[pos] = idx;
        }
      }
    }
    if (size == want) {
      const double bound = __dadd_rn(inner, __dmul_rn(static_cast<double>(r), G.cell));
      if (bd[want - 1] < __dmul_rn(bound, bound)) {
        break;
      }
    }
  }
}

/// PCA normal and cornerness of every scan point from its k nearest
/// neighbours (normals.cpp:70-160): the mean and the covariance sums in
/// neighbour order, the closed-form smaller eigenvector oriented toward the
/// sensor, cornerness max(ev_min, 0) / max(ev_max, 1e-12). per_scan: the
/// neighbours come from the point's own scan in the sensor frame (grid f of
/// grids, points xy) and the normal is rotated into the world; else from all
/// world points (grid 0, points world) with the frame's position as the
/// sensor.
template <int KMAX>
__global__ void __launch_bounds__(128) KScanNormals(const KnnGridDev* __restrict__ grids,
                                                    const int32_t* __restrict__ start,
                                                    const int32_t* __restrict__ items,
                                                    const double2* __restrict__ xy,
                                                    const double2* __restrict__ world,
                                                    const int32_t* __restrict__ frame_of,
                                                    const double* __restrict__ frame_trig, int64_t n, int k,
                                                    int per_scan, double2* snorm, double* scorner) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) {
    return;
  }
  const int f = frame_of[i];
  const KnnGridDev G = grids[per_scan != 0 ? f : 0];
  const double2* pts = per_scan != 0 ? xy + G.pt_off : world;
  const double2 q = pts[i - G.pt_off];
  const int want = min(k, G.count);
  double bd[KMAX];
  int bi[KMAX];
  KnnSearch<KMAX>(G, start, items, pts, q.x, q.y, want, bd, bi);
  double mx = 0.0;
  double my = 0.0;
  for (int j = 0; j < want; ++j) {
    const double2 p = pts[bi[j]];
    mx = __dadd_rn(mx, p.x);
    my = __dadd_rn(my, p.y);
  }
  mx = __ddiv_rn(mx, static_cast<double>(want));
  my = __ddiv_rn(my, static_cast<double>(want));
  double sxx = 0.0;
  double sxy = 0.0;
  double syy = 0.0;
  for (int j = 0; j < want; ++j) {
    const double2 p = pts[bi[j]];
    const double dx = __dsub_rn(p.x, mx);
    const double dy = __dsub_rn(p.y, my);
    sxx = __dadd_rn(sxx, __dmul_rn(dx, dx));
    sxy = __dadd_rn(sxy, __dmul_rn(dx, dy));
    syy = __dadd_rn(syy, __dmul_rn(dy, dy));
  }
  const double half_tr = __dmul_rn(0.5, __dadd_rn(sxx, syy));
  const double half_diff = __dmul_rn(0.5, __dsub_rn(sxx, syy));
  const double disc = __dsqrt_rn(__dadd_rn(__dmul_rn(half_diff, half_diff), __dmul_rn(sxy, sxy)));
  const double ev_min = __dsub_rn(half_tr, disc);
  const double ev_max = __dadd_rn(half_tr, disc);
  double vx;
  double vy;
  if (half_diff >= 0.0) {
    vx = sxy;
    vy = __dsub_rn(ev_min, sxx);
  } else {
    vx = __dsub_rn(ev_min, syy);
    vy = sxy;
  }
  double vn = __dsqrt_rn(__dadd_rn(__dmul_rn(vx, vx), __dmul_rn(vy, vy)));
  if (!(vn > 0.0)) {
    vx = 1.0;
    vy = 0.0;
    vn = 1.0;
  }
  double nx = __ddiv_rn(vx, vn);
  double ny = __ddiv_rn(vy, vn);
  const double lmin = 0.0 < ev_min ? ev_min : 0.0;
  const double lmax = 1e-12 < ev_max ? ev_max : 1e-12;
  const double* t = frame_trig + 4 * static_cast<int64_t>(f);
  const double ox = per_scan != 0 ? 0.0 : t[2];
  const double oy = per_scan != 0 ? 0.0 : t[3];
  if (__dadd_rn(__dmul_rn(nx, __dsub_rn(ox, q.x)), __dmul_rn(ny, __dsub_rn(oy, q.y))) < 0.0) {
    nx = -nx;
    ny = -ny;
  }
  if (per_scan != 0) {
    const double c = t[0];
    const double sn = t[1];
    snorm[i] = make_double2(__dadd_rn(__dmul_rn(c, nx), __dmul_rn(-sn, ny)),
                            __dadd_rn(__dmul_rn(sn, nx), __dmul_rn(c, ny)));
  } else {
    snorm[i] = make_double2(nx, ny);
  }
  scorner[i] = __ddiv_rn(lmin, lmax);
}

struct NodeNormalArgs {
  int method;  // 0 pca, 1 hybrid, 2 weighted
  double corner_threshold;
};

/// Per-node normal and Eikonal scale from the nearest world scan point
/// (normals.cpp:162-220): its PCA normal (method 0), blended toward the
/// direction to it by the clamped cornerness (method 1), or kept with scale
/// 1 - cornerness (method 2). With no scan points: (0, 0) and scale 1.
__global__ void KNodeNormals(KnnGridDev G, const int32_t* __restrict__ start, const int32_t* __restrict__ items,
                             const double2* __restrict__ world, const double2* __restrict__ snorm,
                             const double* __restrict__ scorner, GridArgs g, NodeNormalArgs a, double2* node_normal,
                             double* node_scale) {
  const int64_t id = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (id >= static_cast<int64_t>(g.nx) * g.ny) {
    return;
  }
  if (G.count == 0) {
    node_normal[id] = make_double2(0.0, 0.0);
    node_scale[id] = 1.0;
    return;
  }
  const int w = static_cast<int>(id % g.nx);
  const int h = static_cast<int>(id / g.nx);
  const double qx = __dadd_rn(g.min_x, __dmul_rn(static_cast<double>(w), g.dx));
  const double qy = __dadd_rn(g.min_y, __dmul_rn(static_cast<double>(h), g.dy));
  double bd[1];
  int bi[1];
  KnnSearch<1>(G, start, items, world, qx, qy, 1, bd, bi);
  const int nearest = bi[0];
  const double2 npca = snorm[nearest];
  // std::clamp(scorner / threshold, 0, 1)
  const double v = __ddiv_rn(scorner[nearest], a.corner_threshold);
  const double corner = v < 0.0 ? 0.0 : (1.0 < v ? 1.0 : v);
  double2 out = npca;
  double scale = 1.0;
  if (a.method == 1) {
    const double2 p = world[nearest];
    const double tx = __dsub_rn(p.x, qx);
    const double ty = __dsub_rn(p.y, qy);
    const double tn = __dsqrt_rn(__dadd_rn(__dmul_rn(tx, tx), __dmul_rn(ty, ty)));
    if (!(tn < 1e-9)) {
      double cx = __ddiv_rn(tx, tn);
      double cy = __ddiv_rn(ty, tn);
      if (__dadd_rn(__dmul_rn(cx, npca.x), __dmul_rn(cy, npca.y)) < 0.0) {
        cx = -cx;
        cy = -cy;
      }
      const double keep = __dsub_rn(1.0, corner);
      const double bx = __dadd_rn(__dmul_rn(keep, npca.x), __dmul_rn(corner, cx));
      const double by = __dadd_rn(__dmul_rn(keep, npca.y), __dmul_rn(corner, cy));
      const double bn = __dsqrt_rn(__dadd_rn(__dmul_rn(bx, bx), __dmul_rn(by, by)));
      if (bn > 1e-9) {
        out = make_double2(__ddiv_rn(bx, bn), __ddiv_rn(by, bn));
      }
    }
  } else if (a.method == 2) {
    scale = __dsub_rn(1.0, corner);
  }
  node_normal[id] = out;
  node_scale[id] = scale;
}

/// The grids flattened for the device: descriptors, concatenated start
/// offsets and concatenated items (each grid's items at its pt_off).
struct FlatGrids {
  std::vector<KnnGridDev> desc;
  std::vector<int32_t> start;
  std::vector<int32_t> items;
};

void AppendGrid(const KnnBuckets& b, int64_t pt_off, FlatGrids* f) {
  KnnGridDev d{};
  d.ox = b.ox;
  d.oy = b.oy;
  d.cell = b.cell;
  d.gx = b.gx;
  d.gy = b.gy;
  d.start_off = static_cast<int64_t>(f->start.size());
  d.pt_off = pt_off;
  d.count = static_cast<int>(b.items.size());
  f->desc.push_back(d);
  f->start.insert(f->start.end(), b.start.begin(), b.start.end());
  if (static_cast<int64_t>(f->items.size()) < pt_off + d.count) {
    f->items.resize(static_cast<size_t>(pt_off + d.count));
  }
  std::copy(b.items.begin(), b.items.end(), f->items.begin() + pt_off);
}

template <typename T>
void Download(std::vector<T>& dst, const T* src, size_t count, cudaStream_t s) {
  dst.resize(count);
  if (count > 0) {
    CudaCheck(cudaMemcpyAsync(dst.data(), src, count * sizeof(T), cudaMemcpyDeviceToHost, s), "download");
  }
}

}  // namespace

void DeviceBuildSpecs(HostProblem& hp, int num_frames, const int32_t* scan_offsets, const double* scan_xy,
                      const sdfgpu_problem_options& o, bool download_rows) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    Fail(SDFGPU_ERR_CUDA, "the device builder needs a CUDA device");
  }
  cudaStream_t s = nullptr;
  CudaCheck(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  } guard{s};
  const int nx = hp.nx;
  const int ny = hp.ny;
  const int64_t nodes = static_cast<int64_t>(nx) * ny;
  const int64_t n = scan_offsets[num_frames];
  // host inputs: the frame of every scan point, the poses' cos / sin (the
  // host builder's values) and the square roots of the weights
  std::vector<int32_t> frame_of(static_cast<size_t>(n));
  for (int f = 0; f < num_frames; ++f) {
    std::fill(frame_of.begin() + scan_offsets[f], frame_of.begin() + scan_offsets[f + 1], f);
  }
  std::vector<double> trig(4 * static_cast<size_t>(num_frames));
  for (int f = 0; f < num_frames; ++f) {
    const double* pose = &hp.poses[3 * static_cast<size_t>(f)];
    trig[4 * f] = std::cos(pose[2]);
    trig[4 * f + 1] = std::sin(pose[2]);
    trig[4 * f + 2] = pose[0];
    trig[4 * f + 3] = pose[1];
  }
  const int k = std::max(2, o.normals_k_neighbors);
  if (n > 0) {
    // the checks the host builder makes while it computes the normals
    if (o.normals_method < 0 || o.normals_method > 2) {
      Fail(SDFGPU_ERR_INVALID_ARGUMENT, "unknown normals.method");
    }
    if (k > kMaxNeighbors) {
      Fail(SDFGPU_ERR_INVALID_ARGUMENT, "the device builder supports normals.k_neighbors up to 64");
    }
    for (int64_t q = 0; q < 2 * n; ++q) {
      if (!std::isfinite(scan_xy[q])) {
        Fail(SDFGPU_ERR_INVALID_ARGUMENT, "the device builder needs finite scan points");
      }
    }
    for (double v : hp.poses) {
      if (!std::isfinite(v)) {
        Fail(SDFGPU_ERR_INVALID_ARGUMENT, "the device builder needs finite poses");
      }
    }
  }
  ExpandArgs a{};
  a.per_side = o.hallucination_points_per_scan_point > 0
                   ? o.hallucination_points_per_scan_point / (o.hallucination_both_directions ? 2 : 1)
                   : 0;
  a.both = o.hallucination_both_directions != 0 ? 1 : 0;
  a.rows_per = a.per_side * (a.both != 0 ? 2 : 1);
  a.step = o.hallucination_step_size;
  a.sqrt_ws = std::sqrt(o.weight_scan);
  a.sqrt_wh = std::sqrt(o.weight_hallucination);

  DevBuf<double> d_xy;
  DevBuf<int32_t> d_frame_of;
  DevBuf<int32_t> d_offsets;
  DevBuf<int32_t> d_hal;
  DevBuf<int32_t> d_hal_before;
  DevBuf<int32_t> d_sums;
  d_xy.Alloc(2 * static_cast<size_t>(std::max<int64_t>(n, 1)));
  if (n > 0) {
    CudaCheck(cudaMemcpyAsync(d_xy.get(), scan_xy, 2 * static_cast<size_t>(n) * sizeof(double),
                              cudaMemcpyHostToDevice, s),
              "scans");
  }
  d_frame_of.Upload(frame_of, s);
  d_offsets.Upload(std::vector<int32_t>(scan_offsets, scan_offsets + num_frames + 1), s);
  d_hal.Alloc(static_cast<size_t>(std::max<int64_t>(n, 1)));
  d_hal_before.Alloc(static_cast<size_t>(std::max<int64_t>(n, 1)));
  const auto* xy2 = reinterpret_cast<const double2*>(d_xy.get());
  int64_t hallucinating = 0;
  if (n > 0) {
    KHallucinating<<<Grid(n, 256), 256, 0, s>>>(xy2, n, d_hal.get());
    hallucinating = ExclusiveScan(d_hal.get(), n, d_hal_before.get(), d_sums, s);
  }
  const int64_t rows = n + (a.per_side > 0 ? static_cast<int64_t>(a.rows_per) * hallucinating : 0);
  if (rows >= (int64_t{1} << 31)) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT, "too many point rows");
  }
  DevBuf<int32_t> d_pt_frame;
  DevBuf<double> d_pt_xy;
  DevBuf<double> d_pt_exp;
  DevBuf<double> d_pt_sw;
  d_pt_frame.Alloc(static_cast<size_t>(std::max<int64_t>(rows, 1)));
  d_pt_xy.Alloc(2 * static_cast<size_t>(std::max<int64_t>(rows, 1)));
  d_pt_exp.Alloc(static_cast<size_t>(std::max<int64_t>(rows, 1)));
  d_pt_sw.Alloc(static_cast<size_t>(std::max<int64_t>(rows, 1)));
  if (n > 0) {
    KExpandPoints<<<Grid(n, 256), 256, 0, s>>>(xy2, d_frame_of.get(), d_offsets.get(), d_hal_before.get(),
                                               d_hal.get(), n, a, d_pt_frame.get(),
                                               reinterpret_cast<double2*>(d_pt_xy.get()), d_pt_exp.get(),
                                               d_pt_sw.get());
  }
  // active-region maps
  DevBuf<int32_t> d_active;
  DevBuf<int32_t> d_prefix;
  DevBuf<int32_t> d_n2a;
  DevBuf<int32_t> d_a2n;
  DevBuf<double> d_trig;
  d_active.Alloc(static_cast<size_t>(nodes));
  d_prefix.Alloc(static_cast<size_t>(nodes));
  d_n2a.Alloc(static_cast<size_t>(nodes));
  d_a2n.Alloc(static_cast<size_t>(nodes));
  d_trig.Upload(trig, s);
  if (o.active_region != 0) {
    CudaCheck(cudaMemsetAsync(d_active.get(), 0, static_cast<size_t>(nodes) * sizeof(int32_t), s), "active");
    const GridArgs g{nx, ny, hp.min_x, hp.min_y, hp.dx(), hp.dy()};
    if (rows > 0) {
      KActiveMark<<<Grid(rows, 256), 256, 0, s>>>(d_pt_frame.get(), reinterpret_cast<const double2*>(d_pt_xy.get()),
                                                  rows, d_trig.get(), g, o.active_margin, d_active.get());
    }
  } else {
    std::vector<int32_t> ones(static_cast<size_t>(nodes), 1);
    d_active.Upload(ones, s);
  }
  const int64_t num_active = ExclusiveScan(d_active.get(), nodes, d_prefix.get(), d_sums, s);
  KNodeMaps<<<Grid(nodes, 256), 256, 0, s>>>(d_active.get(), d_prefix.get(), nodes, d_n2a.get(), d_a2n.get());
  // Eikonal spec list
  const int64_t cells = static_cast<int64_t>(nx - 1) * (ny - 1);
  DevBuf<double> d_nn;
  DevBuf<double> d_scale;
  DevBuf<int32_t> d_eflag;
  DevBuf<int32_t> d_eprefix;
  {
    // scan-point normals, then per-node normals and scales
    NormalGrids ng;
    const bool per_scan = o.normals_per_scan != 0;
    PrepareNormalGrids(hp, num_frames, scan_offsets, scan_xy, per_scan, &ng);
    FlatGrids world_flat;
    AppendGrid(ng.world_grid, 0, &world_flat);
    FlatGrids frame_flat;
    for (int f = 0; f < num_frames && per_scan; ++f) {
      AppendGrid(ng.frame_grids[static_cast<size_t>(f)], scan_offsets[f], &frame_flat);
    }
    const FlatGrids& scan_flat = per_scan ? frame_flat : world_flat;
    DevBuf<double> d_world;
    DevBuf<KnnGridDev> d_grids;
    DevBuf<int32_t> d_start;
    DevBuf<int32_t> d_items;
    DevBuf<int32_t> d_wstart;
    DevBuf<int32_t> d_witems;
    DevBuf<double> d_snorm;
    DevBuf<double> d_scorner;
    d_world.Alloc(std::max<size_t>(ng.world.size(), 2));
    d_snorm.Alloc(2 * static_cast<size_t>(std::max<int64_t>(n, 1)));
    d_scorner.Alloc(static_cast<size_t>(std::max<int64_t>(n, 1)));
    if (n > 0) {
      d_world.Upload(ng.world, s);
      d_grids.Upload(scan_flat.desc, s);
      d_start.Upload(scan_flat.start, s);
      d_items.Upload(scan_flat.items, s);
      const unsigned blocks = static_cast<unsigned>((n + 127) / 128);
      auto* world2 = reinterpret_cast<const double2*>(d_world.get());
      auto* snorm2 = reinterpret_cast<double2*>(d_snorm.get());
      if (k <= 16) {
        KScanNormals<16><<<blocks, 128, 0, s>>>(d_grids.get(), d_start.get(), d_items.get(), xy2, world2,
                                                d_frame_of.get(), d_trig.get(), n, k, per_scan ? 1 : 0, snorm2,
                                                d_scorner.get());
      } else {
        KScanNormals<kMaxNeighbors><<<blocks, 128, 0, s>>>(d_grids.get(), d_start.get(), d_items.get(), xy2, world2,
                                                           d_frame_of.get(), d_trig.get(), n, k, per_scan ? 1 : 0,
                                                           snorm2, d_scorner.get());
      }
      if (per_scan) {
        d_wstart.Upload(world_flat.start, s);
        d_witems.Upload(world_flat.items, s);
      }
    }
    d_nn.Alloc(2 * static_cast<size_t>(nodes));
    d_scale.Alloc(static_cast<size_t>(nodes));
    const GridArgs g{nx, ny, hp.min_x, hp.min_y, hp.dx(), hp.dy()};
    KnnGridDev wg = world_flat.desc[0];
    if (n == 0) {
      wg.count = 0;
    }
    KNodeNormals<<<Grid(nodes, 128), 128, 0, s>>>(
        wg, per_scan ? d_wstart.get() : d_start.get(), per_scan ? d_witems.get() : d_items.get(),
        reinterpret_cast<const double2*>(d_world.get()), reinterpret_cast<const double2*>(d_snorm.get()),
        d_scorner.get(), g, NodeNormalArgs{o.normals_method, o.normals_corner_threshold},
        reinterpret_cast<double2*>(d_nn.get()), d_scale.get());
    CudaCheck(cudaStreamSynchronize(s), "normals");
  }
  d_eflag.Alloc(static_cast<size_t>(cells));
  d_eprefix.Alloc(static_cast<size_t>(cells));
  KEikonalFlags<<<Grid(cells, 256), 256, 0, s>>>(d_n2a.get(), d_scale.get(), nx, ny, d_eflag.get());
  const int64_t num_eik = ExclusiveScan(d_eflag.get(), cells, d_eprefix.get(), d_sums, s);
  DevBuf<int32_t> d_eik_wh;
  DevBuf<double> d_eik_n;
  DevBuf<double> d_eik_sw;
  d_eik_wh.Alloc(2 * static_cast<size_t>(std::max<int64_t>(num_eik, 1)));
  d_eik_n.Alloc(2 * static_cast<size_t>(std::max<int64_t>(num_eik, 1)));
  d_eik_sw.Alloc(static_cast<size_t>(std::max<int64_t>(num_eik, 1)));
  KEikonalSpecs<<<Grid(cells, 256), 256, 0, s>>>(d_eflag.get(), d_eprefix.get(), d_nn.get(), d_scale.get(), nx, ny,
                                                 std::sqrt(o.weight_eikonal), d_eik_wh.get(), d_eik_n.get(),
                                                 d_eik_sw.get());
  CudaCheck(cudaGetLastError(), "device builder kernels");
  if (download_rows) {
    Download(hp.pt_frame, d_pt_frame.get(), static_cast<size_t>(rows), s);
    Download(hp.pt_xy, d_pt_xy.get(), 2 * static_cast<size_t>(rows), s);
    Download(hp.pt_expected, d_pt_exp.get(), static_cast<size_t>(rows), s);
    Download(hp.pt_sqrtw, d_pt_sw.get(), static_cast<size_t>(rows), s);
  }
  Download(hp.node_to_active, d_n2a.get(), static_cast<size_t>(nodes), s);
  Download(hp.active_to_node, d_a2n.get(), static_cast<size_t>(num_active), s);
  Download(hp.eik_wh, d_eik_wh.get(), 2 * static_cast<size_t>(num_eik), s);
  Download(hp.eik_n, d_eik_n.get(), 2 * static_cast<size_t>(num_eik), s);
  Download(hp.eik_sqrtw, d_eik_sw.get(), static_cast<size_t>(num_eik), s);
  CudaCheck(cudaStreamSynchronize(s), "device builder");
}

}  // namespace sdfgpu
