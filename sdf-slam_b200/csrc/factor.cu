// Multifrontal supernodal LDL^T of the damped normal equations and its
// triangular solves, level by level over the assembly tree. Fronts are FP64;
// in a mixed-precision solve the grid supernodes are factored in FP32 copies
// (every kernel picks the element type per supernode) while the dense pose
// root stays FP64; the solve vectors are always FP64.
//
// Replaces ParallelSimplicialLdlt::FactorizeParallel / Eigen's solve
// (src/solvers/parallel_ldlt.hpp:44-51,150-244; src/solvers/lm_solver.cpp:
// 352-364) with dense frontal work: every supernode's front is assembled from
// J^T J (written in place by the column kernels) plus its children's update
// matrices, its pivot columns are factored in panels of kPanel columns, and
// the Schur complement of the remaining rows is one rank-k update.
//
// Storage of a front (column major, leading dimension F = k + m): the lower
// triangle holds the assembled values, then L below each panel's diagonal
// block. The strictly lower part of each kPanel x kPanel diagonal block of L
// is stored transposed in the block's upper triangle, and D in `dvec`
// (permuted order), so the lower triangle of a diagonal block is never
// written while other blocks of the same panel still read it.
#include <cuda_runtime.h>

#include "device.cuh"

namespace sdfgpu {

constexpr int kPanel = 32;
constexpr int kTile = 64;
constexpr int kPanelRowsPerBlock = 128;

/// Work front of supernode S in the element type it is factored in.
template <typename T>
__device__ __forceinline__ T* WorkFront(const DeviceView& V, const SupernodeRec& S);
template <>
__device__ __forceinline__ double* WorkFront<double>(const DeviceView& V, const SupernodeRec& S) {
  return V.fronts + S.front_off;
}
template <>
__device__ __forceinline__ float* WorkFront<float>(const DeviceView& V, const SupernodeRec& S) {
  return V.fronts32 + S.front_off;
}

/// 1 / d by Newton-Raphson iteration x <- x + x (1 - d x), seeded with the
/// hardware's approximate reciprocal (two steps square its ~2^-23 error
/// below FP64 precision). Much shorter latency than a correctly rounded
/// division on the pivot chain; the result may differ from 1.0 / d in the
/// last bit.
__device__ __forceinline__ double Recip(double d) {
  double x;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(x) : "d"(d));
  double e = fma(-d, x, 1.0);
  x = fma(x, e, x);
  e = fma(-d, x, 1.0);
  return fma(x, e, x);
}
__device__ __forceinline__ float Recip(float d) { return 1.0f / d; }

/// LDL^T of the w x w (w <= 32) diagonal block at B (row r, column c at
/// B[r * ld + c], lower triangle) by the block's first four warps (threads
/// 0..127): lane i owns row i, warp q owns columns 8q..8q+7 in registers. At
/// pivot j the owning warp inverts d_j (Newton reciprocal) and publishes
/// W(:, j) and L(:, j) in shared memory (two buffers, alternating with j),
/// one named barrier (id 1, 128 threads) later every warp subtracts
/// W(i, j) L(c, j) from its columns; lanes that must not change a column
/// subtract zero (a per-column branch costs more than the multiply-add).
/// Measured on B200 for a 32x32 block: 10.7k cycles against 28k for one warp
/// holding whole rows. Writes L below the diagonal and D on it; returns true
/// when a pivot is exactly zero (in the four warps).
template <typename T>
__device__ __forceinline__ bool DiagonalBlockLdlt(T* B, int ld, int w, T (*lbuf)[kPanel], T (*wbuf)[kPanel]) {
  const int lane = threadIdx.x & 31;
  const int q = threadIdx.x >> 5;
  T col[8];
#pragma unroll
  for (int t = 0; t < 8; ++t) {
    const int c = 8 * q + t;
    col[t] = (lane < w && c <= lane) ? B[lane * ld + c] : (c == lane ? T(1) : T(0));
  }
  bool zero = false;
  for (int jb = 0; jb < 4; ++jb) {
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      const int j = 8 * jb + t;
      if (j < w) {
        const int b = j & 1;
        if (q == jb) {
          const T dj = __shfl_sync(0xffffffffu, col[t], j);
          const T wij = col[t];
          const T lij = wij * Recip(dj);
          lbuf[b][lane] = lij;
          wbuf[b][lane] = wij;
          if (lane < w && lane >= j) {
            B[lane * ld + j] = lane == j ? dj : lij;
          }
        }
        asm volatile("bar.sync 1, 128;" ::: "memory");
        zero = zero || (wbuf[b][j] == T(0));
        const T m = lane > j ? wbuf[b][lane] : T(0);
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const int c = 8 * q + u;
          const T mu = (c > j && c <= lane) ? m : T(0);
          col[u] = fma(-mu, lbuf[b][c], col[u]);
        }
      }
    }
  }
  return zero;
}

/// Adds one child's update columns [cbeg, cend) into the parent front.
template <typename TP, typename TC>
__device__ __forceinline__ void ExtendAddChild(TP* Fp, int PF, const TC* U, int CF, const int32_t* rel, int m,
                                               int cbeg, int cend) {
  const int lane = threadIdx.x & 31;
  const int nwarps = blockDim.x >> 5;
  for (int cc = cbeg + (threadIdx.x >> 5); cc < cend; cc += nwarps) {
    TP* __restrict__ dst = Fp + static_cast<int64_t>(rel[cc]) * PF;
    const TC* __restrict__ src = U + static_cast<int64_t>(cc) * CF;
#pragma unroll 4
    for (int r = cc + lane; r < m; r += 32) {
      dst[rel[r]] += static_cast<TP>(src[r]);
    }
  }
}

template <typename TP>
__device__ __forceinline__ void ExtendAddBody(const DeviceView& V, const SupernodeRec& P, const int32_t* ranges) {
  TP* Fp = WorkFront<TP>(V, P);
  for (int ci = 0; ci < P.child_count; ++ci) {
    const SupernodeRec C = V.sn[V.child_list[P.child_begin + ci]];
    const int32_t* rel = V.sn_rel + C.rows_off;
    // update columns of this child that land in the task's parent columns
    const int cbeg = ranges[2 * ci];
    const int cend = ranges[2 * ci + 1];
    const int64_t uoff = static_cast<int64_t>(C.ncols) * C.F + C.ncols;
    if (Fp32Front(V, C)) {
      ExtendAddChild<TP, float>(Fp, P.F, WorkFront<float>(V, C) + uoff, C.F, rel, C.nrows, cbeg, cend);
    } else {
      ExtendAddChild<TP, double>(Fp, P.F, WorkFront<double>(V, C) + uoff, C.F, rel, C.nrows, cbeg, cend);
    }
    __syncthreads();
  }
}

/// Adds the children's update matrices into each parent front. A task owns a
/// range of parent columns, so no two blocks write the same entry; children
/// are added in their fixed order.
__global__ void KExtendAdd(DeviceView V, const int32_t* tasks, const int32_t* child_ranges) {
  const int32_t* t = tasks + 4 * static_cast<int64_t>(blockIdx.x);
  const SupernodeRec P = V.sn[t[0]];
  if (V.active[P.instance] == 0) {
    return;
  }
  if (Fp32Front(V, P)) {
    ExtendAddBody<float>(V, P, child_ranges + t[3]);
  } else {
    ExtendAddBody<double>(V, P, child_ranges + t[3]);
  }
}

template <typename T>
__device__ __forceinline__ void PanelBody(const DeviceView& V, const SupernodeRec& S, int panel, int row_begin,
                                          int rows, double* dvec, T (*D)[kPanel + 1], T (*lbuf)[kPanel],
                                          T (*wbuf)[kPanel]) {
  const int F = S.F;
  const int c0 = panel * kPanel;
  const int w = min(kPanel, S.ncols - c0);
  const int c1 = c0 + w;
  T* Fs = WorkFront<T>(V, S);
  const int tid = threadIdx.x;
  for (int idx = tid; idx < kPanel * kPanel; idx += blockDim.x) {
    const int i = idx % kPanel;
    const int j = idx / kPanel;
    T v;
    if (i < w && j < w) {
      v = i >= j ? Fs[static_cast<int64_t>(c0 + j) * F + (c0 + i)] : T(0);
    } else {
      v = (i == j) ? T(1) : T(0);
    }
    D[i][j] = v;
  }
  __syncthreads();
  __shared__ T dinv[kPanel];
  const bool zero_pivot = DiagonalBlockLdlt<T>(&D[0][0], kPanel + 1, w, lbuf, wbuf);
  if (tid < kPanel) {
    dinv[tid] = Recip(D[tid][tid]);
  }
  __syncthreads();
  if (row_begin == c1) {
    // first block of the panel: D into dvec, L11 transposed into the upper
    // triangle of the diagonal block
    if (tid < w) {
      dvec[S.first_col + c0 + tid] = static_cast<double>(D[tid][tid]);
    }
    for (int idx = tid; idx < kPanel * kPanel; idx += blockDim.x) {
      const int i = idx % kPanel;
      const int j = idx / kPanel;
      if (i > j && i < w) {
        Fs[static_cast<int64_t>(c0 + i) * F + (c0 + j)] = D[i][j];
      }
    }
    if (tid == 0 && zero_pivot) {
      atomicOr(V.status + S.instance, kStatusZeroPivot);
    }
  }
  const int r = row_begin + tid;
  if (tid < rows && r < F && r >= c1) {
    T y[kPanel];
#pragma unroll
    for (int j = 0; j < kPanel; ++j) {
      y[j] = j < w ? Fs[static_cast<int64_t>(c0 + j) * F + r] : T(0);
    }
#pragma unroll
    for (int j = 1; j < kPanel; ++j) {
#pragma unroll
      for (int l = 0; l < j; ++l) {
        y[j] -= y[l] * D[j][l];
      }
    }
#pragma unroll
    for (int j = 0; j < kPanel; ++j) {
      if (j < w) {
        Fs[static_cast<int64_t>(c0 + j) * F + r] = y[j] * dinv[j];
      }
    }
  }
}

/// Panel factorization: LDL^T of the panel's diagonal block (redundantly in
/// every block of the panel, written back by the first), then
/// L(r, panel) = A(r, panel) L11^-T D^-1 for a chunk of `rows` rows below it.
/// Launched with kPanelRowsPerBlock (128) threads: the diagonal block needs
/// four warps.
__global__ void __launch_bounds__(kPanelRowsPerBlock) KPanel(DeviceView V, const int32_t* tasks, double* dvec,
                                                             int rows) {
  const int32_t* t = tasks + 3 * static_cast<int64_t>(blockIdx.x);
  const SupernodeRec S = V.sn[t[0]];
  if (V.active[S.instance] == 0) {
    return;
  }
  __shared__ double buf[kPanel * (kPanel + 1)];
  __shared__ double lw[4][kPanel];
  if (Fp32Front(V, S)) {
    auto* l = reinterpret_cast<float(*)[kPanel]>(&lw[0][0]);
    PanelBody<float>(V, S, t[1], t[2], rows, dvec, reinterpret_cast<float(*)[kPanel + 1]>(buf), l, l + 2);
  } else {
    PanelBody<double>(V, S, t[1], t[2], rows, dvec, reinterpret_cast<double(*)[kPanel + 1]>(buf), lw, lw + 2);
  }
}

/// Pivot block of a front with at most kSmallPivots columns, factored in
/// one block: blocked LDL^T of the k x k pivot block in shared memory (warp 0
/// factors each 32-wide diagonal block, all threads solve the rows below it
/// inside the pivot block and apply the rank-32 update), then the rows below
/// the pivot block, `row_begin` onwards, get L(r, :) = A(r, :) L11^-T D^-1,
/// panel by panel, in registers. Every block of a front repeats the pivot
/// factorization; the one with row_begin == k writes L11 (the transposed
/// storage of the diagonal panel blocks) and D. Shared memory holds the pivot
/// block padded to a multiple of 32 rows and columns (the padding is zero, so
/// a narrow last panel needs no per-entry tests in the unrolled loops) and
/// the reciprocals of the pivots.
constexpr int kSmallPivots = 128;

/// Dynamic shared memory of KFactorFront for fronts of at most k pivots.
__host__ __device__ constexpr size_t FactorFrontSmem(int k) {
  const size_t kpad = static_cast<size_t>((k + kPanel - 1) / kPanel * kPanel);
  return (kpad * (kpad + 1) + kpad) * sizeof(double);
}

template <typename T>
__device__ __forceinline__ void FactorFrontBody(const DeviceView& V, const SupernodeRec& S, int row_begin, int rows,
                                                double* dvec, T* D, T (*lbuf)[kPanel], T (*wbuf)[kPanel]) {
  const int k = S.ncols;
  const int F = S.F;
  const int kpad = (k + kPanel - 1) / kPanel * kPanel;
  const int ld = kpad + 1;
  T* dinv = D + kpad * ld;
  T* Fs = WorkFront<T>(V, S);
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int nwarps = static_cast<int>(blockDim.x >> 5);
  const int lane = tid & 31;
  // one warp per column: coalesced loads of the column's lower part
  for (int c = warp; c < k; c += nwarps) {
    const T* src = Fs + static_cast<int64_t>(c) * F;
#pragma unroll 4
    for (int r = c + lane; r < k; r += 32) {
      D[r * ld + c] = src[r];
    }
  }
  for (int idx = k * ld + tid; idx < kpad * ld; idx += blockDim.x) {
    D[idx] = T(0);
  }
  __syncthreads();
  bool zero_pivot = false;
  for (int p0 = 0; p0 < k; p0 += kPanel) {
    const int w = min(kPanel, k - p0);
    if (warp < 4) {
      zero_pivot = DiagonalBlockLdlt<T>(D + p0 * ld + p0, ld, w, lbuf, wbuf) || zero_pivot;
      if (tid < w) {
        dinv[p0 + tid] = Recip(D[(p0 + tid) * ld + p0 + tid]);
      }
    }
    __syncthreads();
    // rows of the pivot block below this diagonal block (registers; the
    // panel is full width here because a later row exists)
    for (int r = p0 + w + tid; r < k; r += blockDim.x) {
      T* row = D + r * ld + p0;
      T y[kPanel];
#pragma unroll
      for (int j = 0; j < kPanel; ++j) {
        y[j] = row[j];
      }
#pragma unroll
      for (int j = 1; j < kPanel; ++j) {
#pragma unroll
        for (int l = 0; l < j; ++l) {
          y[j] -= y[l] * D[(p0 + j) * ld + p0 + l];
        }
      }
#pragma unroll
      for (int j = 0; j < kPanel; ++j) {
        row[j] = y[j] * dinv[p0 + j];
      }
    }
    __syncthreads();
    // rank-w update of the trailing pivot block: thread per column c with
    // d_l L(c, l) in registers, rows r >= c read as broadcasts (the panel is
    // full width here because a trailing column exists)
    for (int c = p0 + w + tid; c < k; c += blockDim.x) {
      T wc[kPanel];
#pragma unroll
      for (int l = 0; l < kPanel; ++l) {
        wc[l] = D[c * ld + p0 + l] * D[(p0 + l) * ld + p0 + l];
      }
      for (int r = c; r < k; ++r) {
        const T* lr = D + r * ld + p0;
        T a0 = T(0);
        T a1 = T(0);
#pragma unroll
        for (int l = 0; l < kPanel; l += 2) {
          a0 = fma(lr[l], wc[l], a0);
          a1 = fma(lr[l + 1], wc[l + 1], a1);
        }
        D[r * ld + c] -= a0 + a1;
      }
    }
    __syncthreads();
  }
  if (row_begin == k) {
    // L11 goes to the pivot block's upper triangle only: the other tasks of
    // this front may still be reading its lower triangle (the assembled A11)
    for (int r = warp; r < k; r += nwarps) {
      T* dst = Fs + static_cast<int64_t>(r) * F;
      for (int c = lane; c < r; c += 32) {
        dst[c] = D[r * ld + c];
      }
    }
    for (int j = tid; j < k; j += blockDim.x) {
      dvec[S.first_col + j] = static_cast<double>(D[j * ld + j]);
    }
    if (tid == 0 && zero_pivot) {
      atomicOr(V.status + S.instance, kStatusZeroPivot);
    }
  }
  // rows below the pivot block: thread per row, panel by panel
  const int r = row_begin + tid;
  if (r >= F || tid >= rows) {
    return;
  }
  for (int p0 = 0; p0 < k; p0 += kPanel) {
    const int w = min(kPanel, k - p0);
    T y[kPanel];
#pragma unroll
    for (int j = 0; j < kPanel; ++j) {
      y[j] = j < w ? Fs[static_cast<int64_t>(p0 + j) * F + r] : T(0);
    }
    // contributions of the earlier panels (each panel's 32 values of this
    // row loaded together, then 32 x 32 multiply-adds)
    for (int q0 = 0; q0 < p0; q0 += kPanel) {
      T yq[kPanel];
#pragma unroll
      for (int l = 0; l < kPanel; ++l) {
        yq[l] = Fs[static_cast<int64_t>(q0 + l) * F + r];
      }
#pragma unroll
      for (int l = 0; l < kPanel; ++l) {
        const T yl = yq[l] * D[(q0 + l) * ld + q0 + l];
#pragma unroll
        for (int j = 0; j < kPanel; ++j) {
          // rows p0 + j >= k (a narrow last panel) are the zero padding
          y[j] -= yl * D[(p0 + j) * ld + q0 + l];
        }
      }
    }
    // this panel's triangle (padding rows leave y[j >= w] unchanged)
#pragma unroll
    for (int j = 1; j < kPanel; ++j) {
#pragma unroll
      for (int l = 0; l < j; ++l) {
        y[j] -= y[l] * D[(p0 + j) * ld + p0 + l];
      }
    }
#pragma unroll
    for (int j = 0; j < kPanel; ++j) {
      if (j < w) {
        Fs[static_cast<int64_t>(p0 + j) * F + r] = y[j] * dinv[p0 + j];
      }
    }
  }
}

__global__ void __launch_bounds__(256) KFactorFront(DeviceView V, const int32_t* tasks, double* dvec) {
  extern __shared__ double sm[];
  const int32_t* t = tasks + 3 * static_cast<int64_t>(blockIdx.x);
  const SupernodeRec S = V.sn[t[0]];
  if (V.active[S.instance] == 0) {
    return;
  }
  __shared__ double lw[4][kPanel];
  if (Fp32Front(V, S)) {
    auto* l = reinterpret_cast<float(*)[kPanel]>(&lw[0][0]);
    FactorFrontBody<float>(V, S, t[1], t[2], dvec, reinterpret_cast<float*>(sm), l, l + 2);
  } else {
    FactorFrontBody<double>(V, S, t[1], t[2], dvec, sm, lw, lw + 2);
  }
}

template <typename T>
__device__ __forceinline__ void UpdateBody(const DeviceView& V, const SupernodeRec& S, int panel, int ti, int tj,
                                           const double* dvec, T (*As)[kTile], T (*Bs)[kTile]) {
  const int F = S.F;
  int kb;
  int ke;
  int r0;
  int cc0;
  int clim;
  if (panel >= 0) {
    kb = panel * kPanel;
    ke = min(S.ncols, kb + kPanel);
    r0 = ke + ti * kTile;
    cc0 = ke + tj * kTile;
    clim = S.ncols;
  } else {
    kb = 0;
    ke = S.ncols;
    r0 = S.ncols + ti * kTile;
    cc0 = S.ncols + tj * kTile;
    clim = F;
  }
  T* Fs = WorkFront<T>(V, S);
  const double* d = dvec + S.first_col;
  const int tid = threadIdx.x;
  const int tx = tid % 16;
  const int ty = tid / 16;
  T acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a) {
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      acc[a][b] = T(0);
    }
  }
  // the tile's current values, loaded now so that their latency hides
  // behind the K loop (no other block touches this tile)
  T cur[4][4];
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    const int c = cc0 + ty + 16 * b;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int r = r0 + tx + 16 * a;
      cur[a][b] = (c < clim && r < F && r >= c) ? Fs[static_cast<int64_t>(c) * F + r] : T(0);
    }
  }
  // K chunks of kPanel columns: the next chunk is loaded into registers
  // while the current one is multiplied out of shared memory
  constexpr int kPerThread = (kPanel * kTile) / 256;
  T ra[kPerThread];
  T rb[kPerThread];
  auto load_chunk = [&](int kk) {
    const int kw = min(kPanel, ke - kk);
#pragma unroll
    for (int q = 0; q < kPerThread; ++q) {
      const int idx = tid + 256 * q;
      const int rr = idx % kTile;
      const int l = idx / kTile;
      T av = T(0);
      T bv = T(0);
      if (l < kw) {
        const int64_t colbase = static_cast<int64_t>(kk + l) * F;
        if (r0 + rr < F) {
          av = Fs[colbase + r0 + rr] * static_cast<T>(d[kk + l]);
        }
        if (cc0 + rr < clim) {
          bv = Fs[colbase + cc0 + rr];
        }
      }
      ra[q] = av;
      rb[q] = bv;
    }
  };
  if (kb < ke) {
    load_chunk(kb);
  }
  for (int kk = kb; kk < ke; kk += kPanel) {
#pragma unroll
    for (int q = 0; q < kPerThread; ++q) {
      const int idx = tid + 256 * q;
      As[idx / kTile][idx % kTile] = ra[q];
      Bs[idx / kTile][idx % kTile] = rb[q];
    }
    __syncthreads();
    if (kk + kPanel < ke) {
      load_chunk(kk + kPanel);
    }
#pragma unroll 8
    for (int l = 0; l < kPanel; ++l) {
      T av[4];
      T bv[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        av[a] = As[l][tx + 16 * a];
        bv[a] = Bs[l][ty + 16 * a];
      }
#pragma unroll
      for (int a = 0; a < 4; ++a) {
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          acc[a][b] = fma(av[a], bv[b], acc[a][b]);
        }
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    const int c = cc0 + ty + 16 * b;
    if (c >= clim) {
      continue;
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int r = r0 + tx + 16 * a;
      if (r < F && r >= c) {
        Fs[static_cast<int64_t>(c) * F + r] = cur[a][b] - acc[a][b];
      }
    }
  }
}

/// Tiled rank-k update C -= L_I D L_J^T (lower part only). panel >= 0:
/// update of the remaining pivot columns by one panel; panel == -1: Schur
/// complement of the trailing m x m block by all k pivots.
__global__ void __launch_bounds__(256, 2) KUpdate(DeviceView V, const int32_t* tasks, const double* dvec) {
  const int32_t* t = tasks + 4 * static_cast<int64_t>(blockIdx.x);
  const SupernodeRec S = V.sn[t[0]];
  if (V.active[S.instance] == 0) {
    return;
  }
  __shared__ double as_buf[kPanel * kTile];
  __shared__ double bs_buf[kPanel * kTile];
  if (Fp32Front(V, S)) {
    UpdateBody<float>(V, S, t[1], t[2], t[3], dvec, reinterpret_cast<float(*)[kTile]>(as_buf),
                      reinterpret_cast<float(*)[kTile]>(bs_buf));
  } else {
    UpdateBody<double>(V, S, t[1], t[2], t[3], dvec, reinterpret_cast<double(*)[kTile]>(as_buf),
                       reinterpret_cast<double(*)[kTile]>(bs_buf));
  }
}

template <typename T>
__device__ __forceinline__ void ForwardBody(const DeviceView& V, const SupernodeRec& S, const double* dvec,
                                            double* v) {
  const int k = S.ncols;
  const int F = S.F;
  const T* Fs = WorkFront<T>(V, S);
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  for (int j = threadIdx.x; j < F; j += blockDim.x) {
    v[j] = j < k ? V.rhs[V.perm[S.first_col + j]] : 0.0;
  }
  __syncthreads();
  for (int ci = 0; ci < S.child_count; ++ci) {
    const SupernodeRec C = V.sn[V.child_list[S.child_begin + ci]];
    const int32_t* rel = V.sn_rel + C.rows_off;
    const double* u = V.upd + C.upd_off;
    for (int r = threadIdx.x; r < C.nrows; r += blockDim.x) {
      v[rel[r]] += u[r];
    }
    __syncthreads();
  }
  for (int p0 = 0; p0 < k; p0 += kPanel) {
    const int w = min(kPanel, k - p0);
    if (warp == 0) {
      // lane i preloads row i of the panel's unit triangle (same panel:
      // transposed storage), then the sequential sweep runs on registers
      double lrow[kPanel];
#pragma unroll
      for (int j = 0; j < kPanel; ++j) {
        lrow[j] = (j < lane && lane < w) ? static_cast<double>(Fs[static_cast<int64_t>(p0 + lane) * F + (p0 + j)])
                                         : 0.0;
      }
      double y = lane < w ? v[p0 + lane] : 0.0;
#pragma unroll
      for (int j = 0; j < kPanel; ++j) {
        const double yj = __shfl_sync(0xffffffffu, y, j);
        y -= lrow[j] * yj;
      }
      if (lane < w) {
        v[p0 + lane] = y;
      }
    }
    __syncthreads();
    for (int r = p0 + w + threadIdx.x; r < F; r += blockDim.x) {
      double acc = v[r];
      if (S.upper_l11 != 0 && r < k) {
        const T* lr = Fs + static_cast<int64_t>(r) * F + p0;
        for (int j = 0; j < w; ++j) {
          acc -= static_cast<double>(lr[j]) * v[p0 + j];
        }
      } else {
        for (int j = 0; j < w; ++j) {
          acc -= static_cast<double>(Fs[static_cast<int64_t>(p0 + j) * F + r]) * v[p0 + j];
        }
      }
      v[r] = acc;
    }
    __syncthreads();
  }
  for (int r = threadIdx.x; r < F - k; r += blockDim.x) {
    V.upd[S.upd_off + r] = v[k + r];
  }
  for (int j = threadIdx.x; j < k; j += blockDim.x) {
    V.xs[S.first_col + j] = (1.0 / dvec[S.first_col + j]) * v[j];
  }
}

/// Forward solve of one level: gathers the children's update vectors,
/// solves L11 y = v in 32-wide panels (warp 0 solves each panel's unit
/// triangle with shuffles, then all threads update every row below it,
/// including the front's m rows), stores the parent's update vector
/// u = v_m - L21 y and D^-1 y (Eigen's solve applies the inverse diagonal
/// between the two triangular sweeps). Vectors are FP64 whatever the
/// front's element type.
__global__ void __launch_bounds__(256) KForward(DeviceView V, const int32_t* level_sn, const double* dvec) {
  extern __shared__ double v[];
  const SupernodeRec S = V.sn[level_sn[blockIdx.x]];
  if (V.active[S.instance] == 0) {
    return;
  }
  if (Fp32Front(V, S)) {
    ForwardBody<float>(V, S, dvec, v);
  } else {
    ForwardBody<double>(V, S, dvec, v);
  }
}

template <typename T>
__device__ __forceinline__ void BackwardBody(const DeviceView& V, const SupernodeRec& S, double* z) {
  const int k = S.ncols;
  const int m = S.nrows;
  const int F = S.F;
  const T* Fs = WorkFront<T>(V, S);
  const int32_t* rows = V.sn_rows + S.rows_off;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  // the ancestors' solution at this front's rows, gathered once into shared
  // memory behind the k pivot slots (the gather's latency is paid once, not
  // once per column)
  double* xr = z + k;
  for (int r = threadIdx.x; r < m; r += blockDim.x) {
    xr[r] = V.xs[rows[r]];
  }
  __syncthreads();
  for (int j = warp; j < k; j += nwarps) {
    double acc = 0.0;
    const T* col = Fs + static_cast<int64_t>(j) * F + k;
    for (int r = lane; r < m; r += 32) {
      acc += static_cast<double>(col[r]) * xr[r];
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      acc += __shfl_down_sync(0xffffffffu, acc, off);
    }
    if (lane == 0) {
      z[j] = V.xs[S.first_col + j] - acc;
    }
  }
  __syncthreads();
  const int last = ((k - 1) / kPanel) * kPanel;
  for (int p0 = last; p0 >= 0; p0 -= kPanel) {
    const int w = min(kPanel, k - p0);
    // later pivots of this front: z[p0 + j] -= sum_{i >= p0 + w} L(i, p0 + j) x_i
    for (int j = warp; j < w; j += nwarps) {
      double acc = 0.0;
      if (S.upper_l11 != 0) {
        for (int i = p0 + w + lane; i < k; i += 32) {
          acc += static_cast<double>(Fs[static_cast<int64_t>(i) * F + p0 + j]) * z[i];
        }
      } else {
        const T* col = Fs + static_cast<int64_t>(p0 + j) * F;
        for (int i = p0 + w + lane; i < k; i += 32) {
          acc += static_cast<double>(col[i]) * z[i];
        }
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        acc += __shfl_down_sync(0xffffffffu, acc, off);
      }
      if (lane == 0) {
        z[p0 + j] -= acc;
      }
    }
    __syncthreads();
    if (warp == 0) {
      // lane i preloads column i of the panel's unit triangle: L(j, i) for
      // j > i (same panel: transposed storage)
      double lcolv[kPanel];
#pragma unroll
      for (int j = 0; j < kPanel; ++j) {
        lcolv[j] = (lane < j && j < w) ? static_cast<double>(Fs[static_cast<int64_t>(p0 + j) * F + (p0 + lane)])
                                       : 0.0;
      }
      double x = lane < w ? z[p0 + lane] : 0.0;
#pragma unroll
      for (int j = kPanel - 1; j >= 0; --j) {
        const double xj = __shfl_sync(0xffffffffu, x, j);
        x -= lcolv[j] * xj;
      }
      if (lane < w) {
        z[p0 + lane] = x;
      }
    }
    __syncthreads();
  }
  for (int j = threadIdx.x; j < k; j += blockDim.x) {
    V.xs[S.first_col + j] = z[j];
    V.step[V.perm[S.first_col + j]] = z[j];
  }
}

/// Backward solve of one level (root first): z = x_k - L21^T x_R with one
/// warp per column, then L11^T x = z in 32-wide panels from the last (all
/// threads subtract the later pivots' contribution, warp 0 solves the
/// panel's unit upper triangle with shuffles); writes the step in natural
/// order.
__global__ void __launch_bounds__(256) KBackward(DeviceView V, const int32_t* level_sn) {
  extern __shared__ double z[];
  const SupernodeRec S = V.sn[level_sn[blockIdx.x]];
  if (V.active[S.instance] == 0) {
    return;
  }
  if (Fp32Front(V, S)) {
    BackwardBody<float>(V, S, z);
  } else {
    BackwardBody<double>(V, S, z);
  }
}

}  // namespace sdfgpu

// ------------------------------------------------------------ launchers --

#include <mutex>

#include "engine.h"

namespace sdfgpu {

void ConfigureSolveKernels(int max_front) {
  // The attribute belongs to the kernel, not to an engine: it only grows, so
  // an engine with smaller fronts never lowers another engine's limit.
  static std::mutex mu;
  static int configured = 48 * 1024;
  static bool front_configured = false;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (!front_configured) {
      const int bytes = static_cast<int>(FactorFrontSmem(kSmallPivots));
      CudaCheck(cudaFuncSetAttribute(KFactorFront, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes), "smem attr");
      front_configured = true;
    }
  }
  const int smem = max_front * static_cast<int>(sizeof(double));
  if (smem > 227 * 1024) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT, "front too large for the solve kernels");
  }
  std::lock_guard<std::mutex> lk(mu);
  if (smem > configured) {
    CudaCheck(cudaFuncSetAttribute(KForward, cudaFuncAttributeMaxDynamicSharedMemorySize, smem), "smem attr");
    CudaCheck(cudaFuncSetAttribute(KBackward, cudaFuncAttributeMaxDynamicSharedMemorySize, smem), "smem attr");
    configured = smem;
  }
}

int LaunchFactorLevels(const Symbolic& S, const DeviceView& V, const FactorPlan& P, cudaStream_t stream) {
  // the diagonal blocks are factored by four warps of every factor block
  if (S.front_rows < 128 || S.front_rows > 256 || S.panel_rows < 1 || S.panel_rows > kPanelRowsPerBlock) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT, "factorization schedule out of range");
  }
  int launches = 0;
  for (int l = 0; l < S.num_levels; ++l) {
    const TaskRange ea = S.ea_range[static_cast<size_t>(l)];
    if (ea.count > 0) {
      KExtendAdd<<<static_cast<unsigned>(ea.count), 256, 0, stream>>>(V, P.ea_tasks + 4 * ea.begin, P.ea_child);
      ++launches;
    }
    const TaskRange sm = S.small_range[static_cast<size_t>(l)];
    if (sm.count > 0) {
      const int kmax = S.small_max_k[static_cast<size_t>(l)];
      const size_t bytes = FactorFrontSmem(kmax);
      KFactorFront<<<static_cast<unsigned>(sm.count), S.front_rows, bytes, stream>>>(V, P.small_tasks + 3 * sm.begin,
                                                                                  P.dvec);
      ++launches;
    }
    for (int t = 0; t < S.level_panels[static_cast<size_t>(l)]; ++t) {
      const size_t slot = static_cast<size_t>(S.panel_index_base[static_cast<size_t>(l)] + t);
      const TaskRange pr = S.panel_range[slot];
      if (pr.count > 0) {
        KPanel<<<static_cast<unsigned>(pr.count), kPanelRowsPerBlock, 0, stream>>>(V, P.panel_tasks + 3 * pr.begin,
                                                                                   P.dvec, S.panel_rows);
        ++launches;
      }
      const TaskRange ur = S.update_range[slot];
      if (ur.count > 0) {
        KUpdate<<<static_cast<unsigned>(ur.count), 256, 0, stream>>>(V, P.update_tasks + 4 * ur.begin, P.dvec);
        ++launches;
      }
    }
    const TaskRange sr = S.update_range[static_cast<size_t>(S.panel_index_base.back() + l)];
    if (sr.count > 0) {
      KUpdate<<<static_cast<unsigned>(sr.count), 256, 0, stream>>>(V, P.update_tasks + 4 * sr.begin, P.dvec);
      ++launches;
    }
  }
  CudaCheck(cudaGetLastError(), "factor kernels");
  return launches;
}

int LaunchSolveLevels(const Symbolic& S, const DeviceView& V, const FactorPlan& P, cudaStream_t stream) {
  int launches = 0;
  const size_t smem = static_cast<size_t>(P.max_front) * sizeof(double);
  for (int l = 0; l < S.num_levels; ++l) {
    const int b = S.level_begin[static_cast<size_t>(l)];
    const int e = S.level_begin[static_cast<size_t>(l) + 1];
    if (e > b) {
      KForward<<<static_cast<unsigned>(e - b), 256, smem, stream>>>(V, P.level_sn + b, P.dvec);
      ++launches;
    }
  }
  for (int l = S.num_levels - 1; l >= 0; --l) {
    const int b = S.level_begin[static_cast<size_t>(l)];
    const int e = S.level_begin[static_cast<size_t>(l) + 1];
    if (e > b) {
      KBackward<<<static_cast<unsigned>(e - b), 256, smem, stream>>>(V, P.level_sn + b);
      ++launches;
    }
  }
  CudaCheck(cudaGetLastError(), "solve kernels");
  return launches;
}

}  // namespace sdfgpu
