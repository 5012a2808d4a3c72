// Tiled LDL^T of the dense pose roots: one persistent launch per level.
//
// A pose root is the dense block of an instance's pose variables with no
// rows below it (the last front of the assembly tree; its LDL^T is the
// final, and for many poses the largest, step of the reference's
// factorization: src/solvers/parallel_ldlt.hpp:150-244). Factored panel by
// panel, its ceil(n / 32) panels form a chain of dependent launches. Here
// the front is cut into 64 x 64 tiles and factored right-looking as a task
// graph that every block of one launch works through:
//
//   FACTOR(k)      LDL^T of diagonal tile k (two 32-column halves), D into
//                  dvec, L^-1 of the tile into the inverse workspace; for
//                  k >= 1 it first does
//                  SOLVE(k, k - 1) and UPDATE(k, k, k - 1) itself (the
//                  critical path: no hand-over between those three);
//   SOLVE(i, k)    L(i, k) = A(i, k) L(k, k)^-T D(k)^-1, as a product with
//                  the stored inverse (i >= k + 2);
//   UPDATE(i,j,k)  A(i, j) -= L(i, k) D(k) L(j, k)^T, j <= i (lower part;
//                  not (k + 1, k + 1, k)).
//
// Each tile (i, j) has a counter: the updates applied to it (k of them before
// step k), plus one once it is factored (i == j) or solved (i > j); FACTOR(k)
// publishes tile (k, k - 1) as solved before it goes on. A task
// waits (one thread polling with acquire loads, bounded) until its inputs'
// counters reach their values and publishes its own with a release store
// after the block's writes; updates of a tile are applied in ascending k, so
// every entry is a fixed sequence of operations and the factor is the same
// bits from run to run. Blocks take tasks from a counter in an order sorted
// by bottom level (the longest path of task weights to the end of the
// graph), which lists every task after the tasks it waits for, so a waiting
// task's inputs are already taken by running blocks: the launch cannot
// deadlock whatever number of its blocks is resident. A wait that runs out
// marks the instance (kStatusWaitTimeout) and raises the abort flag, after
// which every remaining task is skipped.
//
// Output layout (what the solve and the diagonal-block inversion read, the
// same as the panel path's): L below each 32 x 32 diagonal block in the
// lower triangle, the strictly lower part of each 32 x 32 diagonal block of L
// transposed into its upper triangle, D in dvec.
#include "dense_root.h"

#include <algorithm>
#include <mutex>

#include "engine.h"
#include "front_ops.cuh"

namespace sdfgpu {
namespace {

constexpr int kDT = kDenseTileCols;
constexpr int kDThreads = 256;
constexpr int kDChunk = 32;
constexpr int kTLd = kDT + 1;
constexpr int kHLd = 33;
// FACTOR: the tile, L11^-1, A21 L11^-T, L22^-1 (32 x 33 each), 1 / d, the
// diagonal-block LDL^T's broadcast buffers and a flag
constexpr int kFactorDoubles = kDT * kTLd + 3 * 32 * kHLd + kDT + 4 * 32 + 2;
// SOLVE / UPDATE: two 32 x 64 staging buffers
constexpr int kGemmDoubles = 2 * kDChunk * kDT;
constexpr size_t kDenseSmem =
    static_cast<size_t>(kFactorDoubles > kGemmDoubles ? kFactorDoubles : kGemmDoubles) * sizeof(double);

__device__ __forceinline__ bool WaitTile(const int32_t* word, int32_t expected, const int32_t* abort,
                                         uint32_t limit) {
  for (uint32_t it = 0; it < limit; ++it) {
    int32_t v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(word) : "memory");
    if (v >= expected) {
      return true;
    }
    if (*reinterpret_cast<const volatile int32_t*>(abort) != 0) {
      return false;
    }
    __nanosleep(64);
  }
  return false;
}

__device__ __forceinline__ uint64_t GlobalTimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void PublishTile(int32_t* word, int32_t value) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(word), "r"(value) : "memory");
}

/// acc[a][b] += sum over l < kw of X(tx + 16 a, l) s_l Y(ty + 16 b, l) with
/// X(r, l) = X[l * ldx + r] (r < xr, else 0), Y(c, l) = Y[l * ldy + c]
/// (c < yr, else 0) and s = xscale (1 when null). K in chunks of 32 staged in
/// shared memory, the next chunk loaded into registers while the current
/// one is multiplied. Starts and ends with a block barrier.
__device__ __forceinline__ void TileProduct(const double* X, int64_t ldx, int xr, const double* Y, int64_t ldy,
                                            int yr, int kw, const double* xscale, double* sm, double acc[4][4]) {
  double(*As)[kDT] = reinterpret_cast<double(*)[kDT]>(sm);
  double(*Bs)[kDT] = reinterpret_cast<double(*)[kDT]>(sm + kDChunk * kDT);
  const int tid = threadIdx.x;
  const int tx = tid & 15;
  const int ty = tid >> 4;
  double ra[8];
  double rb[8];
  auto load = [&](int l0) {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int e = tid + kDThreads * q;
      const int l = l0 + (e >> 6);
      const int r = e & 63;
      const bool in = l < kw;
      const double s = (in && xscale != nullptr) ? xscale[l] : 1.0;
      ra[q] = (in && r < xr) ? X[static_cast<int64_t>(l) * ldx + r] * s : 0.0;
      rb[q] = (in && r < yr) ? Y[static_cast<int64_t>(l) * ldy + r] : 0.0;
    }
  };
  load(0);
  for (int l0 = 0; l0 < kw; l0 += kDChunk) {
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int e = tid + kDThreads * q;
      As[e >> 6][e & 63] = ra[q];
      Bs[e >> 6][e & 63] = rb[q];
    }
    __syncthreads();
    if (l0 + kDChunk < kw) {
      load(l0 + kDChunk);
    }
#pragma unroll 8
    for (int l = 0; l < kDChunk; ++l) {
      double av[4];
      double bv[4];
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
  }
  __syncthreads();
}

/// Columns c of M = L^-1 for the unit lower 32 x 32 triangle at T
/// (row-major, ld kTLd, L(i, j) = T[i][j] for i > j), one warp: lane c
/// solves L m = e_c by forward substitution (unrolled: a loop over the
/// pivots with the register vector indexed at run time measured three
/// times slower). M(i, c) -> Mo[i * kHLd + c].
__device__ __forceinline__ void InvertUnitLower32(const double* T, double* Mo) {
  const int lane = threadIdx.x & 31;
  double m[32];
#pragma unroll
  for (int i = 0; i < 32; ++i) {
    m[i] = i == lane ? 1.0 : 0.0;
  }
#pragma unroll
  for (int j = 0; j < 32; ++j) {
#pragma unroll
    for (int i = j + 1; i < 32; ++i) {
      m[i] = fma(-T[i * kTLd + j], m[j], m[i]);
    }
  }
#pragma unroll
  for (int i = 0; i < 32; ++i) {
    Mo[i * kHLd + lane] = m[i];
  }
}

/// out(r, c) = sum over l < 32 of X[r * xld + l] Y[c * yld + l] for the
/// 32 x 32 block: thread (r = lane, c = warp + 8 q), four outputs each.
template <typename F>
__device__ __forceinline__ void Small32(const double* X, int xld, const double* Y, int yld, F&& sink) {
  const int r = threadIdx.x & 31;
  const int c0 = threadIdx.x >> 5;
  double s[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 8
  for (int l = 0; l < 32; ++l) {
    const double x = X[r * xld + l];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      s[q] = fma(x, Y[(c0 + 8 * q) * yld + l], s[q]);
    }
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    sink(r, c0 + 8 * q, s[q]);
  }
}

/// FACTOR(k) on the tile already in T (shared, row-major, lower triangle,
/// the identity beyond w): LDL^T as two 32-column halves (the second
/// updated by the first's L21 D1 L21^T), D into dvec, L into the front and,
/// when tiles below exist, L^-1 into the inverse workspace.
__device__ void FactorLoaded(const DeviceView& V, const SupernodeRec& S, int k, int nt, const DenseArgs& A,
                             double* sm) {
  const int64_t F = S.F;
  const int c0 = k * kDT;
  const int w = min(kDT, S.ncols - c0);
  double* Fs = V.fronts + S.front_off;
  double(*T)[kTLd] = reinterpret_cast<double(*)[kTLd]>(sm);
  double* M1 = sm + kDT * kTLd;  // L11^-1 (zero above the diagonal)
  double* Y = M1 + 32 * kHLd;    // A21 L11^-T = L21 D1, then L21 L11^-1
  double* M2 = Y + 32 * kHLd;    // L22^-1
  double* dinv = M2 + 32 * kHLd;
  double(*lbuf)[kPanel] = reinterpret_cast<double(*)[kPanel]>(dinv + kDT);
  double(*wbuf)[kPanel] = lbuf + 2;
  int* zflag = reinterpret_cast<int*>(dinv + kDT + 4 * kPanel);
  const int tid = threadIdx.x;
  if (tid < 128) {
    const bool z = DiagonalBlockLdlt<double>(&T[0][0], kTLd, min(32, w), lbuf, wbuf);
    if (tid == 0) {
      *zflag = z ? 1 : 0;
    }
  }
  __syncthreads();
  if (w > 32) {
    if (tid < 32) {
      InvertUnitLower32(&T[0][0], M1);
    } else if (tid < 64) {
      dinv[tid - 32] = Recip(T[tid - 32][tid - 32]);
    }
    __syncthreads();
    // Y = A21 M1^T
    Small32(&T[32][0], kTLd, M1, kHLd, [&](int r, int c, double v) { Y[r * kHLd + c] = v; });
    __syncthreads();
    // L21 = Y D1^-1 over A21; A22 -= L21 Y^T (lower part)
    {
      const int r = tid & 31;
      const int cb = tid >> 5;
      double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 8
      for (int j = 0; j < 32; ++j) {
        const double lr = Y[r * kHLd + j] * dinv[j];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          acc[q] = fma(lr, Y[(cb + 8 * q) * kHLd + j], acc[q]);
        }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int c = cb + 8 * q;
        T[32 + r][c] = Y[r * kHLd + c] * dinv[c];
        if (r >= c) {
          T[32 + r][32 + c] -= acc[q];
        }
      }
    }
    __syncthreads();
    if (tid < 128) {
      const bool z = DiagonalBlockLdlt<double>(&T[32][32], kTLd, w - 32, lbuf, wbuf);
      if (tid == 0 && z) {
        *zflag = 1;
      }
    }
    __syncthreads();
  }
  if (tid < w) {
    A.dvec[S.first_col + c0 + tid] = T[tid][tid];
  }
  // L of the tile into the front
  for (int e = tid; e < kDT * kDT; e += kDThreads) {
    const int j = e >> 6;
    const int i = e & 63;
    if (i < w && j < i) {
      if ((i >> 5) == (j >> 5)) {
        Fs[static_cast<int64_t>(c0 + i) * F + c0 + j] = T[i][j];
      } else {
        Fs[static_cast<int64_t>(c0 + j) * F + c0 + i] = T[i][j];
      }
    }
  }
  if (tid == 0 && *zflag != 0) {
    atomicOr(V.status + S.instance, kStatusZeroPivot);
  }
  {
    // L^-1 = [M1 0; -M2 L21 M1  M2] of the tile (the identity beyond w),
    // column major 64 x 64 into the workspace: the SOLVE tasks below the
    // tile and the solve's 64-row panels multiply by it
    double* Mo = A.inv + S.dense_inv + static_cast<int64_t>(k) * kDT * kDT;
    if (w <= 32) {
      // a narrow last tile: L11^-1 was not needed above
      if (tid < 32) {
        InvertUnitLower32(&T[0][0], M1);
      }
      __syncthreads();
    }
    if (tid < 32) {
      InvertUnitLower32(&T[32][32], M2);
    }
    // P = L21 M1 into Y: P(r, c) = sum_l L21(r, l) M1(l, c), with M1
    // column c read as a row of its transpose
    __syncthreads();
    {
      const int r = tid & 31;
      const int cb = tid >> 5;
      double p[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 8
      for (int l = 0; l < 32; ++l) {
        const double x = T[32 + r][l];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          p[q] = fma(x, M1[l * kHLd + cb + 8 * q], p[q]);
        }
      }
      __syncthreads();
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        Y[r * kHLd + cb + 8 * q] = p[q];
      }
    }
    __syncthreads();
    {
      const int r = tid & 31;
      const int cb = tid >> 5;
      double m[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 8
      for (int l = 0; l < 32; ++l) {
        const double x = M2[r * kHLd + l];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          m[q] = fma(x, Y[l * kHLd + cb + 8 * q], m[q]);
        }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int c = cb + 8 * q;
        Mo[static_cast<int64_t>(c) * kDT + 32 + r] = -m[q];
        Mo[static_cast<int64_t>(c) * kDT + r] = M1[r * kHLd + c];
        Mo[static_cast<int64_t>(32 + c) * kDT + 32 + r] = M2[r * kHLd + c];
        Mo[static_cast<int64_t>(32 + c) * kDT + r] = 0.0;
      }
    }
  }
}

/// Loads diagonal tile k's lower triangle into T (the identity beyond w),
/// subtracting sub(r, c) when given (the update folded into the task).
__device__ __forceinline__ void LoadDiagonal(const SupernodeRec& S, const double* Fs, int k, double* sm) {
  const int64_t F = S.F;
  const int c0 = k * kDT;
  const int w = min(kDT, S.ncols - c0);
  double(*T)[kTLd] = reinterpret_cast<double(*)[kTLd]>(sm);
  for (int e = threadIdx.x; e < kDT * kDT; e += kDThreads) {
    const int j = e >> 6;
    const int i = e & 63;
    double v;
    if (i < w && j < w) {
      v = i >= j ? Fs[static_cast<int64_t>(c0 + j) * F + c0 + i] : 0.0;
    } else {
      v = i == j ? 1.0 : 0.0;
    }
    T[i][j] = v;
  }
  __syncthreads();
}

/// SOLVE(i, k): L(i, k) = A(i, k) M^T D^-1 with M = L(k, k)^-1.
__device__ void SolveTile(const DeviceView& V, const SupernodeRec& S, int i, int k, const DenseArgs& A,
                          double* sm) {
  const int64_t F = S.F;
  const int c0 = k * kDT;
  const int r0 = i * kDT;
  const int w = min(kDT, S.ncols - c0);
  const int h = min(kDT, S.ncols - r0);
  double* Fs = V.fronts + S.front_off;
  const double* Mo = A.inv + S.dense_inv + static_cast<int64_t>(k) * kDT * kDT;
  double acc[4][4] = {};
  TileProduct(Fs + static_cast<int64_t>(c0) * F + r0, F, h, Mo, kDT, w, w, nullptr, sm, acc);
  const int tx = threadIdx.x & 15;
  const int ty = threadIdx.x >> 4;
  const double* d = A.dvec + S.first_col + c0;
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    const int c = ty + 16 * b;
    if (c < w) {
      const double di = Recip(d[c]);
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        const int r = tx + 16 * a;
        if (r < h) {
          Fs[static_cast<int64_t>(c0 + c) * F + r0 + r] = acc[a][b] * di;
        }
      }
    }
  }
}

/// acc = L(i, k) D(k) L(j, k)^T for output tile (i, j).
__device__ __forceinline__ void UpdateProduct(const SupernodeRec& S, const double* Fs, int i, int j, int k,
                                              const DenseArgs& A, double* sm, double acc[4][4]) {
  const int64_t F = S.F;
  const int c0 = k * kDT;
  const int w = min(kDT, S.ncols - c0);
  const int hi = min(kDT, S.ncols - i * kDT);
  const int hj = min(kDT, S.ncols - j * kDT);
  TileProduct(Fs + static_cast<int64_t>(c0) * F + i * kDT, F, hi, Fs + static_cast<int64_t>(c0) * F + j * kDT, F, hj,
              w, A.dvec + S.first_col + c0, sm, acc);
}

/// UPDATE(i, j, k): A(i, j) -= L(i, k) D(k) L(j, k)^T, lower part.
__device__ void UpdateTile(const DeviceView& V, const SupernodeRec& S, int i, int j, int k, const DenseArgs& A,
                           double* sm) {
  const int64_t F = S.F;
  const int ri = i * kDT;
  const int rj = j * kDT;
  const int hi = min(kDT, S.ncols - ri);
  const int hj = min(kDT, S.ncols - rj);
  double* Fs = V.fronts + S.front_off;
  double acc[4][4] = {};
  UpdateProduct(S, Fs, i, j, k, A, sm, acc);
  const int tx = threadIdx.x & 15;
  const int ty = threadIdx.x >> 4;
  // all sixteen reads, then the writes
  double old[4][4];
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    const int c = ty + 16 * b;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int r = tx + 16 * a;
      const bool in = r < hi && c < hj && (i != j || r >= c);
      old[a][b] = in ? Fs[static_cast<int64_t>(rj + c) * F + ri + r] : 0.0;
    }
  }
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    const int c = ty + 16 * b;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int r = tx + 16 * a;
      if (r < hi && c < hj && (i != j || r >= c)) {
        Fs[static_cast<int64_t>(rj + c) * F + ri + r] = old[a][b] - acc[a][b];
      }
    }
  }
}

/// FACTOR(k). For k >= 1 the task first does the two steps that feed it:
/// SOLVE(k, k - 1) (published as soon as it is written, for the other
/// updates of step k - 1) and UPDATE(k, k, k - 1), whose result goes
/// straight into the shared-memory tile instead of the front.
__device__ void FactorTask(const DeviceView& V, const SupernodeRec& S, int k, int nt, const DenseArgs& A,
                           int32_t* cnt, double* sm) {
  double* Fs = V.fronts + S.front_off;
  if (k == 0) {
    LoadDiagonal(S, Fs, 0, sm);
  } else {
    SolveTile(V, S, k, k - 1, A, sm);
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      PublishTile(cnt + k * nt + (k - 1), k);
    }
    double acc[4][4] = {};
    UpdateProduct(S, Fs, k, k, k - 1, A, sm, acc);
    const int64_t F = S.F;
    const int c0 = k * kDT;
    const int w = min(kDT, S.ncols - c0);
    double(*T)[kTLd] = reinterpret_cast<double(*)[kTLd]>(sm);
    const int tx = threadIdx.x & 15;
    const int ty = threadIdx.x >> 4;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int c = ty + 16 * b;
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        const int r = tx + 16 * a;
        double v;
        if (r < w && c < w) {
          v = r >= c ? Fs[static_cast<int64_t>(c0 + c) * F + c0 + r] - acc[a][b] : 0.0;
        } else {
          v = r == c ? 1.0 : 0.0;
        }
        T[r][c] = v;
      }
    }
    __syncthreads();
  }
  FactorLoaded(V, S, k, nt, A, sm);
}

__global__ void __launch_bounds__(kDThreads, 1) KDenseRoot(DeviceView V, DenseArgs A) {
  extern __shared__ double dense_sm[];
  __shared__ int task;
  __shared__ int go;
  const int tid = threadIdx.x;
  for (;;) {
    __syncthreads();
    if (tid == 0) {
      task = atomicAdd(A.claim, 1);
    }
    __syncthreads();
    const int64_t t = task;
    if (t >= A.count) {
      return;
    }
    const int32_t* q = A.tasks + 4 * t;
    const int s = q[0];
    const int i = q[1];
    const int j = q[2];
    const int k = q[3];
    const SupernodeRec S = V.sn[s];
    if (V.active[S.instance] == 0) {
      continue;
    }
    const int nt = (S.ncols + kDT - 1) / kDT;
    int32_t* cnt = A.cnt + S.dense_cnt;
    if (tid == 0) {
      if (A.trace != nullptr) {
        A.trace[3 * t] = GlobalTimer();
      }
      bool ok;
      if (i == k) {
        // FACTOR(k) with SOLVE(k, k - 1) and UPDATE(k, k, k - 1) folded in
        ok = k == 0 || (WaitTile(cnt + (k - 1) * nt + (k - 1), k, A.abort, A.wait_limit) &&
                        WaitTile(cnt + k * nt + (k - 1), k - 1, A.abort, A.wait_limit) &&
                        WaitTile(cnt + k * nt + k, k - 1, A.abort, A.wait_limit));
      } else if (j == k) {
        ok = WaitTile(cnt + k * nt + k, k + 1, A.abort, A.wait_limit) &&
             WaitTile(cnt + i * nt + k, k, A.abort, A.wait_limit);
      } else {
        ok = WaitTile(cnt + i * nt + k, k + 1, A.abort, A.wait_limit) &&
             (i == j || WaitTile(cnt + j * nt + k, k + 1, A.abort, A.wait_limit)) &&
             WaitTile(cnt + i * nt + j, k, A.abort, A.wait_limit);
      }
      if (!ok) {
        atomicOr(V.status + S.instance, kStatusWaitTimeout);
        atomicExch(A.abort, 1);
      }
      go = ok ? 1 : 0;
      if (A.trace != nullptr) {
        A.trace[3 * t + 1] = GlobalTimer();
      }
    }
    __syncthreads();
    if (go == 0) {
      continue;
    }
    if (i == k) {
      FactorTask(V, S, k, nt, A, cnt, dense_sm);
    } else if (j == k) {
      SolveTile(V, S, i, k, A, dense_sm);
    } else {
      UpdateTile(V, S, i, j, k, A, dense_sm);
    }
    __syncthreads();
    if (tid == 0) {
      __threadfence();
      PublishTile(cnt + i * nt + j, k + 1);
      if (A.trace != nullptr) {
        A.trace[3 * t + 2] = GlobalTimer();
      }
    }
  }
}

}  // namespace

int LaunchDenseRoots(const DeviceView& V, const DenseArgs& args, cudaStream_t stream) {
  if (args.count <= 0) {
    return 0;
  }
  static std::mutex mu;
  static int blocks_per_sm[64] = {};
  static int sms[64] = {};
  int dev = 0;
  CudaCheck(cudaGetDevice(&dev), "device");
  if (dev < 0 || dev >= 64) {
    Fail(SDFGPU_ERR_CUDA, "device index out of range");
  }
  const std::lock_guard<std::mutex> lock(mu);
  if (blocks_per_sm[dev] == 0) {
    CudaCheck(cudaFuncSetAttribute(KDenseRoot, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(kDenseSmem)),
              "dense root smem attr");
    int per_sm = 0;
    CudaCheck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, KDenseRoot, kDThreads, kDenseSmem),
              "dense root occupancy");
    CudaCheck(cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, dev), "sm count");
    blocks_per_sm[dev] = per_sm > 0 ? per_sm : 1;
  }
  const int64_t grid = std::min<int64_t>(args.count, static_cast<int64_t>(blocks_per_sm[dev]) * sms[dev]);
  KDenseRoot<<<static_cast<unsigned>(grid), kDThreads, kDenseSmem, stream>>>(V, args);
  CudaCheck(cudaGetLastError(), "dense root launch");
  return 1;
}

}  // namespace sdfgpu
