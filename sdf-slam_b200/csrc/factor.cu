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
#include "front_ops.cuh"

namespace sdfgpu {

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

/// Adds one child's update columns [cbeg, cend) in place into the parent
/// front (fronts too wide to stage): warp per column, lanes over rows.
template <typename TP, typename TC>
__device__ __forceinline__ void ExtendAddDirect(TP* Fp, int64_t PF, const TC* U, int CF, const int32_t* rel, int m,
                                                int cbeg, int cend) {
  const int lane = threadIdx.x & 31;
  const int nwarps = static_cast<int>(blockDim.x >> 5);
  constexpr int kBatchRows = 8;
  for (int cc = cbeg + static_cast<int>(threadIdx.x >> 5); cc < cend; cc += nwarps) {
    TP* __restrict__ dst = Fp + rel[cc] * PF;
    const TC* __restrict__ src = U + static_cast<int64_t>(cc) * CF;
    // a child's rows land on distinct parent rows: all reads of a batch,
    // then all writes, so the batch's read-modify-writes overlap instead of
    // each waiting for the one before
    for (int r0 = cc + lane; r0 < m; r0 += 32 * kBatchRows) {
      int d[kBatchRows];
      TC u[kBatchRows];
#pragma unroll
      for (int q = 0; q < kBatchRows; ++q) {
        const int r = r0 + 32 * q;
        d[q] = r < m ? rel[r] : -1;
        u[q] = r < m ? src[r] : TC(0);
      }
      TP old[kBatchRows];
#pragma unroll
      for (int q = 0; q < kBatchRows; ++q) {
        old[q] = d[q] >= 0 ? dst[d[q]] : TP(0);
      }
#pragma unroll
      for (int q = 0; q < kBatchRows; ++q) {
        if (d[q] >= 0) {
          dst[d[q]] = old[q] + static_cast<TP>(u[q]);
        }
      }
    }
  }
}

/// Adds one child's update columns [cbeg, cend) into the staged parent
/// columns (stage: `rows` values per parent column from row c). Four entries
/// per thread per batch, their loads issued together.
template <typename TP, typename TC>
__device__ __forceinline__ void ExtendAddStaged(TP* stage, int c, int rows, const TC* U, int CF,
                                                const int32_t* rel, int m, int cbeg, int cend) {
  const int nthreads = static_cast<int>(blockDim.x);
  const int items = (cend - cbeg) * m;
  for (int base = threadIdx.x; base < items; base += 4 * nthreads) {
    int dst[4];
    TC val[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int idx = base + u * nthreads;
      const int cq = idx / m;
      const int r = idx - cq * m;
      const int cc = cbeg + cq;
      const bool ok = idx < items && r >= cc;
      dst[u] = ok ? (rel[cc] - c) * rows + (rel[r] - c) : -1;
      val[u] = ok ? U[static_cast<int64_t>(cc) * CF + r] : TC(0);
    }
    // one child's entries are distinct: all reads, then all writes
    TP old[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      old[u] = dst[u] >= 0 ? stage[dst[u]] : TP(0);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if (dst[u] >= 0) {
        stage[dst[u]] = old[u] + static_cast<TP>(val[u]);
      }
    }
  }
}

/// Extend-add of one task, parent columns [c, chi): with `stage` the
/// columns' lower part is copied into shared memory (one coalesced pass),
/// every child's entries are added there in the children's fixed order and
/// the columns are written back, so each entry sees the same additions in
/// the same order as an in-place add without a chain of dependent global
/// read-modify-writes; without it (a front too wide to stage) the children
/// are added in place.
/// A child whose update matrix is left in its own front for the extend-add:
/// the wide FP32 fronts whose Schur complement the tensor cores compute in
/// place. Every other front's Schur complement is added into its parent by
/// the Schur update itself.
__device__ __forceinline__ bool UpdateLeftInPlace(const DeviceView& V, const SupernodeRec& C) {
  return C.tc_pack >= 0 && V.tc_schur != 0 && Fp32Front(V, C);
}

template <typename TP>
__device__ __forceinline__ void ExtendAddBody(const DeviceView& V, const SupernodeRec& P, const int32_t* t,
                                              const int32_t* ranges, TP* stage) {
  const int tid = threadIdx.x;
  const int nthreads = static_cast<int>(blockDim.x);
  if (stage == nullptr) {
    for (int ci = 0; ci < P.child_count; ++ci) {
      const SupernodeRec C = V.sn[V.child_list[P.child_begin + ci]];
      if (!UpdateLeftInPlace(V, C)) {
        continue;
      }
      const int32_t* rel = V.sn_rel + C.rows_off;
      const int64_t uoff = static_cast<int64_t>(C.ncols) * C.F + C.ncols;
      if (Fp32Front(V, C)) {
        ExtendAddDirect<TP, float>(WorkFront<TP>(V, P), P.F, WorkFront<float>(V, C) + uoff, C.F, rel, C.nrows,
                                   ranges[2 * ci], ranges[2 * ci + 1]);
      } else {
        ExtendAddDirect<TP, double>(WorkFront<TP>(V, P), P.F, WorkFront<double>(V, C) + uoff, C.F, rel, C.nrows,
                                    ranges[2 * ci], ranges[2 * ci + 1]);
      }
      __syncthreads();
    }
    return;
  }
  const int c = t[1];
  const int width = t[2] - c;
  const int rows = P.F - c;
  const int n = width * rows;
  const int64_t PF = P.F;
  TP* Fp = WorkFront<TP>(V, P) + c * PF + c;
  for (int base = tid; base < n; base += 4 * nthreads) {
    TP v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int idx = base + u * nthreads;
      const int jj = idx / rows;
      const int ii = idx - jj * rows;
      v[u] = (idx < n && ii >= jj) ? Fp[jj * PF + ii] : TP(0);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int idx = base + u * nthreads;
      if (idx < n) {
        stage[idx] = v[u];
      }
    }
  }
  __syncthreads();
  for (int ci = 0; ci < P.child_count; ++ci) {
    const SupernodeRec C = V.sn[V.child_list[P.child_begin + ci]];
    if (!UpdateLeftInPlace(V, C)) {
      continue;
    }
    const int32_t* rel = V.sn_rel + C.rows_off;
    const int64_t uoff = static_cast<int64_t>(C.ncols) * C.F + C.ncols;
    if (Fp32Front(V, C)) {
      ExtendAddStaged<TP, float>(stage, c, rows, WorkFront<float>(V, C) + uoff, C.F, rel, C.nrows,
                                 ranges[2 * ci], ranges[2 * ci + 1]);
    } else {
      ExtendAddStaged<TP, double>(stage, c, rows, WorkFront<double>(V, C) + uoff, C.F, rel, C.nrows,
                                  ranges[2 * ci], ranges[2 * ci + 1]);
    }
    __syncthreads();
  }
  for (int idx = tid; idx < n; idx += nthreads) {
    const int jj = idx / rows;
    const int ii = idx - jj * rows;
    if (ii >= jj) {
      Fp[jj * PF + ii] = stage[idx];
    }
  }
}

/// Adds the children's update matrices into each parent front. A task owns a
/// range of parent columns, so no two blocks write the same entry; children
/// are added in their fixed order. staged != 0: the launch's dynamic shared
/// memory holds the columns of every task whose front is at most
/// kEaStageMaxF wide.
__global__ void KExtendAdd(DeviceView V, const int32_t* tasks, const int32_t* child_ranges, int staged) {
  extern __shared__ double stage[];
  const int32_t* t = tasks + 4 * static_cast<int64_t>(blockIdx.x);
  const SupernodeRec P = V.sn[t[0]];
  if (V.active[P.instance] == 0) {
    return;
  }
  // the task's columns are staged when the front is narrow enough (the
  // symbolic analysis sized the launch's shared memory for those)
  const bool use_stage = staged != 0 && P.F <= kEaStageMaxF;
  if (Fp32Front(V, P)) {
    ExtendAddBody<float>(V, P, t, child_ranges + t[3], use_stage ? reinterpret_cast<float*>(stage) : nullptr);
  } else {
    ExtendAddBody<double>(V, P, t, child_ranges + t[3], use_stage ? stage : nullptr);
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

/// Outer-block factorization of a front with more than small_pivots pivots:
/// the LDL^T of one outer block of kBlockCols pivot columns (after the
/// updates of every earlier block) and L for a chunk of kBlockRows rows
/// below it, in one CTA of 256 threads. Every CTA of a block factors the
/// block's diagonal tile itself (no CTA waits for another; the first
/// chunk's CTA writes the tile's L and D):
///  * the tile right-looking with its entries in registers (thread (tx, ty)
///    owns rows tx + 16 a and columns ty + 16 b), one pivot per step: the
///    owners of column j publish it to shared memory (two buffers
///    alternating with j, one barrier per step), every thread updates its
///    entries and scales its part of column j;
///  * the chunk's rows by forward substitution against L D: four threads
///    per row, each summing every fourth earlier column, a fixed butterfly
///    of two shuffles.
/// L of the tile's 32 x 32 diagonal blocks goes transposed into their upper
/// triangles, like the panel kernels store it; the rest of L column major.
constexpr int kBlockCols = kOuterPanels * kPanel;  // 128
constexpr int kBlockThreads = 256;
constexpr int kBlockLd = kBlockCols + 1;

/// Dynamic shared memory of KPanelBlock: W = L D of the tile, the chunk's
/// rows, the column buffers and the pivots (FP64 sizes).
__host__ __device__ constexpr size_t PanelBlockSmem() {
  return (static_cast<size_t>(kBlockCols) * kBlockLd + static_cast<size_t>(kBlockRows) * kBlockLd +
          3 * kBlockCols) *
         sizeof(double);
}

template <typename T>
__device__ __forceinline__ void PanelBlockBody(const DeviceView& V, const SupernodeRec& S, int block, int row_begin,
                                               double* dvec, T* smem) {
  const int F = S.F;
  const int64_t F64 = F;
  const int c0 = block * kBlockCols;
  const int w = min(kBlockCols, S.ncols - c0);
  const int c1 = c0 + w;
  const int rows = max(0, min(kBlockRows, F - row_begin));
  T* Fs = WorkFront<T>(V, S);
  T* Wt = smem;                          // kBlockCols x kBlockLd: W(j, l) = L(j, l) d_l, row major
  T* R = Wt + kBlockCols * kBlockLd;     // kBlockRows x kBlockLd: the chunk's rows, then their L
  T* colbuf = R + kBlockRows * kBlockLd; // 2 x kBlockCols
  T* dv = colbuf + 2 * kBlockCols;       // pivots
  const int tid = threadIdx.x;
  const int tx = tid & 15;
  const int ty = tid >> 4;
  // the chunk's rows (read down the front's columns)
  for (int e = tid; e < kBlockRows * kBlockCols; e += kBlockThreads) {
    const int l = e / kBlockRows;
    const int r = e % kBlockRows;
    R[r * kBlockLd + l] = (r < rows && l < w) ? Fs[(c0 + l) * F64 + row_begin + r] : T(0);
  }
  // the tile in registers (lower part; identity past w)
  T a[8][8];
#pragma unroll
  for (int ia = 0; ia < 8; ++ia) {
#pragma unroll
    for (int ib = 0; ib < 8; ++ib) {
      const int i = tx + 16 * ia;
      const int l = ty + 16 * ib;
      T v;
      if (i < w && l < w) {
        v = i >= l ? Fs[(c0 + l) * F64 + c0 + i] : T(0);
      } else {
        v = i == l ? T(1) : T(0);
      }
      a[ia][ib] = v;
    }
  }
  bool zero = false;
  for (int j = 0; j < kBlockCols; ++j) {
    T* cb = colbuf + (j & 1) * kBlockCols;
    const int jb = j >> 4;
    if (ty == (j & 15)) {
      // publish column j (entries on and below the diagonal)
#pragma unroll
      for (int ib = 0; ib < 8; ++ib) {
        if (ib == jb) {
#pragma unroll
          for (int ia = 0; ia < 8; ++ia) {
            cb[tx + 16 * ia] = a[ia][ib];
          }
        }
      }
    }
    __syncthreads();
    const T d = cb[j];
    zero = zero || d == T(0);
    const T di = Recip(d);
    T tl[8];
#pragma unroll
    for (int ib = 0; ib < 8; ++ib) {
      const int l = ty + 16 * ib;
      tl[ib] = l > j ? cb[l] * di : T(0);
    }
#pragma unroll
    for (int ia = 0; ia < 8; ++ia) {
      const int i = tx + 16 * ia;
      if (i > j) {
        const T ti = cb[i];
#pragma unroll
        for (int ib = 0; ib < 8; ++ib) {
          const int l = ty + 16 * ib;
          if (l > j && l <= i) {
            a[ia][ib] -= ti * tl[ib];
          }
        }
      }
    }
    // the owners of column j keep L(i, j) = A(i, j) / d below the diagonal
    if (ty == (j & 15)) {
#pragma unroll
      for (int ib = 0; ib < 8; ++ib) {
        if (ib == jb) {
#pragma unroll
          for (int ia = 0; ia < 8; ++ia) {
            if (tx + 16 * ia > j) {
              a[ia][ib] *= di;
            }
          }
        }
      }
    }
    if (tid == 0) {
      dv[j] = d;
    }
  }
  __syncthreads();
  // W = L D for the substitution (diagonal: d)
#pragma unroll
  for (int ia = 0; ia < 8; ++ia) {
#pragma unroll
    for (int ib = 0; ib < 8; ++ib) {
      const int i = tx + 16 * ia;
      const int l = ty + 16 * ib;
      if (l <= i) {
        Wt[i * kBlockLd + l] = l < i ? a[ia][ib] * dv[l] : dv[i];
      }
    }
  }
  __syncthreads();
  // rows below: L(r, j) = (A(r, j) - sum_{l<j} L(r, l) W(j, l)) / d_j
  {
    const int r = tid >> 2;
    const int q = tid & 3;
    T* Rr = R + r * kBlockLd;
    for (int j = 0; j < w; ++j) {
      const T* Wj = Wt + j * kBlockLd;
      T part = T(0);
      for (int l = q; l < j; l += 4) {
        part = fma(Rr[l], Wj[l], part);
      }
      part += __shfl_xor_sync(0xffffffffu, part, 1);
      part += __shfl_xor_sync(0xffffffffu, part, 2);
      if (q == 0) {
        Rr[j] = (Rr[j] - part) * Recip(Wj[j]);
      }
      __syncwarp();
    }
  }
  __syncthreads();
  if (row_begin == c1) {
    // the first chunk's CTA writes the tile's D and L
    for (int j = tid; j < w; j += kBlockThreads) {
      dvec[S.first_col + c0 + j] = static_cast<double>(dv[j]);
    }
#pragma unroll
    for (int ia = 0; ia < 8; ++ia) {
#pragma unroll
      for (int ib = 0; ib < 8; ++ib) {
        const int i = tx + 16 * ia;
        const int l = ty + 16 * ib;
        if (i < w && l < i) {
          if (i / kPanel == l / kPanel) {
            Fs[(c0 + i) * F64 + c0 + l] = a[ia][ib];  // transposed in the diagonal block
          } else {
            Fs[(c0 + l) * F64 + c0 + i] = a[ia][ib];
          }
        }
      }
    }
    if (tid == 0 && zero) {
      atomicOr(V.status + S.instance, kStatusZeroPivot);
    }
  }
  for (int e = tid; e < rows * w; e += kBlockThreads) {
    const int l = e / rows;
    const int rr = e % rows;
    Fs[(c0 + l) * F64 + row_begin + rr] = R[rr * kBlockLd + l];
  }
}

/// Tasks (sn, outer block, first row of the chunk below it).
__global__ void __launch_bounds__(kBlockThreads, 1) KPanelBlock(DeviceView V, const int32_t* tasks, double* dvec) {
  extern __shared__ double block_smem[];
  const int32_t* t = tasks + 3 * static_cast<int64_t>(blockIdx.x);
  const SupernodeRec S = V.sn[t[0]];
  if (V.active[S.instance] == 0) {
    return;
  }
  if (Fp32Front(V, S)) {
    PanelBlockBody<float>(V, S, t[1], t[2], dvec, reinterpret_cast<float*>(block_smem));
  } else {
    PanelBlockBody<double>(V, S, t[1], t[2], dvec, block_smem);
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

/// Dynamic shared memory of KFactorFront for fronts of at most k pivots: the
/// padded pivot block, the pivots' reciprocals and W = L D of one panel for
/// the trailing update (kPanel rows of kpad + 1).
__host__ __device__ constexpr size_t FactorFrontSmem(int k) {
  const size_t kpad = static_cast<size_t>((k + kPanel - 1) / kPanel * kPanel);
  return (kpad * (kpad + 1) + kpad + static_cast<size_t>(kPanel) * (kpad + 1)) * sizeof(double);
}

/// Rows per block up to which the rows below a pivot block are shared by
/// eight threads each.
constexpr int kRowsShared = 32;

/// Rows below the pivot block, eight threads per row (row = tid / 8 of a
/// pass over blockDim / 8 rows, the thread owning columns 4g..4g+3 of every
/// panel, g = tid % 8): per panel
/// the earlier panels' L values of the row (kept in shared memory) are
/// subtracted, then the panel's triangle is solved with the pivot values
/// passed between the row's threads by shuffles, then scaled by D^-1. Every
/// entry sees the same operations in the same order as the thread-per-row
/// path. Y: rows x (kpad + 1) values in shared memory.
template <typename T>
__device__ __forceinline__ void RowsBelowShared(T* Fs, int F, int k, int kpad, int ld, int row_begin, int rows,
                                                const T* D, const T* dinv, T* Y) {
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int g = tid & 7;
  const int base = lane & ~7;
  const int ldy = kpad + 1;
  const int np = (k + kPanel - 1) / kPanel;
  const int64_t F64 = F;
  const int per_pass = static_cast<int>(blockDim.x) >> 3;
  for (int rb = 0; rb < rows; rb += per_pass) {
    const int ri = rb + (tid >> 3);
    const int r = row_begin + ri;
    const bool live = ri < rows && r < F;
    // the row's assembled values in this thread's columns of every panel
    T a[kSmallPivots / kPanel][4];
#pragma unroll
    for (int p = 0; p < kSmallPivots / kPanel; ++p) {
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int j = p * kPanel + 4 * g + i;
        a[p][i] = (live && j < k) ? Fs[j * F64 + r] : T(0);
      }
    }
    T* yrow = Y + (live ? ri : 0) * ldy;
#pragma unroll
    for (int p = 0; p < kSmallPivots / kPanel; ++p) {
      if (p >= np) {
        break;
      }
      const int p0 = p * kPanel;
      T acc[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        acc[i] = a[p][i];
      }
      const T* drow = D + (p0 + 4 * g) * ld;
      // contributions of the earlier panels
      for (int q = 0; q < p; ++q) {
        const int q0 = q * kPanel;
#pragma unroll 8
        for (int l = 0; l < kPanel; ++l) {
          const T yl = yrow[q0 + l] * D[(q0 + l) * ld + q0 + l];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            acc[i] -= yl * drow[i * ld + q0 + l];
          }
        }
      }
      // this panel's triangle: pivot l's final value comes from its owner
#pragma unroll
      for (int l = 0; l < kPanel; ++l) {
        const T yl = __shfl_sync(0xffffffffu, acc[l & 3], base + (l >> 2));
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          if (4 * g + i > l) {
            acc[i] -= yl * drow[i * ld + p0 + l];
          }
        }
      }
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int j = p0 + 4 * g + i;
        if (j < k && live) {
          const T v = acc[i] * dinv[j];
          yrow[j] = v;
          Fs[j * F64 + r] = v;
        }
      }
      __syncwarp();
    }
  }
}

template <typename T>
__device__ __forceinline__ void FactorFrontBody(const DeviceView& V, const SupernodeRec& S, int row_begin, int rows,
                                                double* dvec, T* D, T (*lbuf)[kPanel], T (*wbuf)[kPanel]) {
  const int k = S.ncols;
  const int F = S.F;
  const int kpad = (k + kPanel - 1) / kPanel * kPanel;
  const int ld = kpad + 1;
  T* dinv = D + kpad * ld;
  T* W = dinv + kpad;  // [kPanel][ld]: W(c, l) = L(c, p0 + l) d_l at W[l * ld + c]
  T* Fs = WorkFront<T>(V, S);
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int nwarps = static_cast<int>(blockDim.x >> 5);
  const int lane = tid & 31;
  const int nthreads = static_cast<int>(blockDim.x);
  // the pivot block's lower triangle, column by column over all threads
  // (coalesced), eight loads in flight per thread
  {
    const int kk = k * k;
    for (int base = tid; base < kk; base += 8 * nthreads) {
      T val[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int i = base + u * nthreads;
        const int c = i / k;
        const int r = i - c * k;
        val[u] = (i < kk && r >= c) ? Fs[static_cast<int64_t>(c) * F + r] : T(0);
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int i = base + u * nthreads;
        const int c = i / k;
        const int r = i - c * k;
        if (i < kk && r >= c) {
          D[r * ld + c] = val[u];
        }
      }
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
    // rank-w update of the trailing pivot block (the panel is full width
    // here because a trailing column exists): W = L(:, panel) D first, then
    // one item per (4-row block, column) over all threads, rows read as
    // broadcasts and W along the columns; even and odd l accumulate
    // separately, as two chains per entry
    const int t0 = p0 + w;
    const int nt = k - t0;
    if (nt > 0) {
      for (int idx = tid; idx < kPanel * nt; idx += nthreads) {
        const int l = idx / nt;
        const int ci = idx - l * nt;
        W[l * ld + ci] = D[(t0 + ci) * ld + p0 + l] * D[(p0 + l) * ld + p0 + l];
      }
      __syncthreads();
      const int nrb = (nt + 3) / 4;
      for (int idx = tid; idx < nrb * nt; idx += nthreads) {
        const int rb = idx / nt;
        const int ci = idx - rb * nt;
        if (4 * rb + 3 < ci) {
          continue;  // the four rows lie above the diagonal
        }
        T a0[4];
        T a1[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          a0[u] = T(0);
          a1[u] = T(0);
        }
        const T* l0 = D + (t0 + 4 * rb) * ld + p0;
#pragma unroll
        for (int l = 0; l < kPanel; l += 2) {
          const T w0 = W[l * ld + ci];
          const T w1 = W[(l + 1) * ld + ci];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            a0[u] = fma(l0[u * ld + l], w0, a0[u]);
            a1[u] = fma(l0[u * ld + l + 1], w1, a1[u]);
          }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int r = 4 * rb + u;
          if (r < nt && r >= ci) {
            D[(t0 + r) * ld + t0 + ci] -= a0[u] + a1[u];
          }
        }
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
  if (rows <= kRowsShared && k <= kSmallPivots) {
    RowsBelowShared<T>(Fs, F, k, kpad, ld, row_begin, rows, D, dinv, W);
    return;
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

/// Adds one 64 x 64 tile of a front's Schur complement (cur - acc over the
/// front's trailing rows r and columns c, r >= c; rows and columns counted
/// from the front's first row, k pivots) into the parent front at the rows
/// rel[r - k], rel[c - k]. All sixteen parent reads first, then the writes.
template <typename TP, typename T>
__device__ __forceinline__ void ScatterSchur(TP* Fp, int64_t PF, const int32_t* rel, int k, int F, int r0, int cc0,
                                             const T (&cur)[4][4], const T (&acc)[4][4]) {
  const int tx = threadIdx.x % 16;
  const int ty = threadIdx.x / 16;
  int64_t pos[4][4];
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    const int c = cc0 + ty + 16 * b;
    const int64_t pc = c < F ? static_cast<int64_t>(rel[c - k]) * PF : -1;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int r = r0 + tx + 16 * a;
      pos[a][b] = (pc >= 0 && r < F && r >= c) ? pc + rel[r - k] : -1;
    }
  }
  TP old[4][4];
#pragma unroll
  for (int b = 0; b < 4; ++b) {
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      old[a][b] = pos[a][b] >= 0 ? Fp[pos[a][b]] : TP(0);
    }
  }
#pragma unroll
  for (int b = 0; b < 4; ++b) {
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      if (pos[a][b] >= 0) {
        Fp[pos[a][b]] = old[a][b] + static_cast<TP>(static_cast<T>(cur[a][b] - acc[a][b]));
      }
    }
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
  } else if (panel <= -2) {
    // outer blocks of kOuterPanels panels (UpdateCodeInner / Outer): a
    // panel's update within its outer block, or the finished block's
    // rank-(kOuterPanels * kPanel) update of the pivot columns past it
    const int x = -2 - panel;
    const int outer = kOuterPanels * kPanel;
    if ((x & 1) == 0) {
      kb = (x >> 1) * kPanel;
      ke = min(S.ncols, kb + kPanel);
      clim = min(S.ncols, (kb / outer + 1) * outer);
    } else {
      kb = (x >> 1) * outer;
      ke = min(S.ncols, kb + outer);
      clim = S.ncols;
    }
    r0 = ke + ti * kTile;
    cc0 = ke + tj * kTile;
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
  // behind the K loop (no other block touches this tile); a leaf's trailing
  // block holds no child contribution and is taken as zero, not loaded
  const bool fresh = panel == -1 && S.child_count == 0;
  T cur[4][4];
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    const int c = cc0 + ty + 16 * b;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int r = r0 + tx + 16 * a;
      cur[a][b] = (!fresh && c < clim && r < F && r >= c) ? Fs[static_cast<int64_t>(c) * F + r] : T(0);
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
  if (panel == -1 && S.parent >= 0) {
    // the Schur complement goes straight into the parent's front (what the
    // extend-add did with the update matrix), T-rounded as it was stored
    const SupernodeRec P = V.sn[S.parent];
    const int32_t* rel = V.sn_rel + S.rows_off;
    if (Fp32Front(V, P)) {
      ScatterSchur<float, T>(WorkFront<float>(V, P), P.F, rel, S.ncols, F, r0, cc0, cur, acc);
    } else {
      ScatterSchur<double, T>(WorkFront<double>(V, P), P.F, rel, S.ncols, F, r0, cc0, cur, acc);
    }
    return;
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

/// Tiled rank-k update C -= L_I D L_J^T (lower part only). panel <= -2: the
/// outer-block updates (UpdateCodeInner / Outer). panel >= 0:
/// update of the remaining pivot columns by one panel; panel == -1: Schur
/// complement of the trailing m x m block by all k pivots.
__global__ void __launch_bounds__(256, 2) KUpdate(DeviceView V, const int32_t* tasks, const double* dvec) {
  const int32_t* t = tasks + 4 * static_cast<int64_t>(blockIdx.x);
  const SupernodeRec S = V.sn[t[0]];
  if (V.active[S.instance] == 0) {
    return;
  }
  if (t[1] == -1) {
    return;  // Schur tiles: KSchur, KSchurF32; wide FP32 fronts: the tensor cores
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

/// Schur complement tiles added into the parent front (the task list of the
/// Schur update, panel -1), FP64 fronts and the FP32 fronts of a mixed solve
/// that the tensor cores do not take, built for occupancy: the K chunks are
/// copied global -> shared with cp.async (element-sized copies: a front's
/// columns start at any element offset), two chunks in flight, so no
/// staging registers; each thread then scales the A entries it copied by d
/// (the same product the register path forms); the tile's current values
/// are read after the K loop. Three blocks per SM (64 KB of shared memory
/// each; an FP32 tile uses half) against two for KUpdate.
constexpr int kSchurK = 32;
constexpr int kSchurBlocksPerSm = 3;
constexpr int kSchurPerThread = kSchurK * 64 / 256;  // entries of a chunk each thread copies
constexpr size_t kSchurSmem = 2 * 2 * static_cast<size_t>(kSchurK) * 64 * sizeof(double);

__device__ __forceinline__ void CpAsync(double* dst, const double* src) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void CpAsync(float* dst, const float* src) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}

/// The end of a KSchur tile: C - acc added into the parent front (or written
/// in place for a front with no parent), one column group of four entries at
/// a time, all parent reads of a group before its writes. kLoadC false: C is
/// known to be zero and is not read.
template <bool kLoadC>
__device__ __forceinline__ void SchurEpilogue(const DeviceView& V, const SupernodeRec& S, const double* Fs, int r0,
                                              int c0, const double (&acc)[4][4]) {
  const int k = S.ncols;
  const int F = S.F;
  const int tx = threadIdx.x & 15;
  const int ty = threadIdx.x >> 4;
  const bool scatter = S.parent >= 0;
  const SupernodeRec P = scatter ? V.sn[S.parent] : S;
  const int32_t* rel = V.sn_rel + S.rows_off;
  double* Fp = scatter ? V.fronts + P.front_off : V.fronts + S.front_off;
  const int64_t PF = P.F;
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    const int c = c0 + ty + 16 * b;
    double cur[4];
    int64_t pos[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int r = r0 + tx + 16 * a;
      const bool in = c < F && r < F && r >= c;
      cur[a] = (kLoadC && in) ? Fs[static_cast<int64_t>(c) * F + r] : 0.0;
      pos[a] = !in ? -1
                   : (scatter ? static_cast<int64_t>(rel[c - k]) * PF + rel[r - k] : static_cast<int64_t>(c) * F + r);
    }
    double old[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      old[a] = (scatter && pos[a] >= 0) ? Fp[pos[a]] : 0.0;
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      if (pos[a] >= 0) {
        Fp[pos[a]] = scatter ? old[a] + (cur[a] - acc[a][b]) : cur[a] - acc[a][b];
      }
    }
  }
}

/// The end of a KSchur tile of an FP32 front (the SIMT Schur complement of
/// a mixed solve): the tile's values (zero for a leaf, not loaded) minus
/// acc, added into the parent front Fp (FP32, or the FP64 pose root), or
/// written in place for a front with no parent (Fp is then the front
/// itself); one column group of four entries at a time, all parent reads of
/// a group before its writes; the same roundings as KUpdate's FP32 tiles.
template <typename TP>
__device__ __forceinline__ void SchurEpilogueF32(TP* Fp, int64_t PF, const int32_t* rel, const float* Fs, int k,
                                                 int F, int r0, int c0, const float (&acc)[4][4]) {
  const int tx = threadIdx.x & 15;
  const int ty = threadIdx.x >> 4;
  const bool scatter = rel != nullptr;
  const bool load = k < F && Fs != nullptr;
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    const int c = c0 + ty + 16 * b;
    float cur[4];
    int64_t pos[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int r = r0 + tx + 16 * a;
      const bool in = c < F && r < F && r >= c;
      cur[a] = (load && in) ? Fs[static_cast<int64_t>(c) * F + r] : 0.0f;
      pos[a] = !in ? -1
                   : (scatter ? static_cast<int64_t>(rel[c - k]) * PF + rel[r - k] : static_cast<int64_t>(c) * F + r);
    }
    TP old[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      old[a] = (scatter && pos[a] >= 0) ? Fp[pos[a]] : TP(0);
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      if (pos[a] >= 0) {
        const float v = cur[a] - acc[a][b];
        Fp[pos[a]] = scatter ? old[a] + static_cast<TP>(v) : static_cast<TP>(v);
      }
    }
  }
}

/// One 64 x 64 Schur complement tile of a front held in T (double: the
/// plain path and the pose root; float: a mixed solve's grid fronts that
/// the tensor cores do not take): K chunks staged by cp.async, two in
/// flight, A scaled by d in shared memory, acc accumulated in T in
/// ascending pivot order.
template <typename T>
__device__ __forceinline__ void SchurTile(const DeviceView& V, const SupernodeRec& S, const int32_t* t,
                                          const double* dvec, T* sm) {
  auto As = reinterpret_cast<T(*)[kSchurK][64]>(sm);
  auto Bs = reinterpret_cast<T(*)[kSchurK][64]>(sm + 2 * kSchurK * 64);
  const int k = S.ncols;
  const int F = S.F;
  const int r0 = k + t[2] * 64;
  const int c0 = k + t[3] * 64;
  T* Fs = WorkFront<T>(V, S);
  const double* d = dvec + S.first_col;
  const int tid = threadIdx.x;
  const int tx = tid & 15;
  const int ty = tid >> 4;
  auto issue = [&](int kk, int buf) {
#pragma unroll
    for (int q = 0; q < kSchurPerThread; ++q) {
      const int e = tid + 256 * q;
      const int l = e >> 6;
      const int rr = e & 63;
      const int col = kk + l;
      const int64_t base = static_cast<int64_t>(col) * F;
      if (col < k && r0 + rr < F) {
        CpAsync(&As[buf][l][rr], Fs + base + r0 + rr);
      } else {
        As[buf][l][rr] = T(0);
      }
      if (col < k && c0 + rr < F) {
        CpAsync(&Bs[buf][l][rr], Fs + base + c0 + rr);
      } else {
        Bs[buf][l][rr] = T(0);
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  T acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a) {
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      acc[a][b] = T(0);
    }
  }
  const int chunks = (k + kSchurK - 1) / kSchurK;
  issue(0, 0);
  if (chunks > 1) {
    issue(kSchurK, 1);
  }
  for (int ch = 0; ch < chunks; ++ch) {
    const int buf = ch & 1;
    if (ch + 1 < chunks) {
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    // the A entries this thread copied, times d (its own copies are
    // complete; the barrier below publishes them)
#pragma unroll
    for (int q = 0; q < kSchurPerThread; ++q) {
      const int e = tid + 256 * q;
      const int l = e >> 6;
      const int col = ch * kSchurK + l;
      if (col < k) {
        As[buf][l][e & 63] *= static_cast<T>(d[col]);
      }
    }
    __syncthreads();
#pragma unroll 8
    for (int l = 0; l < kSchurK; ++l) {
      T av[4];
      T bv[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        av[a] = As[buf][l][tx + 16 * a];
        bv[a] = Bs[buf][l][ty + 16 * a];
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
    if (ch + 2 < chunks) {
      issue((ch + 2) * kSchurK, buf);
    }
  }
  if constexpr (sizeof(T) == sizeof(double)) {
    // C - acc, added into the parent (or written in place for a front with
    // no parent); a leaf's C is zero (no child adds into it) and is not
    // loaded
    if (S.child_count == 0) {
      SchurEpilogue<false>(V, S, Fs, r0, c0, acc);
    } else {
      SchurEpilogue<true>(V, S, Fs, r0, c0, acc);
    }
  } else {
    // a leaf's C is zero (no child adds into it) and is not loaded
    const float* C = S.child_count > 0 ? Fs : nullptr;
    if (S.parent < 0) {
      SchurEpilogueF32<float>(Fs, F, nullptr, C, k, F, r0, c0, acc);
    } else {
      const SupernodeRec P = V.sn[S.parent];
      const int32_t* rel = V.sn_rel + S.rows_off;
      if (Fp32Front(V, P)) {
        SchurEpilogueF32<float>(WorkFront<float>(V, P), P.F, rel, C, k, F, r0, c0, acc);
      } else {
        SchurEpilogueF32<double>(WorkFront<double>(V, P), P.F, rel, C, k, F, r0, c0, acc);
      }
    }
  }
}

__global__ void __launch_bounds__(256, kSchurBlocksPerSm)
    KSchur(DeviceView V, const int32_t* tasks, const double* dvec) {
  const int32_t* t = tasks + 4 * static_cast<int64_t>(blockIdx.x);
  const SupernodeRec S = V.sn[t[0]];
  if (V.active[S.instance] == 0 || Fp32Front(V, S)) {
    return;  // FP32 fronts of a mixed solve: KSchurF32 or the tensor cores
  }
  extern __shared__ __align__(16) double schur_sm[];
  SchurTile<double>(V, S, t, dvec, schur_sm);
}

/// The same tiles for the FP32 fronts of a mixed solve that the tensor
/// cores do not take (a kernel of its own, so that neither variant's
/// registers limit the other's).
__global__ void __launch_bounds__(256, kSchurBlocksPerSm)
    KSchurF32(DeviceView V, const int32_t* tasks, const double* dvec) {
  const int32_t* t = tasks + 4 * static_cast<int64_t>(blockIdx.x);
  const SupernodeRec S = V.sn[t[0]];
  if (V.active[S.instance] == 0 || !Fp32Front(V, S) || (S.tc_pack >= 0 && V.tc_schur != 0)) {
    return;
  }
  extern __shared__ __align__(16) double schur_sm[];
  SchurTile<float>(V, S, t, dvec, reinterpret_cast<float*>(schur_sm));
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
      // L2 loads: another block of the same launch may have written them
      v[rel[r]] += __ldcg(u + r);
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
  // (L2 loads: another block of the same launch may have written them)
  for (int r = threadIdx.x; r < m; r += blockDim.x) {
    xr[r] = __ldcg(V.xs + rows[r]);
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
      z[j] = __ldcg(V.xs + S.first_col + j) - acc;
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

/// Doubles per inverted diagonal block: M = L^-1 of the block's unit lower
/// triangle, column major, then M^T, column major.
constexpr int kInvBlock = 2 * kPanel * kPanel;

/// Inverts the unit lower triangle of every kPanel-column diagonal block of
/// L (one warp per block, four per thread block): lane c solves L m = e_c
/// by forward substitution in registers, reading L from shared memory as
/// broadcasts. Columns of a narrow last panel beyond the pivots invert to
/// the identity. tasks: (sn, panel) pairs in panel_base order.
__global__ void __launch_bounds__(128) KInvertDiagonal(DeviceView V, const int32_t* tasks, int count, double* inv) {
  __shared__ double Ls[4][kPanel][kPanel + 1];
  const int wib = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int b = blockIdx.x * 4 + wib;
  if (b >= count) {
    return;
  }
  const SupernodeRec S = V.sn[tasks[2 * b]];
  if (V.active[S.instance] == 0) {
    return;
  }
  const int p0 = tasks[2 * b + 1] * kPanel;
  const int w = min(kPanel, S.ncols - p0);
  const int64_t F = S.F;
  double(*L)[kPanel + 1] = Ls[wib];
  // L(p0 + i, p0 + j), i > j, lives transposed in the block's upper
  // triangle: row i of L is contiguous
  if (Fp32Front(V, S)) {
    const float* Fs = V.fronts32 + S.front_off;
    for (int i = 0; i < kPanel; ++i) {
      L[i][lane] = (i < w && lane < i) ? static_cast<double>(Fs[(p0 + i) * F + p0 + lane]) : 0.0;
    }
  } else {
    const double* Fs = V.fronts + S.front_off;
    for (int i = 0; i < kPanel; ++i) {
      L[i][lane] = (i < w && lane < i) ? Fs[(p0 + i) * F + p0 + lane] : 0.0;
    }
  }
  __syncwarp();
  // right-looking: once m[j] is final it is subtracted from every later
  // row, so each step waits on one multiply-add only (each m[i] still sees
  // its terms in ascending j)
  double m[kPanel];
#pragma unroll
  for (int i = 0; i < kPanel; ++i) {
    m[i] = i == lane ? 1.0 : 0.0;
  }
#pragma unroll
  for (int j = 0; j < kPanel; ++j) {
#pragma unroll
    for (int i = j + 1; i < kPanel; ++i) {
      m[i] = fma(-L[i][j], m[j], m[i]);
    }
  }
  double* out = inv + static_cast<int64_t>(S.panel_base + p0 / kPanel) * kInvBlock;
  // M^T column major: (i, j) of M^T = M(j, i) = m[j] of lane i
#pragma unroll
  for (int j = 0; j < kPanel; ++j) {
    out[kPanel * kPanel + j * kPanel + lane] = m[j];
  }
  // M column major through shared memory: lane c holds column c
  __syncwarp();
#pragma unroll
  for (int i = 0; i < kPanel; ++i) {
    L[i][lane] = m[i];
  }
  __syncwarp();
  for (int j = 0; j < kPanel; ++j) {
    out[j * kPanel + lane] = L[lane][j];
  }
}

/// Issues an asynchronous copy of one kPanel x kPanel block of doubles
/// (16-byte chunks, L2 only) into shared memory and commits it as a group.
__device__ __forceinline__ void CopyBlockAsync(double* dst, const double* src) {
  for (int c = threadIdx.x; c < kPanel * kPanel / 2; c += blockDim.x) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst + 2 * c));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src + 2 * c) : "memory");
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
}

/// Waits for this thread's asynchronous copies.
__device__ __forceinline__ void WaitBlockCopies() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

/// Global loads a thread of the solve issues before using the first one.
constexpr int kBatch = 16;

/// Rows (or columns) of a panel update that lane pairs of the 224 threads
/// past warp 0 take with early loads.
constexpr int kPairRows = 112;

/// Doubles of shared memory the one-launch solve needs for fronts of at
/// most max_front rows: two inverted blocks, then the front's vector.
__host__ __device__ constexpr size_t SolveTreeSmem(int max_front) {
  return (2 * static_cast<size_t>(kPanel) * kPanel + static_cast<size_t>(max_front)) * sizeof(double);
}

/// L(r, c) of a front for a pivot-block row r below column c's panel:
/// transposed storage (row r contiguous) in single-kernel fronts, column
/// major otherwise.
template <typename T>
__device__ __forceinline__ T PivotL(const T* Fs, int64_t F, bool upper, int r, int c) {
  return upper ? Fs[r * F + c] : Fs[c * F + r];
}

/// u = v_m - L21 y over rows [r0, r1) of the rows below the pivot block:
/// thread per row, L21 column major (coalesced over rows), 16 loads in
/// flight per batch. v = y (k values); v_m(r) from vm[r], or from upd when
/// vm is null.
template <typename T>
__device__ __forceinline__ void ForwardRowsU(const DeviceView& V, const SupernodeRec& S, const T* Fs,
                                             const double* v, const double* vm, int r0, int r1) {
  const int k = S.ncols;
  const int64_t F64 = S.F;
  for (int r = r0 + static_cast<int>(threadIdx.x); r < r1; r += blockDim.x) {
    const T* col = Fs + k + r;
    double a0 = vm != nullptr ? vm[r] : V.upd[S.upd_off + r];
    double a1 = 0.0;
    for (int j0 = 0; j0 < k; j0 += kBatch) {
      T lv[kBatch];
#pragma unroll
      for (int j = 0; j < kBatch; ++j) {
        lv[j] = j0 + j < k ? col[(j0 + j) * F64] : T(0);
      }
#pragma unroll
      for (int j = 0; j < kBatch; j += 2) {
        a0 = fma(-static_cast<double>(lv[j]), j0 + j < k ? v[j0 + j] : 0.0, a0);
        a1 = fma(-static_cast<double>(lv[j + 1]), j0 + j + 1 < k ? v[j0 + j + 1] : 0.0, a1);
      }
    }
    V.upd[S.upd_off + r] = a0 + a1;
  }
}

/// Forward solve of one front for the one-launch solve. Gathers the
/// right-hand side and the children's update vectors, then per panel: warp 0
/// forms y_p = M_p v_p (M_p the inverted diagonal block, copied into shared
/// memory during the previous panel) while the threads that update the
/// later pivot rows load their L values; after a barrier those rows
/// subtract L(r, p) y_p. The m rows below the pivot block get
/// u = v_m - L21 y in one pass at the end; D^-1 y goes to xs. Every sum
/// runs in a fixed order. buf: two blocks for M, then F doubles for v.
template <typename T>
__device__ __forceinline__ void ForwardTreeBody(const DeviceView& V, const SupernodeRec& S, const double* dvec,
                                                const double* inv, double* buf, double* ys) {
  const int k = S.ncols;
  const int F = S.F;
  const int64_t F64 = F;
  const T* Fs = WorkFront<T>(V, S);
  const bool upper = S.upper_l11 != 0;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int nthreads = blockDim.x;
  double* Ms = buf;
  double* v = buf + 2 * kPanel * kPanel;
  const double* Mb = inv + static_cast<int64_t>(S.panel_base) * kInvBlock;
  CopyBlockAsync(Ms, Mb);
  for (int j = tid; j < F; j += nthreads) {
    v[j] = j < k ? V.rhs[V.perm[S.first_col + j]] : 0.0;
  }
  __syncthreads();
  for (int ci = 0; ci < S.child_count; ++ci) {
    const SupernodeRec C = V.sn[V.child_list[S.child_begin + ci]];
    const int32_t* rel = V.sn_rel + C.rows_off;
    const double* u = V.upd + C.upd_off;
    for (int r = tid; r < C.nrows; r += nthreads) {
      v[rel[r]] += __ldcg(u + r);
    }
    __syncthreads();
  }
  WaitBlockCopies();
  __syncthreads();
  for (int p0 = 0, q = 0; p0 < k; p0 += kPanel, ++q) {
    if (p0 + kPanel < k) {
      CopyBlockAsync(Ms + ((q + 1) & 1) * kPanel * kPanel, Mb + static_cast<int64_t>(q + 1) * kInvBlock);
    }
    // later pivot rows: lane pairs of warps 1.. own one row each (16 of its
    // L values per lane, loaded before the barrier); rows past the first
    // kPairRows loop below without the early loads
    const int r = p0 + kPanel + ((tid - 32) >> 1);
    const int half = (tid & 1) * (kPanel / 2);
    T lr[kPanel / 2];
    if (warp > 0 && r < k) {
      const T* src = upper ? Fs + r * F64 + p0 + half : Fs + (p0 + half) * F64 + r;
      const int64_t step = upper ? 1 : F64;
#pragma unroll
      for (int j = 0; j < kPanel / 2; ++j) {
        lr[j] = *src;
        src += step;
      }
    }
    if (warp == 0) {
      const double* M = Ms + (q & 1) * kPanel * kPanel;
      double a0 = 0.0;
      double a1 = 0.0;
#pragma unroll
      for (int j = 0; j < kPanel; j += 2) {
        // past the pivots (a narrow last panel) M is the identity's zero part
        const double v0 = p0 + j < k ? v[p0 + j] : 0.0;
        const double v1 = p0 + j + 1 < k ? v[p0 + j + 1] : 0.0;
        a0 = fma(M[j * kPanel + lane], v0, a0);
        a1 = fma(M[(j + 1) * kPanel + lane], v1, a1);
      }
      __syncwarp();
      if (p0 + lane < k) {
        v[p0 + lane] = a0 + a1;
      }
    }
    __syncthreads();
    if (warp > 0) {
      double part = 0.0;
      if (r < k) {
#pragma unroll
        for (int j = 0; j < kPanel / 2; ++j) {
          part = fma(static_cast<double>(lr[j]), v[p0 + half + j], part);
        }
      }
      part += __shfl_xor_sync(0xffffffffu, part, 1);
      if (half == 0 && r < k) {
        v[r] -= part;
      }
      for (int r2 = p0 + kPanel + kPairRows + tid - 32; r2 < k; r2 += nthreads - 32) {
        const T* src = upper ? Fs + r2 * F64 + p0 : Fs + p0 * F64 + r2;
        const int64_t step = upper ? 1 : F64;
        T l2[kPanel];
#pragma unroll
        for (int j = 0; j < kPanel; ++j) {
          l2[j] = *src;
          src += step;
        }
        double acc = 0.0;
#pragma unroll
        for (int j = 0; j < kPanel; ++j) {
          acc = fma(static_cast<double>(l2[j]), v[p0 + j], acc);
        }
        v[r2] -= acc;
      }
    }
    WaitBlockCopies();
    __syncthreads();
  }
  if (ys != nullptr) {
    // a wide front: v_m and y go out, KSolveTree's row-chunk tasks form u
    for (int r = tid; r < F - k; r += nthreads) {
      V.upd[S.upd_off + r] = v[k + r];
    }
    for (int j = tid; j < k; j += nthreads) {
      ys[S.first_col + j] = v[j];
    }
  } else {
    ForwardRowsU<T>(V, S, Fs, v, v + k, 0, F - k);
  }
  for (int j = tid; j < k; j += nthreads) {
    V.xs[S.first_col + j] = (1.0 / dvec[S.first_col + j]) * v[j];
  }
}

/// u = v_m - L21 y for the wide front's rows [r0, r1) (one row-chunk task):
/// v_m from upd, y from ys.
template <typename T>
__device__ __forceinline__ void ForwardRowsTask(const DeviceView& V, const SupernodeRec& S, const double* ys,
                                                int part, double* buf) {
  const int k = S.ncols;
  for (int j = threadIdx.x; j < k; j += blockDim.x) {
    buf[j] = ys[S.first_col + j];
  }
  __syncthreads();
  const int r0 = part * kSolveRowChunk;
  ForwardRowsU<T>(V, S, WorkFront<T>(V, S), buf, nullptr, r0, min(S.nrows, r0 + kSolveRowChunk));
}

/// Backward solve of one front for the one-launch solve: z = x_k - L21^T x_R
/// (warps over columns, four columns per pass, lanes over the m rows), then
/// panels from the last: warp 0 forms x_p = M_p^T z_p, and after a barrier
/// every earlier pivot column c subtracts L(p, c)^T x_p (its L values loaded
/// before the barrier). Writes xs and the step in natural order. buf: two
/// blocks for M^T, then F doubles (z, then the gathered x_R).
/// acc[q] = sum over rows r in [r0, r1) of L21(r, j0 + q) x_R(r), q < 4, for
/// one warp (lanes over rows, four rows per lane per batch: 16 loads in
/// flight), reduced by a fixed butterfly; xr indexed by r - r0.
template <typename T>
__device__ __forceinline__ void L21tColumns4(const T* Fs, int64_t F64, int k, int j0, int r0, int r1,
                                             const double* xr, double (&acc)[4]) {
  const int lane = threadIdx.x & 31;
  acc[0] = acc[1] = acc[2] = acc[3] = 0.0;
  for (int rb = r0; rb < r1; rb += 128) {
    T lv[4][4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int r = rb + 32 * u + lane;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        lv[u][q] = (r < r1 && j0 + q < k) ? Fs[(j0 + q) * F64 + k + r] : T(0);
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int r = rb + 32 * u + lane;
      const double x = r < r1 ? xr[r - r0] : 0.0;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        acc[q] = fma(static_cast<double>(lv[u][q]), x, acc[q]);
      }
    }
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], off);
    }
  }
}

/// Backward row-chunk task of a wide front: the partial products
/// L21(r0:r1, :)^T x_R(r0:r1) of its k pivot columns into zpart.
template <typename T>
__device__ __forceinline__ void BackwardRowsTask(const DeviceView& V, const SupernodeRec& S, int part,
                                                 double* zpart, double* buf) {
  const int k = S.ncols;
  const int r0 = part * kSolveRowChunk;
  const int r1 = min(S.nrows, r0 + kSolveRowChunk);
  const int32_t* rows = V.sn_rows + S.rows_off;
  for (int r = r0 + static_cast<int>(threadIdx.x); r < r1; r += blockDim.x) {
    buf[r - r0] = __ldcg(V.xs + rows[r]);
  }
  __syncthreads();
  const T* Fs = WorkFront<T>(V, S);
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int nwarps = blockDim.x >> 5;
  double* out = zpart + static_cast<int64_t>(part) * k;
  for (int j0 = 4 * warp; j0 < k; j0 += 4 * nwarps) {
    double acc[4];
    L21tColumns4<T>(Fs, S.F, k, j0, r0, r1, buf, acc);
    if (lane < 4 && j0 + lane < k) {
      out[j0 + lane] = lane == 0 ? acc[0] : lane == 1 ? acc[1] : lane == 2 ? acc[2] : acc[3];
    }
  }
}

/// Backward solve of one front; zpart (parts > 0): the front's row-chunk
/// partial products of L21^T x_R, summed in chunk order, in place of its own
/// pass over L21.
template <typename T>
__device__ __forceinline__ void BackwardTreeBody(const DeviceView& V, const SupernodeRec& S, const double* inv,
                                                 double* buf, const double* zpart, int parts) {
  const int k = S.ncols;
  const int m = S.nrows;
  const int64_t F64 = S.F;
  const T* Fs = WorkFront<T>(V, S);
  const bool upper = S.upper_l11 != 0;
  const int32_t* rows = V.sn_rows + S.rows_off;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int nthreads = blockDim.x;
  const int nwarps = nthreads >> 5;
  double* Ms = buf;
  double* z = buf + 2 * kPanel * kPanel;
  double* xr = z + k;
  const int last_q = (k - 1) / kPanel;
  // M^T of panel q at Mb + q * kInvBlock
  const double* Mb = inv + static_cast<int64_t>(S.panel_base) * kInvBlock + kPanel * kPanel;
  CopyBlockAsync(Ms + (last_q & 1) * kPanel * kPanel, Mb + static_cast<int64_t>(last_q) * kInvBlock);
  if (parts > 0) {
    for (int j = tid; j < k; j += nthreads) {
      double a = 0.0;
      for (int p = 0; p < parts; ++p) {
        a += __ldcg(zpart + static_cast<int64_t>(p) * k + j);
      }
      z[j] = __ldcg(V.xs + S.first_col + j) - a;
    }
  } else {
    for (int r = tid; r < m; r += nthreads) {
      xr[r] = __ldcg(V.xs + rows[r]);
    }
    __syncthreads();
    for (int j0 = 4 * warp; j0 < k; j0 += 4 * nwarps) {
      double acc[4];
      L21tColumns4<T>(Fs, F64, k, j0, 0, m, xr, acc);
      if (lane < 4 && j0 + lane < k) {
        const double a = lane == 0 ? acc[0] : lane == 1 ? acc[1] : lane == 2 ? acc[2] : acc[3];
        z[j0 + lane] = __ldcg(V.xs + S.first_col + j0 + lane) - a;
      }
    }
  }
  WaitBlockCopies();
  __syncthreads();
  for (int q = last_q; q >= 0; --q) {
    const int p0 = q * kPanel;
    if (q > 0) {
      CopyBlockAsync(Ms + ((q - 1) & 1) * kPanel * kPanel, Mb + static_cast<int64_t>(q - 1) * kInvBlock);
    }
    // earlier pivot columns c < p0: lane pairs of warps 1.. own one column
    // each (16 of its L values per lane, loaded before the barrier); columns
    // past the first kPairRows loop below without the early loads
    const int c = (tid - 32) >> 1;
    const int half = (tid & 1) * (kPanel / 2);
    T lc[kPanel / 2];
    if (warp > 0 && c < p0) {
      const T* src = upper ? Fs + (p0 + half) * F64 + c : Fs + c * F64 + p0 + half;
      const int64_t step = upper ? F64 : 1;
#pragma unroll
      for (int i = 0; i < kPanel / 2; ++i) {
        lc[i] = (p0 + half + i < k) ? *src : T(0);
        src += step;
      }
    }
    if (warp == 0) {
      const double* M = Ms + (q & 1) * kPanel * kPanel;
      double a0 = 0.0;
      double a1 = 0.0;
#pragma unroll
      for (int j = 0; j < kPanel; j += 2) {
        // past the pivots z holds x_R: weight zero there
        const double z0 = p0 + j < k ? z[p0 + j] : 0.0;
        const double z1 = p0 + j + 1 < k ? z[p0 + j + 1] : 0.0;
        a0 = fma(M[j * kPanel + lane], z0, a0);
        a1 = fma(M[(j + 1) * kPanel + lane], z1, a1);
      }
      __syncwarp();
      if (p0 + lane < k) {
        z[p0 + lane] = a0 + a1;
      }
    }
    __syncthreads();
    if (warp > 0) {
      double part = 0.0;
      if (c < p0) {
#pragma unroll
        for (int i = 0; i < kPanel / 2; ++i) {
          part = fma(static_cast<double>(lc[i]), p0 + half + i < k ? z[p0 + half + i] : 0.0, part);
        }
      }
      part += __shfl_xor_sync(0xffffffffu, part, 1);
      if (half == 0 && c < p0) {
        z[c] -= part;
      }
      for (int c2 = kPairRows + tid - 32; c2 < p0; c2 += nthreads - 32) {
        const T* src = upper ? Fs + p0 * F64 + c2 : Fs + c2 * F64 + p0;
        const int64_t step = upper ? F64 : 1;
        T l2[kPanel];
#pragma unroll
        for (int i = 0; i < kPanel; ++i) {
          l2[i] = (p0 + i < k) ? *src : T(0);
          src += step;
        }
        double acc = 0.0;
#pragma unroll
        for (int i = 0; i < kPanel; ++i) {
          acc = fma(static_cast<double>(l2[i]), p0 + i < k ? z[p0 + i] : 0.0, acc);
        }
        z[c2] -= acc;
      }
    }
    WaitBlockCopies();
    __syncthreads();
  }
  for (int j = tid; j < k; j += nthreads) {
    V.xs[S.first_col + j] = z[j];
    V.step[V.perm[S.first_col + j]] = z[j];
  }
}

/// Iterations of a bounded wait on another block's flag (about a second).
constexpr uint32_t kWaitLimit = 1u << 21;

/// Thread-level bounded wait until *word >= expected (acquire at GPU
/// scope), at most `limit` polls; false when the limit ran out.
__device__ __forceinline__ bool WaitCount(const uint32_t* word, uint32_t expected, uint32_t limit) {
  for (uint32_t it = 0; it < limit; ++it) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(word) : "memory");
    if (v >= expected) {
      return true;
    }
    __nanosleep(100);
  }
  return false;
}

/// Adds one to *word (release at GPU scope): a task's part is published.
__device__ __forceinline__ void Publish(uint32_t* word) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(word), "r"(1u) : "memory");
}

/// What the one-launch solve's tasks read besides the view.
struct SolveArgs {
  const int32_t* tasks;   // (type, sn, part, 0) quads
  int num_tasks;
  const int32_t* parts;   // per sn: forward, backward parts
  const int64_t* zoff;    // per sn: first partial-product double, or -1
  double* ys;             // per pivot: y of wide fronts, v then y of panel-split roots
  double* zpart;          // backward partial products of wide fronts
  const double* dvec;
  const double* inv;
  const double* dense_inv;  // tile inverses of the tiled dense roots (64-row panels)
  uint32_t* sync;         // counter, then fdone, bdone, ydone, zdone per sn, then two flags per diagonal block
  int num_sn;
  int num_inv;
  int withhold;
  uint32_t wait_limit;
};

/// Whole-block bounded wait: thread 0 polls, every thread learns whether
/// the wait succeeded; a wait that ran out marks the instance.
__device__ __forceinline__ bool BlockWait(const DeviceView& V, const SupernodeRec& S, const uint32_t* word,
                                          uint32_t expected, uint32_t limit) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok = WaitCount(word, expected, limit) ? 1 : 0;
    if (ok == 0) {
      atomicOr(V.status + S.instance, kStatusWaitTimeout);
    }
  }
  __syncthreads();
  return ok != 0;
}

/// Forward panel q of a tiled dense root (64-row panels, FP64): v_q -=
/// L(q, p) y_p for every earlier panel p as its flag arrives (four threads
/// per row, sixteen columns each, summed in a fixed order), then y_q = M_q
/// v_q with M_q the tile inverse the factorization stored, D^-1 y_q into xs.
__device__ __forceinline__ void RootForwardPanel64(const DeviceView& V, const SupernodeRec& S, const SolveArgs& A,
                                                   int q, uint32_t* pflag, double* buf) {
  constexpr int kW = kDenseTileCols;
  const int k = S.ncols;
  const int64_t F64 = S.F;
  const double* Fs = V.fronts + S.front_off;
  const int p0 = q * kW;
  const int w = min(kW, k - p0);
  const int tid = threadIdx.x;
  double* vq = buf;           // kW
  double* yp = buf + kW;      // kW
  double* part = buf + 2 * kW;  // 4 x kW
  const int i = tid & (kW - 1);
  const int g = tid >> 6;  // four groups of sixteen columns
  if (tid < kW) {
    vq[tid] = tid < w ? A.ys[S.first_col + p0 + tid] : 0.0;
  }
  for (int p = 0; p < q; ++p) {
    double l[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) {
      l[c] = i < w ? Fs[static_cast<int64_t>(p * kW + 16 * g + c) * F64 + p0 + i] : 0.0;
    }
    BlockWait(V, S, pflag + S.panel_base + p, 1u, A.wait_limit);
    if (tid < kW) {
      yp[tid] = __ldcg(A.ys + S.first_col + p * kW + tid);
    }
    __syncthreads();
    double acc = 0.0;
#pragma unroll
    for (int c = 0; c < 16; ++c) {
      acc = fma(l[c], yp[16 * g + c], acc);
    }
    part[g * kW + i] = acc;
    __syncthreads();
    if (tid < kW) {
      vq[i] -= (part[i] + part[kW + i]) + (part[2 * kW + i] + part[3 * kW + i]);
    }
  }
  __syncthreads();
  // y = M v: thread (row i, group g) sums sixteen columns of M
  const double* M = A.dense_inv + S.dense_inv + static_cast<int64_t>(q) * kW * kW;
  double acc = 0.0;
#pragma unroll
  for (int c = 0; c < 16; ++c) {
    const int j = 16 * g + c;
    acc = fma(M[static_cast<int64_t>(j) * kW + i], vq[j], acc);
  }
  part[g * kW + i] = acc;
  __syncthreads();
  if (tid < w) {
    const double y = (part[i] + part[kW + i]) + (part[2 * kW + i] + part[3 * kW + i]);
    A.ys[S.first_col + p0 + tid] = y;
    V.xs[S.first_col + p0 + tid] = (1.0 / A.dvec[S.first_col + p0 + tid]) * y;
  }
}

/// Backward panel q of a tiled dense root: z_q = (D^-1 y)_q minus
/// L(p, q)^T x_p for every later panel p as its flag arrives, then x_q =
/// M_q^T z_q into xs and the step.
__device__ __forceinline__ void RootBackwardPanel64(const DeviceView& V, const SupernodeRec& S, const SolveArgs& A,
                                                    int q, uint32_t* bflag, double* buf) {
  constexpr int kW = kDenseTileCols;
  const int k = S.ncols;
  const int64_t F64 = S.F;
  const double* Fs = V.fronts + S.front_off;
  const int np = (k + kW - 1) / kW;
  const int p0 = q * kW;
  const int w = min(kW, k - p0);
  const int tid = threadIdx.x;
  double* zq = buf;
  double* xp = buf + kW;
  double* part = buf + 2 * kW;
  // thread (row i of z, group g of sixteen rows of panel p)
  const int i = tid >> 2;
  const int g = tid & 3;
  if (tid < kW) {
    zq[tid] = tid < w ? __ldcg(V.xs + S.first_col + p0 + tid) : 0.0;
  }
  for (int p = np - 1; p > q; --p) {
    const int wp = min(kW, k - p * kW);
    double l[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) {
      const int r = 16 * g + c;
      l[c] = (i < w && r < wp) ? Fs[static_cast<int64_t>(p0 + i) * F64 + p * kW + r] : 0.0;
    }
    BlockWait(V, S, bflag + S.panel_base + p, 1u, A.wait_limit);
    if (tid < kW) {
      xp[tid] = tid < wp ? __ldcg(V.xs + S.first_col + p * kW + tid) : 0.0;
    }
    __syncthreads();
    double acc = 0.0;
#pragma unroll
    for (int c = 0; c < 16; ++c) {
      acc = fma(l[c], xp[16 * g + c], acc);
    }
    part[g * kW + i] = acc;
    __syncthreads();
    if (tid < kW) {
      zq[tid] -= (part[tid] + part[kW + tid]) + (part[2 * kW + tid] + part[3 * kW + tid]);
    }
  }
  __syncthreads();
  // x = M^T z: thread (row i, group g) sums sixteen entries of column i of M
  const double* M = A.dense_inv + S.dense_inv + static_cast<int64_t>(q) * kW * kW;
  double acc = 0.0;
#pragma unroll
  for (int c = 0; c < 16; ++c) {
    const int j = 16 * g + c;
    acc = fma(M[static_cast<int64_t>(i) * kW + j], zq[j], acc);
  }
  part[g * kW + i] = acc;
  __syncthreads();
  if (tid < w) {
    const double x = (part[tid] + part[kW + tid]) + (part[2 * kW + tid] + part[3 * kW + tid]);
    V.xs[S.first_col + p0 + tid] = x;
    V.step[V.perm[S.first_col + p0 + tid]] = x;
  }
}

/// Right-hand side of a panel-split root: v = rhs plus the children's
/// update vectors (children in their fixed order), into ys.
__device__ __forceinline__ void RootGather(const DeviceView& V, const SupernodeRec& S, double* ys, double* v) {
  const int k = S.ncols;
  for (int j = threadIdx.x; j < k; j += blockDim.x) {
    v[j] = V.rhs[V.perm[S.first_col + j]];
  }
  __syncthreads();
  for (int ci = 0; ci < S.child_count; ++ci) {
    const SupernodeRec C = V.sn[V.child_list[S.child_begin + ci]];
    const int32_t* rel = V.sn_rel + C.rows_off;
    const double* u = V.upd + C.upd_off;
    for (int r = threadIdx.x; r < C.nrows; r += blockDim.x) {
      v[rel[r]] += __ldcg(u + r);
    }
    __syncthreads();
  }
  for (int j = threadIdx.x; j < k; j += blockDim.x) {
    ys[S.first_col + j] = v[j];
  }
}

/// Forward panel q of a panel-split root (FP64, column-major L below the
/// diagonal blocks): v_q -= L(q, p) y_p for every earlier panel p as its
/// flag arrives (eight threads per row, four columns each, summed in a fixed
/// order), then y_q = M_q v_q, D^-1 y_q into xs.
template <typename T>
__device__ __forceinline__ void RootForwardPanel(const DeviceView& V, const SupernodeRec& S, const SolveArgs& A,
                                                 int q, uint32_t* pflag, double* buf) {
  const int k = S.ncols;
  const int64_t F64 = S.F;
  const T* Fs = WorkFront<T>(V, S);
  const int p0 = q * kPanel;
  const int w = min(kPanel, k - p0);
  const int tid = threadIdx.x;
  double* vq = buf;                    // kPanel
  double* yp = buf + kPanel;           // kPanel
  double* part = buf + 2 * kPanel;     // 8 x kPanel
  double* M = buf + 10 * kPanel;       // kPanel x kPanel
  if (tid < kPanel) {
    vq[tid] = tid < w ? A.ys[S.first_col + p0 + tid] : 0.0;
  }
  const int i = tid & (kPanel - 1);
  const int g = tid >> 5;  // eight groups of four columns
  for (int p = 0; p < q; ++p) {
    // L(q, p) values of this thread, loaded before the wait
    double l[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      l[c] = i < w ? static_cast<double>(Fs[static_cast<int64_t>(p * kPanel + 4 * g + c) * F64 + p0 + i]) : 0.0;
    }
    BlockWait(V, S, pflag + S.panel_base + p, 1u, A.wait_limit);
    if (tid < kPanel) {
      yp[tid] = __ldcg(A.ys + S.first_col + p * kPanel + tid);
    }
    __syncthreads();
    double acc = 0.0;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      acc = fma(l[c], yp[4 * g + c], acc);
    }
    part[g * kPanel + i] = acc;
    __syncthreads();
    if (tid < kPanel) {
      const double s01 = part[i] + part[kPanel + i];
      const double s23 = part[2 * kPanel + i] + part[3 * kPanel + i];
      const double s45 = part[4 * kPanel + i] + part[5 * kPanel + i];
      const double s67 = part[6 * kPanel + i] + part[7 * kPanel + i];
      vq[i] -= (s01 + s23) + (s45 + s67);
    }
  }
  const double* Mb = A.inv + static_cast<int64_t>(S.panel_base + q) * kInvBlock;
  for (int e = tid; e < kPanel * kPanel; e += blockDim.x) {
    M[e] = Mb[e];
  }
  __syncthreads();
  if (tid < kPanel) {
    double a0 = 0.0;
    double a1 = 0.0;
#pragma unroll
    for (int j = 0; j < kPanel; j += 2) {
      a0 = fma(M[j * kPanel + tid], vq[j], a0);
      a1 = fma(M[(j + 1) * kPanel + tid], vq[j + 1], a1);
    }
    if (tid < w) {
      const double y = a0 + a1;
      A.ys[S.first_col + p0 + tid] = y;
      V.xs[S.first_col + p0 + tid] = (1.0 / A.dvec[S.first_col + p0 + tid]) * y;
    }
  }
}

/// Backward panel q of a panel-split root: z_q = (D^-1 y)_q minus
/// L(p, q)^T x_p for every later panel p as its flag arrives, then
/// x_q = M_q^T z_q into xs and the step.
template <typename T>
__device__ __forceinline__ void RootBackwardPanel(const DeviceView& V, const SupernodeRec& S, const SolveArgs& A,
                                                  int q, uint32_t* bflag, double* buf) {
  const int k = S.ncols;
  const int64_t F64 = S.F;
  const T* Fs = WorkFront<T>(V, S);
  const int np = (k + kPanel - 1) / kPanel;
  const int p0 = q * kPanel;
  const int w = min(kPanel, k - p0);
  const int tid = threadIdx.x;
  double* zq = buf;
  double* xp = buf + kPanel;
  double* part = buf + 2 * kPanel;
  double* M = buf + 10 * kPanel;
  if (tid < kPanel) {
    zq[tid] = tid < w ? __ldcg(V.xs + S.first_col + p0 + tid) : 0.0;
  }
  // thread (row i of z, group g of four rows of panel p)
  const int i = tid >> 3;
  const int g = tid & 7;
  for (int p = np - 1; p > q; --p) {
    const int wp = min(kPanel, k - p * kPanel);
    double l[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int r = 4 * g + c;
      l[c] = (i < w && r < wp) ? static_cast<double>(Fs[static_cast<int64_t>(p0 + i) * F64 + p * kPanel + r]) : 0.0;
    }
    BlockWait(V, S, bflag + S.panel_base + p, 1u, A.wait_limit);
    if (tid < kPanel) {
      xp[tid] = tid < wp ? __ldcg(V.xs + S.first_col + p * kPanel + tid) : 0.0;
    }
    __syncthreads();
    double acc = 0.0;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      acc = fma(l[c], xp[4 * g + c], acc);
    }
    part[g * kPanel + i] = acc;
    __syncthreads();
    if (tid < kPanel) {
      const double s01 = part[tid] + part[kPanel + tid];
      const double s23 = part[2 * kPanel + tid] + part[3 * kPanel + tid];
      const double s45 = part[4 * kPanel + tid] + part[5 * kPanel + tid];
      const double s67 = part[6 * kPanel + tid] + part[7 * kPanel + tid];
      zq[tid] -= (s01 + s23) + (s45 + s67);
    }
  }
  // M_q^T, stored after M_q in the inverted block
  const double* Mb = A.inv + static_cast<int64_t>(S.panel_base + q) * kInvBlock + kPanel * kPanel;
  for (int e = tid; e < kPanel * kPanel; e += blockDim.x) {
    M[e] = Mb[e];
  }
  __syncthreads();
  if (tid < kPanel) {
    double a0 = 0.0;
    double a1 = 0.0;
#pragma unroll
    for (int j = 0; j < kPanel; j += 2) {
      a0 = fma(M[j * kPanel + tid], zq[j], a0);
      a1 = fma(M[(j + 1) * kPanel + tid], zq[j + 1], a1);
    }
    if (tid < w) {
      const double x = a0 + a1;
      V.xs[S.first_col + p0 + tid] = x;
      V.step[V.perm[S.first_col + p0 + tid]] = x;
    }
  }
}

/// Whole solve (forward sweep, diagonal, backward sweep) in one launch, with
/// the inverted diagonal blocks of KInvertDiagonal. Blocks take the tasks of
/// A.tasks in order from a counter (see Symbolic::solve_tasks): every task
/// waits only on tasks taken before it by running blocks, so the launch
/// completes whatever the number of resident blocks, and no level boundary
/// holds fast fronts behind slow ones. A front's forward parts done counter
/// (fdone) is what its parent waits for, its backward parts done (bdone)
/// what its children wait for; ydone says a wide front's y (or a split
/// root's right-hand side) is out, zdone counts a wide front's backward row
/// chunks; a split root's panels publish one flag each per direction. A wait
/// that runs out of its limit marks the instance kStatusWaitTimeout and lets
/// the task's dependents go. withhold: a supernode whose forward parts are
/// never published (-1: none), the test hook that makes a wait run out.
__global__ void __launch_bounds__(256, 1) KSolveTree(DeviceView V, SolveArgs A) {
  extern __shared__ double buf[];
  __shared__ int task;
  __shared__ int go;
  uint32_t* fdone = A.sync + 2;
  uint32_t* bdone = fdone + A.num_sn;
  uint32_t* ydone = bdone + A.num_sn;
  uint32_t* zdone = ydone + A.num_sn;
  uint32_t* pflag = zdone + A.num_sn;
  uint32_t* bflag = pflag + A.num_inv;
  if (V.refine_left != nullptr && *V.refine_left == 0) {
    return;  // a refinement round after every instance's step became final
  }
  for (;;) {
    if (threadIdx.x == 0) {
      task = static_cast<int>(atomicAdd(A.sync, 1u));
    }
    __syncthreads();
    const int t = task;
    if (t >= A.num_tasks) {
      return;
    }
    const int type = A.tasks[4 * t];
    const int s = A.tasks[4 * t + 1];
    const int part = A.tasks[4 * t + 2];
    const SupernodeRec S = V.sn[s];
    // refinement rounds skip the instances whose step is final
    const bool active = V.active[S.instance] != 0 && (V.refine_done == nullptr || V.refine_done[S.instance] == 0);
    if (threadIdx.x == 0) {
      bool ready = true;
      if (active) {
        switch (type) {
          case kTaskForward:
          case kTaskRootGather:
            for (int ci = 0; ci < S.child_count && ready; ++ci) {
              const int c = V.child_list[S.child_begin + ci];
              ready = WaitCount(fdone + c, static_cast<uint32_t>(A.parts[2 * c]), A.wait_limit);
            }
            break;
          case kTaskForwardRows:
          case kTaskRootForward:
            ready = WaitCount(ydone + s, 1u, A.wait_limit);
            break;
          case kTaskRootBackward:
            ready = WaitCount(fdone + s, static_cast<uint32_t>(A.parts[2 * s]), A.wait_limit);
            break;
          case kTaskBackwardRows:
            ready = WaitCount(bdone + S.parent, static_cast<uint32_t>(A.parts[2 * S.parent + 1]), A.wait_limit);
            break;
          default:  // kTaskBackward
            if (A.zoff[s] >= 0) {
              ready = WaitCount(zdone + s, static_cast<uint32_t>(A.parts[2 * s] - 1), A.wait_limit);
            } else if (S.parent >= 0) {
              ready = WaitCount(bdone + S.parent, static_cast<uint32_t>(A.parts[2 * S.parent + 1]), A.wait_limit);
            } else {
              ready = WaitCount(fdone + s, static_cast<uint32_t>(A.parts[2 * s]), A.wait_limit);
            }
            break;
        }
        if (!ready) {
          atomicOr(V.status + S.instance, kStatusWaitTimeout);
        }
      }
      go = active && ready ? 1 : 0;
    }
    __syncthreads();
    const bool f32 = Fp32Front(V, S);
    if (go != 0) {
      switch (type) {
        case kTaskForward: {
          double* ys = A.zoff[s] >= 0 ? A.ys : nullptr;
          if (f32) {
            ForwardTreeBody<float>(V, S, A.dvec, A.inv, buf, ys);
          } else {
            ForwardTreeBody<double>(V, S, A.dvec, A.inv, buf, ys);
          }
          break;
        }
        case kTaskForwardRows:
          if (f32) {
            ForwardRowsTask<float>(V, S, A.ys, part, buf);
          } else {
            ForwardRowsTask<double>(V, S, A.ys, part, buf);
          }
          break;
        case kTaskRootGather:
          RootGather(V, S, A.ys, buf);
          break;
        case kTaskRootForward:
          if (S.dense_cnt >= 0) {
            RootForwardPanel64(V, S, A, part, pflag, buf);
          } else if (f32) {
            RootForwardPanel<float>(V, S, A, part, pflag, buf);
          } else {
            RootForwardPanel<double>(V, S, A, part, pflag, buf);
          }
          break;
        case kTaskRootBackward:
          if (S.dense_cnt >= 0) {
            RootBackwardPanel64(V, S, A, part, bflag, buf);
          } else if (f32) {
            RootBackwardPanel<float>(V, S, A, part, bflag, buf);
          } else {
            RootBackwardPanel<double>(V, S, A, part, bflag, buf);
          }
          break;
        case kTaskBackwardRows:
          if (f32) {
            BackwardRowsTask<float>(V, S, part, A.zpart + A.zoff[s], buf);
          } else {
            BackwardRowsTask<double>(V, S, part, A.zpart + A.zoff[s], buf);
          }
          break;
        default: {
          const int parts = A.zoff[s] >= 0 ? A.parts[2 * s] - 1 : 0;
          const double* zp = parts > 0 ? A.zpart + A.zoff[s] : nullptr;
          if (f32) {
            BackwardTreeBody<float>(V, S, A.inv, buf, zp, parts);
          } else {
            BackwardTreeBody<double>(V, S, A.inv, buf, zp, parts);
          }
          break;
        }
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      switch (type) {
        case kTaskForward:
          if (A.zoff[s] >= 0) {
            Publish(ydone + s);
          }
          if (s != A.withhold) {
            Publish(fdone + s);
          }
          break;
        case kTaskForwardRows:
          if (s != A.withhold) {
            Publish(fdone + s);
          }
          break;
        case kTaskRootGather:
          Publish(ydone + s);
          break;
        case kTaskRootForward:
          Publish(pflag + S.panel_base + part);
          if (s != A.withhold) {
            Publish(fdone + s);
          }
          break;
        case kTaskRootBackward:
          Publish(bflag + S.panel_base + part);
          Publish(bdone + s);
          break;
        case kTaskBackwardRows:
          Publish(zdone + s);
          break;
        default:
          Publish(bdone + s);
          break;
      }
    }
  }
}

}  // namespace sdfgpu

// ------------------------------------------------------------ launchers --

#include <mutex>

#include "dense_root.h"
#include "engine.h"

namespace sdfgpu {

static_assert(kInvBlock == kInvBlockDoubles, "inverted block size");

/// Dynamic shared memory a block may use on B200.
constexpr int kMaxSmem = 227 * 1024;

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
      CudaCheck(cudaFuncSetAttribute(KExtendAdd, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     kEaStageDoubles * static_cast<int>(sizeof(double))),
                "smem attr");
      front_configured = true;
    }
  }
  const int smem = max_front * static_cast<int>(sizeof(double));
  if (smem > kMaxSmem) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT, "front too large for the solve kernels");
  }
  std::lock_guard<std::mutex> lk(mu);
  if (smem > configured) {
    CudaCheck(cudaFuncSetAttribute(KForward, cudaFuncAttributeMaxDynamicSharedMemorySize, smem), "smem attr");
    CudaCheck(cudaFuncSetAttribute(KBackward, cudaFuncAttributeMaxDynamicSharedMemorySize, smem), "smem attr");
    configured = smem;
  }
  static int tree_configured = 48 * 1024;
  const int tree = static_cast<int>(SolveTreeSmem(max_front));
  if (tree <= kMaxSmem && tree > tree_configured) {
    CudaCheck(cudaFuncSetAttribute(KSolveTree, cudaFuncAttributeMaxDynamicSharedMemorySize, tree), "smem attr");
    tree_configured = tree;
  }
}

int LaunchFactorLevels(const Symbolic& S, const DeviceView& V, const FactorPlan& P, cudaStream_t stream) {
  {
    // the block factorization's shared memory (a per-device attribute)
    static std::mutex mu;
    static bool configured[64] = {};
    int dev = 0;
    CudaCheck(cudaGetDevice(&dev), "device");
    const std::lock_guard<std::mutex> lock(mu);
    if (dev < 0 || dev >= 64 || !configured[dev]) {
      CudaCheck(cudaFuncSetAttribute(KPanelBlock, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(PanelBlockSmem())),
                "block smem attr");
      CudaCheck(cudaFuncSetAttribute(KSchur, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(kSchurSmem)),
                "schur smem attr");
      if (dev >= 0 && dev < 64) {
        configured[dev] = true;
      }
    }
  }
  // the diagonal blocks are factored by four warps of every factor block
  if (S.front_rows < 128 || S.front_rows > 256 || S.panel_rows < 0 || S.panel_rows > kPanelRowsPerBlock) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT, "factorization schedule out of range");
  }
  int launches = 0;
  // algorithmic work of a level's launches (flops: 2 per multiply-add, the
  // dense LDL^T operation counts; bytes for the memory-bound classes), for
  // the kernel timer
  auto level_sum = [&S](int l, auto&& f) {
    double w = 0.0;
    for (int q = S.level_begin[static_cast<size_t>(l)]; q < S.level_begin[static_cast<size_t>(l) + 1]; ++q) {
      w += f(S.sn[static_cast<size_t>(S.level_sn[static_cast<size_t>(q)])]);
    }
    return w;
  };
  if (P.dense_sync != nullptr && S.dense_cnt_words > 0) {
    CudaCheck(cudaMemsetAsync(P.dense_sync, 0, DenseSyncWords(S) * sizeof(int32_t), stream), "dense sync reset");
  }
  for (int l = 0; l < S.num_levels; ++l) {
    // the extend-add only for update matrices the tensor cores left in place
    const TaskRange ea = S.ea_range[static_cast<size_t>(l)];
    if (ea.count > 0 && P.tc_map != nullptr) {
      // staged in shared memory unless a front of the level is too wide
      const size_t stage = static_cast<size_t>(S.ea_stage[static_cast<size_t>(l)]) * sizeof(double);
      const bool staged = stage <= static_cast<size_t>(kEaStageDoubles) * sizeof(double);
      const TimedLaunch tl(P.timer, KernelTimer::kExtendAdd, stream, [&] {
        // each child's update entry read, its parent entry read and written
        return level_sum(l, [&S](const SupernodeRec& r) {
          double b = 0.0;
          for (int ci = 0; ci < r.child_count; ++ci) {
            const double m = S.sn[static_cast<size_t>(S.child_list[static_cast<size_t>(r.child_begin + ci)])].nrows;
            b += 24.0 * m * (m + 1.0) / 2.0;
          }
          return b;
        });
      });
      KExtendAdd<<<static_cast<unsigned>(ea.count), 256, staged ? stage : 0, stream>>>(
          V, P.ea_tasks + 4 * ea.begin, P.ea_child, staged ? 1 : 0);
      ++launches;
    }
    const TaskRange sm = S.small_range[static_cast<size_t>(l)];
    if (sm.count > 0) {
      const int kmax = S.small_max_k[static_cast<size_t>(l)];
      const size_t bytes = FactorFrontSmem(kmax);
      const TimedLaunch tl(P.timer, KernelTimer::kFactorFront, stream, [&] {
        return level_sum(l, [&S](const SupernodeRec& r) {
          const double k = r.ncols;
          return r.ncols <= S.small_pivots ? 2.0 * k * k * k / 3.0 + static_cast<double>(r.nrows) * k * k : 0.0;
        });
      });
      KFactorFront<<<static_cast<unsigned>(sm.count), S.small_threads[static_cast<size_t>(l)], bytes, stream>>>(
          V, P.small_tasks + 3 * sm.begin, P.dvec);
      ++launches;
    }
    const TaskRange dr = S.dense_range[static_cast<size_t>(l)];
    if (dr.count > 0 && P.dense_tasks != nullptr && P.dense_sync != nullptr) {
      const TimedLaunch tl(P.timer, KernelTimer::kDenseRoot, stream, [&] {
        return level_sum(l, [](const SupernodeRec& r) {
          const double n = r.ncols;
          return r.dense_cnt >= 0 ? 2.0 * n * n * n / 3.0 : 0.0;
        });
      });
      DenseArgs A{};
      A.tasks = P.dense_tasks + 4 * dr.begin;
      A.count = dr.count;
      A.claim = P.dense_sync + l;
      A.abort = P.dense_sync + S.num_levels;
      A.cnt = P.dense_sync + S.num_levels + 1;
      A.inv = P.dense_inv;
      A.dvec = P.dvec;
      A.wait_limit = kWaitLimit;
      A.trace = nullptr;
      launches += LaunchDenseRoots(V, A, stream);
    }
    for (int t = 0; t < S.level_panels[static_cast<size_t>(l)]; ++t) {
      const size_t slot = static_cast<size_t>(S.panel_index_base[static_cast<size_t>(l)] + t);
      const TaskRange pr = S.panel_range[slot];
      if (pr.count > 0) {
        const bool blocks = S.panel_rows == 0;
        const TimedLaunch tl(P.timer, KernelTimer::kPanel, stream, [&] {
          return level_sum(l, [&S, t, blocks](const SupernodeRec& r) {
            const int width = blocks ? kBlockCols : kPanel;
            const int c0 = t * width;
            if (r.ncols <= S.small_pivots || c0 >= r.ncols || r.dense_cnt >= 0) {
              return 0.0;
            }
            // the block's LDL^T and the rows below it solved against it
            const double w = std::min(width, r.ncols - c0);
            return 2.0 * w * w * w / 3.0 + static_cast<double>(r.F - c0 - w) * w * w;
          });
        });
        if (blocks) {
          KPanelBlock<<<static_cast<unsigned>(pr.count), kBlockThreads, PanelBlockSmem(), stream>>>(
              V, P.panel_tasks + 3 * pr.begin, P.dvec);
        } else {
          KPanel<<<static_cast<unsigned>(pr.count), kPanelRowsPerBlock, 0, stream>>>(V, P.panel_tasks + 3 * pr.begin,
                                                                                     P.dvec, S.panel_rows);
        }
        ++launches;
      }
      const TaskRange ur = S.update_range[slot];
      if (ur.count > 0) {
        const TimedLaunch tl(P.timer, KernelTimer::kUpdatePanel, stream, [&] {
          return level_sum(l, [&S, t](const SupernodeRec& r) {
            if (r.ncols <= S.small_pivots || r.dense_cnt >= 0) {
              return 0.0;
            }
            // lower-part entries of the pivot columns [a, b) over rows [a, F)
            auto entries = [&r](double a, double b) { return (b - a) * r.F - (a + b - 1.0) * (b - a) / 2.0; };
            const int outer = kOuterPanels * kPanel;
            if (S.panel_rows == 0) {
              const int c0 = t * outer;
              const int c1 = std::min(r.ncols, c0 + outer);
              return c0 < r.ncols && c1 < r.ncols ? 2.0 * (c1 - c0) * entries(c1, r.ncols) : 0.0;
            }
            const int c0 = t * kPanel;
            if (c0 >= r.ncols) {
              return 0.0;
            }
            const int c1 = std::min(r.ncols, c0 + kPanel);
            const int cend = std::min(r.ncols, (c0 / outer + 1) * outer);
            if (c1 < cend) {
              return 2.0 * (c1 - c0) * entries(c1, cend);
            }
            const int b0 = c0 / outer * outer;
            return cend < r.ncols ? 2.0 * (cend - b0) * entries(cend, r.ncols) : 0.0;
          });
        });
        KUpdate<<<static_cast<unsigned>(ur.count), 256, 0, stream>>>(V, P.update_tasks + 4 * ur.begin, P.dvec);
        ++launches;
      }
    }
    if (P.tc_map != nullptr) {
      // Schur complements of the level's wide FP32 fronts on the tensor
      // cores (KUpdate skips their SIMT tiles)
      const TaskRange pk = S.pack_range[static_cast<size_t>(l)];
      const TaskRange tr = S.tc_range[static_cast<size_t>(l)];
      double pack_bytes = 0.0;
      double tc_flops = 0.0;
      if (P.timer != nullptr) {
        level_sum(l, [&](const SupernodeRec& r) {
          if (r.tc_pack >= 0) {
            const double m = r.nrows;
            const double k = r.ncols;
            pack_bytes += 4.0 * m * k + 4.0 * static_cast<double>(TcPackRows(r.ncols, r.nrows)) * kTcChunk;
            tc_flops += k * m * (m + 1.0);
          }
          return 0.0;
        });
      }
      launches += LaunchSchurTc(*P.tc_map, P.tc, P.pack_tasks + 3 * pk.begin, pk.count, P.tc_tasks + 3 * tr.begin,
                                tr.count, stream, P.timer, pack_bytes, tc_flops);
    }
    for (int q = S.schur_base[static_cast<size_t>(l)]; q < S.schur_base[static_cast<size_t>(l) + 1]; ++q) {
      const TaskRange sr = S.schur_range[static_cast<size_t>(q)];
      if (sr.count == 0) {
        continue;
      }
      // the wide FP32 fronts of a mixed solve are on the tensor cores; the
      // level's work is counted with its first sibling slot
      const bool tc = P.tc_map != nullptr;
      const bool first = q == S.schur_base[static_cast<size_t>(l)];
      const TimedLaunch tl(P.timer, KernelTimer::kUpdateSchur, stream, [&] {
        return first ? level_sum(l, [tc](const SupernodeRec& r) {
          const double m = r.nrows;
          return tc && r.tc_pack >= 0 ? 0.0 : static_cast<double>(r.ncols) * m * (m + 1.0);
        }) : 0.0;
      });
      KSchur<<<static_cast<unsigned>(sr.count), 256, kSchurSmem, stream>>>(V, P.update_tasks + 4 * sr.begin,
                                                                            P.dvec);
      ++launches;
      if (P.fp32_fronts) {
        // the FP32 fronts of a mixed solve that the tensor cores do not take
        KSchurF32<<<static_cast<unsigned>(sr.count), 256, kSchurSmem / 2, stream>>>(
            V, P.update_tasks + 4 * sr.begin, P.dvec);
        ++launches;
      }
    }
  }
  if (P.inv != nullptr && P.num_inv > 0) {
    // inverted diagonal blocks for the one-launch solve
    const TimedLaunch tl(P.timer, KernelTimer::kInvertDiagonal, stream,
                         [&] { return static_cast<double>(P.num_inv) * (8.0 + 16.0) * 1024.0; });
    KInvertDiagonal<<<static_cast<unsigned>((P.num_inv + 3) / 4), 128, 0, stream>>>(V, P.inv_tasks, P.num_inv,
                                                                                   P.inv);
    ++launches;
  }
  CudaCheck(cudaGetLastError(), "factor kernels");
  return launches;
}

int LaunchSolveLevels(const Symbolic& S, const DeviceView& V, const FactorPlan& P, cudaStream_t stream) {
  int launches = 0;
  const size_t smem = static_cast<size_t>(P.max_front) * sizeof(double);
  const int num_sn = static_cast<int>(S.sn.size());
  const size_t tree_smem = SolveTreeSmem(P.max_front);
  if (P.solve_sync != nullptr && P.inv != nullptr && P.solve_tasks != nullptr &&
      tree_smem <= static_cast<size_t>(kMaxSmem)) {
    if (num_sn == 0) {
      return 0;
    }
    static const int sms = [] {
      int dev = 0;
      int count = 0;
      CudaCheck(cudaGetDevice(&dev), "device");
      CudaCheck(cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev), "SM count");
      return count;
    }();
    // one resident block per SM (the kernel's register bound); blocks that
    // find no task left return at once
    const int blocks = std::min(P.num_solve_tasks, sms);
    CudaCheck(cudaMemsetAsync(P.solve_sync, 0, SolveSyncWords(num_sn, P.num_inv) * sizeof(uint32_t), stream),
              "solve flags");
    const TimedLaunch tl(P.timer, KernelTimer::kSolveTree, stream, [&] {
      // every entry of L read twice (forward, backward), FP32 in the grid
      // fronts of a mixed solve, and the inverted diagonal blocks
      double b = static_cast<double>(P.num_inv) * 2.0 * 8.0 * 1024.0;
      for (const SupernodeRec& r : S.sn) {
        const double k = r.ncols;
        const double elem = (P.tc_map != nullptr && r.pose_root == 0) ? 4.0 : 8.0;
        b += 2.0 * elem * (k * (k + 1.0) / 2.0 + static_cast<double>(r.nrows) * k);
      }
      return b;
    });
    SolveArgs A{};
    A.tasks = P.solve_tasks;
    A.num_tasks = P.num_solve_tasks;
    A.parts = P.solve_parts;
    A.zoff = P.zpart_off;
    A.ys = P.ys;
    A.zpart = P.zpart;
    A.dvec = P.dvec;
    A.inv = P.inv;
    A.dense_inv = P.dense_inv;
    A.sync = P.solve_sync;
    A.num_sn = num_sn;
    A.num_inv = P.num_inv;
    A.withhold = P.solve_withhold;
    A.wait_limit = P.solve_wait_polls > 0 ? P.solve_wait_polls : kWaitLimit;
    KSolveTree<<<static_cast<unsigned>(blocks), 256, tree_smem, stream>>>(V, A);
    CudaCheck(cudaGetLastError(), "solve kernel");
    return 1;
  }
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
