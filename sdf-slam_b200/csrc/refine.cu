// Mixed-precision support: FP32 copies of the grid fronts and the FP64
// iterative refinement of the LM step.
//
// A mixed solve assembles the damped normal matrix A = J^T J + damping in FP64
// (asm_fronts, the same kernels and summation order as the plain path),
// factors the grid supernodes from FP32 copies (the dense pose root from an
// FP64 copy), and refines the step: r = rhs - A delta with A read in FP64
// from the assembled fronts, delta += (LDL^T)^-1 r. Each round multiplies the
// error by about cond(A) * 2^-24.
#include <cuda_runtime.h>

#include "device.cuh"

namespace sdfgpu {

/// Copies the assembled FP64 fronts into the factorization work fronts: FP32
/// for a mixed solve's grid supernodes, FP64 otherwise. It copies exactly
/// the entries KZeroFronts clears before assembly, with the same tasks (sn,
/// first of kZeroCols columns; one warp per column, rows c..F-1): the lower
/// triangles, and the leaf fronts' trailing columns only when a tensor-core
/// Schur complement is computed in place. No factor kernel reads a work
/// front's entry outside that region before writing it, as on the plain
/// path, where the work fronts are the assembled ones.
__global__ void KConvertFronts(DeviceView V, const int32_t* tasks) {
  const int32_t* t = tasks + 2 * static_cast<int64_t>(blockIdx.x);
  const SupernodeRec S = V.sn[t[0]];
  const int c = t[1] + static_cast<int>(threadIdx.x >> 5);
  const int lane = static_cast<int>(threadIdx.x & 31);
  if (c >= S.F) {
    return;
  }
  const int64_t col = S.front_off + static_cast<int64_t>(c) * S.F;
  const double* src = V.asm_fronts + col;
  if (Fp32Front(V, S)) {
    float* dst = V.fronts32 + col;
    for (int r = c + lane; r < S.F; r += 32) {
      dst[r] = static_cast<float>(src[r]);
    }
  } else {
    double* dst = V.fronts + col;
    for (int r = c + lane; r < S.F; r += 32) {
      dst[r] = src[r];
    }
  }
}

/// True when instance i takes no further refinement round.
__device__ __forceinline__ bool RefineDone(const DeviceView& V, int i) {
  return V.refine_done != nullptr && V.refine_done[i] != 0;
}

/// Opens the refinement rounds of a solve: no instance done, maxima zero.
__global__ void KRefineReset(DeviceView V) {
  for (int i = threadIdx.x; i < V.num_inst; i += blockDim.x) {
    V.refine_done[i] = 0;
    V.refine_max[2 * i] = 0ull;
    V.refine_max[2 * i + 1] = 0ull;
  }
  if (threadIdx.x == 0) {
    *V.refine_left = 1;
  }
}

/// After a round: an instance whose largest correction is at most its
/// refine_tol times its largest step entry is done (the next round would
/// change its step by a fraction of that); the maxima restart and
/// refine_left says whether any mixed instance still refines. One block.
__global__ void KRefineCheck(DeviceView V) {
  __shared__ int left;
  if (threadIdx.x == 0) {
    left = 0;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < V.num_inst; i += blockDim.x) {
    const double mc = __longlong_as_double(static_cast<long long>(V.refine_max[2 * i]));
    const double ms = __longlong_as_double(static_cast<long long>(V.refine_max[2 * i + 1]));
    if (V.refine_done[i] == 0 && mc <= V.inst[i].refine_tol * ms) {
      V.refine_done[i] = 1;
    }
    V.refine_max[2 * i] = 0ull;
    V.refine_max[2 * i + 1] = 0ull;
    if (V.refine_done[i] == 0 && V.inst[i].mixed != 0 && V.active[i] != 0) {
      left = 1;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    *V.refine_left = left;
  }
}

/// y = A x over the map columns of mixed instances (natural order), A read
/// in FP64 from the assembled fronts: the 9-point map stencil (mm_off) and
/// the node's map-pose blocks (mp_*). One warp per column: lanes 0-8 take
/// one stencil slot each, then the lanes stride over the column's coupled
/// frames (a node of a revisited area couples to hundreds of frames), and a
/// fixed butterfly sums the lanes, so every sum runs in a fixed order.
__global__ void KNormalMatVecMap(DeviceView V, const double* x, double* y) {
  const int64_t wid = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (wid >= V.n) {
    return;
  }
  const int c = static_cast<int>(wid);
  const int node = V.col_node[c];
  if (node < 0) {
    return;
  }
  const int i = V.col_inst[c];
  const InstDev& I = V.inst[i];
  if (I.mixed == 0 || V.active[i] == 0 || RefineDone(V, i)) {
    return;
  }
  const double* A = V.asm_fronts;
  const int pose0 = I.col_off + I.num_active;
  double acc = 0.0;
  if (lane < 9) {
    const int64_t ln = node - I.node_off;
    const int w = static_cast<int>(ln % I.nx);
    const int h = static_cast<int>(ln / I.nx);
    const int dh = lane / 3 - 1;
    const int dw = lane % 3 - 1;
    if (w + dw >= 0 && w + dw < I.nx && h + dh >= 0 && h + dh < I.ny) {
      const int c2 = V.node_col[node + static_cast<int64_t>(dh) * I.nx + dw];
      if (c2 >= 0) {
        int64_t off = V.mm_off[static_cast<int64_t>(c) * 9 + lane];
        if (off < 0) {
          off = V.mm_off[static_cast<int64_t>(c2) * 9 + (8 - lane)];
        }
        if (off >= 0) {
          acc = A[off] * x[c2];
        }
      }
    }
  }
  for (int64_t e = V.mp_ptr[c] + lane; e < V.mp_ptr[c + 1]; e += 32) {
    const int64_t off = V.mp_off[e];
    const int pc = pose0 + 3 * (V.mp_frame[e] - 1);
    acc += A[off] * x[pc] + A[off + 1] * x[pc + 1] + A[off + 2] * x[pc + 2];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    acc += __shfl_xor_sync(0xffffffffu, acc, o);
  }
  if (lane == 0) {
    y[c] = acc;
  }
}

/// y = A x over the pose columns of mixed instances: one warp per pose
/// variable (frame, component), lanes strided over the frame's coupled node
/// columns (fmp_*) and over the dense pose block (lower triangle of the pose
/// root), then a fixed butterfly.
__global__ void KNormalMatVecPose(DeviceView V, const double* x, double* y) {
  const int64_t wid = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (wid >= 3 * static_cast<int64_t>(V.total_frames)) {
    return;
  }
  const int gf = static_cast<int>(wid / 3);
  const int a = static_cast<int>(wid % 3);
  const int fc = V.frame_col[gf];
  if (fc < 0) {
    return;
  }
  const int c = fc + a;
  const int i = V.col_inst[c];
  const InstDev& I = V.inst[i];
  if (I.mixed == 0 || V.active[i] == 0 || RefineDone(V, i)) {
    return;
  }
  const double* A = V.asm_fronts;
  const int pose0 = I.col_off + I.num_active;
  double acc = 0.0;
  for (int64_t e = V.fmp_ptr[gf] + lane; e < V.fmp_ptr[gf + 1]; e += 32) {
    acc += A[V.fmp_off[e] + a] * x[V.fmp_col[e]];
  }
  const int np = I.num_params - I.num_active;
  const double* R = A + I.pp_base;
  const int64_t ld = I.pp_ld;
  const int p = I.pp_first + (c - pose0);
  for (int q = lane; q < np; q += 32) {
    const int rq = I.pp_first + q;
    const double aij = p >= rq ? R[rq * ld + p] : R[static_cast<int64_t>(p) * ld + rq];
    acc += aij * x[pose0 + q];
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    acc += __shfl_xor_sync(0xffffffffu, acc, off);
  }
  if (lane == 0) {
    y[c] = acc;
  }
}

/// r = rhs - y for the columns of mixed instances, 0 elsewhere.
__global__ void KRefineResidual(DeviceView V, const double* y, double* r) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= V.n) {
    return;
  }
  const int i = V.col_inst[c];
  r[c] = (V.inst[i].mixed != 0 && V.active[i] != 0 && !RefineDone(V, i)) ? V.rhs[c] - y[c] : 0.0;
}

/// step += correction for the columns of mixed instances.
__global__ void KAddCorrection(DeviceView V, const double* corr) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= V.n) {
    return;
  }
  const int i = V.col_inst[c];
  if (V.inst[i].mixed != 0 && V.active[i] != 0 && !RefineDone(V, i)) {
    const double s = V.step[c] + corr[c];
    V.step[c] = s;
    if (V.refine_max != nullptr) {
      atomicMax(V.refine_max + 2 * i, static_cast<unsigned long long>(__double_as_longlong(fabs(corr[c]))));
      atomicMax(V.refine_max + 2 * i + 1, static_cast<unsigned long long>(__double_as_longlong(fabs(s))));
    }
  }
}

}  // namespace sdfgpu
