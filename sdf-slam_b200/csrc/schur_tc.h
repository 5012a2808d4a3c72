// Tensor-core (tcgen05, split TF32) Schur complement of the FP32 fronts of a
// mixed-precision solve (schur_tc.cu).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "device.cuh"
#include "kernel_timer.h"

namespace sdfgpu {

/// Output tile (rows = columns) and K chunk (FP32 elements, one 128-byte
/// swizzle row) of the tensor-core Schur kernels.
constexpr int kTcTile = 128;
constexpr int kTcChunk = 32;

/// What the tensor-core kernels read: supernodes, FP32 work fronts, D, the
/// per-instance running / precision flags, the status words and the packed
/// operand buffer.
struct TcArgs {
  const SupernodeRec* sn;
  float* fronts32;
  const double* dvec;
  const int32_t* active;
  const InstDev* inst;
  int32_t* status;
  float* pack;
};

/// Packed operand rows (kTcChunk FP32 each) of a front with k pivots and m
/// rows below: four operands x row tiles x K chunks x kTcTile rows.
inline int64_t TcPackRows(int k, int m) {
  const int64_t nT = (m + kTcTile - 1) / kTcTile;
  const int64_t nC = (k + kTcChunk - 1) / kTcChunk;
  return 4 * nT * nC * kTcTile;
}

/// Tensor map of the packed buffer (`rows` rows of kTcChunk FP32).
void EncodePackMap(CUtensorMap* map, float* pack, int64_t rows);
/// Dynamic shared memory of KSchurTc.
size_t SchurTcSmemBytes();
/// KPackSchur over (sn, row tile, chunk) triples, then KSchurTc over
/// (sn, tile i, tile j) triples. Returns the kernels launched. work_pack
/// (bytes) and work_flops (useful flops) are what a timer records.
int LaunchSchurTc(const CUtensorMap& map, const TcArgs& A, const int32_t* pack_tasks, int64_t pack_count,
                  const int32_t* tc_tasks, int64_t tc_count, cudaStream_t stream, KernelTimer* timer,
                  double work_pack, double work_flops);

}  // namespace sdfgpu
