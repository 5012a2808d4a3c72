// Tiled LDL^T of the dense pose roots by one persistent launch per level.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "device.cuh"

namespace sdfgpu {

/// What one dense-root launch reads besides the view.
struct DenseArgs {
  const int32_t* tasks;  // (sn, i, j, k) quads of the level, in the order blocks take them
  int64_t count;
  int32_t* claim;        // the launch's task counter (zero before the launch)
  int32_t* abort;        // set when a wait ran out: every later task is skipped
  int32_t* cnt;          // per dense front (SupernodeRec::dense_cnt): tile counters, zero before the factorization
  double* inv;           // per dense front (SupernodeRec::dense_inv): L^-1 of each diagonal tile, 64 x 64
  double* dvec;
  uint32_t wait_limit;
  /// Optional task trace (null: off): per task, the global timer in ns when
  /// a block took it, when its inputs were ready and when it published.
  uint64_t* trace;
};

/// Launches the persistent tiled factorization over args.count tasks on
/// `stream` (one block per SM, never more blocks than tasks).
/// Returns the launches made (0 or 1).
int LaunchDenseRoots(const DeviceView& V, const DenseArgs& args, cudaStream_t stream);

}  // namespace sdfgpu
