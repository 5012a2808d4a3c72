// Schur complement of the FP32 fronts of a mixed-precision solve on the
// fifth-generation tensor cores (tcgen05, kind::tf32), with the split-TF32
// ("TF32x3") products that keep FP32 accuracy:
//
//   C -= L21 D L21^T,  A = L21 D = Ah + Al,  B = L21 = Bh + Bl,
//   C -= Ah Bh^T + Ah Bl^T + Al Bh^T
//
// (Ah, Bh the operands rounded to TF32, Al, Bl the TF32 roundings of the
// remainders; the dropped Al Bl^T term is below FP32 rounding). This is the
// rank-k update that ParallelSimplicialLdlt's row kernel applies entry by
// entry (src/solvers/parallel_ldlt.hpp:165-206) and CHOLMOD's supernodal
// update (src/solvers/lm_solver.cpp:342-358), done per front as one dense
// contraction; FP64 iterative refinement of the step against the FP64 normal
// matrix wins the accuracy back.
//
// Two kernels per level of the assembly tree:
//  * KPackSchur: per (front, 128-row tile, 32-column chunk) of L21, the four
//    operand tiles Ah, Al, Bh, Bl as 128 rows x 32 FP32 (K-major, 128 B per
//    row) into a packed buffer;
//  * KSchurTc: per 128 x 128 tile of the front's trailing block (lower part),
//    one CTA of four warps: a producer thread streams the operand tiles of
//    each 32-wide K chunk into a three-stage shared-memory ring with TMA
//    (cp.async.bulk.tensor, 128-byte swizzle, one tensor map over the packed
//    buffer), one thread issues the 12 tcgen05.mma of a chunk (3 products x
//    4 steps of K = 8) into a 128 x 128 FP32 accumulator in tensor memory,
//    and the four warps read the accumulator back (tcgen05.ld) and subtract
//    it from the front's lower triangle.
// Every wait on an mbarrier has an iteration limit; a wait that runs out
// marks the instance kStatusWaitTimeout, lets the copies in flight land,
// frees the tensor memory and returns (the solve then fails with a timeout).
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "engine.h"
#include "schur_tc.h"

namespace sdfgpu {

namespace {

constexpr int kRowsTile = kTcTile;                 // M = N = 128
constexpr int kChunk = kTcChunk;                   // K per chunk (FP32 elements)
constexpr int kStages = 3;
constexpr int kTileBytes = kRowsTile * kChunk * 4;  // 16 KB
constexpr int kStageBytes = 4 * kTileBytes;         // Ah, Al, Bh, Bl
constexpr uint32_t kTmemCols = 128;
constexpr uint32_t kWaitLimit = 1u << 24;

__device__ __forceinline__ uint32_t SmemAddr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void MbarInit(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(SmemAddr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void MbarArriveExpectTx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(SmemAddr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool MbarTestWait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(SmemAddr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

/// Waits for the phase of `parity` to complete, at most kWaitLimit polls;
/// gives up early when another role raised `abort`. Returns false (and
/// raises abort) when the limit ran out.
__device__ __forceinline__ bool MbarWait(uint64_t* bar, uint32_t parity, volatile int* abort) {
  for (uint32_t i = 0; i < kWaitLimit; ++i) {
    if (MbarTestWait(bar, parity)) {
      return true;
    }
    if (*abort != 0) {
      return false;
    }
  }
  *abort = 1;
  return false;
}

/// Same, ignoring `abort`: for the copies that must land before the CTA
/// exits.
__device__ __forceinline__ bool MbarDrain(uint64_t* bar, uint32_t parity) {
  for (uint32_t i = 0; i < kWaitLimit; ++i) {
    if (MbarTestWait(bar, parity)) {
      return true;
    }
  }
  return false;
}

__device__ __forceinline__ void TmaLoadTile(void* dst, const CUtensorMap* map, int row, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          SmemAddr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(row), "r"(SmemAddr(bar))
      : "memory");
}

__device__ __forceinline__ void TcFenceBefore() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void TcFenceAfter() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

/// Shared-memory matrix descriptor of a K-major operand tile with 128-byte
/// swizzle: rows of 128 B, 8-row groups 1024 B apart (the stride byte
/// offset); the leading byte offset is not used by swizzled K-major layouts.
__device__ __forceinline__ uint64_t SmemDescSw128(uint32_t saddr) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((saddr & 0x3FFFFu) >> 4);
  d |= static_cast<uint64_t>(16u >> 4) << 16;
  d |= static_cast<uint64_t>(1024u >> 4) << 32;
  d |= static_cast<uint64_t>(1) << 46;  // descriptor version of sm_100
  d |= static_cast<uint64_t>(2) << 61;  // 128-byte swizzle
  return d;
}

/// Instruction descriptor of kind::tf32: FP32 accumulator, TF32 A and B,
/// both K-major, M = N = 128.
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((kRowsTile >> 3) << 17) | ((kRowsTile >> 4) << 24);

__device__ __forceinline__ void MmaTf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate)
      : "memory");
}

/// Arrives on `bar` when every tcgen05.mma this thread issued has completed.
__device__ __forceinline__ void MmaCommit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(SmemAddr(bar))
               : "memory");
}

__device__ __forceinline__ void TmemLoad16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ float ToTf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

__device__ __forceinline__ bool TcFront(const TcArgs& A, const SupernodeRec& S) {
  return S.tc_pack >= 0 && S.pose_root == 0 && A.active[S.instance] != 0 && A.inst[S.instance].mixed != 0;
}

}  // namespace

/// Operand tiles of one (front, row tile t, K chunk c): L21 rows
/// [t*128, t*128 + 128) of pivot columns [c*32, c*32 + 32), read coalesced
/// along the column-major front, transposed in shared memory, split into
/// TF32 halves and written row-major (zero past m rows and k columns).
__global__ void __launch_bounds__(256) KPackSchur(TcArgs A, const int32_t* tasks) {
  const int32_t* t = tasks + 3 * static_cast<int64_t>(blockIdx.x);
  const SupernodeRec S = A.sn[t[0]];
  if (!TcFront(A, S)) {
    return;
  }
  __shared__ float tile[kChunk][kRowsTile + 1];
  __shared__ float dk[kChunk];
  const int k = S.ncols;
  const int m = S.nrows;
  const int64_t F = S.F;
  const int nT = (m + kRowsTile - 1) / kRowsTile;
  const int nC = (k + kChunk - 1) / kChunk;
  const int rt = t[1];
  const int c = t[2];
  const float* Fs = A.fronts32 + S.front_off;
  const int tid = threadIdx.x;
  if (tid < kChunk) {
    const int l = c * kChunk + tid;
    dk[tid] = l < k ? static_cast<float>(A.dvec[S.first_col + l]) : 0.0f;
  }
  for (int idx = tid; idx < kChunk * kRowsTile; idx += blockDim.x) {
    const int i = idx % kRowsTile;
    const int l = idx / kRowsTile;
    const int r = rt * kRowsTile + i;
    const int col = c * kChunk + l;
    tile[l][i] = (r < m && col < k) ? Fs[col * F + k + r] : 0.0f;
  }
  __syncthreads();
  float* base = A.pack + S.tc_pack * kChunk;
  const int64_t tile_floats = static_cast<int64_t>(kRowsTile) * kChunk;
  float* ah = base + ((0 * static_cast<int64_t>(nT) + rt) * nC + c) * tile_floats;
  float* al = base + ((1 * static_cast<int64_t>(nT) + rt) * nC + c) * tile_floats;
  float* bh = base + ((2 * static_cast<int64_t>(nT) + rt) * nC + c) * tile_floats;
  float* bl = base + ((3 * static_cast<int64_t>(nT) + rt) * nC + c) * tile_floats;
  for (int idx = tid; idx < kChunk * kRowsTile; idx += blockDim.x) {
    const int i = idx / kChunk;
    const int l = idx % kChunk;
    const float b = tile[l][i];
    const float a = b * dk[l];
    const float a_hi = ToTf32(a);
    const float b_hi = ToTf32(b);
    ah[idx] = a_hi;
    al[idx] = ToTf32(a - a_hi);
    bh[idx] = b_hi;
    bl[idx] = ToTf32(b - b_hi);
  }
}

/// One 128 x 128 tile (ti, tj), ti >= tj, of the front's trailing block:
/// C(ti, tj) -= A(ti) B(tj)^T over all K chunks (see the file comment).
__global__ void __launch_bounds__(128, 1) KSchurTc(const __grid_constant__ CUtensorMap tmap, TcArgs A,
                                                   const int32_t* tasks) {
  const int32_t* t = tasks + 3 * static_cast<int64_t>(blockIdx.x);
  const SupernodeRec S = A.sn[t[0]];
  if (!TcFront(A, S)) {
    return;
  }
  extern __shared__ uint8_t smem_raw[];
  uint8_t* ring = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t{1023});
  __shared__ uint64_t full[kStages];
  __shared__ uint64_t empty[kStages];
  __shared__ uint64_t done;
  __shared__ uint32_t tmem_base;
  __shared__ int abort_flag;
  volatile int* abort = &abort_flag;
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int k = S.ncols;
  const int m = S.nrows;
  const int64_t F = S.F;
  const int nT = (m + kRowsTile - 1) / kRowsTile;
  const int nC = (k + kChunk - 1) / kChunk;
  const int ti = t[1];
  const int tj = t[2];
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      MbarInit(&full[s], 1);
      MbarInit(&empty[s], 1);
    }
    MbarInit(&done, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmap)) : "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(SmemAddr(&tmem_base)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  TcFenceBefore();
  __syncthreads();
  TcFenceAfter();
  const uint32_t tmem = tmem_base;
  // first packed row of operand o's tile (row tile rt, chunk c)
  auto tile_row = [&](int o, int rt, int c) {
    return static_cast<int>(S.tc_pack + ((static_cast<int64_t>(o) * nT + rt) * nC + c) * kRowsTile);
  };
  if (warp == 0 && lane == 0) {
    // producer: TMA loads of each chunk's four tiles into the ring
    int issued = 0;
    for (int c = 0; c < nC; ++c) {
      const int s = c % kStages;
      if (c >= kStages && !MbarWait(&empty[s], static_cast<uint32_t>((c / kStages - 1) & 1), abort)) {
        break;
      }
      uint8_t* st = ring + s * kStageBytes;
      MbarArriveExpectTx(&full[s], kStageBytes);
      TmaLoadTile(st, &tmap, tile_row(0, ti, c), &full[s]);
      TmaLoadTile(st + kTileBytes, &tmap, tile_row(1, ti, c), &full[s]);
      TmaLoadTile(st + 2 * kTileBytes, &tmap, tile_row(2, tj, c), &full[s]);
      TmaLoadTile(st + 3 * kTileBytes, &tmap, tile_row(3, tj, c), &full[s]);
      ++issued;
    }
    if (*abort != 0) {
      // the last load of each stage may still be in flight: let it land
      for (int c = (issued > kStages ? issued - kStages : 0); c < issued; ++c) {
        MbarDrain(&full[c % kStages], static_cast<uint32_t>((c / kStages) & 1));
      }
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer: 3 products x 4 K steps per chunk into the accumulator
    for (int c = 0; c < nC; ++c) {
      const int s = c % kStages;
      if (!MbarWait(&full[s], static_cast<uint32_t>((c / kStages) & 1), abort)) {
        break;
      }
      TcFenceAfter();
      const uint32_t base = SmemAddr(ring + s * kStageBytes);
      const uint64_t ah = SmemDescSw128(base);
      const uint64_t al = SmemDescSw128(base + kTileBytes);
      const uint64_t bh = SmemDescSw128(base + 2 * kTileBytes);
      const uint64_t bl = SmemDescSw128(base + 3 * kTileBytes);
#pragma unroll
      for (int kk = 0; kk < kChunk / 8; ++kk) {
        // K step kk: 8 TF32 = 32 bytes further along each 128-byte row
        const uint64_t step = static_cast<uint64_t>(kk * 32 / 16);
        MmaTf32(tmem, ah + step, bh + step, (c | kk) != 0 ? 1u : 0u);
        MmaTf32(tmem, ah + step, bl + step, 1u);
        MmaTf32(tmem, al + step, bh + step, 1u);
      }
      MmaCommit(&empty[s]);
    }
    MmaCommit(&done);
  }
  __syncwarp();
  // epilogue: warp w reads accumulator lanes (rows) 32w..32w+31
  const bool ok = MbarWait(&done, 0u, abort);
  __syncwarp();
  TcFenceAfter();
  if (ok && *abort == 0) {
    float* Fs = A.fronts32 + S.front_off;
    const int row = ti * kRowsTile + warp * 32 + lane;
    const uint32_t taddr = tmem + (static_cast<uint32_t>(warp * 32) << 16);
    // 32 columns per batch: the batch's C values are read before any is
    // written (the compiler cannot prove the columns apart), so the reads
    // overlap instead of each waiting for the previous write
    for (int j0 = 0; j0 < kRowsTile; j0 += 32) {
      float cv[32];
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        const int col = tj * kRowsTile + j0 + j;
        cv[j] = (row < m && col <= row) ? Fs[(k + col) * F + k + row] : 0.0f;
      }
      uint32_t r[32];
      TmemLoad16(taddr + static_cast<uint32_t>(j0), *reinterpret_cast<uint32_t(*)[16]>(r));
      TmemLoad16(taddr + static_cast<uint32_t>(j0 + 16), *reinterpret_cast<uint32_t(*)[16]>(r + 16));
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        const int col = tj * kRowsTile + j0 + j;
        if (row < m && col <= row) {
          Fs[(k + col) * F + k + row] = cv[j] - __uint_as_float(r[j]);
        }
      }
    }
  }
  TcFenceBefore();
  __syncthreads();
  TcFenceAfter();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
  if (threadIdx.x == 0 && *abort != 0) {
    atomicOr(A.status + S.instance, kStatusWaitTimeout);
  }
}

namespace {

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn EncodeTiled() {
  static EncodeTiledFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    CudaCheck(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q), "driver entry point");
    if (q != cudaDriverEntryPointSuccess || p == nullptr) {
      Fail(SDFGPU_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
    }
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  return fn;
}

}  // namespace

void EncodePackMap(CUtensorMap* map, float* pack, int64_t rows) {
  // the packed buffer as rows of kChunk FP32 (128 B); one box = one operand
  // tile of 128 rows, swizzled in 16-byte units within each 128-byte row
  const cuuint64_t dims[2] = {static_cast<cuuint64_t>(kChunk), static_cast<cuuint64_t>(rows < 1 ? 1 : rows)};
  const cuuint64_t strides[1] = {static_cast<cuuint64_t>(kChunk) * sizeof(float)};
  const cuuint32_t box[2] = {static_cast<cuuint32_t>(kChunk), static_cast<cuuint32_t>(kRowsTile)};
  const cuuint32_t elem[2] = {1, 1};
  const CUresult r = EncodeTiled()(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, pack, dims, strides, box, elem,
                                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    Fail(SDFGPU_ERR_CUDA, "cuTensorMapEncodeTiled failed for the packed Schur operands");
  }
}

size_t SchurTcSmemBytes() { return static_cast<size_t>(kStages) * kStageBytes + 1024; }

int LaunchSchurTc(const CUtensorMap& map, const TcArgs& A, const int32_t* pack_tasks, int64_t pack_count,
                  const int32_t* tc_tasks, int64_t tc_count, cudaStream_t stream, KernelTimer* timer,
                  double work_pack, double work_flops) {
  // the shared memory limit is a per-device attribute of the kernel
  static bool configured[64] = {};
  int dev = 0;
  CudaCheck(cudaGetDevice(&dev), "device");
  if (dev < 0 || dev >= 64 || !configured[dev]) {
    CudaCheck(cudaFuncSetAttribute(KSchurTc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(SchurTcSmemBytes())),
              "tc smem attr");
    if (dev >= 0 && dev < 64) {
      configured[dev] = true;
    }
  }
  int launches = 0;
  if (pack_count > 0) {
    const TimedLaunch tl(timer, KernelTimer::kPackSchur, stream, [&] { return work_pack; });
    KPackSchur<<<static_cast<unsigned>(pack_count), 256, 0, stream>>>(A, pack_tasks);
    ++launches;
  }
  if (tc_count > 0) {
    const TimedLaunch tl(timer, KernelTimer::kSchurTc, stream, [&] { return work_flops; });
    KSchurTc<<<static_cast<unsigned>(tc_count), 128, SchurTcSmemBytes(), stream>>>(map, A, tc_tasks);
    ++launches;
  }
  CudaCheck(cudaGetLastError(), "tensor-core Schur kernels");
  return launches;
}

}  // namespace sdfgpu
