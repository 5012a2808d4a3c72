// Allocation-free dense LDL^T solve.
//
// Some callers cannot allocate device memory at the time they need a solve:
// a host framework whose caching allocator has already reserved the device's
// free memory (a cudaMalloc would fail or fragment its pool), or a real-time
// loop that forbids allocation after start-up. For them this entry point
// solves A x = b for a dense symmetric A with the same panel-factorization,
// update and triangular-solve kernels as the sparse path, but every device
// buffer it touches (the front holding A and L, D, the right-hand side, the
// solution, the task lists) lives in one file-scope __device__ array of fixed
// size. The caller passes host arrays for A, b and x; nothing is allocated.
//
// Limits and sharing: n <= SDFGPU_NOALLOC_MAX_N. The array (about 8.6 MB) is
// resident on every GPU that loads the library until the process exits. All
// calls share it and it keeps the last call's contents, so each call
// overwrites the whole front and clears the status word it reads; two calls
// whose work overlaps on the GPU (from two host threads, for example) race on
// the array and must be serialised by the caller. The first call on a device
// looks up the array's device address (cudaGetSymbolAddress) with that device
// current; with CUDA's lazy module loading that lookup also loads this code
// and reserves the array, so the first call belongs at start-up, before the
// host framework's allocator takes the free memory and before any stream
// capture. The work runs on the calling thread's per-thread default stream,
// which does not wait for the host application's other streams.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "device.cuh"
#include "engine.h"

namespace sdfgpu {

__global__ void KPanel(DeviceView V, const int32_t* tasks, double* dvec, int rows);
__global__ void KUpdate(DeviceView V, const int32_t* tasks, const double* dvec);
__global__ void KForward(DeviceView V, const int32_t* level_sn, const double* dvec);
__global__ void KBackward(DeviceView V, const int32_t* level_sn);

namespace {

constexpr int kMaxN = SDFGPU_NOALLOC_MAX_N;
constexpr int kPanelW = 32;       // panel width of KPanel / KUpdate
constexpr int kTileW = 64;        // tile of KUpdate
constexpr int kPanelRows = 128;   // rows per KPanel block
constexpr int kMaxPanels = (kMaxN + kPanelW - 1) / kPanelW;
constexpr int kMaxPanelTasks = kMaxPanels * ((kMaxN + kPanelRows - 1) / kPanelRows);
constexpr int kMaxUpdateTasks = kMaxPanels * ((kMaxN + kTileW - 1) / kTileW) * ((kMaxN + kTileW - 1) / kTileW);

// Layout of the scratch array, in doubles.
constexpr size_t kFrontOff = 0;
constexpr size_t kDvecOff = kFrontOff + static_cast<size_t>(kMaxN) * kMaxN;
constexpr size_t kRhsOff = kDvecOff + kMaxN;
constexpr size_t kStepOff = kRhsOff + kMaxN;
constexpr size_t kXsOff = kStepOff + kMaxN;
constexpr size_t kUpdOff = kXsOff + kMaxN;
constexpr size_t kSnOff = kUpdOff + 32;                       // one SupernodeRec
constexpr size_t kIntOff = kSnOff + 32;                       // int32 region follows
constexpr size_t kIntCount = static_cast<size_t>(kMaxN)      // perm
                             + 4                               // level_sn, status, active, child
                             + 3 * static_cast<size_t>(kMaxPanelTasks) + 4 * static_cast<size_t>(kMaxUpdateTasks);
constexpr size_t kScratchDoubles = kIntOff + (kIntCount + 1) / 2;

static_assert(sizeof(SupernodeRec) <= 32 * sizeof(double), "supernode record slot too small");

__device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

/// Device address of g_noalloc_scratch on the current device, looked up once
/// per device.
double* ScratchAddress() {
  static std::mutex mu;
  static void* cached[64] = {};
  int dev = 0;
  CudaCheck(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= 64) {
    Fail(SDFGPU_ERR_CUDA, "device index out of range for the scratch table");
  }
  std::lock_guard<std::mutex> lk(mu);
  if (cached[dev] == nullptr) {
    void* ptr = nullptr;
    CudaCheck(cudaGetSymbolAddress(&ptr, g_noalloc_scratch), "cudaGetSymbolAddress");
    cached[dev] = ptr;
  }
  return static_cast<double*>(cached[dev]);
}

}  // namespace

/// Solves A x = b in the static scratch; throws Error on bad sizes or a zero
/// pivot. A is n x n column major; only its lower triangle is read.
void DenseLdltSolveNoAlloc(int n, const double* a, const double* b, double* x) {
  if (n < 1 || n > kMaxN) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT,
         "n = " + std::to_string(n) + " is outside 1.." + std::to_string(kMaxN) +
             " (the size of the allocation-free scratch)");
  }
  if (a == nullptr || b == nullptr || x == nullptr) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT, "a, b and x are required");
  }
  double* base = ScratchAddress();
  int32_t* ints = reinterpret_cast<int32_t*>(base + kIntOff);
  int32_t* d_perm = ints;
  int32_t* d_level = ints + kMaxN;
  int32_t* d_status = d_level + 1;
  int32_t* d_active = d_level + 2;
  int32_t* d_child = d_level + 3;
  int32_t* d_ptasks = d_level + 4;
  int32_t* d_utasks = d_ptasks + 3 * kMaxPanelTasks;

  // host-side task lists and constants, on the stack
  SupernodeRec rec{};
  rec.front_off = 0;
  rec.rows_off = 0;
  rec.upd_off = 0;
  rec.first_col = 0;
  rec.ncols = n;
  rec.nrows = 0;
  rec.F = n;
  rec.child_begin = 0;
  rec.child_count = 0;
  rec.parent = -1;
  rec.instance = 0;
  int32_t perm[kMaxN];
  for (int i = 0; i < n; ++i) {
    perm[i] = i;
  }
  int32_t consts[4] = {0, 0, 1, 0};  // level list {supernode 0}, status 0, active 1, no child
  // the calling thread's per-thread default stream: no stream object is
  // created and the host application's streams are not waited for
  cudaStream_t s = cudaStreamPerThread;
  const size_t nn = static_cast<size_t>(n);
  CudaCheck(cudaMemcpyAsync(base + kFrontOff, a, nn * nn * sizeof(double), cudaMemcpyHostToDevice, s), "A");
  CudaCheck(cudaMemcpyAsync(base + kRhsOff, b, nn * sizeof(double), cudaMemcpyHostToDevice, s), "b");
  CudaCheck(cudaMemcpyAsync(base + kSnOff, &rec, sizeof(rec), cudaMemcpyHostToDevice, s), "record");
  CudaCheck(cudaMemcpyAsync(d_perm, perm, nn * sizeof(int32_t), cudaMemcpyHostToDevice, s), "perm");
  CudaCheck(cudaMemcpyAsync(d_level, consts, sizeof(consts), cudaMemcpyHostToDevice, s), "consts");
  // Task lists of each panel, built in small stack buffers and copied into
  // the panel's own region of the scratch (copies from pageable memory have
  // consumed the buffer when cudaMemcpyAsync returns).
  constexpr int kRowChunks = (kMaxN + kPanelRows - 1) / kPanelRows;
  constexpr int kTiles = (kMaxN + kTileW - 1) / kTileW;
  int32_t ptask[3 * kRowChunks];
  int32_t utask[4 * kTiles * kTiles];
  int panel_count[kMaxPanels];
  int update_count[kMaxPanels];
  const int panels = (n + kPanelW - 1) / kPanelW;
  for (int t = 0; t < panels; ++t) {
    const int c1 = std::min(n, (t + 1) * kPanelW);
    const int chunks = std::max(1, (n - c1 + kPanelRows - 1) / kPanelRows);
    for (int ch = 0; ch < chunks; ++ch) {
      ptask[3 * ch] = 0;
      ptask[3 * ch + 1] = t;
      ptask[3 * ch + 2] = c1 + ch * kPanelRows;
    }
    int nu = 0;
    const int rest = n - c1;
    for (int tj = 0; tj * kTileW < rest; ++tj) {
      for (int ti = 0; ti * kTileW < rest; ++ti) {
        if ((ti + 1) * kTileW - 1 < tj * kTileW) {
          continue;
        }
        utask[4 * nu] = 0;
        utask[4 * nu + 1] = t;
        utask[4 * nu + 2] = ti;
        utask[4 * nu + 3] = tj;
        ++nu;
      }
    }
    panel_count[t] = chunks;
    update_count[t] = nu;
    CudaCheck(cudaMemcpyAsync(d_ptasks + 3 * kRowChunks * t, ptask, static_cast<size_t>(3 * chunks) * sizeof(int32_t),
                              cudaMemcpyHostToDevice, s),
              "panel tasks");
    if (nu > 0) {
      CudaCheck(cudaMemcpyAsync(d_utasks + 4 * kTiles * kTiles * t, utask, static_cast<size_t>(4 * nu) * sizeof(int32_t),
                                cudaMemcpyHostToDevice, s),
                "update tasks");
    }
  }
  DeviceView V{};
  V.num_inst = 1;
  V.n = n;
  V.perm = d_perm;
  V.sn = reinterpret_cast<const SupernodeRec*>(base + kSnOff);
  V.child_list = d_child;
  V.sn_rows = d_child;
  V.sn_rel = d_child;
  V.fronts = base + kFrontOff;
  V.upd = base + kUpdOff;
  V.rhs = base + kRhsOff;
  V.step = base + kStepOff;
  V.xs = base + kXsOff;
  V.status = d_status;
  V.active = d_active;
  double* dvec = base + kDvecOff;
  for (int t = 0; t < panels; ++t) {
    KPanel<<<static_cast<unsigned>(panel_count[t]), kPanelRows, 0, s>>>(V, d_ptasks + 3 * kRowChunks * t, dvec,
                                                                        kPanelRows);
    if (update_count[t] > 0) {
      KUpdate<<<static_cast<unsigned>(update_count[t]), 256, 0, s>>>(V, d_utasks + 4 * kTiles * kTiles * t, dvec);
    }
  }
  const size_t smem = nn * sizeof(double);
  KForward<<<1, 256, smem, s>>>(V, d_level, dvec);
  KBackward<<<1, 256, smem, s>>>(V, d_level);
  CudaCheck(cudaGetLastError(), "allocation-free solve kernels");
  int32_t status = 0;
  CudaCheck(cudaMemcpyAsync(&status, d_status, sizeof(status), cudaMemcpyDeviceToHost, s), "status");
  CudaCheck(cudaMemcpyAsync(x, base + kStepOff, nn * sizeof(double), cudaMemcpyDeviceToHost, s), "x");
  CudaCheck(cudaStreamSynchronize(s), "allocation-free solve");
  if ((status & kStatusZeroPivot) != 0) {
    Fail(SDFGPU_ERR_NUMERICAL, "sparse Cholesky factorization failed");
  }
}

}  // namespace sdfgpu
