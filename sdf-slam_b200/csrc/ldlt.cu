// Factor-only sparse LDL^T (see ldlt.h).
#include "ldlt.h"

namespace sdfgpu {

namespace {

/// Scatters the input values into their front positions (lower triangle of
/// the permuted matrix; the upper copies are skipped).
__global__ void KScatterValues(const double* values, const int64_t* off, int64_t nnz, double* fronts) {
  const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (p < nnz) {
    const int64_t o = off[p];
    if (o >= 0) {
      fronts[o] = values[p];
    }
  }
}

}  // namespace

LdltEngine::LdltEngine(int n, const int32_t* outer, const int32_t* inner, const int32_t* perm) : n_(n) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    Fail(SDFGPU_ERR_CUDA, "no CUDA device available (the GPU backend has no CPU fallback)");
  }
  nnz_ = outer[n];
  for (int j = 0; j < n; ++j) {
    if (outer[j + 1] < outer[j]) {
      Fail(SDFGPU_ERR_INVALID_ARGUMENT, "CSC outer index must not decrease");
    }
    for (int p = outer[j]; p < outer[j + 1]; ++p) {
      if (inner[p] < 0 || inner[p] >= n) {
        Fail(SDFGPU_ERR_INVALID_ARGUMENT, "CSC row index out of range");
      }
    }
  }
  std::vector<int32_t> pv;
  if (perm != nullptr) {
    pv.assign(perm, perm + n);
  }
  std::vector<int64_t> offs;
  sym_ = AnalyzeGeneral(n, outer, inner, pv, 32, 64, offs);
  CudaCheck(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "stream");
  cudaStream_t s = stream_;
  perm_.Upload(sym_.perm, s);
  sn_.Upload(sym_.sn, s);
  sn_rows_.Upload(sym_.sn_rows, s);
  sn_rel_.Upload(sym_.sn_rel, s);
  child_list_.Upload(sym_.child_list, s);
  level_sn_.Upload(sym_.level_sn, s);
  ea_tasks_.Upload(sym_.ea_tasks, s);
  ea_child_.Upload(sym_.ea_child, s);
  panel_tasks_.Upload(sym_.panel_tasks, s);
  update_tasks_.Upload(sym_.update_tasks, s);
  small_tasks_.Upload(sym_.small_tasks, s);
  value_off_.Upload(offs, s);
  values_.Alloc(static_cast<size_t>(nnz_));
  fronts_.Alloc(static_cast<size_t>(sym_.front_doubles));
  upd_.Alloc(static_cast<size_t>(std::max<int64_t>(1, sym_.update_doubles)));
  dvec_.Alloc(static_cast<size_t>(n));
  rhs_.Alloc(static_cast<size_t>(n));
  step_.Alloc(static_cast<size_t>(n));
  xs_.Alloc(static_cast<size_t>(n));
  status_.Upload(std::vector<int32_t>{0}, s);
  active_.Upload(std::vector<int32_t>{1}, s);
  int max_front = 1;
  for (const SupernodeRec& r : sym_.sn) {
    max_front = std::max(max_front, r.F);
  }
  ConfigureSolveKernels(max_front);
  V_.num_inst = 1;
  V_.n = n;
  V_.perm = perm_.get();
  V_.sn = sn_.get();
  V_.sn_rows = sn_rows_.get();
  V_.sn_rel = sn_rel_.get();
  V_.child_list = child_list_.get();
  V_.fronts = fronts_.get();
  V_.upd = upd_.get();
  V_.rhs = rhs_.get();
  V_.step = step_.get();
  V_.xs = xs_.get();
  V_.status = status_.get();
  V_.active = active_.get();
  plan_.small_tasks = small_tasks_.get();
  plan_.ea_tasks = ea_tasks_.get();
  plan_.ea_child = ea_child_.get();
  plan_.panel_tasks = panel_tasks_.get();
  plan_.update_tasks = update_tasks_.get();
  plan_.level_sn = level_sn_.get();
  plan_.dvec = dvec_.get();
  plan_.max_front = max_front;
  solve_sync_.Alloc(SolveSyncWords(static_cast<int>(sym_.sn.size()), static_cast<int>(sym_.inv_tasks.size() / 2)));
  plan_.solve_sync = solve_sync_.get();
  solve_tasks_.Upload(sym_.solve_tasks, s);
  solve_parts_.Upload(sym_.solve_parts, s);
  zpart_off_.Upload(sym_.zpart_off, s);
  ys_.Alloc(static_cast<size_t>(std::max(n, 1)));
  zpart_.Alloc(static_cast<size_t>(std::max<int64_t>(1, sym_.zpart_doubles)));
  dense_tasks_.Upload(sym_.dense_tasks, s);
  dense_sync_.Alloc(DenseSyncWords(sym_));
  dense_inv_.Alloc(static_cast<size_t>(std::max<int64_t>(1, sym_.dense_inv_doubles)));
  plan_.dense_tasks = dense_tasks_.get();
  plan_.dense_sync = dense_sync_.get();
  plan_.dense_inv = dense_inv_.get();
  plan_.solve_tasks = solve_tasks_.get();
  plan_.num_solve_tasks = static_cast<int>(sym_.solve_tasks.size() / 4);
  plan_.solve_parts = solve_parts_.get();
  plan_.zpart_off = zpart_off_.get();
  plan_.ys = ys_.get();
  plan_.zpart = zpart_.get();
  inv_tasks_.Upload(sym_.inv_tasks, s);
  inv_.Alloc(std::max<size_t>(1, sym_.inv_tasks.size() / 2) * kInvBlockDoubles);
  plan_.inv_tasks = inv_tasks_.get();
  plan_.num_inv = static_cast<int>(sym_.inv_tasks.size() / 2);
  plan_.inv = inv_.get();
  CudaCheck(cudaStreamSynchronize(s), "ldlt analyze");
}

LdltEngine::~LdltEngine() {
  if (stream_ != nullptr) {
    cudaStreamSynchronize(stream_);
    cudaStreamDestroy(stream_);
  }
}

void LdltEngine::Factorize(const double* values) {
  cudaStream_t s = stream_;
  factored_ = false;
  CudaCheck(cudaMemcpyAsync(values_.get(), values, static_cast<size_t>(nnz_) * sizeof(double),
                            cudaMemcpyHostToDevice, s),
            "values");
  CudaCheck(cudaMemsetAsync(fronts_.get(), 0, static_cast<size_t>(sym_.front_doubles) * sizeof(double), s),
            "fronts");
  CudaCheck(cudaMemsetAsync(status_.get(), 0, sizeof(int32_t), s), "status");
  if (nnz_ > 0) {
    KScatterValues<<<static_cast<unsigned>((nnz_ + 255) / 256), 256, 0, s>>>(values_.get(), value_off_.get(), nnz_,
                                                                              fronts_.get());
  }
  LaunchFactorLevels(sym_, V_, plan_, s);
  int32_t st = 0;
  CudaCheck(cudaMemcpyAsync(&st, status_.get(), sizeof(int32_t), cudaMemcpyDeviceToHost, s), "status");
  CudaCheck(cudaStreamSynchronize(s), "factorize");
  if ((st & kStatusZeroPivot) != 0) {
    Fail(SDFGPU_ERR_NUMERICAL, "sparse Cholesky factorization failed");
  }
  factored_ = true;
}

void LdltEngine::Solve(const double* b, double* x) {
  if (!factored_) {
    Fail(SDFGPU_ERR_INVALID_ARGUMENT, "solve needs a successful factorization");
  }
  cudaStream_t s = stream_;
  CudaCheck(cudaMemcpyAsync(rhs_.get(), b, static_cast<size_t>(n_) * sizeof(double), cudaMemcpyHostToDevice, s),
            "b");
  CudaCheck(cudaMemsetAsync(status_.get(), 0, sizeof(int32_t), s), "status");
  LaunchSolveLevels(sym_, V_, plan_, s);
  int32_t st = 0;
  CudaCheck(cudaMemcpyAsync(&st, status_.get(), sizeof(int32_t), cudaMemcpyDeviceToHost, s), "status");
  CudaCheck(cudaMemcpyAsync(x, step_.get(), static_cast<size_t>(n_) * sizeof(double), cudaMemcpyDeviceToHost, s),
            "x");
  CudaCheck(cudaStreamSynchronize(s), "solve");
  if ((st & kStatusWaitTimeout) != 0) {
    Fail(SDFGPU_ERR_TIMEOUT, "a wait of the solve kernel ran out of its limit");
  }
}

}  // namespace sdfgpu
