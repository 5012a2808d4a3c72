// Factor-only sparse LDL^T on the GPU for any symmetric matrix: the
// interface of ParallelSimplicialLdlt (src/solvers/parallel_ldlt.hpp:38-51)
// plus Eigen's solve, on the multifrontal kernels of the LM path.
#pragma once

#include <vector>

#include "engine.h"

namespace sdfgpu {

class LdltEngine {
 public:
  /// Symbolic analysis of a full symmetric CSC pattern (sorted rows);
  /// perm: new -> old or NULL for the natural order.
  LdltEngine(int n, const int32_t* outer, const int32_t* inner, const int32_t* perm);
  ~LdltEngine();
  LdltEngine(const LdltEngine&) = delete;
  LdltEngine& operator=(const LdltEngine&) = delete;
  /// Numeric factorization; SDFGPU_ERR_NUMERICAL on a zero pivot.
  void Factorize(const double* values);
  /// x = A^-1 b after a successful Factorize.
  void Solve(const double* b, double* x);

 private:
  int n_{0};
  int64_t nnz_{0};
  bool factored_{false};
  Symbolic sym_;
  cudaStream_t stream_{nullptr};
  DeviceView V_{};
  FactorPlan plan_{};
  DevBuf<int32_t> perm_, sn_rows_, sn_rel_, child_list_, level_sn_, ea_tasks_, ea_child_, panel_tasks_, update_tasks_,
      small_tasks_;
  DevBuf<SupernodeRec> sn_;
  DevBuf<int64_t> value_off_;
  DevBuf<double> values_, fronts_, upd_, dvec_, rhs_, step_, xs_;
  DevBuf<int32_t> status_, active_;
  DevBuf<uint32_t> solve_sync_;
  DevBuf<int32_t> solve_tasks_, solve_parts_, dense_tasks_, dense_sync_;
  DevBuf<double> dense_inv_;
  DevBuf<int64_t> zpart_off_;
  DevBuf<double> ys_, zpart_;
  DevBuf<int32_t> inv_tasks_;
  DevBuf<double> inv_;
};

}  // namespace sdfgpu
