// Engine: device-resident state, symbolic structure and LM driver of one
// sdfgpu handle (one or several independent problems).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <future>
#include <memory>
#include <string>
#include <vector>

#include "device.cuh"
#include "internal.h"
#include "schur_tc.h"

namespace sdfgpu {

[[noreturn]] void ThrowCuda(cudaError_t e, const char* what);

inline void CudaCheck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    ThrowCuda(e, what);
  }
}

/// Block allocators with a per-device cache of freed blocks (alloc.cpp):
/// `got` receives the block's size (the request rounded up to its class),
/// `device` (when given) the device it lives on, which its free must name,
/// whichever device is current then. A block may only be freed once no
/// enqueued work uses it.
void* CachedDeviceAlloc(size_t bytes, size_t* got, int* device = nullptr);
void CachedDeviceFree(void* p, size_t bytes, int device);
/// Returns the current device's cached blocks and its pool's reserve to the
/// driver.
void ReleaseCachedDeviceMemory();
/// FP64 FMA throughput of the current device in TFLOP/s (peak.cu).
double MeasureFp64PeakTflops();
void* CachedHostAlloc(size_t bytes, size_t* got);
void CachedHostFree(void* p, size_t bytes);

/// Host-to-device copy of `bytes` from pageable memory, enqueued on `s`.
/// Large copies go through two pinned staging buffers, one filled (by the
/// host pool's threads) while the other's transfer runs; `src` may be
/// reused as soon as this returns.
void UploadAsync(void* dst, const void* src, size_t bytes, cudaStream_t s);

/// Owning device buffer. Owners free (or grow) it only after their stream
/// has drained.
template <typename T>
class DevBuf {
 public:
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { Free(); }
  void Free() {
    if (ptr_ != nullptr) {
      CachedDeviceFree(ptr_, bytes_, device_);
      ptr_ = nullptr;
      count_ = 0;
      bytes_ = 0;
    }
  }
  void Alloc(size_t count) {
    if (count <= count_ && ptr_ != nullptr) {
      return;
    }
    // a buffer that has to grow (a re-analysis widened the pattern) gets a
    // quarter of headroom, so that the next growth reuses it
    const bool regrow = ptr_ != nullptr;
    Free();
    if (regrow) {
      count += count / 4;
    }
    const size_t bytes = std::max<size_t>(1, count) * sizeof(T);
    ptr_ = static_cast<T*>(CachedDeviceAlloc(bytes, &bytes_, &device_));
    count_ = bytes_ / sizeof(T);
  }
  /// As Alloc, but a fresh block is a quarter larger than asked for from the
  /// first allocation on (the front buffers: a re-analysis that widens a
  /// pattern by two cells adds about a fifth more front entries, which then
  /// fit in place instead of mapping a new multi-gigabyte block while the
  /// solve waits).
  void AllocGrowable(size_t count) {
    if (count <= count_ && ptr_ != nullptr) {
      return;
    }
    Free();
    const size_t want = std::max<size_t>(1, count + count / 4);
    ptr_ = static_cast<T*>(CachedDeviceAlloc(want * sizeof(T), &bytes_, &device_));
    count_ = bytes_ / sizeof(T);
  }
  template <typename A>
  void Upload(const std::vector<T, A>& v, cudaStream_t s) {
    Alloc(v.size());
    if (!v.empty()) {
      UploadAsync(ptr_, v.data(), v.size() * sizeof(T), s);
    }
  }
  /// Holds src[0, count) afterwards, of which [0, keep) is on the device
  /// already: a buffer that has to grow copies that prefix over (with a
  /// quarter of headroom), then src[keep, count) is uploaded.
  void UploadKeep(const T* src, size_t count, size_t keep, cudaStream_t s) {
    keep = std::min(keep, count);
    if (ptr_ == nullptr) {
      keep = 0;
    }
    if (count > count_ || ptr_ == nullptr) {
      size_t got = 0;
      int dev = 0;
      const size_t want = count + count / 4;
      T* fresh = static_cast<T*>(CachedDeviceAlloc(std::max<size_t>(1, want) * sizeof(T), &got, &dev));
      if (keep > 0) {
        CudaCheck(cudaMemcpyAsync(fresh, ptr_, keep * sizeof(T), cudaMemcpyDeviceToDevice, s), "keep");
        // the old block goes back to the cache only after the copy read it
        CudaCheck(cudaStreamSynchronize(s), "keep");
      }
      Free();
      ptr_ = fresh;
      bytes_ = got;
      device_ = dev;
      count_ = got / sizeof(T);
    }
    if (count > keep) {
      UploadAsync(ptr_ + keep, src + keep, (count - keep) * sizeof(T), s);
    }
  }
  T* get() const { return ptr_; }
  [[nodiscard]] size_t size() const { return count_; }

 private:
  T* ptr_{nullptr};
  size_t count_{0};
  size_t bytes_{0};
  int device_{0};  // the device the block was allocated on
};

/// Device task lists of a symbolic analysis plus the launch parameters of
/// the factorization and solve kernels.
struct FactorPlan {
  const int32_t* small_tasks{nullptr};
  const int32_t* ea_tasks{nullptr};
  const int32_t* ea_child{nullptr};
  const int32_t* panel_tasks{nullptr};
  const int32_t* update_tasks{nullptr};
  const int32_t* level_sn{nullptr};
  double* dvec{nullptr};
  int max_front{1};
  /// Counter and flags of the one-launch solve (SolveSyncWords words), its
  /// task list and scratch (Symbolic::solve_tasks); the solve runs level by
  /// level when these or inv are null.
  uint32_t* solve_sync{nullptr};
  const int32_t* solve_tasks{nullptr};
  int num_solve_tasks{0};
  const int32_t* solve_parts{nullptr};
  const int64_t* zpart_off{nullptr};
  double* ys{nullptr};
  double* zpart{nullptr};
  /// (sn, panel) pairs of the diagonal blocks and their inverses
  /// (kInvBlockDoubles each), written after every factorization.
  const int32_t* inv_tasks{nullptr};
  int num_inv{0};
  double* inv{nullptr};
  /// Tensor-core Schur complements of the mixed solve's wide FP32 fronts:
  /// the packed operands' tensor map (null: every Schur update on the SIMT
  /// tiles), the task lists and what the kernels read.
  const CUtensorMap* tc_map{nullptr};
  const int32_t* pack_tasks{nullptr};
  const int32_t* tc_tasks{nullptr};
  TcArgs tc{};
  /// Whether any front may be factored in FP32 (a mixed instance): their
  /// Schur tiles take KUpdate, the FP64 ones KSchur.
  bool fp32_fronts{false};
  /// Tiled dense roots: task quads (Symbolic::dense_tasks), the sync words
  /// (a claim counter per level, the abort flag, then the tile counters;
  /// zeroed at the start of every factorization) and the inverse workspace.
  const int32_t* dense_tasks{nullptr};
  int32_t* dense_sync{nullptr};
  double* dense_inv{nullptr};
  /// Test hook of the one-launch solve: a supernode whose forward flag is
  /// never published (-1: none) and the polls a wait may take (0: the
  /// default of about a second).
  int solve_withhold{-1};
  uint32_t solve_wait_polls{0};
  /// Per-kernel device time of the launches (null: not timed).
  KernelTimer* timer{nullptr};
};

/// Words of the tiled dense roots' sync area: a claim counter per level,
/// the abort flag, the tile counters.
inline size_t DenseSyncWords(const Symbolic& S) {
  return static_cast<size_t>(S.num_levels) + 1 + static_cast<size_t>(S.dense_cnt_words);
}

/// Doubles per inverted 32 x 32 diagonal block (the inverse and its
/// transpose).
constexpr int kInvBlockDoubles = 2 * 32 * 32;

/// Words of the one-launch solve's counter and flags for num_sn supernodes
/// and num_inv diagonal blocks.
inline size_t SolveSyncWords(int num_sn, int num_inv) {
  return 2 + 4 * static_cast<size_t>(num_sn) + 2 * static_cast<size_t>(num_inv);
}

/// Level-scheduled multifrontal LDL^T of the assembled fronts.
/// Returns the number of kernels launched.
int LaunchFactorLevels(const Symbolic& S, const DeviceView& V, const FactorPlan& P, cudaStream_t stream);
/// Forward sweep, diagonal, backward sweep: V.step = A^-1 V.rhs (natural order).
int LaunchSolveLevels(const Symbolic& S, const DeviceView& V, const FactorPlan& P, cudaStream_t stream);
/// Raises the dynamic shared memory limit of the solve kernels.
void ConfigureSolveKernels(int max_front);

/// Pinned host buffer.
template <typename T>
class HostBuf {
 public:
  HostBuf() = default;
  HostBuf(const HostBuf&) = delete;
  HostBuf& operator=(const HostBuf&) = delete;
  ~HostBuf() {
    if (ptr_ != nullptr) {
      CachedHostFree(ptr_, bytes_);
    }
  }
  void Alloc(size_t count) {
    if (count <= count_ && ptr_ != nullptr) {
      return;
    }
    if (ptr_ != nullptr) {
      CachedHostFree(ptr_, bytes_);
      ptr_ = nullptr;
    }
    ptr_ = static_cast<T*>(CachedHostAlloc(std::max<size_t>(1, count) * sizeof(T), &bytes_));
    count_ = bytes_ / sizeof(T);
  }
  T* get() const { return ptr_; }
  T& operator[](size_t i) const { return ptr_[i]; }

 private:
  T* ptr_{nullptr};
  size_t count_{0};
  size_t bytes_{0};
};

struct IterTimes {
  double assemble{0};
  double normal{0};
  double factor{0};
  double solve{0};
  double update{0};
  int iterations{0};
  double span{0};        // device time from the first iteration's start to the last one's end
  int64_t launches{0};   // kernels launched by the iterations
  int reanalyses{0};     // symbolic re-analyses (a state left its pattern)
  double reanalysis_host{0};  // host seconds in re-analyses (analysis, upload)
  double capture_host{0};     // host seconds capturing and instantiating graphs
};

class Engine {
 public:
  explicit Engine(std::vector<HostProblem> problems);
  /// One problem with its symbolic analysis done already (AnalyzeInstance
  /// of a problem with the same columns, frames and point rows; the
  /// iterations re-analyse if the state leaves its pattern).
  Engine(HostProblem problem, SymPiece piece);
  /// Several problems with their analyses done already (one piece per
  /// problem, as AnalyzeInstance returns them).
  Engine(std::vector<HostProblem> problems, std::vector<SymPiece> pieces);
  /// Replaces this engine's single problem by `next` on the same grid with
  /// the same active columns, whose first `keep_rows` point rows are the
  /// current problem's (they stay on the device; the rest is uploaded). The
  /// state becomes next's. piece: its analysis, or null to analyse here.
  void Replace(HostProblem next, SymPiece* piece, int64_t keep_rows);
  /// True when Replace accepts `next`.
  [[nodiscard]] bool CanReplace(const HostProblem& next) const;
  ~Engine();
  Engine(const Engine&) = delete;
  Engine& operator=(const Engine&) = delete;

  [[nodiscard]] int count() const { return static_cast<int>(host_.size()); }
  [[nodiscard]] const HostProblem& host(int i) const { return host_[static_cast<size_t>(i)]; }
  [[nodiscard]] int64_t DeviceBytes() const { return device_bytes_; }

  void GetState(int i, double* map_values, double* poses);
  void SetState(int i, const double* map_values, const double* poses);
  double Cost(int i);
  void ApplyStep(int i, const double* step);

  void Linearize(int i, double lambda, bool marquardt, bool compute_step);
  void LinearizationSizes(int64_t* sizes) const;
  void LinearizationGet(double* residuals, int32_t* point_cell, int32_t* j_outer, int32_t* j_inner,
                        double* j_values, int32_t* n_outer, int32_t* n_inner, double* n_values, double* rhs,
                        double* step) const;

  void Solve(const std::vector<sdfgpu_solver_options>& options, sdfgpu_solve_result* results,
             double* cost_history, int capacity);

  // Split LM driver (used by Solve and by the serving loop, which interleaves
  // the iterations of several engines on the device):
  /// Starts a solve: options per instance, initial cost (synchronous).
  void BeginSolve(const std::vector<sdfgpu_solver_options>& options);
  /// True when every instance has finished.
  [[nodiscard]] bool SolveDone() const;
  /// Enqueues one LM iteration of every running instance (asynchronous).
  void LaunchIteration();
  /// Waits for the iteration, re-runs it after a pattern re-analysis if a
  /// point left its pose's analysed cells, and applies the LM control logic.
  void FinishIteration();
  /// Copies results and cost histories (rows of `capacity`).
  void EndSolve(sdfgpu_solve_result* results, double* cost_history, int capacity);
  /// True once instance i's solve has ended (converged, failed or out of
  /// iterations); its result as EndSolve would report it.
  [[nodiscard]] bool InstanceDone(int i) const;
  [[nodiscard]] sdfgpu_solve_result InstanceResult(int i) const;
  [[nodiscard]] cudaStream_t stream() const { return stream_; }
  /// True when an instance's state left its pattern and the next
  /// LaunchIteration would re-analyse it first.
  [[nodiscard]] bool NeedsReanalysis() const { return !pending_.empty(); }
  /// Runs that re-analysis now (the serving loop does it off its own thread).
  void ReanalyzeNow() { ReanalyzePending(); }
  /// True when the iteration enqueued by LaunchIteration has finished on the
  /// device (FinishIteration will not wait).
  [[nodiscard]] bool IterationReady() const;
  /// Times the factorization of the current state's normal matrix under each
  /// candidate schedule and keeps the fastest (also across re-analyses).
  /// When the last solve was mixed, it then times that solve's factor and
  /// refined solve with and without the tensor-core Schur complements and
  /// keeps the faster (Schedule::tc_min_rows). Returns the fastest FP64
  /// factorization time in ms; trials receives every candidate's time.
  double Autotune(std::vector<std::pair<Schedule, double>>* trials);
  /// Installs a factorization schedule (checked against the ranges the
  /// kernels support) for the later solves, also across re-analyses.
  void SetSchedule(const Schedule& sched);
  [[nodiscard]] const Schedule& schedule() const { return sched_; }
  /// Mixed factor + solve time of the last autotune with (true) or without
  /// the tensor-core Schur complements, ms (0: not timed).
  [[nodiscard]] double tc_trial_ms(bool with) const { return tc_trial_ms_[with ? 0 : 1]; }
  [[nodiscard]] const IterTimes& times() const { return times_; }
  [[nodiscard]] int64_t factor_flops() const { return sym_.total_flops; }
  [[nodiscard]] const Symbolic& symbolic() const { return sym_; }
  /// Test hook: the next solves' one-launch triangular solve never
  /// publishes supernode `withhold`'s forward flag (-1: normal) and a wait
  /// takes at most `wait_polls` polls (0: the default).
  void SetSolveFault(int withhold, uint32_t wait_polls);
  /// Times the launches of the kernel classes in `mask` (KernelTimer) from
  /// the next iteration on, with zeroed totals; 0 stops timing.
  void SetKernelTiming(uint32_t mask);
  [[nodiscard]] const KernelTimer& kernel_timer() const { return timer_; }

 private:
  void Init(std::vector<SymPiece>* pieces);
  /// The analysis of host_ (or the given pieces' structure, one per
  /// instance) while the problem uploads (keep_rows of its point rows are on
  /// the device).
  void AnalyzeAndUpload(std::vector<SymPiece>* pieces, int64_t keep_rows);
  void BuildLayout();
  void UploadProblem(int64_t keep_rows = 0);
  /// Symbolic analysis of every instance at its current state (host only).
  void AnalyzeHost();
  /// Global structure of the current pieces (a single piece is taken over).
  Symbolic GlobalStructure();
  void UploadSymbolic();
  void UploadSchedule();
  void InstallSchedule();          // sched_ into the structure, task lists and view
  double TimeMixedFactorSolve();   // fastest of three mixed factor + solve runs, ms
  /// The one-launch solve's task list and its scratch.
  void UploadSolveTasks(cudaStream_t s);
  /// Per-instance precision of the coming solve (1: mixed) and refinement
  /// rounds; re-uploads flags and drops the graphs when they change.
  // refine_tol: per instance (missing entries: kDefaultRefineTol)
  void SetMode(const std::vector<int32_t>& mixed, int refine_steps, const std::vector<double>& refine_tol = {});
  void AllocMixed();
  void RefreshView();
  void SetActive(const std::vector<int32_t>& active);
  void SetLambda(const std::vector<double>& lam, const std::vector<int32_t>& marquardt);
  void ClearStatus();
  std::vector<int32_t> DownloadStatus();
  void LaunchRows();
  int64_t ZeroTaskCount() const;  // front-clearing (and conversion) tasks of this iteration
  void LaunchNormal();
  void LaunchFactor();
  void LaunchSolve();
  void LaunchStepAndCost(bool backup);
  /// ApplyStep of the running instances (KApplyStep, provisional angles on
  /// the device) and the copy of the moved frames' angles to the host.
  void LaunchApplyStep();
  /// With the stream drained: the exact angles of the last step's moved
  /// frames (the platform libm's WrapAngle, cos and sin), uploaded and
  /// committed, except for the instances `revert` marks.
  void CommitAngles(const std::vector<int32_t>* revert);
  /// (cos, sin) of frames [frame_off, frame_off + frames) from host poses.
  void UploadPoseTrig(const double* poses, int frame_off, int frames);
  void LaunchCost(std::vector<double>& cost);
  /// Re-analyses the listed instances at the current state (with a wider
  /// coupling margin) and rebuilds the global structure.
  void Reanalyze(const std::vector<int>& which);
  /// Re-analyses the instances whose state left their pattern (pending_).
  void ReanalyzePending();
  /// A pattern re-centred ahead of time: an instance whose accepted state
  /// brought a point within a few cells of its pattern's edge is analysed
  /// again (same margin) on a host thread from that state, while the
  /// iterations go on with the current pattern, and the analysis replaces
  /// its pattern a fixed number of its own iterations later (so that no
  /// result depends on host timing or on the other instances of a batch).
  struct Speculation {
    int inst{0};
    int margin{0};
    std::vector<double> poses;  // the state analysed
    SymPiece piece;
    // a single-instance engine's global structure, built on the same thread
    // under `sched` (the piece is consumed)
    Symbolic structure;
    Schedule sched;
    bool has_structure{false};
    std::future<void> done;
    int64_t adopt_at{0};  // iters_[inst] at which the analysis is installed
  };
  /// At the start of an iteration: drops the speculations of instances
  /// that are about to be re-analysed synchronously, installs the ones that
  /// are due, starts one for each instance near its pattern's edge.
  void StepSpeculations();
  void StartSpeculation(int i, const std::vector<double>& poses);
  /// Waits for the speculations of the instances in `which` (all of them
  /// when null) and discards them.
  void DropSpeculations(const std::vector<int>* which);
  void EnqueueIteration();
  int AssembleWithPattern();
  [[nodiscard]] FactorPlan Plan();
  void SegmentSum(const double* x, const int64_t* seg_begin, const int64_t* seg_end, int segments, double* out);

  std::vector<HostProblem> host_;
  std::vector<InstanceLayout> layout_;
  std::vector<SymPiece> pieces_;   // per-instance analyses (local numbering)
  std::vector<int> margin_;        // per instance: coupling margin of its piece
  std::vector<int> pending_;       // instances whose current state overflows their pattern
  std::vector<std::unique_ptr<Speculation>> specs_;  // background re-analyses in flight
  std::vector<int> near_;          // instances whose last accepted state nears their pattern's edge
  std::vector<int64_t> iters_;     // per instance: iterations launched with it active, over the engine's life
  std::vector<int64_t> analysed_at_;  // per instance: iters_ at its last analysis
  Schedule sched_;                 // factorization schedule (autotuned or default)
  double tc_trial_ms_[2]{0.0, 0.0};
  Symbolic sym_;
  cudaStream_t stream_{nullptr};
  cudaEvent_t ev_[6]{};
  cudaEvent_t span_[2]{};
  bool span_started_{false};
  int device_{0};
  int64_t device_bytes_{0};
  DeviceView V_{};
  IterTimes times_;
  int64_t total_cells_{0};
  int64_t pass_begin_[5]{};   // colour class p's cells: pass_cells_[pass_begin_[p], pass_begin_[p + 1])
  int64_t total_points_{0};
  int64_t total_eik_{0};
  int64_t total_odom_{0};
  int64_t total_nodes_{0};
  int total_frames_{0};
  int n_{0};
  int max_front_{0};

  // problem buffers
  DevBuf<InstDev> inst_;
  DevBuf<int32_t> node_col_, col_node_, col_inst_, frame_inst_, frame_col_;
  DevBuf<int32_t> pt_frame_;
  DevBuf<double2> pt_xy_;
  DevBuf<double> pt_exp_, pt_sw_;
  DevBuf<int32_t> eik_node_, eik_index_;
  DevBuf<double2> eik_n_;
  DevBuf<double> eik_sw_;
  DevBuf<int32_t> odom_fi_, odom_fj_;
  DevBuf<double> odom_meas_, odom_sw_;
  DevBuf<int64_t> frame_rows_ptr_, frame_odom_ptr_, pair_ptr_;
  DevBuf<int32_t> frame_rows_, frame_odom_, pair_f_, pair_g_, pair_spec_;
  int num_pairs_{0};
  bool frame_rows_identity_{false};  // frame_rows_ holds 0, 1, 2, ... (rows ordered by frame)
  // state and per-iteration buffers
  DevBuf<double> map_, poses_, map_backup_, poses_backup_;
  DevBuf<double2> pose_cs_, pose_cs_backup_;
  DevBuf<double> theta_pre_, theta_out_;
  DevBuf<int32_t> theta_upd_;
  std::vector<int32_t> frame_inst_host_;  // global frame -> instance
  HostBuf<double> h_theta_pre_, h_theta_out_;
  HostBuf<int32_t> h_theta_upd_;
  DevBuf<double> pt_rec_, eik_rec_, odom_rec_;
  DevBuf<int64_t> pt_poff_;
  DevBuf<int32_t> pt_cell_, cell_start_, sort_keys_a_, sort_vals_a_, sort_keys_b_, sort_vals_b_, sort_hist_;
  DevBuf<int64_t> pass_cells_;
  DevBuf<double> rhs_, step_, xs_, lam_, dvec_;
  DevBuf<int32_t> marq_, status_, active_, revert_;
  DevBuf<double> terms_, sq_terms_, pred_terms_, seg_out_, seg_partial_;
  DevBuf<int64_t> seg_begin_, seg_end_, step_seg_begin_, step_seg_end_;
  // symbolic buffers
  DevBuf<int32_t> perm_, pinv_, sn_rows_, sn_rel_, child_list_, level_sn_;
  DevBuf<SupernodeRec> sn_;
  DevBuf<int64_t> mm_off_, mp_ptr_, mp_off_;
  DevBuf<int32_t> mp_frame_;
  DevBuf<uint32_t> allow_bits_;
  DevBuf<int32_t> ea_tasks_, ea_child_, panel_tasks_, update_tasks_, small_tasks_;
  DevBuf<double> fronts_, upd_;
  DevBuf<int32_t> dense_tasks_, dense_sync_;  // tiled dense roots
  DevBuf<int32_t> zero_tasks_;                // lower-triangle clearing of the fronts
  DevBuf<double> dense_inv_;
  DevBuf<uint32_t> solve_sync_;  // counter and flags of the one-launch solve
  DevBuf<int32_t> solve_tasks_, solve_parts_;
  DevBuf<int64_t> zpart_off_;
  DevBuf<double> ys_, zpart_;
  DevBuf<int32_t> inv_tasks_;     // diagonal blocks of L and their inverses
  DevBuf<double> inv_;
  // mixed precision: assembled FP64 normal matrix, FP32 work fronts and the
  // refinement vectors (the conversion runs over zero_tasks_)
  DevBuf<double> amat_;
  DevBuf<float> fronts32_;
  DevBuf<double> res_, ax_, corr_;
  DevBuf<int32_t> refine_done_, refine_left_;
  DevBuf<unsigned long long> refine_max_;
  // tensor-core Schur update of the wide FP32 fronts: packed operands of one
  // level and their tensor map (re-encoded when the buffer moves)
  DevBuf<int32_t> pack_tasks_, tc_tasks_;
  DevBuf<float> pack_;
  CUtensorMap tc_map_{};
  const float* tc_map_base_{nullptr};
  int64_t tc_map_rows_{0};
  int solve_withhold_{-1};
  uint32_t solve_wait_polls_{0};
  KernelTimer timer_;
  bool timing_phase_{false};  // EnqueuePhase is inside the factor or solve phase
  DevBuf<int64_t> fmp_ptr_, fmp_off_;
  DevBuf<int32_t> fmp_col_;
  std::vector<int32_t> mixed_;
  int refine_steps_{0};
  std::vector<double> refine_tol_;
  bool any_mixed_{false};
  std::vector<InstDev> inst_host_;
  int32_t* cell_rows_ptr_{nullptr};
  HostBuf<double> h_seg_;      // 5 per instance: cost parts x3, |delta|^2, prediction
  HostBuf<int32_t> h_status_;
  HostBuf<int32_t> h_active_;  // per-iteration parameters read by the graph's copies
  HostBuf<int32_t> h_marq_;
  HostBuf<double> h_lam_;
  // CUDA graphs of one LM iteration, one per phase (fixed per symbolic
  // analysis); the phase events are recorded between the graph launches
  cudaGraphExec_t graph_exec_[5]{};
  bool graph_backup_{false};
  bool use_graph_{true};
  int64_t graph_launches_{0};
  void EnqueuePhase(int phase);
  void DropGraph();

  // LM control state of the current solve (lm_solver.cpp:201-434)
  struct LmInst {
    sdfgpu_solver_options opt{};
    double lam{1.0};
    double prev{0.0};
    double nu{2.0};
    int32_t active{0};
    int32_t revert{0};
    sdfgpu_solve_result res{};
    std::vector<double> hist;
  };
  std::vector<LmInst> lm_;
  int iter_{0};
  bool need_backup_{false};
  std::chrono::steady_clock::time_point t_start_;

  // linearization snapshot (host)
  struct Lin {
    int instance{-1};
    std::vector<double> residuals;
    std::vector<int32_t> point_cell;
    std::vector<int32_t> j_outer, j_inner, n_outer, n_inner;
    std::vector<double> j_values, n_values, rhs, step;
  } lin_;
};

}  // namespace sdfgpu
