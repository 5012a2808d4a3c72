// Device time per kernel class of the factorization and the solves, from
// CUDA events recorded on the launching stream around each timed launch
// (inside a captured iteration they become event nodes of its graph).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <utility>
#include <vector>

namespace sdfgpu {

class KernelTimer {
 public:
  enum Class {
    kExtendAdd,
    kFactorFront,
    kPanel,
    kUpdatePanel,   // KUpdate: outer-block and panel updates of the later pivot columns
    kUpdateSchur,   // KSchur / KSchurF32: the fronts' Schur complements
    kPackSchur,
    kSchurTc,
    kInvertDiagonal,
    kSolveTree,
    kDenseRoot,     // tiled LDL^T of the dense pose roots
    kClasses
  };
  static const char* Name(int c);

  KernelTimer() = default;
  KernelTimer(const KernelTimer&) = delete;
  KernelTimer& operator=(const KernelTimer&) = delete;
  ~KernelTimer();

  /// Classes to time (bit c for class c; 0 disables) and zero totals. The
  /// launches that follow record events; marks made under a previous mask
  /// are dropped.
  void SetMask(uint32_t mask);
  [[nodiscard]] bool On(int c) const { return ((mask_ >> c) & 1u) != 0; }
  /// Forgets the launches recorded so far (a fresh enqueue or capture of the
  /// timed phases follows).
  void NewSequence() { marks_.clear(); next_ = 0; }
  /// Records the start of a launch of class c on s doing `work` units of
  /// algorithmic work (flops, or bytes for the memory-bound classes);
  /// returns its mark.
  int Begin(int c, cudaStream_t s, double work);
  void End(int mark, cudaStream_t s);
  /// Adds the elapsed time of every recorded launch (the stream has drained).
  void Accumulate();
  [[nodiscard]] double Ms(int c) const { return ms_[c]; }
  [[nodiscard]] int64_t Launches(int c) const { return count_[c]; }
  [[nodiscard]] double Work(int c) const { return work_[c]; }
  /// True for the classes whose work is counted in bytes (else flops).
  static bool ByteBound(int c);

 private:
  uint32_t mask_{0};
  std::vector<cudaEvent_t> pool_;
  struct Mark {
    int cls;
    int first;  // first of its two events
    double work;
  };
  std::vector<Mark> marks_;
  int next_{0};
  double ms_[kClasses]{};
  int64_t count_[kClasses]{};
  double work_[kClasses]{};
};

/// Brackets one launch when its class is timed (timer may be null).
class TimedLaunch {
 public:
  /// work: a function returning the launch's algorithmic work, called only
  /// when the class is timed.
  template <typename Work>
  TimedLaunch(KernelTimer* t, int c, cudaStream_t s, Work work) : t_(t), s_(s) {
    if (t_ != nullptr && t_->On(c)) {
      mark_ = t_->Begin(c, s_, static_cast<double>(work()));
    }
  }
  ~TimedLaunch() {
    if (mark_ >= 0) {
      t_->End(mark_, s_);
    }
  }
  TimedLaunch(const TimedLaunch&) = delete;
  TimedLaunch& operator=(const TimedLaunch&) = delete;

 private:
  KernelTimer* t_;
  cudaStream_t s_;
  int mark_{-1};
};

}  // namespace sdfgpu
