// KernelTimer (kernel_timer.h).
#include "kernel_timer.h"

#include "engine.h"

namespace sdfgpu {

const char* KernelTimer::Name(int c) {
  static const char* const kNames[kClasses] = {"KExtendAdd",     "KFactorFront", "KPanel",
                                               "KUpdate",        "KSchur",         "KPackSchur",
                                               "KSchurTc",       "KInvertDiagonal", "KSolveTree",
                                               "KDenseRoot"};
  return c >= 0 && c < kClasses ? kNames[c] : "";
}

bool KernelTimer::ByteBound(int c) {
  return c == kExtendAdd || c == kPackSchur || c == kInvertDiagonal || c == kSolveTree;
}

KernelTimer::~KernelTimer() {
  for (cudaEvent_t e : pool_) {
    cudaEventDestroy(e);
  }
}

void KernelTimer::SetMask(uint32_t mask) {
  mask_ = mask;
  NewSequence();
  for (int c = 0; c < kClasses; ++c) {
    ms_[c] = 0.0;
    count_[c] = 0;
    work_[c] = 0.0;
  }
}

namespace {

/// Records e on s; inside a stream capture as an event record node of the
/// graph (an event recorded there without cudaEventRecordExternal would
/// only order the capture's streams and never be recorded).
void Record(cudaEvent_t e, cudaStream_t s) {
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  CudaCheck(cudaStreamIsCapturing(s, &st), "capture status");
  if (st == cudaStreamCaptureStatusActive) {
    CudaCheck(cudaEventRecordWithFlags(e, s, cudaEventRecordExternal), "timer event");
  } else {
    CudaCheck(cudaEventRecord(e, s), "timer event");
  }
}

}  // namespace

int KernelTimer::Begin(int c, cudaStream_t s, double work) {
  while (static_cast<int>(pool_.size()) < next_ + 2) {
    cudaEvent_t e = nullptr;
    CudaCheck(cudaEventCreate(&e), "timer event");
    pool_.push_back(e);
  }
  const int mark = next_;
  next_ += 2;
  marks_.push_back(Mark{c, mark, work});
  Record(pool_[static_cast<size_t>(mark)], s);
  return mark;
}

void KernelTimer::End(int mark, cudaStream_t s) { Record(pool_[static_cast<size_t>(mark) + 1], s); }

void KernelTimer::Accumulate() {
  for (const Mark& m : marks_) {
    float ms = 0.0f;
    CudaCheck(cudaEventElapsedTime(&ms, pool_[static_cast<size_t>(m.first)], pool_[static_cast<size_t>(m.first) + 1]),
              "timer elapsed");
    ms_[m.cls] += ms;
    ++count_[m.cls];
    work_[m.cls] += m.work;
  }
}

}  // namespace sdfgpu
