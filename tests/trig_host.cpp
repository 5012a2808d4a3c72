// Host build of the library's correctly rounded sin/cos (the same header the
// CUDA kernels include) for tests/test_trig.py.
#include "trig.cuh"

extern "C" void sincos_rn_host(const double* x, int n, double* s, double* c) {
  for (int i = 0; i < n; ++i) {
    sdfgpu::SinCosRn(x[i], s + i, c + i);
  }
}
