// Host build of the distance epilogue's logarithm (csharp_b200/csrc/swg_log.cuh) for the CPU
// tests: the same source the device code runs.
#include "../csharp_b200/csrc/swg_log.cuh"

extern "C" void cr_log_many(const double* x, double* y, long n) {
  for (long k = 0; k < n; k++) y[k] = swg::cr_log(x[k]);
}
