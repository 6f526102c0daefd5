// FP64 fused multiply-add throughput of the device, for the FP64 roofline.
//
// The stage kernels are bound by FP64 issue and latency rather than by HBM
// bandwidth, so their roofline is the FP64 pipe's peak. This kernel measures
// that peak on the GPU at hand: every thread runs eight independent DFMA
// chains (enough to cover the pipe's latency at full occupancy), and the
// caller times the launch with CUDA events. FLOPs per launch =
// 2 x 8 x iters x ctas x 256.
#include <cuda_runtime.h>

#include "pangu_b200.h"

namespace {

constexpr int kPeakThreads = 256;
constexpr int kPeakChains = 8;

__global__ void __launch_bounds__(kPeakThreads) k_dfma_peak(int iters, double a, double b,
                                                            double *sink) {
  double x[kPeakChains];
#pragma unroll
  for (int c = 0; c < kPeakChains; ++c) x[c] = 1e-3 * threadIdx.x + c;
#pragma unroll 4
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int c = 0; c < kPeakChains; ++c) x[c] = __fma_rn(x[c], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < kPeakChains; ++c) s += x[c];
  // never true for the arguments the caller passes; keeps the chains live
  if (s == -1.0) sink[blockIdx.x] = s;
}

}  // namespace

extern "C" int pangu_fp64_peak(int ctas, int iters, double *sink, void *stream) {
  if (ctas < 1 || iters < 1 || !sink) return PANGU_EINVAL;
  k_dfma_peak<<<ctas, kPeakThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      iters, 0.999999999, 1e-9, sink);
  return cudaGetLastError() == cudaSuccess ? PANGU_OK : PANGU_ECUDA;
}

extern "C" double pangu_fp64_peak_flops(int ctas, int iters) {
  return 2.0 * kPeakChains * (double)iters * (double)ctas * kPeakThreads;
}
