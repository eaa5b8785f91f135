// k_peak.cu -- arithmetic-pipe throughput probes, the FP64 / FP32 denominators of the operator roofline.
//
// The fused operator kernels are bounded by min(HBM bandwidth, FP64 or FP32 pipe rate).  The HBM peak is a measured
// copy bandwidth; this file gives the pipe side the same footing: a kernel of independent fused multiply-add chains
// (eight per thread, enough to cover the pipe latency), sized to a few milliseconds, whose FMA count is returned so the
// caller can divide by its own CUDA-event time.  Nothing here is on the operator path.
#include <cuda_runtime.h>
#include <stdint.h>

#include "honee_b200.h"

namespace {

constexpr int kChains = 8;
constexpr int kThreads = 256;

template <typename T>
__global__ void __launch_bounds__(kThreads) k_fma_probe(T *sink, int iters, T y, T z) {
  T x[kChains];
#pragma unroll
  for (int c = 0; c < kChains; c++) x[c] = T(threadIdx.x + c);
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int c = 0; c < kChains; c++) x[c] = fma(x[c], y, z);
  }
  T s = 0;
#pragma unroll
  for (int c = 0; c < kChains; c++) s += x[c];
  // never true for the inputs the host passes (|x| stays below 2 for y < 1, z < 1e-2), but the compiler cannot know
  if (s == T(-12345.5)) sink[blockIdx.x * kThreads + threadIdx.x] = s;
}

}  // namespace

extern "C" int hb_fma_peak_probe(int fp64, int iters, void *d_sink, int64_t sink_elems, int64_t *fma_per_launch, void *stream) {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return HB_ERROR_CUDA;
  if (iters <= 0 || !d_sink || sms <= 0) return HB_ERROR_INVALID;
  const int blocks = 8 * sms;
  if (sink_elems < (int64_t)blocks * kThreads) return HB_ERROR_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  if (fp64) k_fma_probe<double><<<blocks, kThreads, 0, s>>>((double *)d_sink, iters, 0.999, 1e-3);
  else k_fma_probe<float><<<blocks, kThreads, 0, s>>>((float *)d_sink, iters, 0.999f, 1e-3f);
  if (fma_per_launch) *fma_per_launch = (int64_t)blocks * kThreads * kChains * iters;
  return cudaGetLastError() == cudaSuccess ? HB_SUCCESS : HB_ERROR_CUDA;
}
