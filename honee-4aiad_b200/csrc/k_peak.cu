// k_peak.cu -- arithmetic-pipe throughput probes, the FP64 / FP32 denominators of the operator roofline, and the A/B
// probe of the basis-contraction mechanism (shared-memory fibre passes against warp shuffles).
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

// ---------------------------------------------------------------------------------------------------------------------
// Contraction mechanism A/B: the in-plane collocated derivatives of the operator kernels (five FP64 components on the
// Q = 5 point grid of one element), repeated `reps` times as u <- D_x u + D_y u per component, by
//   variant 0: fibre passes over shared memory, the mechanism of the operator kernels: 128 threads per element, one
//              thread per 1D fibre (two per round), basis entries as compile-time operands; then one thread per point
//              combines the two derivatives, as the point-wise phase reads them;
//   variant 1: warp shuffles: 160 threads per element, one z-plane of 25 points per warp (lanes 25-31 idle), each lane
//              holding its point's five values in registers and fetching the fibre's other values with __shfl_sync.
// Both form every output as the same FMA chain in the same order, so their results are bit-identical.

constexpr int kCQ = 5, kCQ2 = kCQ * kCQ, kCQ3 = kCQ2 * kCQ, kCNC = 5;

struct Colo5 {
  double D[kCQ2];
};

__global__ void __launch_bounds__(128) k_contract_shared(const Colo5 b, const double *__restrict__ u, double *__restrict__ out, int num_elem,
                                                        int reps) {
  __shared__ double sU[kCNC * kCQ3], sG[2 * kCNC * kCQ3];
  constexpr int NT = 128, NXY = 2 * kCNC * kCQ2;
  for (int e = blockIdx.x; e < num_elem; e += gridDim.x) {
    for (int t = threadIdx.x; t < kCNC * kCQ3; t += NT) sU[t] = u[(size_t)e * kCNC * kCQ3 + t];
    __syncthreads();
    for (int r = 0; r < reps; r++) {
#pragma unroll 1
      for (int f0 = threadIdx.x; f0 < NXY; f0 += 2 * NT) {
        const bool h1 = f0 + NT < NXY;
        const int f1 = h1 ? f0 + NT : f0;
        const int dir0 = f0 / (kCNC * kCQ2), r0 = f0 % (kCNC * kCQ2), c0 = r0 / kCQ2, rem0 = r0 % kCQ2;
        const int dir1 = f1 / (kCNC * kCQ2), r1 = f1 % (kCNC * kCQ2), c1 = r1 / kCQ2, rem1 = r1 % kCQ2;
        const int base0 = dir0 == 0 ? rem0 * kCQ : (rem0 / kCQ) * kCQ2 + rem0 % kCQ, st0 = dir0 == 0 ? 1 : kCQ;
        const int base1 = dir1 == 0 ? rem1 * kCQ : (rem1 / kCQ) * kCQ2 + rem1 % kCQ, st1 = dir1 == 0 ? 1 : kCQ;
        const double *src0 = sU + c0 * kCQ3 + base0, *src1 = sU + c1 * kCQ3 + base1;
        double *dst0 = sG + (dir0 * kCNC + c0) * kCQ3 + base0, *dst1 = sG + (dir1 * kCNC + c1) * kCQ3 + base1;
        double v0[kCQ], v1[kCQ];
#pragma unroll
        for (int l = 0; l < kCQ; l++) {
          v0[l] = src0[l * st0];
          v1[l] = src1[l * st1];
        }
#pragma unroll
        for (int k = 0; k < kCQ; k++) {
          double d0 = 0, d1 = 0;
#pragma unroll
          for (int l = 0; l < kCQ; l++) {
            d0 = fma(b.D[k * kCQ + l], v0[l], d0);
            d1 = fma(b.D[k * kCQ + l], v1[l], d1);
          }
          dst0[k * st0] = d0;
          if (h1) dst1[k * st1] = d1;
        }
      }
      __syncthreads();
      if (threadIdx.x < kCQ3) {
#pragma unroll
        for (int c = 0; c < kCNC; c++) sU[c * kCQ3 + threadIdx.x] = sG[c * kCQ3 + threadIdx.x] + sG[(kCNC + c) * kCQ3 + threadIdx.x];
      }
      __syncthreads();
    }
    for (int t = threadIdx.x; t < kCNC * kCQ3; t += NT) out[(size_t)e * kCNC * kCQ3 + t] = sU[t];
    __syncthreads();
  }
}

__global__ void __launch_bounds__(160) k_contract_shuffle(const Colo5 b, const double *__restrict__ u, double *__restrict__ out, int num_elem,
                                                         int reps) {
  const int lane = threadIdx.x & 31, k = threadIdx.x >> 5, i = lane % kCQ, j = lane / kCQ;
  const bool act = lane < kCQ2;
  double Di[kCQ], Dj[kCQ];
#pragma unroll
  for (int m = 0; m < kCQ; m++) {
    Di[m] = act ? b.D[i * kCQ + m] : 0.0;
    Dj[m] = act ? b.D[j * kCQ + m] : 0.0;
  }
  for (int e = blockIdx.x; e < num_elem; e += gridDim.x) {
    double v[kCNC];
#pragma unroll
    for (int c = 0; c < kCNC; c++) v[c] = act ? u[(size_t)e * kCNC * kCQ3 + c * kCQ3 + k * kCQ2 + lane] : 0.0;
    for (int r = 0; r < reps; r++) {
#pragma unroll
      for (int c = 0; c < kCNC; c++) {
        double dx = 0, dy = 0;
#pragma unroll
        for (int m = 0; m < kCQ; m++) {
          dx = fma(Di[m], __shfl_sync(0xffffffffu, v[c], j * kCQ + m), dx);
          dy = fma(Dj[m], __shfl_sync(0xffffffffu, v[c], m * kCQ + i), dy);
        }
        v[c] = dx + dy;
      }
    }
    if (act) {
#pragma unroll
      for (int c = 0; c < kCNC; c++) out[(size_t)e * kCNC * kCQ3 + c * kCQ3 + k * kCQ2 + lane] = v[c];
    }
  }
}

}  // namespace

/* Contraction mechanism A/B (no reference counterpart): `reps` rounds of u <- D_x u + D_y u on num_elem elements of five
 * FP64 components at the Q = 5 points ([num_elem][5][125], x fastest), by shared-memory fibre passes (variant 0) or warp
 * shuffles (variant 1); D: the 5 x 5 collocated derivative matrix, row-major.  ctas_per_sm = 0 runs each variant at its
 * own occupancy limit, else that many CTAs per SM (persistent grid).  *fma_per_launch receives the FMA count. */
extern "C" int hb_contraction_probe(int variant, const double *D, const double *d_u, double *d_out, int num_elem, int reps, int ctas_per_sm,
                                    int64_t *fma_per_launch, void *stream) {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return HB_ERROR_CUDA;
  if ((variant != 0 && variant != 1) || !D || !d_u || !d_out || num_elem <= 0 || reps < 0 || ctas_per_sm < 0 || sms <= 0) return HB_ERROR_INVALID;
  Colo5 b;
  for (int t = 0; t < kCQ2; t++) b.D[t] = D[t];
  int occ = 0;
  if (variant == 0) {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_contract_shared, 128, 0) != cudaSuccess) return HB_ERROR_CUDA;
  } else if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_contract_shuffle, 160, 0) != cudaSuccess) return HB_ERROR_CUDA;
  if (occ <= 0) return HB_ERROR_CUDA;
  const int per_sm = ctas_per_sm ? (ctas_per_sm < occ ? ctas_per_sm : occ) : occ;
  const int blocks = per_sm * sms < num_elem ? per_sm * sms : num_elem;
  cudaStream_t s = (cudaStream_t)stream;
  if (variant == 0) k_contract_shared<<<blocks, 128, 0, s>>>(b, d_u, d_out, num_elem, reps);
  else k_contract_shuffle<<<blocks, 160, 0, s>>>(b, d_u, d_out, num_elem, reps);
  if (fma_per_launch) *fma_per_launch = (int64_t)num_elem * reps * 2 * kCNC * kCQ3 * kCQ;
  return cudaGetLastError() == cudaSuccess ? HB_SUCCESS : HB_ERROR_CUDA;
}

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
