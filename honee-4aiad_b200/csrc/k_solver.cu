// k_solver.cu -- device kernels of the implicit time loop: Krylov block operations (multi-dot, multi-axpy) in FP32 or FP64
// with FP64 accumulation, the BDF time-derivative update, and the total-kinetic-energy / CFL monitors.
//
// Monitors restate qfunctions/monitor_totalkineticenergy.h:8-39 (summed as src/monitor_totalkineticenergy.c:134-163) and
// qfunctions/monitor_cfl.h:9-46 with numerics.h:24-29 (min/max times dt, src/monitor_cfl.c:140-164).  Reductions are
// two-stage with fixed block order, so results are deterministic.
#include <cuda_runtime.h>

#include <atomic>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "honee_b200.h"
#include "newtonian_qf.cuh"

namespace {

constexpr int kBS = 256;
constexpr int kMaxK = HB_GMRES_MAX_BASIS;
constexpr int kRedBlocks = 512;

inline unsigned nblocks(int64_t n) {
  const int64_t b = (n + kBS - 1) / kBS;
  return (unsigned)(b > 148 * 32 ? 148 * 32 : (b < 1 ? 1 : b));
}

// h[i] = sum_e V[i][e] w[e], i < k; per-block partials [kRedBlocks][kMaxK]
template <typename T>
__global__ void __launch_bounds__(kBS) k_multidot(const T *__restrict__ V, int64_t ldv, int k, const T *__restrict__ w, int64_t n, double *partial) {
  __shared__ double sh[kMaxK][kBS / 32];
  double acc[kMaxK];
#pragma unroll
  for (int i = 0; i < kMaxK; i++) acc[i] = 0;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const double we = (double)w[e];
#pragma unroll
    for (int i = 0; i < kMaxK; i++)
      if (i < k) acc[i] += (double)V[i * ldv + e] * we;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < kMaxK; i++) {
    if (i >= k) break;
    double v = acc[i];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh[i][warp] = v;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < k; i += blockDim.x) {
    double s = 0;
    for (int wi = 0; wi < kBS / 32; wi++) s += sh[i][wi];
    partial[blockIdx.x * kMaxK + i] = s;
  }
}

__global__ void k_multidot_final(const double *partial, int nblk, int k, double *out) {
  const int i = blockIdx.x;  // one block per output
  __shared__ double sh[kBS];
  double s = 0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) s += partial[b * kMaxK + i];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) sh[threadIdx.x] += sh[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0 && i < k) out[i] = sh[0];
}

struct Coefs {
  double c[kMaxK];
};

// w[e] += sum_{i<k} c[i] V[i][e]
template <typename T, typename TW>
__global__ void __launch_bounds__(kBS) k_multiaxpy(TW *__restrict__ w, const T *__restrict__ V, int64_t ldv, int k, Coefs c, int64_t n) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    double s = 0;
#pragma unroll
    for (int i = 0; i < kMaxK; i++)
      if (i < k) s += c.c[i] * (double)V[i * ldv + e];
    w[e] = TW((double)w[e] + s);
  }
}

// ---------------------------------------------------------------------------------------------------------------------
// Vectorised forms of the two block operations, used when every basis row and w start on a 16-byte boundary: each
// thread moves 16 bytes per vector and step (2 doubles or 4 floats), and the basis size K is a template parameter, so
// the accumulators stay in registers and no predicated slots are issued.  These are pure streams over K + 1 (multi-dot)
// or K + 2 (multi-axpy) vectors and run at the HBM rate in either precision.

template <typename T>
__device__ __forceinline__ void ld16(const T *__restrict__ p, T (&x)[16 / sizeof(T)]) {
  if constexpr (sizeof(T) == 8) {
    const double2 v = __ldg(reinterpret_cast<const double2 *>(p));
    x[0] = v.x;
    x[1] = v.y;
  } else {
    const float4 v = __ldg(reinterpret_cast<const float4 *>(p));
    x[0] = v.x;
    x[1] = v.y;
    x[2] = v.z;
    x[3] = v.w;
  }
}

template <typename T>
__device__ __forceinline__ void st16(T *__restrict__ p, const T (&x)[16 / sizeof(T)]) {
  if constexpr (sizeof(T) == 8) *reinterpret_cast<double2 *>(p) = make_double2(x[0], x[1]);
  else *reinterpret_cast<float4 *>(p) = make_float4(x[0], x[1], x[2], x[3]);
}

// partial[block][i] = sum over this block's elements of V[i][e] w[e], i < K (FP64 accumulation)
template <typename T, int K>
__global__ void __launch_bounds__(kBS) k_multidot_vec(const T *__restrict__ V, int64_t ldv, const T *__restrict__ w, int64_t n, double *partial) {
  constexpr int VW = 16 / sizeof(T);
  __shared__ double sh[K][kBS / 32];
  double acc[K];
#pragma unroll
  for (int i = 0; i < K; i++) acc[i] = 0;
  const int64_t nv = n / VW;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nv; j += (int64_t)gridDim.x * blockDim.x) {
    T wv[VW];
    ld16(w + j * VW, wv);
#pragma unroll
    for (int i = 0; i < K; i++) {
      T x[VW];
      ld16(V + i * ldv + j * VW, x);
#pragma unroll
      for (int u = 0; u < VW; u++) acc[i] += (double)x[u] * (double)wv[u];
    }
  }
  if (blockIdx.x == 0 && threadIdx.x < n - nv * VW) {  // the last n mod VW elements
    const int64_t e = nv * VW + threadIdx.x;
    const double we = (double)w[e];
#pragma unroll
    for (int i = 0; i < K; i++) acc[i] += (double)V[i * ldv + e] * we;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < K; i++) {
    double v = acc[i];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh[i][warp] = v;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < K; i += blockDim.x) {
    double s = 0;
    for (int wi = 0; wi < kBS / 32; wi++) s += sh[i][wi];
    partial[blockIdx.x * kMaxK + i] = s;
  }
}

// w[e] += sum_{i<K} c[i] V[i][e] (w and V of one precision; the sum in FP64)
template <typename T, int K>
__global__ void __launch_bounds__(kBS) k_multiaxpy_vec(T *__restrict__ w, const T *__restrict__ V, int64_t ldv, Coefs c, int64_t n) {
  constexpr int VW = 16 / sizeof(T);
  const int64_t nv = n / VW;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nv; j += (int64_t)gridDim.x * blockDim.x) {
    T wv[VW];
    ld16(w + j * VW, wv);
    double s[VW];
#pragma unroll
    for (int u = 0; u < VW; u++) s[u] = (double)wv[u];
#pragma unroll
    for (int i = 0; i < K; i++) {
      T x[VW];
      ld16(V + i * ldv + j * VW, x);
#pragma unroll
      for (int u = 0; u < VW; u++) s[u] += c.c[i] * (double)x[u];
    }
#pragma unroll
    for (int u = 0; u < VW; u++) wv[u] = T(s[u]);
    st16(w + j * VW, wv);
  }
  if (blockIdx.x == 0 && threadIdx.x < n - nv * VW) {
    const int64_t e = nv * VW + threadIdx.x;
    double s = (double)w[e];
#pragma unroll
    for (int i = 0; i < K; i++) s += c.c[i] * (double)V[i * ldv + e];
    w[e] = T(s);
  }
}

// The same with the coefficients read from device memory, times `sign` (the Gram-Schmidt step passes the multi-dot's
// result, so no host round trip separates the two); sign * c[i] is formed exactly as the host path's negated copy.
template <typename T, int K>
__global__ void __launch_bounds__(kBS) k_multiaxpy_vec_dev(T *__restrict__ w, const T *__restrict__ V, int64_t ldv, const double *__restrict__ dc,
                                                           double sign, int64_t n) {
  constexpr int VW = 16 / sizeof(T);
  double c[K];
#pragma unroll
  for (int i = 0; i < K; i++) c[i] = sign * dc[i];
  const int64_t nv = n / VW;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nv; j += (int64_t)gridDim.x * blockDim.x) {
    T wv[VW];
    ld16(w + j * VW, wv);
    double s[VW];
#pragma unroll
    for (int u = 0; u < VW; u++) s[u] = (double)wv[u];
#pragma unroll
    for (int i = 0; i < K; i++) {
      T x[VW];
      ld16(V + i * ldv + j * VW, x);
#pragma unroll
      for (int u = 0; u < VW; u++) s[u] += c[i] * (double)x[u];
    }
#pragma unroll
    for (int u = 0; u < VW; u++) wv[u] = T(s[u]);
    st16(w + j * VW, wv);
  }
  if (blockIdx.x == 0 && threadIdx.x < n - nv * VW) {
    const int64_t e = nv * VW + threadIdx.x;
    double s = (double)w[e];
#pragma unroll
    for (int i = 0; i < K; i++) s += c[i] * (double)V[i * ldv + e];
    w[e] = T(s);
  }
}
template <typename T>
__global__ void k_multiaxpy_dev(T *w, const T *V, int64_t ldv, int k, const double *dc, double sign, int64_t n) {  // as k_multiaxpy
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    double s = 0;
    for (int i = 0; i < k; i++) s += (sign * dc[i]) * (double)V[i * ldv + e];
    w[e] = T((double)w[e] + s);
  }
}

#define HB_BASIS_SIZES(X)                                                                                               \
  X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16) X(17) X(18) X(19) X(20) X(21) \
  X(22) X(23) X(24) X(25) X(26) X(27) X(28) X(29) X(30) X(31) X(32)
static_assert(kMaxK == 32, "HB_BASIS_SIZES lists every basis size up to the maximum");

template <typename T>
inline bool vec_ok(const T *V, int64_t ldv, const void *w) {
  return ((uintptr_t)V % 16 == 0) && ((uintptr_t)w % 16 == 0) && ((ldv * (int64_t)sizeof(T)) % 16 == 0);
}

// Blocks of one full wave of a grid-stride kernel at kBS threads: the SMs times the blocks resident per SM, lowered to a
// whole multiple of the SM count when that exceeds `cap`.  Every block then starts at once and carries the same share, where
// a fixed grid that is not a whole number of waves leaves a small, slow last wave (the multi-dot's 512 blocks were 1.15 or
// 1.73 waves at three or two resident blocks per SM).
template <typename F>
unsigned full_wave(F kernel, unsigned cap) {
  int dev = 0, sms = 0, occ = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, kBS, 0) != cudaSuccess || sms <= 0 || occ <= 0)
    return cap;
  const unsigned per = (unsigned)sms, g = (unsigned)occ * per;
  if (g <= cap) return g;
  return cap >= per ? cap / per * per : cap;
}

// Full-wave grids of the multi-dot and multi-axpy for every basis size, read on the first call for the element type (so
// before any stream capture that follows a first call; the devices of one process are alike).
template <typename T>
struct Waves {
  unsigned dot[kMaxK + 1], axpy[kMaxK + 1], axpy_dev[kMaxK + 1];
  Waves() {
#define HB_WAVE(KK)                                                  \
  dot[KK] = full_wave(k_multidot_vec<T, KK>, kRedBlocks);            \
  axpy[KK] = full_wave(k_multiaxpy_vec<T, KK>, 148 * 16);            \
  axpy_dev[KK] = full_wave(k_multiaxpy_vec_dev<T, KK>, 148 * 16);
    HB_BASIS_SIZES(HB_WAVE)
#undef HB_WAVE
  }
};
template <typename T>
const Waves<T> &waves() {
  static const Waves<T> w;
  return w;
}

// out[i] = V_i . w for i < k through the per-block partials (at most kRedBlocks x kMaxK doubles)
template <typename T>
void launch_multidot(const T *V, int64_t ldv, int k, const T *w, int64_t n, double *partial, double *out, cudaStream_t s) {
  unsigned nblk = kRedBlocks;
  if (vec_ok(V, ldv, w)) {
    const Waves<T> &wv = waves<T>();
    switch (k) {
#define HB_MDOT_CASE(KK)                                                       \
  case KK:                                                                     \
    nblk = wv.dot[KK];                                                         \
    k_multidot_vec<T, KK><<<nblk, kBS, 0, s>>>(V, ldv, w, n, partial);         \
    break;
      HB_BASIS_SIZES(HB_MDOT_CASE)
#undef HB_MDOT_CASE
    }
  } else {
    k_multidot<T><<<kRedBlocks, kBS, 0, s>>>(V, ldv, k, w, n, partial);
  }
  k_multidot_final<<<k, kBS, 0, s>>>(partial, (int)nblk, k, out);
}

template <typename T>
void launch_multiaxpy(T *w, const T *V, int64_t ldv, int k, const Coefs &c, int64_t n, cudaStream_t s) {
  if (vec_ok(V, ldv, w)) {
    const int64_t nv = n / (16 / (int64_t)sizeof(T));
    const unsigned work = (unsigned)(nv / kBS + 1 > 148 * 16 ? 148 * 16 : nv / kBS + 1);
    const Waves<T> &wv = waves<T>();
    switch (k) {
#define HB_MAXPY_CASE(KK)                                                                         \
  case KK:                                                                                        \
    k_multiaxpy_vec<T, KK><<<work < wv.axpy[KK] ? work : wv.axpy[KK], kBS, 0, s>>>(w, V, ldv, c, n); \
    break;
      HB_BASIS_SIZES(HB_MAXPY_CASE)
#undef HB_MAXPY_CASE
    }
  } else {
    k_multiaxpy<T, T><<<nblocks(n), kBS, 0, s>>>(w, V, ldv, k, c, n);
  }
}

template <typename T>
void launch_multiaxpy_dev(T *w, const T *V, int64_t ldv, int k, const double *dc, double sign, int64_t n, cudaStream_t s) {
  if (vec_ok(V, ldv, w)) {
    const int64_t nv = n / (16 / (int64_t)sizeof(T));
    const unsigned work = (unsigned)(nv / kBS + 1 > 148 * 16 ? 148 * 16 : nv / kBS + 1);
    const Waves<T> &wv = waves<T>();
    switch (k) {
#define HB_MAXPY_DEV_CASE(KK)                                                                                          \
  case KK:                                                                                                             \
    k_multiaxpy_vec_dev<T, KK><<<work < wv.axpy_dev[KK] ? work : wv.axpy_dev[KK], kBS, 0, s>>>(w, V, ldv, dc, sign, n); \
    break;
      HB_BASIS_SIZES(HB_MAXPY_DEV_CASE)
#undef HB_MAXPY_DEV_CASE
    }
  } else {
    k_multiaxpy_dev<T><<<nblocks(n), kBS, 0, s>>>(w, V, ldv, k, dc, sign, n);
  }
}

// q_dot = alpha q + z
__global__ void k_bdf_qdot(const double *__restrict__ q, const double *__restrict__ z, double alpha, double *__restrict__ qdot, int64_t n) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) qdot[e] = alpha * q[e] + z[e];
}

// z = a q1 + b q2 (history combination of the BDF formula)
__global__ void k_combine(const double *__restrict__ q1, const double *__restrict__ q2, double a, double b, double *__restrict__ z, int64_t n) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
    z[e] = a * q1[e] + (q2 ? b * q2[e] : 0.0);
}

// ---------------------------------------------------------------------------------------------------------------------
// Monitors: one CTA per element, q and its reference gradient tabulated at the points by sum factorisation (mon_tabulate).

struct MonBasis {
  double B[HB_MAX_P * HB_MAX_P], G[HB_MAX_P * HB_MAX_P];
};

// physical gradient of the state (StatePhysicalGradientFromReference, newtonian_state.h:581-593) in the state variable sv
__device__ __forceinline__ void mon_gradient(int sv, const hb::PhysConst<double> &pc, const hb::St<double> &s, const hb::SAux<double> &a,
                                             const double gref[3][5], const double X[3][3], hb::St<double> gs[3]) {
  for (int j = 0; j < 3; j++) {
    double dq[5];
    for (int c = 0; c < 5; c++) dq[c] = gref[0][c] * X[0][j] + gref[1][c] * X[1][j] + gref[2][c] * X[2][j];
    hb::state_from_q_fwd_rt(sv, pc, s, a, dq, gs[j]);
  }
}

// q (and, with grads, its reference gradient) at the Q^3 points of one element by sum factorisation in shared memory:
// an x pass (B, and G with grads), a y pass and a z pass, one thread per 1D output fibre: the tensor-product sums
// sum_{pa,pb,pc} B_i B_j B_k u (and G in one direction) evaluated in O(P) instead of O(P^3) operations per point.  sN [P^3][5] node-major; work: T1B, T1G
// [5][P][P][Q], T2BB, T2BG, T2GB [5][P][Q][Q]; out [1 or 4][5][Q^3]: the values, then d/dX0, d/dX1, d/dX2.
__device__ void mon_tabulate(const double *sN, int P, int Q, const MonBasis &b, bool grads, double *work, double *out) {
  const int P2Q = P * P * Q, PQ2 = P * Q * Q, Q2 = Q * Q, Q3 = Q2 * Q;
  double *T1B = work, *T1G = T1B + 5 * P2Q, *T2BB = T1G + (grads ? 5 * P2Q : 0), *T2BG = T2BB + 5 * PQ2, *T2GB = T2BG + 5 * PQ2;
  for (int t = threadIdx.x; t < 5 * P2Q; t += blockDim.x) {  // x pass: [c][pc][pb][i]
    const int c = t / P2Q, r = t % P2Q, pcb = r / Q, i = r % Q;
    const double *u = sN + (pcb * P) * 5 + c;
    double sb = 0, sg = 0;
    for (int pa = 0; pa < P; pa++) {
      sb += b.B[i * P + pa] * u[pa * 5];
      sg += b.G[i * P + pa] * u[pa * 5];
    }
    T1B[t] = sb;
    if (grads) T1G[t] = sg;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < 5 * PQ2; t += blockDim.x) {  // y pass: [c][pc][j][i]
    const int c = t / PQ2, r = t % PQ2, pc = r / Q2, j = (r / Q) % Q, i = r % Q;
    const int base = ((c * P + pc) * P) * Q + i;
    double bb = 0, bg = 0, gb = 0;
    for (int pb = 0; pb < P; pb++) {
      const double x = T1B[base + pb * Q];
      bb += b.B[j * P + pb] * x;
      if (grads) {
        bg += b.G[j * P + pb] * x;
        gb += b.B[j * P + pb] * T1G[base + pb * Q];
      }
    }
    T2BB[t] = bb;
    if (grads) {
      T2BG[t] = bg;
      T2GB[t] = gb;
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < 5 * Q3; t += blockDim.x) {  // z pass: [c][k][j][i]
    const int c = t / Q3, r = t % Q3, k = r / Q2, ji = r % Q2;
    const int base = (c * P) * Q2 + ji;
    double v = 0, dx = 0, dy = 0, dz = 0;
    for (int pc = 0; pc < P; pc++) {
      const double bz = b.B[k * P + pc], x = T2BB[base + pc * Q2];
      v += bz * x;
      if (grads) {
        dz += b.G[k * P + pc] * x;
        dy += bz * T2BG[base + pc * Q2];
        dx += bz * T2GB[base + pc * Q2];
      }
    }
    out[c * Q3 + r] = v;
    if (grads) {
      out[(5 + c) * Q3 + r] = dx;
      out[(10 + c) * Q3 + r] = dy;
      out[(15 + c) * Q3 + r] = dz;
    }
  }
  __syncthreads();
}
__host__ __device__ inline size_t mon_smem_doubles(int P, int Q, bool grads, int nt, int nred) {
  const size_t P3 = (size_t)P * P * P, P2Q = (size_t)P * P * Q, PQ2 = (size_t)P * Q * Q, Q3 = (size_t)Q * Q * Q;
  return 5 * P3 + (grads ? 2 : 1) * 5 * P2Q + (grads ? 3 : 1) * 5 * PQ2 + (grads ? 4 : 1) * 5 * Q3 + (size_t)nred * nt;
}

// per-element partial sums of the five kinetic-energy integrands [num_elem][5] (MonitorTotalKineticEnergy_Conserv/_Prim/
// _Entropy, qfunctions/monitor_totalkineticenergy.h:8-51)
// point_out (may be null): the five integrands at every point, E-vector [elem][5][Q^3], the output of the Ceed-bound
// MonitorTotalKineticEnergy_* operator (src/monitor_totalkineticenergy.c:80-103); elem_sums (may be null): their sums.
__global__ void k_monitor_ke(int P, int Q, const int32_t *__restrict__ offsets, const double *__restrict__ q, const double *__restrict__ qdata,
                             hb::PhysConst<double> pc, int sv, MonBasis b, double *__restrict__ elem_sums, double *__restrict__ point_out) {
  extern __shared__ double sm[];
  const int e = blockIdx.x, P3 = P * P * P, Q3 = Q * Q * Q;
  double *sN = sm, *sW = sN + 5 * P3, *sQ = sW + 2 * 5 * P * P * Q + 3 * 5 * P * Q * Q, *red = sQ + 4 * 5 * Q3;
  for (int t = threadIdx.x; t < 5 * P3; t += blockDim.x) sN[t] = q[offsets[(int64_t)e * P3 + t / 5] + t % 5];
  __syncthreads();
  mon_tabulate(sN, P, Q, b, true, sW, sQ);
  double acc[5] = {0, 0, 0, 0, 0};
  for (int qp = threadIdx.x; qp < Q3; qp += blockDim.x) {
    double qi[5], gref[3][5], X[3][3];
    for (int c = 0; c < 5; c++) {
      qi[c] = sQ[c * Q3 + qp];
      for (int d = 0; d < 3; d++) gref[d][c] = sQ[((1 + d) * 5 + c) * Q3 + qp];
    }
    const double *qd = qdata + (int64_t)e * 10 * Q3;
    const double wdetJ = qd[qp];
    for (int kk = 0; kk < 9; kk++) X[kk / 3][kk % 3] = qd[(1 + kk) * Q3 + qp];
    hb::St<double> s;
    hb::SAux<double> aux;
    hb::state_from_q_rt(sv, pc, qi, s, aux);
    hb::St<double> gs[3];
    mon_gradient(sv, pc, s, aux, gref, X, gs);
    double e6[6], S[3][3];
    hb::km_strain(gs, e6);
    const double w = 1.0 / 1.4142135623730951;
    S[0][0] = e6[0];
    S[1][1] = e6[1];
    S[2][2] = e6[2];
    S[1][2] = S[2][1] = w * e6[3];
    S[0][2] = S[2][0] = w * e6[4];
    S[0][1] = S[1][0] = w * e6[5];
    const double div = e6[0] + e6[1] + e6[2];
    double SS = 0;
    for (int a = 0; a < 3; a++)
      for (int c = 0; c < 3; c++) SS += S[a][c] * S[a][c];
    const double w0 = gs[2].u[1] - gs[1].u[2], w1 = gs[0].u[2] - gs[2].u[0], w2 = gs[1].u[0] - gs[0].u[1];
    const double v[5] = {wdetJ * 0.5 * s.rho * (s.u[0] * s.u[0] + s.u[1] * s.u[1] + s.u[2] * s.u[2]), wdetJ * -2 * pc.mu * SS,
                         wdetJ * -pc.lambda * pc.mu * div * div, wdetJ * s.P * div, wdetJ * pc.mu * (w0 * w0 + w1 * w1 + w2 * w2)};
    for (int c = 0; c < 5; c++) acc[c] += v[c];
    if (point_out)
      for (int c = 0; c < 5; c++) point_out[((int64_t)e * 5 + c) * Q3 + qp] = v[c];
  }
  if (!elem_sums) return;
  for (int c = 0; c < 5; c++) red[c * blockDim.x + threadIdx.x] = acc[c];
  __syncthreads();
  if (threadIdx.x < 5) {
    double s = 0;
    for (int t = 0; t < (int)blockDim.x; t++) s += red[threadIdx.x * blockDim.x + t];
    elem_sums[(int64_t)e * 5 + threadIdx.x] = s;
  }
}

// per-element min/max over points of sqrt(u . g u) with g = 0.25 dXdx^T dXdx (MonitorCFL_3D_Conserv/_Prim/_Entropy,
// qfunctions/monitor_cfl.h:9-58)
// point_out (may be null): sqrt(u . g u) at every point, E-vector [elem][Q^3] (the Ceed-bound MonitorCFL_3D_* operator,
// src/monitor_cfl.c:100-110); elem_minmax (may be null): its per-element extremes.
__global__ void k_monitor_cfl(int P, int Q, const int32_t *__restrict__ offsets, const double *__restrict__ q, const double *__restrict__ qdata,
                              hb::PhysConst<double> pc, int sv, MonBasis b, double *__restrict__ elem_minmax, double *__restrict__ point_out) {
  extern __shared__ double sm[];
  const int e = blockIdx.x, P3 = P * P * P, Q3 = Q * Q * Q;
  double *sN = sm, *sW = sN + 5 * P3, *sQ = sW + 5 * P * P * Q + 5 * P * Q * Q, *red = sQ + 5 * Q3;
  for (int t = threadIdx.x; t < 5 * P3; t += blockDim.x) sN[t] = q[offsets[(int64_t)e * P3 + t / 5] + t % 5];
  __syncthreads();
  mon_tabulate(sN, P, Q, b, false, sW, sQ);
  double mn = 1e300, mx = -1e300;
  for (int qp = threadIdx.x; qp < Q3; qp += blockDim.x) {
    double qi[5], X[3][3], g[3][3];
    for (int c = 0; c < 5; c++) qi[c] = sQ[c * Q3 + qp];
    const double *qd = qdata + (int64_t)e * 10 * Q3;
    for (int kk = 0; kk < 9; kk++) X[kk / 3][kk % 3] = qd[(1 + kk) * Q3 + qp];
    hb::St<double> s;
    hb::SAux<double> aux;
    hb::state_from_q_rt(sv, pc, qi, s, aux);
    for (int a = 0; a < 3; a++)
      for (int c = 0; c < 3; c++) g[a][c] = 0.25 * (X[0][a] * X[0][c] + X[1][a] * X[1][c] + X[2][a] * X[2][c]);
    double ugu = 0;
    for (int a = 0; a < 3; a++) ugu += s.u[a] * (g[a][0] * s.u[0] + g[a][1] * s.u[1] + g[a][2] * s.u[2]);
    const double cfl = sqrt(ugu);
    mn = fmin(mn, cfl);
    mx = fmax(mx, cfl);
    if (point_out) point_out[(int64_t)e * Q3 + qp] = cfl;
  }
  if (!elem_minmax) return;
  red[threadIdx.x] = mn;
  red[blockDim.x + threadIdx.x] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 1e300, c = -1e300;
    for (int t = 0; t < (int)blockDim.x; t++) {
      a = fmin(a, red[t]);
      c = fmax(c, red[blockDim.x + t]);
    }
    elem_minmax[(int64_t)e * 2] = a;
    elem_minmax[(int64_t)e * 2 + 1] = c;
  }
}

inline int rc() { return cudaGetLastError() == cudaSuccess ? HB_SUCCESS : HB_ERROR_CUDA; }

}  // namespace

// ---------------------------------------------------------------------------------------------------------------------
// Fixed device scratch for hb_krylov_multidot_f64_static: the per-block partial sums of k_multidot, [kRedBlocks][kMaxK]
// doubles = 512 x 32 x 8 B = 128 KiB, the most any k <= HB_GMRES_MAX_BASIS needs.  Every entry the final pass reads is
// written earlier in the same call by k_multidot, so nothing in it has to start at zero.  One copy per device and per
// loaded module: calls that overlap on one device (two streams, or two host threads without ordering) race on it.
static __device__ __align__(256) double g_multidot_scratch[kRedBlocks * kMaxK];

namespace {
constexpr int kMaxDevices = 64;
std::atomic<double *> g_multidot_scratch_addr[kMaxDevices];

// Address of g_multidot_scratch on the current device, looked up once per device (with that device current) on the first
// call there.  The lookup may load this module on the device, so the first call on each device belongs before any
// stream capture starts.  The cached address does not survive cudaDeviceReset (the reloaded module may place the array
// elsewhere); the header states that the entry point is not for a device whose context was reset.
int multidot_scratch(double **p) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return HB_ERROR_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return HB_ERROR_UNSUPPORTED;
  double *a = g_multidot_scratch_addr[dev].load(std::memory_order_acquire);
  if (!a) {
    void *sym = nullptr;
    if (cudaGetSymbolAddress(&sym, g_multidot_scratch) != cudaSuccess || !sym) return HB_ERROR_CUDA;
    a = (double *)sym;
    g_multidot_scratch_addr[dev].store(a, std::memory_order_release);
  }
  *p = a;
  return HB_SUCCESS;
}
}  // namespace

namespace {

// ---- point-block Jacobi (PCVPBJACOBI on the 5 x 5 node blocks): invert each block once per preconditioner set-up, apply
// y = B^-1 x per node in the Krylov precision.  One thread per node; the set-up kernel is Gauss-Jordan with partial
// pivoting in FP64 (a block whose pivot vanishes or is not finite is counted in *singular and replaced by the identity).
template <typename TO>
__global__ void __launch_bounds__(kBS) k_pb_invert(const double *in, TO *out, int64_t nodes, int *singular) {  // in may equal out
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < nodes; b += (int64_t)gridDim.x * blockDim.x) {
    double A[5][10];
#pragma unroll
    for (int i = 0; i < 5; i++)
#pragma unroll
      for (int j = 0; j < 5; j++) {
        A[i][j]     = in[b * 25 + i * 5 + j];
        A[i][5 + j] = i == j ? 1.0 : 0.0;
      }
    bool ok = true;
    for (int c = 0; c < 5 && ok; c++) {
      int pr = c;
      for (int r = c + 1; r < 5; r++)
        if (fabs(A[r][c]) > fabs(A[pr][c])) pr = r;
      if (!(fabs(A[pr][c]) > 0.0) || !isfinite(A[pr][c])) {
        ok = false;
        break;
      }
      if (pr != c)
        for (int j = 0; j < 10; j++) {
          const double t = A[c][j];
          A[c][j]         = A[pr][j];
          A[pr][j]        = t;
        }
      const double inv = 1.0 / A[c][c];
      for (int j = 0; j < 10; j++) A[c][j] *= inv;
      for (int r = 0; r < 5; r++)
        if (r != c) {
          const double f = A[r][c];
          for (int j = 0; j < 10; j++) A[r][j] -= f * A[c][j];
        }
    }
    if (!ok) atomicAdd(singular, 1);
#pragma unroll
    for (int i = 0; i < 5; i++)
#pragma unroll
      for (int j = 0; j < 5; j++) out[b * 25 + i * 5 + j] = (TO)(ok ? A[i][5 + j] : (i == j ? 1.0 : 0.0));
  }
}

template <typename T>
__global__ void __launch_bounds__(kBS) k_pb_apply(const T *__restrict__ inv, const T *__restrict__ x, T *__restrict__ y, int64_t nodes) {
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < nodes; b += (int64_t)gridDim.x * blockDim.x) {
    T xv[5], yv[5];
#pragma unroll
    for (int j = 0; j < 5; j++) xv[j] = x[b * 5 + j];
#pragma unroll
    for (int i = 0; i < 5; i++) {
      T acc = 0;
#pragma unroll
      for (int j = 0; j < 5; j++) acc += inv[b * 25 + i * 5 + j] * xv[j];
      yv[i] = acc;
    }
#pragma unroll
    for (int i = 0; i < 5; i++) y[b * 5 + i] = yv[i];
  }
}

template <typename TO>
int pb_invert(const double *blocks, TO *inv, int64_t nodes, int *d_singular, int *h_singular, void *s) {
  cudaStream_t st = (cudaStream_t)s;
  if (!blocks || !inv || !d_singular || nodes < 0) return HB_ERROR_INVALID;
  if (cudaMemsetAsync(d_singular, 0, sizeof(int), st) != cudaSuccess) return HB_ERROR_CUDA;
  if (nodes) k_pb_invert<TO><<<nblocks(nodes), kBS, 0, st>>>(blocks, inv, nodes, d_singular);
  if (cudaGetLastError() != cudaSuccess) return HB_ERROR_CUDA;
  if (h_singular) {
    if (cudaMemcpyAsync(h_singular, d_singular, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
      return HB_ERROR_CUDA;
  }
  return HB_SUCCESS;
}

// ---- essential (Dirichlet) DOFs: the constrained entries of the node-interleaved L-vector, which PETSc's DMPlex section
// removes from the global system (the values are inserted into the local state, DMPlexInsertBoundaryValues)
template <typename T>
__global__ void k_constrain_set(T *__restrict__ x, const int32_t *__restrict__ idx, const double *__restrict__ val, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) x[idx[i]] = val ? (T)val[i] : T(0);
}
// rows and columns of the constrained components become those of the identity in their node's 5 x 5 block (two threads of
// one node only ever write the same value to an entry they share)
__global__ void k_pb_constrain(double *__restrict__ blocks, const int32_t *__restrict__ idx, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t node = idx[i] / 5, c = idx[i] % 5;
    double *b = blocks + node * 25;
    for (int k = 0; k < 5; k++) {
      b[c * 5 + k] = 0.0;
      b[k * 5 + c] = 0.0;
    }
    b[c * 6] = 1.0;
  }
}

}  // namespace

extern "C" {

int hb_krylov_multidot_f64(const double *V, int64_t ldv, int k, const double *w, int64_t n, double *d_partial, double *d_out, void *s) {
  if (k < 1 || k > kMaxK) return HB_ERROR_INVALID;
  launch_multidot<double>(V, ldv, k, w, n, d_partial, d_out, (cudaStream_t)s);
  return rc();
}
int hb_krylov_multidot_f32(const float *V, int64_t ldv, int k, const float *w, int64_t n, double *d_partial, double *d_out, void *s) {
  if (k < 1 || k > kMaxK) return HB_ERROR_INVALID;
  launch_multidot<float>(V, ldv, k, w, n, d_partial, d_out, (cudaStream_t)s);
  return rc();
}

// hb_krylov_multidot_f64 without the caller's partial-sum buffer: the same kernels, with the partials in the fixed
// device scratch above.  For callers that have no device work buffer to give and must not create one per call: an inner
// product requested through a vector-library callback that carries only the vectors (a cudaMalloc/cudaFree pair there
// would synchronise the whole device on every Krylov iteration), or a solver that commits all device memory to its Krylov
// basis at set-up and allocates nothing afterwards.  k above HB_GMRES_MAX_BASIS would need more partials than the scratch
// holds and is refused with HB_ERROR_INVALID before anything is launched.
int hb_krylov_multidot_f64_static(const double *V, int64_t ldv, int k, const double *w, int64_t n, double *d_out, void *s) {
  if (k < 1 || k > kMaxK) return HB_ERROR_INVALID;
  double *partial = nullptr;
  const int e = multidot_scratch(&partial);
  if (e) return e;
  launch_multidot<double>(V, ldv, k, w, n, partial, d_out, (cudaStream_t)s);
  return rc();
}
int hb_krylov_multiaxpy_f64(double *w, const double *V, int64_t ldv, int k, const double *c, int64_t n, void *s) {
  if (k < 1 || k > kMaxK) return HB_ERROR_INVALID;
  Coefs cf;
  memset(&cf, 0, sizeof cf);
  memcpy(cf.c, c, sizeof(double) * k);
  launch_multiaxpy<double>(w, V, ldv, k, cf, n, (cudaStream_t)s);
  return rc();
}
int hb_krylov_multiaxpy_f32(float *w, const float *V, int64_t ldv, int k, const double *c, int64_t n, void *s) {
  if (k < 1 || k > kMaxK) return HB_ERROR_INVALID;
  Coefs cf;
  memset(&cf, 0, sizeof cf);
  memcpy(cf.c, c, sizeof(double) * k);
  launch_multiaxpy<float>(w, V, ldv, k, cf, n, (cudaStream_t)s);
  return rc();
}
int hb_krylov_multiaxpy_dev_f64(double *w, const double *V, int64_t ldv, int k, const double *d_c, double sign, int64_t n, void *s) {
  if (k < 1 || k > kMaxK || !d_c) return HB_ERROR_INVALID;
  launch_multiaxpy_dev<double>(w, V, ldv, k, d_c, sign, n, (cudaStream_t)s);
  return rc();
}
int hb_krylov_multiaxpy_dev_f32(float *w, const float *V, int64_t ldv, int k, const double *d_c, double sign, int64_t n, void *s) {
  if (k < 1 || k > kMaxK || !d_c) return HB_ERROR_INVALID;
  launch_multiaxpy_dev<float>(w, V, ldv, k, d_c, sign, n, (cudaStream_t)s);
  return rc();
}
int hb_krylov_multiaxpy_f32_to_f64(double *w, const float *V, int64_t ldv, int k, const double *c, int64_t n, void *s) {
  if (k < 1 || k > kMaxK) return HB_ERROR_INVALID;
  Coefs cf;
  memset(&cf, 0, sizeof cf);
  memcpy(cf.c, c, sizeof(double) * k);
  k_multiaxpy<float, double><<<nblocks(n), kBS, 0, (cudaStream_t)s>>>(w, V, ldv, k, cf, n);
  return rc();
}
int hb_bdf_qdot(const double *q, const double *z, double alpha, double *qdot, int64_t n, void *s) {
  k_bdf_qdot<<<nblocks(n), kBS, 0, (cudaStream_t)s>>>(q, z, alpha, qdot, n);
  return rc();
}
int hb_vec_combine_f64(const double *q1, const double *q2, double a, double b, double *z, int64_t n, void *s) {
  k_combine<<<nblocks(n), kBS, 0, (cudaStream_t)s>>>(q1, q2, a, b, z, n);
  return rc();
}

static hb::PhysConst<double> phys_of(const void *ctx184) {
  HbNewtonianContext c;
  memcpy(&c, ctx184, sizeof c);
  hb::PhysConst<double> p;
  memset(&p, 0, sizeof p);
  p.mu = c.gas.mu;
  p.lambda = c.gas.lambda;
  p.k = c.gas.k;
  p.cv = c.gas.cv;
  p.inv_cv = 1.0 / c.gas.cv;
  p.gm1 = c.gas.cp / c.gas.cv - 1;
  p.Rgas = c.gas.cp - c.gas.cv;
  return p;
}

static MonBasis mon_basis(const HbElemOp *op) {
  MonBasis b;
  memset(&b, 0, sizeof b);
  memcpy(b.B, op->interp1d, sizeof(double) * op->P * op->Q);
  memcpy(b.G, op->grad1d, sizeof(double) * op->P * op->Q);
  return b;
}

// Kinetic-energy monitor sums (not divided by the volume); d_scratch >= 5 * num_elem doubles; synchronises the stream.
static int state_var_of(const void *ctx184, int *sv) {
  HbNewtonianContext c;
  memcpy(&c, ctx184, sizeof c);
  if (c.state_var != HB_STATEVAR_CONSERVATIVE && c.state_var != HB_STATEVAR_PRIMITIVE && c.state_var != HB_STATEVAR_ENTROPY) return HB_ERROR_UNSUPPORTED;
  *sv = c.state_var;
  return HB_SUCCESS;
}

int hb_monitor_ke(const HbElemOp *op, const void *ctx184, const double *q, const double *qdata, double *d_scratch, double sums[5], void *s) {
  int sv = 0;
  if (state_var_of(ctx184, &sv)) return HB_ERROR_UNSUPPORTED;
  const int nt = 128;
  const size_t sm = sizeof(double) * mon_smem_doubles(op->P, op->Q, true, nt, 5);
  if (cudaFuncSetAttribute(k_monitor_ke, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess) return HB_ERROR_CUDA;
  k_monitor_ke<<<op->num_elem, nt, sm, (cudaStream_t)s>>>(op->P, op->Q, op->d_offsets, q, qdata, phys_of(ctx184), sv, mon_basis(op), d_scratch, nullptr);
  if (rc()) return HB_ERROR_CUDA;
  double *h = (double *)malloc(sizeof(double) * 5 * (size_t)op->num_elem);
  if (!h) return HB_ERROR_NOMEM;
  int err = cudaMemcpyAsync(h, d_scratch, sizeof(double) * 5 * (size_t)op->num_elem, cudaMemcpyDeviceToHost, (cudaStream_t)s) != cudaSuccess ||
            cudaStreamSynchronize((cudaStream_t)s) != cudaSuccess;
  for (int c = 0; c < 5; c++) sums[c] = 0;
  for (int64_t e = 0; e < op->num_elem; e++)
    for (int c = 0; c < 5; c++) sums[c] += h[e * 5 + c];
  free(h);
  return err ? HB_ERROR_CUDA : HB_SUCCESS;
}

// CFL monitor: min and max over points of dt * sqrt(u . g u); d_scratch >= 2 * num_elem doubles; synchronises.
int hb_monitor_cfl(const HbElemOp *op, const void *ctx184, const double *q, const double *qdata, double dt, double *d_scratch, double minmax[2],
                   void *s) {
  int sv = 0;
  if (state_var_of(ctx184, &sv)) return HB_ERROR_UNSUPPORTED;
  const int nt = 128;
  const size_t sm = sizeof(double) * mon_smem_doubles(op->P, op->Q, false, nt, 2);
  if (cudaFuncSetAttribute(k_monitor_cfl, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess) return HB_ERROR_CUDA;
  k_monitor_cfl<<<op->num_elem, nt, sm, (cudaStream_t)s>>>(op->P, op->Q, op->d_offsets, q, qdata, phys_of(ctx184), sv, mon_basis(op), d_scratch, nullptr);
  if (rc()) return HB_ERROR_CUDA;
  double *h = (double *)malloc(sizeof(double) * 2 * (size_t)op->num_elem);
  if (!h) return HB_ERROR_NOMEM;
  int err = cudaMemcpyAsync(h, d_scratch, sizeof(double) * 2 * (size_t)op->num_elem, cudaMemcpyDeviceToHost, (cudaStream_t)s) != cudaSuccess ||
            cudaStreamSynchronize((cudaStream_t)s) != cudaSuccess;
  double mn = 1e300, mx = -1e300;
  for (int64_t e = 0; e < op->num_elem; e++) {
    mn = fmin(mn, h[2 * e]);
    mx = fmax(mx, h[2 * e + 1]);
  }
  free(h);
  minmax[0] = mn * dt;
  minmax[1] = mx * dt;
  return err ? HB_ERROR_CUDA : HB_SUCCESS;
}

// Per-point monitor values (the Ceed-bound monitor operators): asynchronous on s.
int hb_monitor_ke_points(const HbElemOp *op, const void *ctx184, const double *q, const double *qdata, double *e_out, void *s) {
  int sv = 0;
  if (state_var_of(ctx184, &sv)) return HB_ERROR_UNSUPPORTED;
  if (op->num_elem == 0) return HB_SUCCESS;
  const int nt = 128;
  const size_t sm = sizeof(double) * mon_smem_doubles(op->P, op->Q, true, nt, 5);
  if (cudaFuncSetAttribute(k_monitor_ke, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess) return HB_ERROR_CUDA;
  k_monitor_ke<<<op->num_elem, nt, sm, (cudaStream_t)s>>>(op->P, op->Q, op->d_offsets, q, qdata, phys_of(ctx184), sv, mon_basis(op), nullptr, e_out);
  return rc();
}
int hb_monitor_cfl_points(const HbElemOp *op, const void *ctx184, const double *q, const double *qdata, double *e_out, void *s) {
  int sv = 0;
  if (state_var_of(ctx184, &sv)) return HB_ERROR_UNSUPPORTED;
  if (op->num_elem == 0) return HB_SUCCESS;
  const int nt = 128;
  const size_t sm = sizeof(double) * mon_smem_doubles(op->P, op->Q, false, nt, 2);
  if (cudaFuncSetAttribute(k_monitor_cfl, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess) return HB_ERROR_CUDA;
  k_monitor_cfl<<<op->num_elem, nt, sm, (cudaStream_t)s>>>(op->P, op->Q, op->d_offsets, q, qdata, phys_of(ctx184), sv, mon_basis(op), nullptr, e_out);
  return rc();
}

int hb_pb_invert_f64(const double *blocks, double *inv, int64_t nodes, int *d_singular, int *h_singular, void *s) {
  return pb_invert<double>(blocks, inv, nodes, d_singular, h_singular, s);
}
int hb_pb_invert_f64_to_f32(const double *blocks, float *inv, int64_t nodes, int *d_singular, int *h_singular, void *s) {
  return pb_invert<float>(blocks, inv, nodes, d_singular, h_singular, s);
}
int hb_pb_apply_f64(const double *inv, const double *x, double *y, int64_t nodes, void *s) {
  if (!inv || !x || !y || x == y) return HB_ERROR_INVALID;
  if (nodes) k_pb_apply<double><<<nblocks(nodes), kBS, 0, (cudaStream_t)s>>>(inv, x, y, nodes);
  return cudaGetLastError() == cudaSuccess ? HB_SUCCESS : HB_ERROR_CUDA;
}
int hb_pb_apply_f32(const float *inv, const float *x, float *y, int64_t nodes, void *s) {
  if (!inv || !x || !y || x == y) return HB_ERROR_INVALID;
  if (nodes) k_pb_apply<float><<<nblocks(nodes), kBS, 0, (cudaStream_t)s>>>(inv, x, y, nodes);
  return cudaGetLastError() == cudaSuccess ? HB_SUCCESS : HB_ERROR_CUDA;
}

int hb_constrain_set_f64(double *x, const int32_t *idx, const double *val, int64_t n, void *s) {
  if (n < 0 || (n && (!x || !idx))) return HB_ERROR_INVALID;
  if (n) k_constrain_set<double><<<nblocks(n), kBS, 0, (cudaStream_t)s>>>(x, idx, val, n);
  return cudaGetLastError() == cudaSuccess ? HB_SUCCESS : HB_ERROR_CUDA;
}
int hb_constrain_set_f32(float *x, const int32_t *idx, const double *val, int64_t n, void *s) {
  if (n < 0 || (n && (!x || !idx))) return HB_ERROR_INVALID;
  if (n) k_constrain_set<float><<<nblocks(n), kBS, 0, (cudaStream_t)s>>>(x, idx, val, n);
  return cudaGetLastError() == cudaSuccess ? HB_SUCCESS : HB_ERROR_CUDA;
}
int hb_pb_constrain(double *blocks, const int32_t *idx, int64_t n, void *s) {
  if (n < 0 || (n && (!blocks || !idx))) return HB_ERROR_INVALID;
  if (n) k_pb_constrain<<<nblocks(n), kBS, 0, (cudaStream_t)s>>>(blocks, idx, n);
  return cudaGetLastError() == cudaSuccess ? HB_SUCCESS : HB_ERROR_CUDA;
}

}  // extern "C"
