// k_sgs.cu -- the learned subgrid-stress closure on the GPU: training data from filtered fields, the model's
// forward / backward / Adam training kernels (FP32), batch inference, and point-wise checks of the closure's maps.
//
// Training step (one launch pair per step):
//   k_mlp_grad   one thread per sample of the batch: forward pass in registers, loss and output error, backward pass;
//                the CTA then forms its weight gradients from the per-sample activations and errors staged in shared
//                memory (each thread owns a few weight entries and sums over the CTA's samples) and writes one partial
//                gradient row -- no atomics, so the gradient is deterministic
//   k_mlp_adam   one thread per weight: sums the partial rows in a fixed order and applies Adam (Kingma & Ba, 2015:
//                m, v moment estimates with bias correction, step lr m^ / (sqrt(v^) + eps))
// Samples are drawn with replacement by a counter-based hash of (seed, step, slot), or taken from an index list.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include "honee_b200.h"
#include "sgs.cuh"

namespace {

constexpr int kTB = 256;  // samples per CTA in the training kernels

inline int rc() { return cudaGetLastError() == cudaSuccess ? HB_SUCCESS : HB_ERROR_CUDA; }

__device__ __forceinline__ uint64_t mix64(uint64_t z) {  // splitmix64 finaliser
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

template <int H1, int H2>
struct Act {  // per-sample values the weight gradients need: inputs, hidden activations and the layer errors
  static constexpr int L2 = H2 > 0 ? H2 : H1;  // width entering the output layer (the first hidden layer when H2 == 0)
  static constexpr int NX = 6, oX = 0, oH1 = oX + NX, oH2 = oH1 + H1, oD3 = oH2 + L2, oD2 = oD3 + 6, oD1 = oD2 + L2, size = oD1 + H1;
};

// partial[blockIdx][p] = d(loss)/d(param p) summed over this CTA's samples; loss_part[blockIdx] = its squared error sum.
// Loss = mean over the batch and the 6 outputs of (y - t)^2.
template <int H1, int H2>
__global__ void __launch_bounds__(kTB) k_mlp_grad(const float *__restrict__ w, float alpha, const float *__restrict__ X, const float *__restrict__ Y,
                                                  int64_t n, const int32_t *__restrict__ idx, int batch, uint64_t seed, float *__restrict__ partial,
                                                  float *__restrict__ loss_part) {
  using S = hb::sgs::MlpShape<H1, H2>;
  using A = Act<H1, H2>;
  constexpr int L2 = S::L2IN;
  extern __shared__ float smem[];
  float *sw_ = smem;             // weights; read through a volatile view so the compiler reloads them (cheap shared
  volatile float *sw = sw_;      // loads) instead of keeping hundreds of them live across the forward and backward passes
  float *sa = smem + S::size;    // [kTB][A::size] activations and errors
  __shared__ float sl[kTB / 32];
  for (int p = threadIdx.x; p < S::size; p += blockDim.x) sw_[p] = w[p];
  __syncthreads();
  const int slot = blockIdx.x * kTB + threadIdx.x;
  const bool live = slot < batch;
  float *a = sa + threadIdx.x * A::size;
  float err = 0.f;
  if (live) {
    const int64_t s = idx ? (int64_t)idx[slot] : (int64_t)(mix64(seed ^ ((uint64_t)slot * 0x2545f4914f6cdd1dull)) % (uint64_t)n);
    float x[6], t[6], h1[H1], z1[H1], h2[L2], z2[L2], y[6];
#pragma unroll
    for (int j = 0; j < 6; j++) {
      x[j] = X[s * 6 + j];
      t[j] = Y[s * 6 + j];
    }
#pragma unroll
    for (int i = 0; i < H1; i++) {
      float z = sw[S::oB1 + i];
#pragma unroll
      for (int j = 0; j < 6; j++) z += sw[S::oW1 + i * 6 + j] * x[j];
      z1[i] = z;
      h1[i] = z < 0.f ? alpha * z : z;
    }
    if constexpr (H2 > 0) {
#pragma unroll
      for (int i = 0; i < H2; i++) {
        float z = sw[S::oB2 + i];
#pragma unroll
        for (int j = 0; j < H1; j++) z += sw[S::oW2 + i * H1 + j] * h1[j];
        z2[i] = z;
        h2[i] = z < 0.f ? alpha * z : z;
      }
    } else {
#pragma unroll
      for (int i = 0; i < L2; i++) {
        z2[i] = z1[i];
        h2[i] = h1[i];
      }
    }
    float d3[6];
    const float scale = 2.f / (6.f * (float)batch);
#pragma unroll
    for (int i = 0; i < 6; i++) {
      float z = sw[S::oB3 + i];
#pragma unroll
      for (int j = 0; j < L2; j++) z += sw[S::oW3 + i * L2 + j] * h2[j];
      y[i] = z;
      const float e = z - t[i];
      err += e * e;
      d3[i] = scale * e;
    }
    // back-propagation: d2 = (W3^T d3) * act'(z2), d1 = (W2^T d2) * act'(z1)
    float d2[L2], d1[H1];
#pragma unroll
    for (int j = 0; j < L2; j++) {
      float s2 = 0.f;
#pragma unroll
      for (int i = 0; i < 6; i++) s2 += sw[S::oW3 + i * L2 + j] * d3[i];
      d2[j] = z2[j] < 0.f ? alpha * s2 : s2;
    }
    if constexpr (H2 > 0) {
#pragma unroll
      for (int j = 0; j < H1; j++) {
        float s1 = 0.f;
#pragma unroll
        for (int i = 0; i < H2; i++) s1 += sw[S::oW2 + i * H1 + j] * d2[i];
        d1[j] = z1[j] < 0.f ? alpha * s1 : s1;
      }
    } else {
#pragma unroll
      for (int j = 0; j < H1; j++) d1[j] = d2[j];
    }
#pragma unroll
    for (int j = 0; j < 6; j++) a[A::oX + j] = x[j];
#pragma unroll
    for (int j = 0; j < H1; j++) {
      a[A::oH1 + j] = h1[j];
      a[A::oD1 + j] = d1[j];
    }
#pragma unroll
    for (int j = 0; j < L2; j++) {
      a[A::oH2 + j] = h2[j];
      a[A::oD2 + j] = d2[j];
    }
#pragma unroll
    for (int j = 0; j < 6; j++) a[A::oD3 + j] = d3[j];
  } else {
    for (int j = 0; j < A::size; j++) a[j] = 0.f;  // a missing sample contributes nothing
  }
  // loss partial
  for (int o = 16; o > 0; o >>= 1) err += __shfl_down_sync(0xffffffffu, err, o);
  if ((threadIdx.x & 31) == 0) sl[threadIdx.x >> 5] = err;
  __syncthreads();
  if (threadIdx.x == 0) {
    float s = 0.f;
    for (int i = 0; i < kTB / 32; i++) s += sl[i];
    loss_part[blockIdx.x] = s;
  }
  // weight gradients: each thread owns parameters p = threadIdx.x + k * kTB and sums over the CTA's samples in order
  for (int p = threadIdx.x; p < S::size; p += kTB) {
    int eo, io;  // offsets (within a sample's record) of the error row and the input row of this parameter; io < 0: bias
    if (p < S::oB1) {
      const int ri = (p - S::oW1) / 6, ci = (p - S::oW1) % 6;
      eo = A::oD1 + ri, io = A::oX + ci;
    } else if (p < S::oW2) {
      eo = A::oD1 + (p - S::oB1), io = -1;
    } else if (H2 > 0 && p < S::oB2) {
      const int ri = (p - S::oW2) / H1, ci = (p - S::oW2) % H1;
      eo = A::oD2 + ri, io = A::oH1 + ci;
    } else if (H2 > 0 && p < S::oW3) {
      eo = A::oD2 + (p - S::oB2), io = -1;
    } else if (p < S::oB3) {
      const int ri = (p - S::oW3) / L2, ci = (p - S::oW3) % L2;
      eo = A::oD3 + ri, io = A::oH2 + ci;
    } else {
      eo = A::oD3 + (p - S::oB3), io = -1;
    }
    float g = 0.f;
    if (io >= 0)
      for (int s = 0; s < kTB; s++) g += sa[s * A::size + eo] * sa[s * A::size + io];
    else
      for (int s = 0; s < kTB; s++) g += sa[s * A::size + eo];
    partial[(int64_t)blockIdx.x * S::size + p] = g;
  }
}

// g = sum of the partial rows; Adam update of w, m, v at step t (1-based); loss[0] = mean squared error of the batch
__global__ void k_mlp_adam(float *__restrict__ w, float *__restrict__ m, float *__restrict__ v, const float *__restrict__ partial, int nparts,
                           int np, float lr, float b1, float b2, float eps, float bc1, float bc2, const float *__restrict__ loss_part,
                           float loss_scale, float *__restrict__ loss, float *__restrict__ grad_out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p == 0) {
    float s = 0.f;
    for (int b = 0; b < nparts; b++) s += loss_part[b];
    loss[0] = s * loss_scale;
  }
  if (p >= np) return;
  float g = 0.f;
  for (int b = 0; b < nparts; b++) g += partial[(int64_t)b * np + p];
  if (grad_out) grad_out[p] = g;
  if (lr == 0.f) return;  // gradient only
  const float mm = b1 * m[p] + (1.f - b1) * g, vv = b2 * v[p] + (1.f - b2) * g * g;
  m[p] = mm;
  v[p] = vv;
  w[p] -= lr * (mm / bc1) / (sqrtf(vv / bc2) + eps);
}

// one sample per thread (no grid-stride loop: the weights would become loop invariants and be hoisted into registers)
template <int H1, int H2>
__global__ void k_mlp_forward(const float *__restrict__ w, float alpha, const float *__restrict__ X, float *__restrict__ Y, int64_t n) {
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= n) return;
  float x[6], y[6];
#pragma unroll
  for (int j = 0; j < 6; j++) x[j] = X[s * 6 + j];
  hb::sgs::mlp_forward<H1, H2>(w, alpha, x, y);
#pragma unroll
  for (int j = 0; j < 6; j++) Y[s * 6 + j] = y[j];
}

// ---------------------------------------------------------------------------------------------------------------------
// Point-wise maps of the closure on arrays of points (FP64), for checking them against the reference QFunctions and for
// callers that build model inputs themselves.

__global__ void k_sgs_anisotropy(int64_t n, const double *__restrict__ dXdx, double *__restrict__ kmA, double *__restrict__ delta) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double X[3][3], a[6], d;
#pragma unroll
    for (int k = 0; k < 9; k++) X[k / 3][k % 3] = dXdx[i * 9 + k];
    hb::sgs::anisotropy(X, a, d);
#pragma unroll
    for (int k = 0; k < 6; k++) kmA[i * 6 + k] = a[k];
    delta[i] = d;
  }
}

__global__ void k_sgs_inputs(int64_t n, const double *__restrict__ G, const double *__restrict__ kmA, const double *__restrict__ delta,
                             const double *__restrict__ nu, double *__restrict__ in, double *__restrict__ E, double *__restrict__ gmag) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double g[3][3], a[6], e[3][3], x[6], m;
#pragma unroll
    for (int k = 0; k < 9; k++) g[k / 3][k % 3] = G[i * 9 + k];
#pragma unroll
    for (int k = 0; k < 6; k++) a[k] = kmA[i * 6 + k];
    hb::sgs::inputs(g, a, delta[i], nu[i], e, x, m);
#pragma unroll
    for (int k = 0; k < 6; k++) in[i * 6 + k] = x[k];
#pragma unroll
    for (int k = 0; k < 9; k++) E[i * 9 + k] = e[k / 3][k % 3];
    gmag[i] = m;
  }
}

struct Bounds {
  float b[6][2];
};

__global__ void k_sgs_stress(int64_t n, const double *__restrict__ out_n, const double *__restrict__ delta, const double *__restrict__ E,
                             const double *__restrict__ gmag, Bounds bd, double *__restrict__ km_tau) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double o[6], e[3][3], t[6];
#pragma unroll
    for (int k = 0; k < 6; k++) o[k] = out_n[i * 6 + k];
#pragma unroll
    for (int k = 0; k < 9; k++) e[k / 3][k % 3] = E[i * 9 + k];
    hb::sgs::outputs_to_stress(o, delta[i], e, bd.b, gmag[i], t);
#pragma unroll
    for (int k = 0; k < 6; k++) km_tau[i * 6 + k] = t[k];
  }
}

// min / max of each of the 6 target columns: per-block partials then one final block
__global__ void k_col_minmax(const float *__restrict__ Y, int64_t n, float *__restrict__ part) {
  float lo[6], hi[6];
#pragma unroll
  for (int c = 0; c < 6; c++) {
    lo[c] = 3.4e38f;
    hi[c] = -3.4e38f;
  }
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
#pragma unroll
    for (int c = 0; c < 6; c++) {
      const float y = Y[i * 6 + c];
      lo[c] = fminf(lo[c], y);
      hi[c] = fmaxf(hi[c], y);
    }
#pragma unroll
  for (int c = 0; c < 6; c++)
    for (int o = 16; o > 0; o >>= 1) {
      lo[c] = fminf(lo[c], __shfl_down_sync(0xffffffffu, lo[c], o));
      hi[c] = fmaxf(hi[c], __shfl_down_sync(0xffffffffu, hi[c], o));
    }
  __shared__ float s[12][8];
  if ((threadIdx.x & 31) == 0)
    for (int c = 0; c < 6; c++) {
      s[2 * c][threadIdx.x >> 5] = lo[c];
      s[2 * c + 1][threadIdx.x >> 5] = hi[c];
    }
  __syncthreads();
  if (threadIdx.x < 12) {
    float v = s[threadIdx.x][0];
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) v = (threadIdx.x & 1) ? fmaxf(v, s[threadIdx.x][w]) : fminf(v, s[threadIdx.x][w]);
    part[blockIdx.x * 12 + threadIdx.x] = v;
  }
}

__global__ void k_normalize_cols(float *__restrict__ Y, int64_t n, Bounds bd) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
#pragma unroll
    for (int c = 0; c < 6; c++) Y[i * 6 + c] = (Y[i * 6 + c] - bd.b[c][0]) / (bd.b[c][1] - bd.b[c][0]);
}

inline unsigned grid1d(int64_t n) {
  const int64_t b = (n + 255) / 256;
  return (unsigned)(b > 148 * 16 ? 148 * 16 : (b < 1 ? 1 : b));
}

}  // namespace

extern "C" {

int hb_mlp_num_params(const HbMlpDesc *d) {
  if (!d) return HB_ERROR_INVALID;
  if (d->hidden1 == 20 && d->hidden2 == 20) return hb::sgs::MlpShape<20, 20>::size;
  if (d->hidden1 == 20 && d->hidden2 == 0) return hb::sgs::MlpShape<20, 0>::size;
  return HB_ERROR_UNSUPPORTED;
}

int hb_mlp_train_step(const HbMlpDesc *d, float *w, float *m, float *v, const float *X, const float *Y, int64_t n, const int32_t *idx, int batch,
                      uint64_t seed, int step, float lr, float *d_work, float *d_loss, float *d_grad, void *stream) {
  const int np = hb_mlp_num_params(d);
  if (np < 0) return np;
  if (batch < 1 || n < 1 || step < 1 || !w || !X || !Y || !d_work || !d_loss) return HB_ERROR_INVALID;
  if (lr != 0.f && (!m || !v)) return HB_ERROR_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  const int nb = (batch + kTB - 1) / kTB;
  float *partial = d_work, *loss_part = d_work + (size_t)nb * np;
  const uint64_t sd = seed ^ ((uint64_t)step * 0x9e3779b97f4a7c15ull);
  if (d->hidden2 == 20) {
    using S = hb::sgs::MlpShape<20, 20>;
    const size_t sm = sizeof(float) * (S::size + (size_t)kTB * Act<20, 20>::size);
    cudaFuncSetAttribute(k_mlp_grad<20, 20>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_mlp_grad<20, 20><<<nb, kTB, sm, s>>>(w, d->leaky_alpha, X, Y, n, idx, batch, sd, partial, loss_part);
  } else {
    using S = hb::sgs::MlpShape<20, 0>;
    const size_t sm = sizeof(float) * (S::size + (size_t)kTB * Act<20, 0>::size);
    cudaFuncSetAttribute(k_mlp_grad<20, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_mlp_grad<20, 0><<<nb, kTB, sm, s>>>(w, d->leaky_alpha, X, Y, n, idx, batch, sd, partial, loss_part);
  }
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float bc1 = 1.f - powf(b1, (float)step), bc2 = 1.f - powf(b2, (float)step);
  k_mlp_adam<<<(np + 255) / 256, 256, 0, s>>>(w, m, v, partial, nb, np, lr, b1, b2, eps, bc1, bc2, loss_part, 1.f / (6.f * (float)batch), d_loss,
                                             d_grad);
  return rc();
}

int hb_mlp_forward(const HbMlpDesc *d, const float *w, const float *X, float *Y, int64_t n, void *stream) {
  const int np = hb_mlp_num_params(d);
  if (np < 0) return np;
  if (n < 0 || !w || !X || !Y) return HB_ERROR_INVALID;
  if (n == 0) return HB_SUCCESS;
  cudaStream_t s = (cudaStream_t)stream;
  const unsigned g = (unsigned)((n + 255) / 256);
  if (d->hidden2 == 20) k_mlp_forward<20, 20><<<g, 256, 0, s>>>(w, d->leaky_alpha, X, Y, n);
  else k_mlp_forward<20, 0><<<g, 256, 0, s>>>(w, d->leaky_alpha, X, Y, n);
  return rc();
}

int hb_sgs_anisotropy(int64_t n, const double *dXdx, double *kmA, double *delta, void *stream) {
  if (n < 0) return HB_ERROR_INVALID;
  if (n) k_sgs_anisotropy<<<grid1d(n), 256, 0, (cudaStream_t)stream>>>(n, dXdx, kmA, delta);
  return rc();
}

int hb_sgs_inputs(int64_t n, const double *G, const double *kmA, const double *delta, const double *nu, double *inputs, double *E, double *gmag,
                  void *stream) {
  if (n < 0) return HB_ERROR_INVALID;
  if (n) k_sgs_inputs<<<grid1d(n), 256, 0, (cudaStream_t)stream>>>(n, G, kmA, delta, nu, inputs, E, gmag);
  return rc();
}

int hb_sgs_stress(int64_t n, const double *out_n, const double *delta, const double *E, const double *gmag, const float bounds[12], double *km_tau,
                  void *stream) {
  if (n < 0 || !bounds) return HB_ERROR_INVALID;
  Bounds bd;
  memcpy(bd.b, bounds, sizeof bd.b);
  if (n) k_sgs_stress<<<grid1d(n), 256, 0, (cudaStream_t)stream>>>(n, out_n, delta, E, gmag, bd, km_tau);
  return rc();
}

int hb_sgs_target_bounds(const float *Y, int64_t n, float *d_work, float bounds[12], void *stream) {
  if (n < 1 || !Y || !d_work || !bounds) return HB_ERROR_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  const unsigned nb = 256;
  k_col_minmax<<<nb, 256, 0, s>>>(Y, n, d_work);
  float h[256 * 12];
  if (cudaMemcpyAsync(h, d_work, sizeof h, cudaMemcpyDeviceToHost, s) != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) return HB_ERROR_CUDA;
  for (int c = 0; c < 12; c++) {
    float v = h[c];
    for (unsigned b = 1; b < nb; b++) v = (c & 1) ? fmaxf(v, h[b * 12 + c]) : fminf(v, h[b * 12 + c]);
    bounds[c] = v;
  }
  return rc();
}

int hb_sgs_normalize_targets(float *Y, int64_t n, const float bounds[12], void *stream) {
  if (n < 0 || !bounds) return HB_ERROR_INVALID;
  Bounds bd;
  memcpy(bd.b, bounds, sizeof bd.b);
  for (int c = 0; c < 6; c++)
    if (!(bd.b[c][1] > bd.b[c][0])) return HB_ERROR_INVALID;
  if (n) k_normalize_cols<<<grid1d(n), 256, 0, (cudaStream_t)stream>>>(Y, n, bd);
  return rc();
}

}  // extern "C"
