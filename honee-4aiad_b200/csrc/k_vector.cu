// k_vector.cu -- device vector kernels and the generic restriction/basis kernels behind the libCEED API.
//
// Vector algebra (set, scale, axpy, norms, precision casts) for CeedVector and for the Krylov solver; element
// restriction gather and a deterministic transpose (sum over a node's element entries in element order, the same
// order as a serial scatter, so E->L results are bit-reproducible); and a direct tensor-basis apply used when a caller
// applies a CeedBasis on its own (CeedBasisApply).  The fused operator kernels live in k_newtonian.cu.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "hb_internal.h"

namespace {

constexpr int kBS = 256;

inline unsigned nblocks(int64_t n, int per = kBS) {
  int64_t b = (n + per - 1) / per;
  return (unsigned)(b > 148 * 64 ? 148 * 64 : (b < 1 ? 1 : b));
}

template <typename T>
__global__ void k_set(T *x, int64_t n, T v) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) x[i] = v;
}
template <typename T>
__global__ void k_scale(T *x, int64_t n, T a) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) x[i] *= a;
}
template <typename T>
__global__ void k_axpby(T *y, T a, T b, const T *x, int64_t n) {  // y = a x + b y
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) y[i] = a * x[i] + b * y[i];
}
template <typename T>
__global__ void k_axpy(T *y, T a, const T *x, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) y[i] += a * x[i];
}
template <typename T>
__global__ void k_pmult(T *w, const T *x, const T *y, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) w[i] = x[i] * y[i];
}
template <typename T>
__global__ void k_recip(T *x, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    if (fabs((double)x[i]) > 2.2e-16) x[i] = T(1) / x[i];
}
template <typename TI, typename TO>
__global__ void k_cast(const TI *x, TO *y, int64_t n, int add) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = add ? TO(y[i] + TO(x[i])) : TO(x[i]);
}

// Two-stage reductions: per-block partials (double accumulation) then one block.  type 0: sum|x|, 1: sum x^2, 2: max|x|,
// 3: dot(x, y).
template <typename T>
__global__ void k_reduce(const T *x, const T *y, int64_t n, int type, double *partial) {
  __shared__ double sh[kBS];
  double acc = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double v = (double)x[i];
    if (type == 0) acc += fabs(v);
    else if (type == 1) acc += v * v;
    else if (type == 2) acc = fmax(acc, fabs(v));
    else acc += v * (double)y[i];
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) sh[threadIdx.x] = type == 2 ? fmax(sh[threadIdx.x], sh[threadIdx.x + s]) : sh[threadIdx.x] + sh[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

// 16-byte vector forms of the kernels in the Krylov inner loop (scale, point-wise multiply, reductions): VW entries per
// load and store where every pointer is 16-byte aligned (checked by the caller), the last n mod VW entries by block 0.
template <typename T>
struct Vec16;
template <>
struct Vec16<float> {
  using V = float4;
  static constexpr int W = 4;
  static __device__ __forceinline__ void get(const V &v, float (&x)[4]) { x[0] = v.x, x[1] = v.y, x[2] = v.z, x[3] = v.w; }
  static __device__ __forceinline__ V make(const float (&x)[4]) { return make_float4(x[0], x[1], x[2], x[3]); }
};
template <>
struct Vec16<double> {
  using V = double2;
  static constexpr int W = 2;
  static __device__ __forceinline__ void get(const V &v, double (&x)[2]) { x[0] = v.x, x[1] = v.y; }
  static __device__ __forceinline__ V make(const double (&x)[2]) { return make_double2(x[0], x[1]); }
};

template <typename T>
__global__ void k_scale_v(T *x, int64_t n, T a) {
  using H = Vec16<T>;
  const int64_t nv = n / H::W;
  typename H::V *xv = reinterpret_cast<typename H::V *>(x);
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nv; j += (int64_t)gridDim.x * blockDim.x) {
    T u[H::W];
    H::get(xv[j], u);
#pragma unroll
    for (int k = 0; k < H::W; k++) u[k] *= a;
    xv[j] = H::make(u);
  }
  if (blockIdx.x == 0 && threadIdx.x < n - nv * H::W) x[nv * H::W + threadIdx.x] *= a;
}
template <typename T>
__global__ void k_pmult_v(T *w, const T *x, const T *y, int64_t n) {
  using H = Vec16<T>;
  const int64_t nv = n / H::W;
  const typename H::V *xv = reinterpret_cast<const typename H::V *>(x), *yv = reinterpret_cast<const typename H::V *>(y);
  typename H::V *wv = reinterpret_cast<typename H::V *>(w);
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nv; j += (int64_t)gridDim.x * blockDim.x) {
    T a[H::W], b[H::W];
    H::get(xv[j], a);
    H::get(yv[j], b);
#pragma unroll
    for (int k = 0; k < H::W; k++) a[k] *= b[k];
    wv[j] = H::make(a);
  }
  if (blockIdx.x == 0 && threadIdx.x < n - nv * H::W) {
    const int64_t i = nv * H::W + threadIdx.x;
    w[i] = x[i] * y[i];
  }
}
template <typename T>
__global__ void k_reduce_v(const T *x, const T *y, int64_t n, int type, double *partial) {
  using H = Vec16<T>;
  __shared__ double sh[kBS];
  const int64_t nv = n / H::W;
  const typename H::V *xv = reinterpret_cast<const typename H::V *>(x), *yv = reinterpret_cast<const typename H::V *>(y);
  double acc = 0;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nv; j += (int64_t)gridDim.x * blockDim.x) {
    T a[H::W], b[H::W];
    H::get(xv[j], a);
    if (type == 3) H::get(yv[j], b);
#pragma unroll
    for (int k = 0; k < H::W; k++) {
      const double v = (double)a[k];
      if (type == 0) acc += fabs(v);
      else if (type == 1) acc += v * v;
      else if (type == 2) acc = fmax(acc, fabs(v));
      else acc += v * (double)b[k];
    }
  }
  if (blockIdx.x == 0 && threadIdx.x < n - nv * H::W) {
    const int64_t i = nv * H::W + threadIdx.x;
    const double v = (double)x[i];
    if (type == 0) acc += fabs(v);
    else if (type == 1) acc += v * v;
    else if (type == 2) acc = fmax(acc, fabs(v));
    else acc += v * (double)y[i];
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) sh[threadIdx.x] = type == 2 ? fmax(sh[threadIdx.x], sh[threadIdx.x + s]) : sh[threadIdx.x] + sh[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

inline bool al16(const void *p) { return p == nullptr || ((uintptr_t)p % 16) == 0; }

// One full wave of a grid-stride kernel at kBS threads (resident blocks per SM x SMs), lowered to a whole multiple of the
// SM count when that exceeds `cap`.
template <typename F>
unsigned wave_blocks(F kernel, unsigned cap) {
  int dev = 0, sms = 0, occ = 0;
  unsigned g = cap;
  if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, kBS, 0) == cudaSuccess && sms > 0 && occ > 0) {
    const unsigned w = (unsigned)occ * (unsigned)sms;
    g = w <= cap ? w : (cap >= (unsigned)sms ? cap / sms * sms : cap);
  }
  return g;
}
template <typename T>
struct VecWaves {
  unsigned scale, pmult, reduce;
  VecWaves()
      : scale(wave_blocks(k_scale_v<T>, 148 * 64)), pmult(wave_blocks(k_pmult_v<T>, 148 * 64)), reduce(wave_blocks(k_reduce_v<T>, 1024)) {}
};
template <typename T>
const VecWaves<T> &vec_waves() {
  static const VecWaves<T> w;
  return w;
}
// blocks for n entries: the full wave, or fewer when n needs fewer (block 0 always exists for the tail)
template <typename T>
unsigned capped(unsigned wave, int64_t n) {
  const int64_t need = (n / Vec16<T>::W + kBS - 1) / kBS;
  return need < 1 ? 1u : (need < (int64_t)wave ? (unsigned)need : wave);
}

__global__ void k_reduce_final(double *partial, int n, int type) {
  __shared__ double sh[kBS];
  double acc = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc = type == 2 ? fmax(acc, partial[i]) : acc + partial[i];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) sh[threadIdx.x] = type == 2 ? fmax(sh[threadIdx.x], sh[threadIdx.x + s]) : sh[threadIdx.x] + sh[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[0] = sh[0];
}

// Restriction gather: e[(el*ncomp + c)*esize + p] = l[off[el*esize+p] + c*cstride]  (offsets) or strided
__global__ void k_restrict(int num_elem, int esize, int ncomp, int cstride, const int32_t *off, const int32_t *strides, const double *l, double *e) {
  const int64_t n = (int64_t)num_elem * esize * ncomp;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const int p = (int)(t % esize);
    const int64_t r = t / esize;
    const int c = (int)(r % ncomp);
    const int64_t el = r / ncomp;
    int64_t li;
    if (off) li = (int64_t)off[el * esize + p] + (int64_t)c * cstride;
    else li = (int64_t)p * strides[0] + (int64_t)c * strides[1] + el * strides[2];
    e[t] = l[li];
  }
}

// Transpose restriction through a CSR map from L-entries to E-entries (sorted by E index): deterministic sums.
__global__ void k_restrict_t_csr(int64_t l_size, const int64_t *ptr, const int64_t *eidx, const double *e, double *l) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < l_size; i += (int64_t)gridDim.x * blockDim.x) {
    double s = l[i];
    for (int64_t k = ptr[i]; k < ptr[i + 1]; k++) s += e[eidx[k]];
    l[i] = s;
  }
}

__global__ void k_restrict_t_strided(int num_elem, int esize, int ncomp, const int32_t *strides, const double *e, double *l) {
  const int64_t n = (int64_t)num_elem * esize * ncomp;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const int p = (int)(t % esize);
    const int64_t r = t / esize;
    const int c = (int)(r % ncomp);
    const int64_t el = r / ncomp;
    l[(int64_t)p * strides[0] + (int64_t)c * strides[1] + el * strides[2]] += e[t];
  }
}

// Direct (non-factorised) tensor basis apply, one thread per output entry.  Used only by CeedBasisApply.
// B, G: [Q][P] 1D matrices in device memory.  emode 1 interp, 2 grad, 16 weight.
__global__ void k_basis(int num_elem, int ncomp, int dim, int P, int Q, int tmode, int emode, const double *B, const double *G, const double *w1,
                        const double *u, double *v) {
  int Pn = 1, Qn = 1;
  for (int d = 0; d < dim; d++) {
    Pn *= P;
    Qn *= Q;
  }
  const int nd = emode == 2 ? dim : 1;
  int64_t nout;
  if (emode == 16) nout = (int64_t)num_elem * Qn;
  else if (tmode) nout = (int64_t)num_elem * ncomp * Pn;  // transpose sums over the nd gradient directions
  else nout = (int64_t)num_elem * ncomp * nd * Qn;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nout; t += (int64_t)gridDim.x * blockDim.x) {
    if (emode == 16) {
      int q = (int)(t % Qn), w = 1;
      double s = 1;
      for (int d = 0; d < dim; d++, w *= Q) s *= w1[(q / w) % Q];
      v[t] = s;
      continue;
    }
    if (!tmode) {  // out [elem][d][comp][Qn] (libCEED E-vector layout at quadrature points per element)
      const int q = (int)(t % Qn);
      int64_t r = t / Qn;
      const int c = (int)(r % ncomp);
      r /= ncomp;
      const int dd = (int)(r % nd);
      const int64_t el = r / nd;
      double s = 0;
      for (int p = 0; p < Pn; p++) {
        double phi = 1;
        int qw = 1, pw = 1;
        for (int d = 0; d < dim; d++, qw *= Q, pw *= P) {
          const int qi = (q / qw) % Q, pi = (p / pw) % P;
          phi *= (emode == 2 && d == dd) ? G[qi * P + pi] : B[qi * P + pi];
        }
        s += phi * u[(el * ncomp + c) * Pn + p];
      }
      v[t] = s;
    } else {  // out [elem][comp][Pn]
      const int p = (int)(t % Pn);
      int64_t r = t / Pn;
      const int c = (int)(r % ncomp);
      const int64_t el = r / ncomp;
      double s = 0;
      for (int dd = 0; dd < nd; dd++)
        for (int q = 0; q < Qn; q++) {
          double phi = 1;
          int qw = 1, pw = 1;
          for (int d = 0; d < dim; d++, qw *= Q, pw *= P) {
            const int qi = (q / qw) % Q, pi = (p / pw) % P;
            phi *= (emode == 2 && d == dd) ? G[qi * P + pi] : B[qi * P + pi];
          }
          s += phi * u[((el * nd + dd) * ncomp + c) * Qn + q];
        }
      v[t] = s;
    }
  }
}

inline int rc() { return cudaGetLastError() == cudaSuccess ? 0 : -5; }

}  // namespace

extern "C" {

int hb_vec_set_f64(double *x, int64_t n, double v, void *s) {
  k_set<<<nblocks(n), kBS, 0, (cudaStream_t)s>>>(x, n, v);
  return rc();
}
int hb_vec_set_f32(float *x, int64_t n, float v, void *s) {
  k_set<<<nblocks(n), kBS, 0, (cudaStream_t)s>>>(x, n, v);
  return rc();
}
int hb_vec_scale_f64(double *x, int64_t n, double a, void *s) {
  if (al16(x)) k_scale_v<<<capped<double>(vec_waves<double>().scale, n), kBS, 0, (cudaStream_t)s>>>(x, n, a);
  else k_scale<<<nblocks(n), kBS, 0, (cudaStream_t)s>>>(x, n, a);
  return rc();
}
int hb_vec_scale_f32(float *x, int64_t n, float a, void *s) {
  if (al16(x)) k_scale_v<<<capped<float>(vec_waves<float>().scale, n), kBS, 0, (cudaStream_t)s>>>(x, n, a);
  else k_scale<<<nblocks(n), kBS, 0, (cudaStream_t)s>>>(x, n, a);
  return rc();
}
int hb_vec_axpy_f64(double *y, double a, const double *x, int64_t n, void *s) {
  k_axpy<<<nblocks(n), kBS, 0, (cudaStream_t)s>>>(y, a, x, n);
  return rc();
}
int hb_vec_axpy_f32(float *y, float a, const float *x, int64_t n, void *s) {
  k_axpy<<<nblocks(n), kBS, 0, (cudaStream_t)s>>>(y, a, x, n);
  return rc();
}
int hb_vec_axpby_f64(double *y, double a, double b, const double *x, int64_t n, void *s) {
  k_axpby<<<nblocks(n), kBS, 0, (cudaStream_t)s>>>(y, a, b, x, n);
  return rc();
}
int hb_vec_axpby_f32(float *y, float a, float b, const float *x, int64_t n, void *s) {
  k_axpby<<<nblocks(n), kBS, 0, (cudaStream_t)s>>>(y, a, b, x, n);
  return rc();
}
int hb_vec_pointwise_mult_f64(double *w, const double *x, const double *y, int64_t n, void *s) {
  if (al16(w) && al16(x) && al16(y)) k_pmult_v<<<capped<double>(vec_waves<double>().pmult, n), kBS, 0, (cudaStream_t)s>>>(w, x, y, n);
  else k_pmult<<<nblocks(n), kBS, 0, (cudaStream_t)s>>>(w, x, y, n);
  return rc();
}
int hb_vec_pointwise_mult_f32(float *w, const float *x, const float *y, int64_t n, void *s) {
  if (al16(w) && al16(x) && al16(y)) k_pmult_v<<<capped<float>(vec_waves<float>().pmult, n), kBS, 0, (cudaStream_t)s>>>(w, x, y, n);
  else k_pmult<<<nblocks(n), kBS, 0, (cudaStream_t)s>>>(w, x, y, n);
  return rc();
}
int hb_vec_reciprocal_f64(double *x, int64_t n, void *s) {
  k_recip<<<nblocks(n), kBS, 0, (cudaStream_t)s>>>(x, n);
  return rc();
}
int hb_vec_f64_to_f32(const double *x, float *y, int64_t n, int add, void *s) {
  k_cast<<<nblocks(n), kBS, 0, (cudaStream_t)s>>>(x, y, n, add);
  return rc();
}
int hb_vec_f32_to_f64(const float *x, double *y, int64_t n, int add, void *s) {
  k_cast<<<nblocks(n), kBS, 0, (cudaStream_t)s>>>(x, y, n, add);
  return rc();
}

// Reductions write the result to *result (host) after synchronising the stream; scratch holds >= 1024 doubles.
static int reduce_common(int type, double *scratch, double *result, void *s) {
  cudaStream_t st = (cudaStream_t)s;
  k_reduce_final<<<1, kBS, 0, st>>>(scratch, 1024, type);
  if (cudaMemcpyAsync(result, scratch, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess) return -5;
  return cudaStreamSynchronize(st) == cudaSuccess ? 0 : -5;
}
int hb_vec_reduce_f64(const double *x, const double *y, int64_t n, int type, double *scratch, double *result, void *s) {
  cudaStream_t st = (cudaStream_t)s;
  cudaMemsetAsync(scratch, 0, 1024 * sizeof(double), st);
  if (al16(x) && al16(y)) k_reduce_v<<<capped<double>(vec_waves<double>().reduce, n), kBS, 0, st>>>(x, y, n, type, scratch);
  else k_reduce<<<1024, kBS, 0, st>>>(x, y, n, type, scratch);
  return reduce_common(type, scratch, result, s);
}
int hb_vec_reduce_f32(const float *x, const float *y, int64_t n, int type, double *scratch, double *result, void *s) {
  cudaStream_t st = (cudaStream_t)s;
  cudaMemsetAsync(scratch, 0, 1024 * sizeof(double), st);
  if (al16(x) && al16(y)) k_reduce_v<<<capped<float>(vec_waves<float>().reduce, n), kBS, 0, st>>>(x, y, n, type, scratch);
  else k_reduce<<<1024, kBS, 0, st>>>(x, y, n, type, scratch);
  return reduce_common(type, scratch, result, s);
}

int hb_restrict_apply(int num_elem, int esize, int ncomp, int cstride, const int32_t *d_off, const int32_t *d_strides, const double *l, double *e,
                      void *s) {
  const int64_t n = (int64_t)num_elem * esize * ncomp;
  k_restrict<<<nblocks(n), kBS, 0, (cudaStream_t)s>>>(num_elem, esize, ncomp, cstride, d_off, d_strides, l, e);
  return rc();
}
int hb_restrict_apply_t_csr(int64_t l_size, const int64_t *d_ptr, const int64_t *d_eidx, const double *e, double *l, void *s) {
  k_restrict_t_csr<<<nblocks(l_size), kBS, 0, (cudaStream_t)s>>>(l_size, d_ptr, d_eidx, e, l);
  return rc();
}
int hb_restrict_apply_t_strided(int num_elem, int esize, int ncomp, const int32_t *d_strides, const double *e, double *l, void *s) {
  const int64_t n = (int64_t)num_elem * esize * ncomp;
  k_restrict_t_strided<<<nblocks(n), kBS, 0, (cudaStream_t)s>>>(num_elem, esize, ncomp, d_strides, e, l);
  return rc();
}
int hb_basis_apply_generic(int num_elem, int ncomp, int dim, int P, int Q, int tmode, int emode, const double *d_B, const double *d_G,
                           const double *d_w, const double *u, double *v, void *s) {
  int64_t Pn = 1, Qn = 1;
  for (int d = 0; d < dim; d++) {
    Pn *= P;
    Qn *= Q;
  }
  const int64_t n = emode == 16 ? (int64_t)num_elem * Qn : (tmode ? (int64_t)num_elem * ncomp * Pn : (int64_t)num_elem * ncomp * (emode == 2 ? dim : 1) * Qn);
  k_basis<<<nblocks(n), kBS, 0, (cudaStream_t)s>>>(num_elem, ncomp, dim, P, Q, tmode, emode, d_B, d_G, d_w, u, v);
  return rc();
}

}  // extern "C"
