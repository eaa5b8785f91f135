// k_newtonian.cu -- fused element kernels of the Newtonian operator for sm_100a.
//
// One kernel launch per element colour.  Each CTA walks a strided slice of that colour's element list and, per
// element, does the whole libCEED operator chain in shared memory:
//   restriction gather (L-vector -> E-vector, int32 offsets, node-interleaved 5 components)
//   -> tensor interpolation and gradient by sum factorisation (x, y, z fibre passes; the gradient uses the collocated
//      derivative D = G B^+ on the quadrature grid, exact for tensor H1 bases with Q >= P)
//   -> point-wise IFunction / IJacobian / linearised diagonal (newtonian_qf.cuh), one thread per quadrature point, with
//      qdata read and jac_data written coalesced in the [elem][comp][qpt] layout
//   -> transpose gradient + interpolation back to the element nodes
//   -> scatter-add into the L-vector without atomics: elements of one colour share no node, colours run in stream order.
// Reference semantics: libCEED CeedOperatorApply / CeedOperatorLinearAssembleDiagonal as called from src/setupts.c:109,
// src/mat-ceed.c:1618,1669 on the operators built in src/setuplibceed.c:209-269.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include "honee_b200.h"
#include "newtonian_qf.cuh"

namespace hb {

constexpr int kMaxP = 8;

template <typename T>
struct Basis1D {
  T B[kMaxP * kMaxP];  // interp  [Q][P]
  T D[kMaxP * kMaxP];  // collocated derivative on the quadrature points [Q][Q]
  T Gx[4];             // unused padding keeps the struct size a multiple of 16 bytes
};

template <typename T>
__host__ __device__ constexpr int nthreads_for(int Q) {
  return ((Q * Q * Q + 31) / 32) * 32;
}

// ---------------------------------------------------------------------------------------------------------------------
// fibre passes over shared-memory tensors.  All arrays are [comp][n2][n1][n0] with n0 fastest.
// M is row-major [rows][cols]; forward passes use out[i] = sum_a M[i][a] in[a], transposed passes out[a] = sum_i M[i][a] in[i].

// along n0: in [NF][NIN] contiguous rows -> out [NF][NOUT]
template <int NF, int NIN, int NOUT, bool TR, int NT, typename T>
__device__ __forceinline__ void pass0(const T *__restrict__ in, T *__restrict__ out, const T *__restrict__ M, int ldm) {
  for (int f = threadIdx.x; f < NF; f += NT) {
    T x[NIN];
#pragma unroll
    for (int a = 0; a < NIN; a++) x[a] = in[f * NIN + a];
#pragma unroll
    for (int i = 0; i < NOUT; i++) {
      T s = 0;
#pragma unroll
      for (int a = 0; a < NIN; a++) s += (TR ? M[a * ldm + i] : M[i * ldm + a]) * x[a];
      out[f * NOUT + i] = s;
    }
  }
}

// along n1: in [NC][N2][NIN][N0] -> out [NC][N2][NOUT][N0]
template <int NC, int N2, int N0, int NIN, int NOUT, bool TR, int NT, typename T>
__device__ __forceinline__ void pass1(const T *__restrict__ in, T *__restrict__ out, const T *__restrict__ M, int ldm) {
  for (int f = threadIdx.x; f < NC * N2 * N0; f += NT) {
    const int x = f % N0, cz = f / N0;
    const T *src = in + cz * NIN * N0 + x;
    T *dst = out + cz * NOUT * N0 + x;
    T v[NIN];
#pragma unroll
    for (int a = 0; a < NIN; a++) v[a] = src[a * N0];
#pragma unroll
    for (int i = 0; i < NOUT; i++) {
      T s = 0;
#pragma unroll
      for (int a = 0; a < NIN; a++) s += (TR ? M[a * ldm + i] : M[i * ldm + a]) * v[a];
      dst[i * N0] = s;
    }
  }
}

// ---------------------------------------------------------------------------------------------------------------------
// kernel arguments

template <typename T>
struct ElemArgs {
  const int32_t *offsets;  // [E][P^3] node*5
  const int32_t *elems;    // element ids of this colour
  int n_elems;
  Basis1D<T> basis;
  PhysConst<T> pc;
  const double *qdata;     // [E][10][Q^3]
  const double *x_elem;    // [E][3][8] vertex coordinates (IDL only), may be null
  int num_jd;              // 14 or 15
};

template <typename T>
__device__ __forceinline__ void load_qdata(const double *__restrict__ qd, int Q3, int q, T &wdetJ, T X[3][3]) {
  wdetJ = T(__ldg(qd + q));
#pragma unroll
  for (int k = 0; k < 9; k++) X[k / 3][k % 3] = T(__ldg(qd + (1 + k) * Q3 + q));
}

// x coordinate of quadrature point (i,j,k) from the element's vertex coordinates (trilinear coordinate field).
template <int Q>
__device__ __forceinline__ double qpt_x0(const double *__restrict__ xe, const double *qref, int i, int j, int k) {
  const double xi[3] = {qref[i], qref[j], qref[k]};
  double s = 0;
#pragma unroll
  for (int v = 0; v < 8; v++) {
    double w = 1;
#pragma unroll
    for (int d = 0; d < 3; d++) w *= ((v >> d) & 1) ? 0.5 * (1 + xi[d]) : 0.5 * (1 - xi[d]);
    s += w * __ldg(xe + v);
  }
  return s;
}

struct QRef {
  double x[kMaxP];
};

// L2 prefetch of the 16-byte-aligned part of [p, p + bytes) with one bulk (TMA-engine) request; issued by one thread.
__device__ __forceinline__ void prefetch_l2_bulk(const void *p, size_t bytes) {
  const uintptr_t a = (uintptr_t)p, lo = (a + 15) & ~(uintptr_t)15, hi = (a + bytes) & ~(uintptr_t)15;
  if (hi > lo) asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(lo), "r"((unsigned)(hi - lo)) : "memory");
}

__device__ __forceinline__ void prefetch_l2(const void *p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// Warm L2 with the next element's node values (all L-vectors it gathers or scatter-adds) and its per-point data.
template <int P, typename TL>
__device__ __forceinline__ void prefetch_element(const int32_t *__restrict__ offsets, int e, const TL *const *vecs, int nvec, const void *blk0,
                                                 size_t bytes0, const void *blk1, size_t bytes1) {
  constexpr int P3 = P * P * P;
  if (threadIdx.x < P3) {
    const int64_t o = __ldg(offsets + (int64_t)e * P3 + threadIdx.x);
    for (int v = 0; v < nvec; v++) {
      const char *a = (const char *)(vecs[v] + o);
      prefetch_l2(a);
      prefetch_l2(a + 5 * sizeof(TL) - 1);
    }
  } else if (threadIdx.x == P3) {
    if (blk0) prefetch_l2_bulk(blk0, bytes0);
    if (blk1) prefetch_l2_bulk(blk1, bytes1);
  }
}

// ---------------------------------------------------------------------------------------------------------------------
// Forward: gather NV input L-vectors (5 comps each) and produce interp [NV*5][Q3] and, for the first vector, the
// reference gradient [3][5][Q3].  Shared layout (doubles or T): sN [NV*5][P3], s1 [NV*5][P][P][Q], s2 [NV*5][P][Q][Q].
template <int P, int Q, int NV, int NT, typename T, typename TL>
__device__ __forceinline__ void forward(const ElemArgs<T> &a, int e, const TL *const *l_in, T *sN, T *s1, T *s2, T *sU, T *sG) {
  constexpr int P3 = P * P * P, Q2 = Q * Q, Q3 = Q2 * Q;
  constexpr int NC = NV * 5;
  const int32_t *off = a.offsets + (int64_t)e * P3;
  for (int t = threadIdx.x; t < P3 * 5; t += NT) {
    const int p = t / 5, c = t % 5;
    const int64_t o = __ldg(off + p) + c;
#pragma unroll
    for (int v = 0; v < NV; v++) sN[(v * 5 + c) * P3 + p] = T(l_in[v][o]);
  }
  __syncthreads();
  pass0<NC * P * P, P, Q, false, NT>(sN, s1, a.basis.B, P);
  __syncthreads();
  pass1<NC, P, Q, P, Q, false, NT>(s1, s2, a.basis.B, P);
  __syncthreads();
  // z pass: interpolate along z and, for the first vector, differentiate along z on the quadrature grid
  for (int f = threadIdx.x; f < NC * Q2; f += NT) {
    const int yx = f % Q2, c = f / Q2;
    T in[P], val[Q];
#pragma unroll
    for (int cz = 0; cz < P; cz++) in[cz] = s2[(c * P + cz) * Q2 + yx];
#pragma unroll
    for (int k = 0; k < Q; k++) {
      T s = 0;
#pragma unroll
      for (int cz = 0; cz < P; cz++) s += a.basis.B[k * P + cz] * in[cz];
      val[k] = s;
      sU[c * Q3 + k * Q2 + yx] = s;
    }
    if (c < 5) {
#pragma unroll
      for (int k = 0; k < Q; k++) {
        T s = 0;
#pragma unroll
        for (int l = 0; l < Q; l++) s += a.basis.D[k * Q + l] * val[l];
        sG[(2 * 5 + c) * Q3 + k * Q2 + yx] = s;
      }
    }
  }
  __syncthreads();
  // x and y derivatives of the first vector on the quadrature grid
  for (int f = threadIdx.x; f < 2 * 5 * Q2; f += NT) {
    const int dir = f / (5 * Q2), r = f % (5 * Q2), c = r / Q2, rem = r % Q2;
    const T *src;
    T *dst;
    int stride;
    if (dir == 0) {  // fibre along x at (k,j) = rem
      src = sU + c * Q3 + rem * Q;
      dst = sG + (0 * 5 + c) * Q3 + rem * Q;
      stride = 1;
    } else {  // fibre along y at (k, i): rem = k*Q + i
      const int k = rem / Q, i = rem % Q;
      src = sU + c * Q3 + k * Q2 + i;
      dst = sG + (1 * 5 + c) * Q3 + k * Q2 + i;
      stride = Q;
    }
    T val[Q];
#pragma unroll
    for (int l = 0; l < Q; l++) val[l] = src[l * stride];
#pragma unroll
    for (int k = 0; k < Q; k++) {
      T s = 0;
#pragma unroll
      for (int l = 0; l < Q; l++) s += a.basis.D[k * Q + l] * val[l];
      dst[k * stride] = s;
    }
  }
  __syncthreads();
}

// Transpose: v [5][Q3] (in sU) and grad_v [3][5][Q3] (in sG) back to the element nodes, then scatter-add into l_out.
// Scratch: sW1 [5][Q3], sW2 [5][Q3], sT2 [5][P][Q][Q], sT1 [5][P][P][Q], sF [P3][5].
template <int P, int Q, int NT, typename T, typename TL>
__device__ __forceinline__ void transpose_scatter(const ElemArgs<T> &a, int e, TL *l_out, const T *sU, const T *sG, T *sW1, T *sW2, T *sT2, T *sT1,
                                                  T *sF) {
  constexpr int P3 = P * P * P, Q2 = Q * Q, Q3 = Q2 * Q;
  for (int f = threadIdx.x; f < 2 * 5 * Q2; f += NT) {
    const int dir = f / (5 * Q2), r = f % (5 * Q2), c = r / Q2, rem = r % Q2;
    int base, stride;
    if (dir == 0) {
      base = rem * Q;
      stride = 1;
    } else {
      base = (rem / Q) * Q2 + (rem % Q);
      stride = Q;
    }
    const T *g = sG + (dir * 5 + c) * Q3 + base;
    T gv[Q];
#pragma unroll
    for (int l = 0; l < Q; l++) gv[l] = g[l * stride];
    if (dir == 0) {
      const T *v = sU + c * Q3 + base;
      T *w = sW1 + c * Q3 + base;
#pragma unroll
      for (int i = 0; i < Q; i++) {
        T s = v[i];
#pragma unroll
        for (int l = 0; l < Q; l++) s += a.basis.D[l * Q + i] * gv[l];
        w[i] = s;
      }
    } else {
      T *w = sW2 + c * Q3 + base;
#pragma unroll
      for (int j = 0; j < Q; j++) {
        T s = 0;
#pragma unroll
        for (int l = 0; l < Q; l++) s += a.basis.D[l * Q + j] * gv[l];
        w[j * Q] = s;
      }
    }
  }
  __syncthreads();
  for (int f = threadIdx.x; f < 5 * Q2; f += NT) {
    const int yx = f % Q2, c = f / Q2;
    T w[Q], gz[Q];
#pragma unroll
    for (int l = 0; l < Q; l++) gz[l] = sG[(2 * 5 + c) * Q3 + l * Q2 + yx];
#pragma unroll
    for (int k = 0; k < Q; k++) {
      T s = sW1[c * Q3 + k * Q2 + yx] + sW2[c * Q3 + k * Q2 + yx];
#pragma unroll
      for (int l = 0; l < Q; l++) s += a.basis.D[l * Q + k] * gz[l];
      w[k] = s;
    }
#pragma unroll
    for (int cz = 0; cz < P; cz++) {
      T s = 0;
#pragma unroll
      for (int k = 0; k < Q; k++) s += a.basis.B[k * P + cz] * w[k];
      sT2[(c * P + cz) * Q2 + yx] = s;
    }
  }
  __syncthreads();
  pass1<5, P, Q, Q, P, true, NT>(sT2, sT1, a.basis.B, P);
  __syncthreads();
  // x pass writes node-major [p][c] for a coalesced scatter
  for (int f = threadIdx.x; f < 5 * P * P; f += NT) {
    const int c = f / (P * P), zb = f % (P * P);
    T in[Q];
#pragma unroll
    for (int i = 0; i < Q; i++) in[i] = sT1[f * Q + i];
#pragma unroll
    for (int pa = 0; pa < P; pa++) {
      T s = 0;
#pragma unroll
      for (int i = 0; i < Q; i++) s += a.basis.B[i * P + pa] * in[i];
      sF[(zb * P + pa) * 5 + c] = s;
    }
  }
  __syncthreads();
  const int32_t *off = a.offsets + (int64_t)e * P3;
  for (int t = threadIdx.x; t < P3 * 5; t += NT) {
    const int p = t / 5, c = t % 5;
    const int64_t o = __ldg(off + p) + c;
    l_out[o] += TL(sF[t]);
  }
}

template <int P, int Q>
struct SmemLayout {
  static constexpr int P3 = P * P * P, Q2 = Q * Q, Q3 = Q2 * Q;
  // forward buffers for up to two input vectors
  static constexpr int nN = 10 * P3, n1 = 10 * P * P * Q, n2 = 10 * P * Q2;
  static constexpr int nU = 10 * Q3, nG = 15 * Q3;
  static constexpr int total = nN + n1 + n2 + nU + nG;
  static_assert(5 * P * Q2 <= nN, "sT2 fits in sN");
  static_assert(5 * P * P * Q <= n1, "sT1 fits in s1");
  static_assert(5 * Q3 <= n2 || 5 * Q3 <= nN + n1, "w2 fits");
};

// ---------------------------------------------------------------------------------------------------------------------
// IFunction

struct IfunctionPtrs {
  const double *q, *q_dot;
  double *jac_data;   // [E][num_jd][Q3], may be null
  float *jac_f32;     // [E][num_jd][Q3] single-precision shadow for the mixed-precision Jacobian, may be null
  double *v;
  QRef qref;
};

template <int P, int Q>
__global__ void __launch_bounds__(nthreads_for<double>(Q), 3) k_ifunction(const ElemArgs<double> a, const IfunctionPtrs p) {
  constexpr int NT = nthreads_for<double>(Q);
  using L = SmemLayout<P, Q>;
  extern __shared__ __align__(16) double smem[];
  double *sN = smem, *s1 = sN + L::nN, *s2 = s1 + L::n1, *sU = s2 + L::n2, *sG = sU + L::nU;
  double *sD = sU + 5 * L::Q3;  // interp of q_dot
  const double *lin[2] = {p.q, p.q_dot};
  const double *pre[3] = {p.q, p.q_dot, p.v};
  for (int idx = blockIdx.x; idx < a.n_elems; idx += gridDim.x) {
    const int e = a.elems[idx];
    if (idx == blockIdx.x)
      prefetch_element<P, double>(a.offsets, e, pre, 3, a.qdata + (int64_t)e * 10 * L::Q3, sizeof(double) * 10 * L::Q3, nullptr, 0);
    if (idx + gridDim.x < a.n_elems) {
      const int en = a.elems[idx + gridDim.x];
      prefetch_element<P, double>(a.offsets, en, pre, 3, a.qdata + (int64_t)en * 10 * L::Q3, sizeof(double) * 10 * L::Q3, nullptr, 0);
    }
    forward<P, Q, 2, NT, double, double>(a, e, lin, sN, s1, s2, sU, sG);
    const int q = threadIdx.x;
    if (q < L::Q3) {
      double qi[5], qd[5], gref[3][5], wdetJ, X[3][3], v[5], gv[3][5], jd[15];
#pragma unroll
      for (int c = 0; c < 5; c++) {
        qi[c] = sU[c * L::Q3 + q];
        qd[c] = sD[c * L::Q3 + q];
#pragma unroll
        for (int d = 0; d < 3; d++) gref[d][c] = sG[(d * 5 + c) * L::Q3 + q];
      }
      load_qdata(a.qdata + (int64_t)e * 10 * L::Q3, L::Q3, q, wdetJ, X);
      double x0 = 0;
      if (a.pc.idl_enable) x0 = qpt_x0<Q>(a.x_elem + (int64_t)e * 24, p.qref.x, q % Q, (q / Q) % Q, q / (Q * Q));
      ifunction_point<double>(a.pc, qi, gref, qd, wdetJ, X, x0, v, gv, jd);
#pragma unroll
      for (int c = 0; c < 5; c++) {
        sU[c * L::Q3 + q] = v[c];
#pragma unroll
        for (int d = 0; d < 3; d++) sG[(d * 5 + c) * L::Q3 + q] = gv[d][c];
      }
      if (p.jac_data) {
        double *jdp = p.jac_data + (int64_t)e * a.num_jd * L::Q3 + q;
#pragma unroll
        for (int c = 0; c < 14; c++) jdp[c * L::Q3] = jd[c];
        if (a.num_jd > 14) jdp[14 * L::Q3] = jd[14];
      }
      if (p.jac_f32) {
        float *jdp = p.jac_f32 + (int64_t)e * a.num_jd * L::Q3 + q;
#pragma unroll
        for (int c = 0; c < 14; c++) jdp[c * L::Q3] = float(jd[c]);
        if (a.num_jd > 14) jdp[14 * L::Q3] = float(jd[14]);
      }
    }
    __syncthreads();
    // transpose scratch: w1 in the q_dot interp slot, w2 in s2, sT2 in sN, sT1 in s1, final node values in s2
    transpose_scatter<P, Q, NT, double, double>(a, e, p.v, sU, sG, sD, s2, sN, s1, s2);
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------------------------------------------------
// IJacobian action (FP64 or FP32 arithmetic; jac_data and L-vectors in the same precision, qdata FP64)

template <typename T>
struct IjacobianPtrs {
  const T *dq;
  const T *jac_data;  // [E][num_jd][Q3]
  T *v;
};

template <int P, int Q, typename T>
__global__ void __launch_bounds__(nthreads_for<T>(Q), 3) k_ijacobian(const ElemArgs<T> a, const IjacobianPtrs<T> p) {
  constexpr int NT = nthreads_for<T>(Q);
  using L = SmemLayout<P, Q>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *smem = reinterpret_cast<T *>(smem_raw);
  T *sN = smem, *s1 = sN + L::nN, *s2 = s1 + L::n1, *sU = s2 + L::n2, *sG = sU + L::nU;
  T *sW1 = sU + 5 * L::Q3;
  const T *lin[1] = {p.dq};
  const T *pre[2] = {p.dq, p.v};
  const size_t jbytes = sizeof(T) * (size_t)a.num_jd * L::Q3;
  for (int idx = blockIdx.x; idx < a.n_elems; idx += gridDim.x) {
    const int e = a.elems[idx];
    if (idx == blockIdx.x)
      prefetch_element<P, T>(a.offsets, e, pre, 2, a.qdata + (int64_t)e * 10 * L::Q3, sizeof(double) * 10 * L::Q3,
                             p.jac_data + (int64_t)e * a.num_jd * L::Q3, jbytes);
    if (idx + gridDim.x < a.n_elems) {
      const int en = a.elems[idx + gridDim.x];
      prefetch_element<P, T>(a.offsets, en, pre, 2, a.qdata + (int64_t)en * 10 * L::Q3, sizeof(double) * 10 * L::Q3,
                             p.jac_data + (int64_t)en * a.num_jd * L::Q3, jbytes);
    }
    forward<P, Q, 1, NT, T, T>(a, e, lin, sN, s1, s2, sU, sG);
    const int q = threadIdx.x;
    if (q < L::Q3) {
      T dq[5], gref[3][5], wdetJ, X[3][3], v[5], gv[3][5], jd[15];
#pragma unroll
      for (int c = 0; c < 5; c++) {
        dq[c] = sU[c * L::Q3 + q];
#pragma unroll
        for (int d = 0; d < 3; d++) gref[d][c] = sG[(d * 5 + c) * L::Q3 + q];
      }
      const T *jdp = p.jac_data + (int64_t)e * a.num_jd * L::Q3 + q;
#pragma unroll
      for (int c = 0; c < 14; c++) jd[c] = jdp[c * L::Q3];
      jd[14] = a.num_jd > 14 ? jdp[14 * L::Q3] : T(0);
      load_qdata(a.qdata + (int64_t)e * 10 * L::Q3, L::Q3, q, wdetJ, X);
      ijacobian_point<T>(a.pc, jd, dq, gref, wdetJ, X, v, gv);
#pragma unroll
      for (int c = 0; c < 5; c++) {
        sU[c * L::Q3 + q] = v[c];
#pragma unroll
        for (int d = 0; d < 3; d++) sG[(d * 5 + c) * L::Q3 + q] = gv[d][c];
      }
    }
    __syncthreads();
    transpose_scatter<P, Q, NT, T, T>(a, e, p.v, sU, sG, sW1, s2, sN, s1, s2);
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------------------------------------------------
// Diagonal of the IJacobian operator (libCEED CeedOperatorLinearAssembleDiagonal semantics): at every quadrature point
// linearise the point-wise Jacobian for each component c with unit inputs in the four eval modes (interp, grad x/y/z),
// keep the 4x4 block A_c[m][n] = d out(m,c) / d in(n,c), and contract sum_q phi_m(q,p) A_c[m][n](q) phi_n(q,p) by sum
// factorisation with products of 1D basis rows.  The 16 (m,n) pairs share 10 distinct product triples.

template <typename T>
struct DiagArgs {
  const T *jac_data;
  T *diag;
  T G1[kMaxP * kMaxP];  // reference 1D gradient [Q][P]
};

template <int P, int Q, typename T>
__global__ void __launch_bounds__(nthreads_for<T>(Q), 2) k_diagonal(const ElemArgs<T> a, const DiagArgs<T> p) {
  constexpr int NT = nthreads_for<T>(Q);
  constexpr int P3 = P * P * P, Q2 = Q * Q, Q3 = Q2 * Q;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *smem = reinterpret_cast<T *>(smem_raw);
  T *sA = smem;                // [10][Q3]
  T *sT1 = sA + 10 * Q3;       // [Q][Q][P]  after x contraction
  T *sT2 = sT1 + Q2 * P;       // [Q][P][P]  after y contraction
  T *sOut = sT2 + Q * P * P;   // [5][P3]
  // product-matrix selectors for the 10 (m,n) combinations: number of x/y/z derivatives (0: B*B, 1: B*G, 2: G*G)
  // combo order: II, IGx, IGy, IGz, GxGx, GyGy, GzGz, GxGy, GxGz, GyGz
  constexpr int cx[10] = {0, 1, 0, 0, 2, 0, 0, 1, 1, 0};
  constexpr int cy[10] = {0, 0, 1, 0, 0, 2, 0, 1, 0, 1};
  constexpr int cz[10] = {0, 0, 0, 1, 0, 0, 2, 0, 1, 1};
  for (int idx = blockIdx.x; idx < a.n_elems; idx += gridDim.x) {
    const int e = a.elems[idx];
    for (int c = 0; c < 5; c++) {
      const int q = threadIdx.x;
      if (q < Q3) {
        T jd[15], wdetJ, X[3][3];
        const T *jdp = p.jac_data + (int64_t)e * a.num_jd * Q3 + q;
#pragma unroll
        for (int k = 0; k < 14; k++) jd[k] = jdp[k * Q3];
        jd[14] = a.num_jd > 14 ? jdp[14 * Q3] : T(0);
        load_qdata(a.qdata + (int64_t)e * 10 * Q3, Q3, q, wdetJ, X);
        T A[4][4];
#pragma unroll 1
        for (int n = 0; n < 4; n++) {
          T dq[5] = {0, 0, 0, 0, 0}, gref[3][5] = {{0, 0, 0, 0, 0}, {0, 0, 0, 0, 0}, {0, 0, 0, 0, 0}}, v[5], gv[3][5];
          if (n == 0) dq[c] = 1;
          else gref[n - 1][c] = 1;
          ijacobian_point<T>(a.pc, jd, dq, gref, wdetJ, X, v, gv);
          A[0][n] = v[c];
          A[1][n] = gv[0][c];
          A[2][n] = gv[1][c];
          A[3][n] = gv[2][c];
        }
        sA[0 * Q3 + q] = A[0][0];
        sA[1 * Q3 + q] = A[0][1] + A[1][0];
        sA[2 * Q3 + q] = A[0][2] + A[2][0];
        sA[3 * Q3 + q] = A[0][3] + A[3][0];
        sA[4 * Q3 + q] = A[1][1];
        sA[5 * Q3 + q] = A[2][2];
        sA[6 * Q3 + q] = A[3][3];
        sA[7 * Q3 + q] = A[1][2] + A[2][1];
        sA[8 * Q3 + q] = A[1][3] + A[3][1];
        sA[9 * Q3 + q] = A[2][3] + A[3][2];
      }
      for (int t = threadIdx.x; t < P3; t += NT) sOut[c * P3 + t] = 0;
      __syncthreads();
#pragma unroll
      for (int m = 0; m < 10; m++) {
        // x: T1[k][j][pa] = sum_i X(i,pa) A[k][j][i]
        for (int f = threadIdx.x; f < Q2 * P; f += NT) {
          const int pa = f % P, kj = f / P;
          T s = 0;
#pragma unroll
          for (int i = 0; i < Q; i++) {
            const T b = a.basis.B[i * P + pa], g = p.G1[i * P + pa];
            const T w = cx[m] == 0 ? b * b : (cx[m] == 1 ? b * g : g * g);
            s += w * sA[m * Q3 + kj * Q + i];
          }
          sT1[kj * P + pa] = s;
        }
        __syncthreads();
        for (int f = threadIdx.x; f < Q * P * P; f += NT) {
          const int pa = f % P, pb = (f / P) % P, k = f / (P * P);
          T s = 0;
#pragma unroll
          for (int j = 0; j < Q; j++) {
            const T b = a.basis.B[j * P + pb], g = p.G1[j * P + pb];
            const T w = cy[m] == 0 ? b * b : (cy[m] == 1 ? b * g : g * g);
            s += w * sT1[(k * Q + j) * P + pa];
          }
          sT2[(k * P + pb) * P + pa] = s;
        }
        __syncthreads();
        for (int f = threadIdx.x; f < P3; f += NT) {
          const int pab = f % (P * P), pc_ = f / (P * P);
          T s = 0;
#pragma unroll
          for (int k = 0; k < Q; k++) {
            const T b = a.basis.B[k * P + pc_], g = p.G1[k * P + pc_];
            const T w = cz[m] == 0 ? b * b : (cz[m] == 1 ? b * g : g * g);
            s += w * sT2[k * P * P + pab];
          }
          sOut[c * P3 + f] += s;
        }
        __syncthreads();
      }
    }
    const int32_t *off = a.offsets + (int64_t)e * P3;
    for (int t = threadIdx.x; t < P3 * 5; t += NT) {
      const int pp = t / 5, c = t % 5;
      p.diag[__ldg(off + pp) + c] += sOut[c * P3 + pp];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------------------------------------------------
// Geometric factors (qfunctions/setupgeo.h:42-56, utils.h:201-216): trilinear coordinates -> w detJ, dX/dx.

__global__ void k_setup_qdata(int num_elem, int Q, const double *__restrict__ x_elem, QRef qref, QRef qw, double *__restrict__ qdata) {
  const int Q3 = Q * Q * Q;
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (int64_t)num_elem * Q3) return;
  const int64_t e = gid / Q3;
  const int q = (int)(gid % Q3);
  const int ii[3] = {q % Q, (q / Q) % Q, q / (Q * Q)};
  const double *xe = x_elem + e * 24;
  double J[3][3];  // J[c][d] = dx_c / dX_d
  for (int c = 0; c < 3; c++)
    for (int d = 0; d < 3; d++) {
      double s = 0;
      for (int v = 0; v < 8; v++) {
        double w = 1;
        for (int dd = 0; dd < 3; dd++) {
          const int bit = (v >> dd) & 1;
          const double xi = qref.x[ii[dd]];
          w *= (dd == d) ? (bit ? 0.5 : -0.5) : (bit ? 0.5 * (1 + xi) : 0.5 * (1 - xi));
        }
        s += w * xe[c * 8 + v];
      }
      J[c][d] = s;
    }
  double A[3][3];
  A[0][0] = J[1][1] * J[2][2] - J[1][2] * J[2][1];
  A[0][1] = J[0][2] * J[2][1] - J[0][1] * J[2][2];
  A[0][2] = J[0][1] * J[1][2] - J[0][2] * J[1][1];
  A[1][0] = J[1][2] * J[2][0] - J[1][0] * J[2][2];
  A[1][1] = J[0][0] * J[2][2] - J[0][2] * J[2][0];
  A[1][2] = J[0][2] * J[1][0] - J[0][0] * J[1][2];
  A[2][0] = J[1][0] * J[2][1] - J[1][1] * J[2][0];
  A[2][1] = J[0][1] * J[2][0] - J[0][0] * J[2][1];
  A[2][2] = J[0][0] * J[1][1] - J[0][1] * J[1][0];
  const double det = J[0][0] * A[0][0] + J[1][0] * A[0][1] + J[2][0] * A[0][2];
  const double inv = 1 / det;
  double *qd = qdata + e * 10 * Q3 + q;
  qd[0] = qw.x[ii[0]] * qw.x[ii[1]] * qw.x[ii[2]] * det;
  for (int k = 0; k < 9; k++) qd[(1 + k) * Q3] = A[k / 3][k % 3] * inv;
}

// ---------------------------------------------------------------------------------------------------------------------
// host side

template <typename T>
static PhysConst<T> make_phys(const HbNewtonianContext &c) {
  PhysConst<T> p;
  p.mu = T(c.gas.mu);
  p.lambda = T(c.gas.lambda);
  p.k = T(c.gas.k);
  p.cv = T(c.gas.cv);
  p.inv_cv = T(1.0 / c.gas.cv);
  p.gm1 = T(c.gas.cp / c.gas.cv - 1);
  p.Rgas = T(c.gas.cp - c.gas.cv);
  for (int i = 0; i < 3; i++) p.g[i] = T(c.g[i]);
  p.shift = T(c.ijacobian_time_shift);
  p.Ctau_C = T(c.tau_coeffs.Ctau_C);
  p.Ctau_M = T(c.tau_coeffs.Ctau_M);
  p.Ctau_E = T(c.tau_coeffs.Ctau_E);
  p.Ctau_v = T(c.tau_coeffs.Ctau_v);
  p.dts = T(c.tau_coeffs.Ctau_t / c.dt);
  p.stab = (int)c.stabilization;
  p.idl_enable = c.idl_enable ? 1 : 0;
  p.idl_amplitude = T(c.idl_amplitude);
  p.idl_start = T(c.idl_start);
  p.idl_length = T(c.idl_length);
  p.idl_pressure = T(c.idl_pressure);
  return p;
}

template <typename T>
static void fill_basis(const HbElemOp *op, Basis1D<T> &b) {
  memset(&b, 0, sizeof b);
  for (int i = 0; i < op->Q * op->P; i++) b.B[i] = T(op->interp1d[i]);
  for (int i = 0; i < op->Q * op->Q; i++) b.D[i] = T(op->colo_grad1d[i]);
}

template <typename T>
static ElemArgs<T> make_args(const HbElemOp *op, const HbNewtonianContext &ctx, const double *qdata, int color) {
  ElemArgs<T> a;
  a.offsets = op->d_offsets;
  a.elems = op->d_color_elem + op->h_color_ptr[color];
  a.n_elems = op->h_color_ptr[color + 1] - op->h_color_ptr[color];
  fill_basis<T>(op, a.basis);
  a.pc = make_phys<T>(ctx);
  a.qdata = qdata;
  a.x_elem = op->d_x_elem;
  a.num_jd = ctx.idl_enable ? 15 : 14;
  return a;
}

static int grid_for(const HbElemOp *op, int n_elems, int ctas_per_sm) {
  const int g = op->num_sms * ctas_per_sm;
  return n_elems < g ? n_elems : g;
}

template <typename T>
static size_t smem_bytes(int P, int Q) {
  const int P3 = P * P * P, Q3 = Q * Q * Q;
  return sizeof(T) * (size_t)(10 * P3 + 10 * P * P * Q + 10 * P * Q * Q + 10 * Q3 + 15 * Q3);
}

template <int P, int Q>
static int launch_ifunction(const HbElemOp *op, const HbNewtonianContext &ctx, const HbIFunctionIO *io, cudaStream_t s) {
  const size_t sm = smem_bytes<double>(P, Q);
  cudaFuncSetAttribute(k_ifunction<P, Q>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  IfunctionPtrs p;
  p.q = io->q;
  p.q_dot = io->q_dot;
  p.jac_data = io->jac_data;
  p.jac_f32 = io->jac_data_f32;
  p.v = io->v;
  for (int i = 0; i < kMaxP; i++) p.qref.x[i] = i < Q ? op->qref1d[i] : 0;
  for (int c = 0; c < op->num_colors; c++) {
    ElemArgs<double> a = make_args<double>(op, ctx, io->qdata, c);
    if (a.n_elems == 0) continue;
    k_ifunction<P, Q><<<grid_for(op, a.n_elems, 3), nthreads_for<double>(Q), sm, s>>>(a, p);
  }
  return cudaGetLastError() == cudaSuccess ? HB_SUCCESS : HB_ERROR_CUDA;
}

template <int P, int Q, typename T>
static int launch_ijacobian(const HbElemOp *op, const HbNewtonianContext &ctx, const double *qdata, const T *jd, const T *dq, T *v,
                            cudaStream_t s) {
  const size_t sm = smem_bytes<T>(P, Q);
  cudaFuncSetAttribute(k_ijacobian<P, Q, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  IjacobianPtrs<T> p{dq, jd, v};
  for (int c = 0; c < op->num_colors; c++) {
    ElemArgs<T> a = make_args<T>(op, ctx, qdata, c);
    if (a.n_elems == 0) continue;
    k_ijacobian<P, Q, T><<<grid_for(op, a.n_elems, 3), nthreads_for<T>(Q), sm, s>>>(a, p);
  }
  return cudaGetLastError() == cudaSuccess ? HB_SUCCESS : HB_ERROR_CUDA;
}

template <int P, int Q, typename T>
static int launch_diagonal(const HbElemOp *op, const HbNewtonianContext &ctx, const double *qdata, const T *jd, T *diag, cudaStream_t s) {
  const int P3 = P * P * P, Q3 = Q * Q * Q;
  const size_t sm = sizeof(T) * (size_t)(10 * Q3 + Q * Q * P + Q * P * P + 5 * P3);
  cudaFuncSetAttribute(k_diagonal<P, Q, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  DiagArgs<T> p;
  p.jac_data = jd;
  p.diag = diag;
  memset(p.G1, 0, sizeof p.G1);
  for (int i = 0; i < Q * P; i++) p.G1[i] = T(op->grad1d[i]);
  for (int c = 0; c < op->num_colors; c++) {
    ElemArgs<T> a = make_args<T>(op, ctx, qdata, c);
    if (a.n_elems == 0) continue;
    k_diagonal<P, Q, T><<<grid_for(op, a.n_elems, 2), nthreads_for<T>(Q), sm, s>>>(a, p);
  }
  return cudaGetLastError() == cudaSuccess ? HB_SUCCESS : HB_ERROR_CUDA;
}

// (P, Q) pairs compiled: polynomial degree 1..5 with q_extra 0 or 1 (Q = P or P + 1); the benchmark configurations use
// (3,3), (4,5) and (5,6).  P=2 with Q=3 is left out because its transpose scratch would not fit the forward buffers.
#define HB_PQ_LIST(X) X(2, 2) X(3, 3) X(3, 4) X(4, 4) X(4, 5) X(5, 5) X(5, 6) X(6, 6) X(6, 7)

}  // namespace hb

using namespace hb;

static int check_op(const HbElemOp *op) {
  if (!op || op->P < 2 || op->P > kMaxP || op->Q < op->P || op->Q > kMaxP) return HB_ERROR_UNSUPPORTED;
  return HB_SUCCESS;
}

extern "C" int hb_ifunction_apply(const HbElemOp *op, const void *ctx184, const HbIFunctionIO *io, void *stream) {
  int err = check_op(op);
  if (err) return err;
  HbNewtonianContext ctx;
  memcpy(&ctx, ctx184, sizeof ctx);
  if (ctx.state_var != HB_STATEVAR_CONSERVATIVE || ctx.divFdiff_method != HB_DIV_DIFF_FLUX_PROJ_NONE) return HB_ERROR_UNSUPPORTED;
  if (ctx.idl_enable && !op->d_x_elem) return HB_ERROR_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  if (!io->add && cudaMemsetAsync(io->v, 0, sizeof(double) * op->l_size, s) != cudaSuccess) return HB_ERROR_CUDA;
#define HB_CASE(PP, QQ) \
  if (op->P == PP && op->Q == QQ) return launch_ifunction<PP, QQ>(op, ctx, io, s);
  HB_PQ_LIST(HB_CASE)
#undef HB_CASE
  return HB_ERROR_UNSUPPORTED;
}

extern "C" int hb_ijacobian_apply_f64(const HbElemOp *op, const void *ctx184, const double *qdata, const double *jac_data, const double *dq,
                                      double *v, int add, void *stream) {
  int err = check_op(op);
  if (err) return err;
  HbNewtonianContext ctx;
  memcpy(&ctx, ctx184, sizeof ctx);
  if (ctx.state_var != HB_STATEVAR_CONSERVATIVE) return HB_ERROR_UNSUPPORTED;
  cudaStream_t s = (cudaStream_t)stream;
  if (!add && cudaMemsetAsync(v, 0, sizeof(double) * op->l_size, s) != cudaSuccess) return HB_ERROR_CUDA;
#define HB_CASE(PP, QQ) \
  if (op->P == PP && op->Q == QQ) return launch_ijacobian<PP, QQ, double>(op, ctx, qdata, jac_data, dq, v, s);
  HB_PQ_LIST(HB_CASE)
#undef HB_CASE
  return HB_ERROR_UNSUPPORTED;
}

extern "C" int hb_ijacobian_apply_f32(const HbElemOp *op, const void *ctx184, const double *qdata, const float *jac_data, const float *dq,
                                      float *v, int add, void *stream) {
  int err = check_op(op);
  if (err) return err;
  HbNewtonianContext ctx;
  memcpy(&ctx, ctx184, sizeof ctx);
  if (ctx.state_var != HB_STATEVAR_CONSERVATIVE) return HB_ERROR_UNSUPPORTED;
  cudaStream_t s = (cudaStream_t)stream;
  if (!add && cudaMemsetAsync(v, 0, sizeof(float) * op->l_size, s) != cudaSuccess) return HB_ERROR_CUDA;
#define HB_CASE(PP, QQ) \
  if (op->P == PP && op->Q == QQ) return launch_ijacobian<PP, QQ, float>(op, ctx, qdata, jac_data, dq, v, s);
  HB_PQ_LIST(HB_CASE)
#undef HB_CASE
  return HB_ERROR_UNSUPPORTED;
}

extern "C" int hb_diagonal_assemble_f64(const HbElemOp *op, const void *ctx184, const double *qdata, const double *jac_data, double *diag, int add,
                                        void *stream) {
  int err = check_op(op);
  if (err) return err;
  HbNewtonianContext ctx;
  memcpy(&ctx, ctx184, sizeof ctx);
  if (ctx.state_var != HB_STATEVAR_CONSERVATIVE) return HB_ERROR_UNSUPPORTED;
  cudaStream_t s = (cudaStream_t)stream;
  if (!add && cudaMemsetAsync(diag, 0, sizeof(double) * op->l_size, s) != cudaSuccess) return HB_ERROR_CUDA;
#define HB_CASE(PP, QQ) \
  if (op->P == PP && op->Q == QQ) return launch_diagonal<PP, QQ, double>(op, ctx, qdata, jac_data, diag, s);
  HB_PQ_LIST(HB_CASE)
#undef HB_CASE
  return HB_ERROR_UNSUPPORTED;
}

extern "C" int hb_diagonal_assemble_f32(const HbElemOp *op, const void *ctx184, const double *qdata, const float *jac_data, float *diag, int add,
                                        void *stream) {
  int err = check_op(op);
  if (err) return err;
  HbNewtonianContext ctx;
  memcpy(&ctx, ctx184, sizeof ctx);
  if (ctx.state_var != HB_STATEVAR_CONSERVATIVE) return HB_ERROR_UNSUPPORTED;
  cudaStream_t s = (cudaStream_t)stream;
  if (!add && cudaMemsetAsync(diag, 0, sizeof(float) * op->l_size, s) != cudaSuccess) return HB_ERROR_CUDA;
#define HB_CASE(PP, QQ) \
  if (op->P == PP && op->Q == QQ) return launch_diagonal<PP, QQ, float>(op, ctx, qdata, jac_data, diag, s);
  HB_PQ_LIST(HB_CASE)
#undef HB_CASE
  return HB_ERROR_UNSUPPORTED;
}

extern "C" int hb_setup_qdata(int num_elem, int Q, const double *qref1d, const double *qweight1d, const double *x_elem, double *qdata, void *stream) {
  if (Q < 1 || Q > kMaxP || num_elem <= 0) return HB_ERROR_INVALID;
  QRef r, w;
  for (int i = 0; i < kMaxP; i++) {
    r.x[i] = i < Q ? qref1d[i] : 0;
    w.x[i] = i < Q ? qweight1d[i] : 0;
  }
  const int64_t n = (int64_t)num_elem * Q * Q * Q;
  const int bs = 256;
  k_setup_qdata<<<(unsigned)((n + bs - 1) / bs), bs, 0, (cudaStream_t)stream>>>(num_elem, Q, x_elem, r, w, qdata);
  return cudaGetLastError() == cudaSuccess ? HB_SUCCESS : HB_ERROR_CUDA;
}
