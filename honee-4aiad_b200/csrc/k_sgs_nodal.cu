// k_sgs_nodal.cu -- the reference's nodal data-driven subgrid-stress (SGS) pipeline on fused kernels.
//
// HONEE evaluates its data-driven closure at the mesh nodes (problems/sgs_dd_model.c:98-200, 508-560, 645-737).  Per
// residual evaluation (SgsDDApplyIFunction, :559-587) it
//   1. projects the velocity gradient onto the nodes: right-hand side int phi wdetJ du_i/dx_j
//      (VelocityGradientProjectionRHS_*, qfunctions/velocity_gradient_projection.h:9-37, src/velocity_gradient_projection.c:44-103)
//      and one row-sum Jacobi step on the 9-component mass matrix (Mass_9, KSPPREONLY + PC_JACOBI_ROWSUM, :105-127);
//   2. evaluates the closure at every element node, with the grid anisotropy tensor projected once at set-up
//      (AnisotropyTensorProjection, qfunctions/grid_anisotropy_tensor.h:35-55; CG + Jacobi on Mass_7,
//      src/grid_anisotropy_tensor.c:49-108), weights each value by the inverse of the node's multiplicity
//      (InverseMultiplicity, src/inverse_multiplicity.c:24-80) and sums it into the node (ComputeSgsDDNodal_*,
//      qfunctions/sgs_dd_model.h:69-96; network :38-53; frame maps sgs_dd_utils.h:58-127);
//   3. adds the flux of the interpolated nodal stress to the residual (IFunction_NodalSgs_*, sgs_dd_model.h:219-243).
//
// Here:
//   * the element operators (the two projection right-hand sides, Mass_N and its diagonal, the SGS residual) run one
//     CTA per element of one colour, so the scatter into the node-interleaved L-vector is a plain read-add-write.  P
//     and Q are run-time values; interpolation is sum-factorised in shared memory (three one-dimensional passes) and
//     gradients are taken on the quadrature points with the collocated derivative D = grad1d interp1d^+, as the
//     Newtonian kernels take them.  These operators are called once per residual, next to an IFunction that costs
//     several times more, so they favour one compact code path over per-(P, Q) specialisation;
//   * the closure runs once per node, not once per element node.  Every element holding a node gathers the same nodal
//     values, so the reference's sum over those elements of (1/multiplicity) f(node) equals w(node) f(node), w being the
//     transposed restriction of the inverse multiplicity (hb_node_weight_sum): the same value up to the rounding of
//     that sum, for the element-node count divided by the node count less closure work (about 3.4x at P = 3).
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include "honee_b200.h"
#include "newtonian_qf.cuh"
#include "sgs.cuh"

namespace {

constexpr int kThreads = 128;
constexpr size_t kMaxSmem = 227 * 1024;

inline int rc() { return cudaGetLastError() == cudaSuccess ? HB_SUCCESS : HB_ERROR_CUDA; }

#define HB_TRY(x)             \
  do {                        \
    const int hb_e_ = (x);    \
    if (hb_e_) return hb_e_;  \
  } while (0)

// interp1d [Q][P], its square, and the collocated derivative [Q][Q] of the element operator
struct NBasis {
  double B[HB_MAX_P * HB_MAX_P], D[HB_MAX_P * HB_MAX_P];
  int P, Q;
};

NBasis nbasis(const HbElemOp *op) {
  NBasis b;
  memset(&b, 0, sizeof b);
  b.P = op->P;
  b.Q = op->Q;
  memcpy(b.B, op->interp1d, sizeof(double) * op->P * op->Q);
  memcpy(b.D, op->colo_grad1d, sizeof(double) * op->Q * op->Q);
  return b;
}

hb::PhysConst<double> state_consts(const HbGasProperties &gas) {
  hb::PhysConst<double> pc;
  memset(&pc, 0, sizeof pc);
  pc.cv = gas.cv;
  pc.inv_cv = 1.0 / gas.cv;
  pc.gm1 = gas.cp / gas.cv - 1;
  pc.Rgas = gas.cp - gas.cv;
  pc.mu = gas.mu;
  return pc;
}

bool valid_sv(int sv) { return sv == HB_STATEVAR_CONSERVATIVE || sv == HB_STATEVAR_PRIMITIVE || sv == HB_STATEVAR_ENTROPY; }

// ---------------------------------------------------------------------------------------------------------------------
// Shared-memory tensor passes (run-time P, Q; nc fields; all threads of the CTA take part, each ends with a barrier)

struct Dims {
  int P, Q, P3, Q3, n1, n2;  // n1 = P P Q, n2 = P Q Q
  __host__ __device__ Dims(int p, int q) : P(p), Q(q), P3(p * p * p), Q3(q * q * q), n1(p * p * q), n2(p * q * q) {}
};

// sU [nc][Q3] = (B x B x B) sN [nc][P3]; t1 [nc][n1], t2 [nc][n2] scratch
__device__ void interp_fwd(const Dims &d, int nc, const double *sB, const double *sN, double *t1, double *t2, double *sU) {
  const int P = d.P, Q = d.Q;
  for (int idx = threadIdx.x; idx < nc * d.n1; idx += blockDim.x) {
    const int c = idx / d.n1, r = idx - c * d.n1, i = r % Q, row = r / Q;  // row = pc P + pb
    const double *x = sN + c * d.P3 + row * P;
    double s = 0;
    for (int a = 0; a < P; a++) s += sB[i * P + a] * x[a];
    t1[idx] = s;  // [c][pc][pb][i]
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < nc * d.n2; idx += blockDim.x) {
    const int c = idx / d.n2, r = idx - c * d.n2, i = r % Q, j = (r / Q) % Q, pc = r / (Q * Q);
    const double *x = t1 + c * d.n1 + pc * P * Q + i;
    double s = 0;
    for (int a = 0; a < P; a++) s += sB[j * P + a] * x[a * Q];
    t2[idx] = s;  // [c][pc][j][i]
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < nc * d.Q3; idx += blockDim.x) {
    const int c = idx / d.Q3, r = idx - c * d.Q3, ji = r % (Q * Q), k = r / (Q * Q);
    const double *x = t2 + c * d.n2 + ji;
    double s = 0;
    for (int a = 0; a < P; a++) s += sB[k * P + a] * x[a * Q * Q];
    sU[idx] = s;  // [c][k][j][i]
  }
  __syncthreads();
}

// sO [nc][P3] = (B x B x B)^T sF [nc][Q3]
__device__ void interp_t(const Dims &d, int nc, const double *sB, const double *sF, double *t2, double *t1, double *sO) {
  const int P = d.P, Q = d.Q;
  for (int idx = threadIdx.x; idx < nc * d.n2; idx += blockDim.x) {
    const int c = idx / d.n2, r = idx - c * d.n2, ji = r % (Q * Q), pc = r / (Q * Q);
    const double *x = sF + c * d.Q3 + ji;
    double s = 0;
    for (int k = 0; k < Q; k++) s += sB[k * P + pc] * x[k * Q * Q];
    t2[idx] = s;  // [c][pc][j][i]
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < nc * d.n1; idx += blockDim.x) {
    const int c = idx / d.n1, r = idx - c * d.n1, i = r % Q, pb = (r / Q) % P, pc = r / (Q * P);
    const double *x = t2 + c * d.n2 + pc * Q * Q + i;
    double s = 0;
    for (int j = 0; j < Q; j++) s += sB[j * P + pb] * x[j * Q];
    t1[idx] = s;  // [c][pc][pb][i]
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < nc * d.P3; idx += blockDim.x) {
    const int c = idx / d.P3, r = idx - c * d.P3, pa = r % P, row = r / P;
    const double *x = t1 + c * d.n1 + row * Q;
    double s = 0;
    for (int i = 0; i < Q; i++) s += sB[i * P + pa] * x[i];
    sO[idx] = s;  // [c][pc][pb][pa]
  }
  __syncthreads();
}

// reference gradient on the points: sG [3][nc][Q3] from sU [nc][Q3]
__device__ void colo_grad(const Dims &d, int nc, const double *sD, const double *sU, double *sG) {
  const int Q = d.Q, Q3 = d.Q3;
  for (int idx = threadIdx.x; idx < 3 * nc * Q3; idx += blockDim.x) {
    const int dir = idx / (nc * Q3), r = idx - dir * nc * Q3, c = r / Q3, p = r - c * Q3;
    const int i = p % Q, j = (p / Q) % Q, k = p / (Q * Q);
    const double *u = sU + c * Q3;
    double s = 0;
    if (dir == 0)
      for (int a = 0; a < Q; a++) s += sD[i * Q + a] * u[(k * Q + j) * Q + a];
    else if (dir == 1)
      for (int a = 0; a < Q; a++) s += sD[j * Q + a] * u[(k * Q + a) * Q + i];
    else
      for (int a = 0; a < Q; a++) s += sD[k * Q + a] * u[(a * Q + j) * Q + i];
    sG[idx] = s;
  }
  __syncthreads();
}

// its transpose: sH [nc][Q3] = sum_dir D_dir^T sGv [dir][nc][Q3]
__device__ void colo_grad_t(const Dims &d, int nc, const double *sD, const double *sGv, double *sH) {
  const int Q = d.Q, Q3 = d.Q3;
  for (int idx = threadIdx.x; idx < nc * Q3; idx += blockDim.x) {
    const int c = idx / Q3, p = idx - c * Q3, i = p % Q, j = (p / Q) % Q, k = p / (Q * Q);
    const double *g0 = sGv + c * Q3, *g1 = sGv + (nc + c) * Q3, *g2 = sGv + (2 * nc + c) * Q3;
    double s = 0;
    for (int a = 0; a < Q; a++) s += sD[a * Q + i] * g0[(k * Q + j) * Q + a];
    for (int a = 0; a < Q; a++) s += sD[a * Q + j] * g1[(k * Q + a) * Q + i];
    for (int a = 0; a < Q; a++) s += sD[a * Q + k] * g2[(a * Q + j) * Q + i];
    sH[idx] = s;
  }
  __syncthreads();
}

__device__ void load_basis(const NBasis &b, double *sB, double *sD, bool squared) {
  for (int i = threadIdx.x; i < b.P * b.Q; i += blockDim.x) sB[i] = squared ? b.B[i] * b.B[i] : b.B[i];
  if (sD)
    for (int i = threadIdx.x; i < b.Q * b.Q; i += blockDim.x) sD[i] = b.D[i];
}

// sN [nc][P3] from the node-interleaved L-vector l [node][ncl], fields c0 .. c0 + nc - 1 (off5 = node * 5 offsets)
__device__ void gather(const Dims &d, const int32_t *off5, int e, const double *l, int ncl, int c0, int nc, double *sN) {
  for (int idx = threadIdx.x; idx < nc * d.P3; idx += blockDim.x) {
    const int c = idx / d.P3, p = idx - c * d.P3;
    sN[idx] = l[(int64_t)(off5[(int64_t)e * d.P3 + p] / 5) * ncl + c0 + c];
  }
}

// l [node][nc] += sO [nc][P3]
__device__ void scatter_add(const Dims &d, const int32_t *off5, int e, const double *sO, int nc, double *l) {
  for (int idx = threadIdx.x; idx < nc * d.P3; idx += blockDim.x) {
    const int c = idx / d.P3, p = idx - c * d.P3;
    l[(int64_t)(off5[(int64_t)e * d.P3 + p] / 5) * nc + c] += sO[idx];
  }
}

__device__ __forceinline__ void load_point(const double *qd, int Q3, int p, double &w, double X[3][3]) {
  w = qd[p];
#pragma unroll
  for (int k = 0; k < 9; k++) X[k / 3][k % 3] = qd[(1 + k) * Q3 + p];
}

// shared-memory carve-up: returns the next free double
struct Carve {
  double *p;
  __device__ double *take(int n) {
    double *r = p;
    p += n;
    return r;
  }
};

// ---------------------------------------------------------------------------------------------------------------------
// 1. velocity-gradient projection right-hand side: v [node][9] += int phi wdetJ du_i/dx_j

size_t smem_velgrad(const Dims &d) {
  return sizeof(double) * (d.P * d.Q + d.Q * d.Q + 5 * d.P3 + 9 * d.n1 + 9 * d.n2 + 5 * d.Q3 + 15 * d.Q3 + 9 * d.Q3 + 9 * d.P3);
}

__global__ void __launch_bounds__(kThreads) k_velgrad_rhs(const int32_t *__restrict__ off5, const int32_t *__restrict__ elems, NBasis b,
                                                          hb::PhysConst<double> pc, int sv, const double *__restrict__ qdata,
                                                          const double *__restrict__ q, double *__restrict__ v) {
  extern __shared__ double smem[];
  const Dims d(b.P, b.Q);
  Carve cv{smem};
  double *sB = cv.take(d.P * d.Q), *sD = cv.take(d.Q * d.Q), *sN = cv.take(5 * d.P3), *t1 = cv.take(9 * d.n1), *t2 = cv.take(9 * d.n2),
         *sU = cv.take(5 * d.Q3), *sG = cv.take(15 * d.Q3), *sF = cv.take(9 * d.Q3), *sO = cv.take(9 * d.P3);
  const int e = elems[blockIdx.x];
  load_basis(b, sB, sD, false);
  gather(d, off5, e, q, 5, 0, 5, sN);
  __syncthreads();
  interp_fwd(d, 5, sB, sN, t1, t2, sU);
  colo_grad(d, 5, sD, sU, sG);
  const double *qd = qdata + (int64_t)e * 10 * d.Q3;
  for (int p = threadIdx.x; p < d.Q3; p += blockDim.x) {
    double qi[5], w, X[3][3];
#pragma unroll
    for (int c = 0; c < 5; c++) qi[c] = sU[c * d.Q3 + p];
    load_point(qd, d.Q3, p, w, X);
    hb::St<double> s;
    hb::SAux<double> aux;
    hb::state_from_q_rt(sv, pc, qi, s, aux);
    // StatePhysicalGradientFromReference (newtonian_state.h:581-593): dq[c][j] = sum_r grad_ref[r][c] dXdx[r][j]
#pragma unroll
    for (int j = 0; j < 3; j++) {
      double dq[5];
#pragma unroll
      for (int c = 0; c < 5; c++) dq[c] = sG[c * d.Q3 + p] * X[0][j] + sG[(5 + c) * d.Q3 + p] * X[1][j] + sG[(10 + c) * d.Q3 + p] * X[2][j];
      hb::St<double> ds;
      hb::state_from_q_fwd_rt(sv, pc, s, aux, dq, ds);
      // VelocityGradient (newtonian_state.h:511-521): grad_velocity[a][j] = d u_a / d x_j, stored at a * 3 + j
#pragma unroll
      for (int a = 0; a < 3; a++) sF[(a * 3 + j) * d.Q3 + p] = w * ds.u[a];
    }
  }
  __syncthreads();
  interp_t(d, 9, sB, sF, t2, t1, sO);
  scatter_add(d, off5, e, sO, 9, v);
}

// ---------------------------------------------------------------------------------------------------------------------
// 2. anisotropy-tensor projection right-hand side: v [node][7] += int phi wdetJ (km A_ij, delta)

size_t smem_aniso(const Dims &d) { return sizeof(double) * (d.P * d.Q + 7 * d.n1 + 7 * d.n2 + 7 * d.Q3 + 7 * d.P3); }

__global__ void __launch_bounds__(kThreads) k_aniso_rhs(const int32_t *__restrict__ off5, const int32_t *__restrict__ elems, NBasis b,
                                                        const double *__restrict__ qdata, double *__restrict__ v) {
  extern __shared__ double smem[];
  const Dims d(b.P, b.Q);
  Carve cv{smem};
  double *sB = cv.take(d.P * d.Q), *t1 = cv.take(7 * d.n1), *t2 = cv.take(7 * d.n2), *sF = cv.take(7 * d.Q3), *sO = cv.take(7 * d.P3);
  const int e = elems[blockIdx.x];
  load_basis(b, sB, nullptr, false);
  const double *qd = qdata + (int64_t)e * 10 * d.Q3;
  for (int p = threadIdx.x; p < d.Q3; p += blockDim.x) {
    double w, X[3][3], kmA[6], delta;
    load_point(qd, d.Q3, p, w, X);
    hb::sgs::anisotropy(X, kmA, delta);  // KMMetricTensor + AnisotropyTensor (15 sweeps) + KMPack
#pragma unroll
    for (int c = 0; c < 6; c++) sF[c * d.Q3 + p] = w * kmA[c];
    sF[6 * d.Q3 + p] = w * delta;
  }
  __syncthreads();
  interp_t(d, 7, sB, sF, t2, t1, sO);
  scatter_add(d, off5, e, sO, 7, v);
}

// ---------------------------------------------------------------------------------------------------------------------
// Mass_N (qfunctions/mass.h, src/honee-mass.c:20-60): v [node][nc] += M u, and the diagonal of M per node and field

size_t smem_mass(const Dims &d, int nc) { return sizeof(double) * (d.P * d.Q + nc * (d.P3 + d.n1 + d.n2 + d.Q3)); }

__global__ void __launch_bounds__(kThreads) k_mass_n(const int32_t *__restrict__ off5, const int32_t *__restrict__ elems, NBasis b, int nc,
                                                     const double *__restrict__ qdata, const double *__restrict__ u, double *__restrict__ v) {
  extern __shared__ double smem[];
  const Dims d(b.P, b.Q);
  Carve cv{smem};
  double *sB = cv.take(d.P * d.Q), *sN = cv.take(nc * d.P3), *t1 = cv.take(nc * d.n1), *t2 = cv.take(nc * d.n2), *sU = cv.take(nc * d.Q3);
  const int e = elems[blockIdx.x];
  load_basis(b, sB, nullptr, false);
  gather(d, off5, e, u, nc, 0, nc, sN);
  __syncthreads();
  interp_fwd(d, nc, sB, sN, t1, t2, sU);
  const double *qd = qdata + (int64_t)e * 10 * d.Q3;
  for (int idx = threadIdx.x; idx < nc * d.Q3; idx += blockDim.x) sU[idx] *= qd[idx % d.Q3];
  __syncthreads();
  interp_t(d, nc, sB, sU, t2, t1, sN);
  scatter_add(d, off5, e, sN, nc, v);
}

// diag [node][nc] += sum_q wdetJ(q) phi_node(q)^2 in every field (the transposed interpolation of wdetJ with B squared)
__global__ void __launch_bounds__(kThreads) k_mass_n_diag(const int32_t *__restrict__ off5, const int32_t *__restrict__ elems, NBasis b, int nc,
                                                          const double *__restrict__ qdata, double *__restrict__ diag) {
  extern __shared__ double smem[];
  const Dims d(b.P, b.Q);
  Carve cv{smem};
  double *sB = cv.take(d.P * d.Q), *sW = cv.take(d.Q3), *t1 = cv.take(d.n1), *t2 = cv.take(d.n2), *sO = cv.take(d.P3);
  const int e = elems[blockIdx.x];
  load_basis(b, sB, nullptr, true);
  const double *qd = qdata + (int64_t)e * 10 * d.Q3;
  for (int p = threadIdx.x; p < d.Q3; p += blockDim.x) sW[p] = qd[p];
  __syncthreads();
  interp_t(d, 1, sB, sW, t2, t1, sO);
  for (int idx = threadIdx.x; idx < nc * d.P3; idx += blockDim.x) {
    const int c = idx / d.P3, p = idx - c * d.P3;
    diag[(int64_t)(off5[(int64_t)e * d.P3 + p] / 5) * nc + c] += sO[p];
  }
}

// ---------------------------------------------------------------------------------------------------------------------
// 3. SGS residual: v [node][5] += int grad phi . (-wdetJ dXdx F_sgs(Y(q), km_sgs))

size_t smem_sgs_if(const Dims &d) {
  return sizeof(double) * (d.P * d.Q + d.Q * d.Q + 11 * d.P3 + 11 * d.n1 + 11 * d.n2 + 11 * d.Q3 + 15 * d.Q3 + 5 * d.Q3);
}

__global__ void __launch_bounds__(kThreads) k_sgs_nodal_ifunction(const int32_t *__restrict__ off5, const int32_t *__restrict__ elems, NBasis b,
                                                                  hb::PhysConst<double> pc, int sv, const double *__restrict__ qdata,
                                                                  const double *__restrict__ q, const double *__restrict__ km,
                                                                  double *__restrict__ v) {
  extern __shared__ double smem[];
  const Dims d(b.P, b.Q);
  Carve cv{smem};
  double *sB = cv.take(d.P * d.Q), *sD = cv.take(d.Q * d.Q), *sN = cv.take(11 * d.P3), *t1 = cv.take(11 * d.n1), *t2 = cv.take(11 * d.n2),
         *sU = cv.take(11 * d.Q3), *sGv = cv.take(15 * d.Q3), *sH = cv.take(5 * d.Q3);
  const int e = elems[blockIdx.x];
  load_basis(b, sB, sD, false);
  gather(d, off5, e, q, 5, 0, 5, sN);
  gather(d, off5, e, km, 6, 0, 6, sN + 5 * d.P3);
  __syncthreads();
  interp_fwd(d, 11, sB, sN, t1, t2, sU);
  const double *qd = qdata + (int64_t)e * 10 * d.Q3;
  for (int p = threadIdx.x; p < d.Q3; p += blockDim.x) {
    double qi[5], kmi[6], w, X[3][3], F[5][3];
#pragma unroll
    for (int c = 0; c < 5; c++) qi[c] = sU[c * d.Q3 + p];
#pragma unroll
    for (int c = 0; c < 6; c++) kmi[c] = sU[(5 + c) * d.Q3 + p];
    load_point(qd, d.Q3, p, w, X);
    hb::St<double> s;
    hb::SAux<double> aux;
    hb::state_from_q_rt(sv, pc, qi, s, aux);
    hb::sgs::flux(s.u, kmi, F);  // FluxSubgridStress (sgs_dd_model.h:205-217)
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
      for (int c = 0; c < 5; c++) sGv[(k * 5 + c) * d.Q3 + p] = -w * (X[k][0] * F[c][0] + X[k][1] * F[c][1] + X[k][2] * F[c][2]);
  }
  __syncthreads();
  colo_grad_t(d, 5, sD, sGv, sH);
  interp_t(d, 5, sB, sH, t2, t1, sN);
  scatter_add(d, off5, e, sN, 5, v);
}

// ---------------------------------------------------------------------------------------------------------------------
// inverse multiplicity and the per-node weight

// e_out [elem][es] = 1 / l_mult [off[elem][es]] (InverseMultiplicity reads component 0 of the multiplicity field)
__global__ void k_inverse_multiplicity(int64_t n, const int32_t *__restrict__ off, const double *__restrict__ mult, double *__restrict__ e_out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) e_out[i] = 1.0 / mult[off[i]];
}

// w [node] += e_vec [elem][P3] over the element nodes of one colour
__global__ void k_node_weight(const int32_t *__restrict__ off5, const int32_t *__restrict__ elems, int n_elems, int P3, const double *__restrict__ e_vec,
                              double *__restrict__ w) {
  const int64_t n = (int64_t)n_elems * P3;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int e = elems[i / P3], p = (int)(i % P3);
    w[off5[(int64_t)e * P3 + p] / 5] += e_vec[(int64_t)e * P3 + p];
  }
}

// ---------------------------------------------------------------------------------------------------------------------
// 4. the closure at the nodes

// The network of SgsDDContext_ (sgs_dd_model.h:16-31): one hidden layer of 20, 6 inputs and outputs, FP64 weights
// (W1 [20][6], W2 [6][20] row-major after the reference's transpose at load, problems/sgs_dd_model.c:633-643), leaky
// ReLU slope alpha, and the min-max bounds of the outputs.
struct NodalNet {
  double b1[20], b2[6], w1[120], w2[120], bounds[6][2];
  double alpha;
};

__device__ __forceinline__ void nodal_closure(const NodalNet &net, const hb::PhysConst<double> &pc, int sv, const double qi[5], const double G[3][3],
                                              const double A7[7], double km_sgs[6]) {
  hb::St<double> s;
  hb::SAux<double> aux;
  hb::state_from_q_rt(sv, pc, qi, s, aux);
  const double kmA[6] = {A7[0], A7[1], A7[2], A7[3], A7[4], A7[5]}, delta = A7[6];
  double E[3][3], in[6], gmag;
  hb::sgs::inputs(G, kmA, delta, pc.mu / s.rho, E, in, gmag);  // ComputeSgsDDInputs (sgs_dd_utils.h:58-96)
  // DataDrivenInference (sgs_dd_model.h:38-53): V = b1 + W1 x; leaky ReLU; y = b2 + W2 V
  double V[20], y[6];
#pragma unroll
  for (int i = 0; i < 20; i++) {
    double dot = 0;
#pragma unroll
    for (int j = 0; j < 6; j++) dot += net.w1[i * 6 + j] * in[j];
    const double h = net.b1[i] + dot;
    V[i] = h * (h < 0 ? net.alpha : 1.);
  }
#pragma unroll
  for (int i = 0; i < 6; i++) {
    double dot = 0;
#pragma unroll
    for (int j = 0; j < 20; j++) dot += net.w2[i * 20 + j] * V[j];
    y[i] = net.b2[i] + dot;
  }
  hb::sgs::outputs_to_stress(y, delta, E, net.bounds, gmag, km_sgs);  // ComputeSgsDDOutputs (sgs_dd_utils.h:107-127)
}

__global__ void k_sgs_nodal_closure(int64_t nodes, NodalNet net, hb::PhysConst<double> pc, int sv, const double *__restrict__ q,
                                    const double *__restrict__ G9, const double *__restrict__ A7, const double *__restrict__ w,
                                    double *__restrict__ km_sgs) {
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nodes; n += (int64_t)gridDim.x * blockDim.x) {
    const double wn = w[n];
    if (wn == 0) continue;  // a node no element holds: the reference evaluates nothing there
    double qi[5], G[3][3], A[7], tau[6];
#pragma unroll
    for (int c = 0; c < 5; c++) qi[c] = q[n * 5 + c];
#pragma unroll
    for (int c = 0; c < 9; c++) G[c / 3][c % 3] = G9[n * 9 + c];
#pragma unroll
    for (int c = 0; c < 7; c++) A[c] = A7[n * 7 + c];
    nodal_closure(net, pc, sv, qi, G, A, tau);
#pragma unroll
    for (int c = 0; c < 6; c++) km_sgs[n * 6 + c] += wn * tau[c];
  }
}

// ---------------------------------------------------------------------------------------------------------------------
// launch helpers

template <typename K>
int prep(K kernel, size_t smem) {
  if (smem > kMaxSmem) return HB_ERROR_UNSUPPORTED;
  if (smem > 48 * 1024 && cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return HB_ERROR_CUDA;
  return HB_SUCCESS;
}

bool op_ok(const HbElemOp *op) { return op && op->P >= 2 && op->Q >= op->P && op->Q <= HB_MAX_P; }

int grid_1d(int64_t n) {
  const int64_t g = (n + 255) / 256;
  return (int)(g < 148 * 16 ? (g > 0 ? g : 1) : 148 * 16);
}

int parse_net(const void *ctx, size_t bytes, NodalNet &net, HbNewtonianContext &newt) {
  if (!ctx || bytes < sizeof(HbSgsDDContext)) return HB_ERROR_INVALID;
  HbSgsDDContext h;
  memcpy(&h, ctx, sizeof h);
  if (h.num_inputs != 6 || h.num_outputs != 6 || h.num_neurons != 20) return HB_ERROR_UNSUPPORTED;  // num_layers is not read (sgs_dd_model.h:38-53)
  const size_t n = (bytes - offsetof(HbSgsDDContext, data)) / sizeof(double);
  const size_t need[5][2] = {{h.offsets.bias1, 20}, {h.offsets.bias2, 6}, {h.offsets.weight1, 120}, {h.offsets.weight2, 120}, {h.offsets.out_scaling, 12}};
  for (int i = 0; i < 5; i++)
    if (need[i][0] + need[i][1] > n) return HB_ERROR_INVALID;
  const double *data = (const double *)((const char *)ctx + offsetof(HbSgsDDContext, data));
  memcpy(net.b1, data + h.offsets.bias1, sizeof net.b1);
  memcpy(net.b2, data + h.offsets.bias2, sizeof net.b2);
  memcpy(net.w1, data + h.offsets.weight1, sizeof net.w1);
  memcpy(net.w2, data + h.offsets.weight2, sizeof net.w2);
  memcpy(net.bounds, data + h.offsets.out_scaling, sizeof net.bounds);
  net.alpha = h.alpha;
  newt = h.newt_ctx;
  return HB_SUCCESS;
}

}  // namespace

extern "C" {

int hb_velocity_gradient_rhs(const HbElemOp *op, const void *ctx184, int state_var, const double *qdata, const double *q, double *v, void *stream) {
  if (!op_ok(op) || !ctx184 || !qdata || !q || !v) return HB_ERROR_INVALID;
  if (!valid_sv(state_var)) return HB_ERROR_UNSUPPORTED;
  HbNewtonianContext c;
  memcpy(&c, ctx184, sizeof c);
  const Dims d(op->P, op->Q);
  const size_t smem = smem_velgrad(d);
  HB_TRY(prep(k_velgrad_rhs, smem));
  const NBasis b = nbasis(op);
  const hb::PhysConst<double> pc = state_consts(c.gas);
  for (int k = 0; k < op->num_colors; k++) {
    const int n = op->h_color_ptr[k + 1] - op->h_color_ptr[k];
    if (n)
      k_velgrad_rhs<<<n, kThreads, smem, (cudaStream_t)stream>>>(op->d_offsets, op->d_color_elem + op->h_color_ptr[k], b, pc, state_var, qdata, q, v);
  }
  return rc();
}

int hb_anisotropy_rhs(const HbElemOp *op, const double *qdata, double *v, void *stream) {
  if (!op_ok(op) || !qdata || !v) return HB_ERROR_INVALID;
  const Dims d(op->P, op->Q);
  const size_t smem = smem_aniso(d);
  HB_TRY(prep(k_aniso_rhs, smem));
  const NBasis b = nbasis(op);
  for (int k = 0; k < op->num_colors; k++) {
    const int n = op->h_color_ptr[k + 1] - op->h_color_ptr[k];
    if (n) k_aniso_rhs<<<n, kThreads, smem, (cudaStream_t)stream>>>(op->d_offsets, op->d_color_elem + op->h_color_ptr[k], b, qdata, v);
  }
  return rc();
}

int hb_mass_n_apply(const HbElemOp *op, int nc, const double *qdata, const double *u, double *v, void *stream) {
  if (!op_ok(op) || nc < 1 || nc > 64 || !qdata || !u || !v) return HB_ERROR_INVALID;
  const Dims d(op->P, op->Q);
  const size_t smem = smem_mass(d, nc);
  HB_TRY(prep(k_mass_n, smem));
  const NBasis b = nbasis(op);
  for (int k = 0; k < op->num_colors; k++) {
    const int n = op->h_color_ptr[k + 1] - op->h_color_ptr[k];
    if (n) k_mass_n<<<n, kThreads, smem, (cudaStream_t)stream>>>(op->d_offsets, op->d_color_elem + op->h_color_ptr[k], b, nc, qdata, u, v);
  }
  return rc();
}

int hb_mass_n_diagonal(const HbElemOp *op, int nc, const double *qdata, double *diag, void *stream) {
  if (!op_ok(op) || nc < 1 || nc > 64 || !qdata || !diag) return HB_ERROR_INVALID;
  const Dims d(op->P, op->Q);
  const size_t smem = sizeof(double) * (d.P * d.Q + d.Q3 + d.n1 + d.n2 + d.P3);
  HB_TRY(prep(k_mass_n_diag, smem));
  const NBasis b = nbasis(op);
  for (int k = 0; k < op->num_colors; k++) {
    const int n = op->h_color_ptr[k + 1] - op->h_color_ptr[k];
    if (n) k_mass_n_diag<<<n, kThreads, smem, (cudaStream_t)stream>>>(op->d_offsets, op->d_color_elem + op->h_color_ptr[k], b, nc, qdata, diag);
  }
  return rc();
}

int hb_sgs_nodal_ifunction(const HbElemOp *op, const void *ctx184, int state_var, const double *qdata, const double *q, const double *km_sgs, double *v,
                           void *stream) {
  if (!op_ok(op) || !ctx184 || !qdata || !q || !km_sgs || !v) return HB_ERROR_INVALID;
  if (!valid_sv(state_var)) return HB_ERROR_UNSUPPORTED;
  HbNewtonianContext c;
  memcpy(&c, ctx184, sizeof c);
  const Dims d(op->P, op->Q);
  const size_t smem = smem_sgs_if(d);
  HB_TRY(prep(k_sgs_nodal_ifunction, smem));
  const NBasis b = nbasis(op);
  const hb::PhysConst<double> pc = state_consts(c.gas);
  for (int k = 0; k < op->num_colors; k++) {
    const int n = op->h_color_ptr[k + 1] - op->h_color_ptr[k];
    if (n)
      k_sgs_nodal_ifunction<<<n, kThreads, smem, (cudaStream_t)stream>>>(op->d_offsets, op->d_color_elem + op->h_color_ptr[k], b, pc, state_var, qdata, q,
                                                                       km_sgs, v);
  }
  return rc();
}

int hb_inverse_multiplicity(int64_t n, const int32_t *offsets, const double *mult, double *e_out, void *stream) {
  if (n < 0 || (n && (!offsets || !mult || !e_out))) return HB_ERROR_INVALID;
  if (n) k_inverse_multiplicity<<<grid_1d(n), 256, 0, (cudaStream_t)stream>>>(n, offsets, mult, e_out);
  return rc();
}

int hb_node_weight_sum(const HbElemOp *op, const double *e_vec, double *w, void *stream) {
  if (!op_ok(op) || !e_vec || !w) return HB_ERROR_INVALID;
  const int P3 = op->P * op->P * op->P;
  for (int k = 0; k < op->num_colors; k++) {
    const int n = op->h_color_ptr[k + 1] - op->h_color_ptr[k];
    if (n) k_node_weight<<<grid_1d((int64_t)n * P3), 256, 0, (cudaStream_t)stream>>>(op->d_offsets, op->d_color_elem + op->h_color_ptr[k], n, P3, e_vec, w);
  }
  return rc();
}

int hb_sgs_nodal_closure(int64_t nodes, const void *sgs_ctx, size_t ctx_bytes, int state_var, const double *q, const double *G, const double *A,
                         const double *w, double *km_sgs, void *stream) {
  if (nodes < 0 || (nodes && (!q || !G || !A || !w || !km_sgs))) return HB_ERROR_INVALID;
  if (!valid_sv(state_var)) return HB_ERROR_UNSUPPORTED;
  NodalNet net;
  HbNewtonianContext newt;
  HB_TRY(parse_net(sgs_ctx, ctx_bytes, net, newt));
  const hb::PhysConst<double> pc = state_consts(newt.gas);
  if (nodes) k_sgs_nodal_closure<<<grid_1d(nodes), 128, 0, (cudaStream_t)stream>>>(nodes, net, pc, state_var, q, G, A, w, km_sgs);
  return rc();
}

}  // extern "C"
