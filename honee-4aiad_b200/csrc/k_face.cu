// k_face.cu -- boundary-face operators: face geometric factors and the free-stream boundary condition (residual and
// Jacobian), the surface sub-operators HONEE adds to its composite IFunction / IJacobian for `bc_freestream`
// (problems/bc_freestream.c, qfunctions/bc_freestream.h:14-138, face qdata qfunctions/setupgeo.h:100-117).
//
// One CTA per face element, one thread per face quadrature point (Q^2 <= 64), 2D tensor contractions evaluated directly;
// faces of one colour per launch, so the scatter into the volume L-vector is a plain read-add-write (faces on different
// box sides share edge nodes, the colouring keeps them apart).  Boundary work is O(E^(2/3)): written plainly.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "hb_internal.h"
#include "riemann.cuh"

namespace {

constexpr int kMaxQ2 = 64, kMaxP2 = 64;

struct FaceBasis {
  double B[HB_MAX_P * HB_MAX_P], G[HB_MAX_P * HB_MAX_P];  // [Q][P]
  double w[HB_MAX_P];
};

struct Exterior {
  double cv, gamma, gm1;
  double U[5], Y[5];  // free-stream State: conservative (rho, m, E) and primitive (P, u, T)
  int hllc;
  int sv;             // state variable of q and of the stored face state (HbStateVariable)
};

inline int rc() { return cudaGetLastError() == cudaSuccess ? HB_SUCCESS : HB_ERROR_CUDA; }

__device__ __forceinline__ double b2(const FaceBasis &b, int P, int q0, int q1, int p0, int p1) { return b.B[q0 * P + p0] * b.B[q1 * P + p1]; }

// qdata_sur [F][10][Q^2]: w detJb, unit normal (3), dX/dx (2 x 3, Moore-Penrose inverse of dx/dX)
__global__ void k_face_setup(int P, int Q, FaceBasis b, const double *__restrict__ xn, double *__restrict__ qd) {
  const int f = blockIdx.x, t = threadIdx.x, P2 = P * P, Q2 = Q * Q;
  if (t >= Q2) return;
  const int q0 = t % Q, q1 = t / Q;
  double J[3][2] = {{0, 0}, {0, 0}, {0, 0}};
  for (int p = 0; p < P2; p++) {
    const int p0 = p % P, p1 = p / P;
    const double g0 = b.G[q0 * P + p0] * b.B[q1 * P + p1], g1 = b.B[q0 * P + p0] * b.G[q1 * P + p1];
    for (int d = 0; d < 3; d++) {
      const double x = xn[((int64_t)f * 3 + d) * P2 + p];
      J[d][0] += g0 * x;
      J[d][1] += g1 * x;
    }
  }
  const double N[3] = {J[1][0] * J[2][1] - J[2][0] * J[1][1], J[2][0] * J[0][1] - J[0][0] * J[2][1], J[0][0] * J[1][1] - J[1][0] * J[0][1]};
  const double detJb = sqrt(N[0] * N[0] + N[1] * N[1] + N[2] * N[2]);
  // dX/dx = (J^T J)^-1 J^T
  const double a = J[0][0] * J[0][0] + J[1][0] * J[1][0] + J[2][0] * J[2][0], c = J[0][1] * J[0][1] + J[1][1] * J[1][1] + J[2][1] * J[2][1];
  const double bb = J[0][0] * J[0][1] + J[1][0] * J[1][1] + J[2][0] * J[2][1];
  const double det = a * c - bb * bb;
  const double inv[2][2] = {{c / det, -bb / det}, {-bb / det, a / det}};
  double *o = qd + (int64_t)f * 10 * Q2 + t;
  o[0] = b.w[q0] * b.w[q1] * detJb;
  for (int d = 0; d < 3; d++) o[(1 + d) * Q2] = N[d] / detJb;
  for (int i = 0; i < 2; i++)
    for (int j = 0; j < 3; j++) o[(4 + i * 3 + j) * Q2] = inv[i][0] * J[j][0] + inv[i][1] * J[j][1];
}

__device__ __forceinline__ void exterior_state(const Exterior &x, hb::St<double> &s) {
  s.rho = x.U[0];
  s.m[0] = x.U[1];
  s.m[1] = x.U[2];
  s.m[2] = x.U[3];
  s.E = x.U[4];
  s.P = x.Y[0];
  s.u[0] = x.Y[1];
  s.u[1] = x.Y[2];
  s.u[2] = x.Y[3];
  s.T_ = x.Y[4];
}

// v += wdetJb * F_riemann(q, S_infty, n) integrated against the face basis; jac_sur [F][5][Q^2] = q at the points
// (Freestream, bc_freestream.h:14-48)
__global__ void k_freestream(int P, int Q, const int32_t *__restrict__ offsets, const int32_t *__restrict__ faces, FaceBasis b,
                             hb::PhysConst<double> pc, Exterior ex, const double *__restrict__ qd, const double *__restrict__ q, double *__restrict__ jac,
                             double *__restrict__ v) {
  __shared__ double sN[5][kMaxP2], sF[5][kMaxQ2];
  const int f = faces[blockIdx.x], t = threadIdx.x, P2 = P * P, Q2 = Q * Q;
  for (int i = t; i < 5 * P2; i += blockDim.x) sN[i % 5][i / 5] = q[offsets[(int64_t)f * P2 + i / 5] + i % 5];
  __syncthreads();
  if (t < Q2) {
    const int q0 = t % Q, q1 = t / Q;
    double U[5] = {0, 0, 0, 0, 0};
    for (int p = 0; p < P2; p++) {
      const double w = b2(b, P, q0, q1, p % P, p / P);
      for (int c = 0; c < 5; c++) U[c] += w * sN[c][p];
    }
    hb::St<double> s, sx;
    hb::SAux<double> aux;
    hb::state_from_q_rt(ex.sv, pc, U, s, aux);
    exterior_state(ex, sx);
    const double *qf = qd + (int64_t)f * 10 * Q2;
    const double wdetJb = qf[t], n[3] = {qf[Q2 + t], qf[2 * Q2 + t], qf[3 * Q2 + t]};
    double F[5];
    if (ex.hllc) hb::riemann::hllc_flux(ex.gamma, ex.cv, s, sx, n, F);
    else hb::riemann::hll_flux(ex.gamma, ex.cv, s, sx, n, F);
    for (int c = 0; c < 5; c++) sF[c][t] = wdetJb * F[c];
    if (jac)
      for (int c = 0; c < 5; c++) jac[((int64_t)f * 5 + c) * Q2 + t] = U[c];
  }
  __syncthreads();
  for (int i = t; i < 5 * P2; i += blockDim.x) {
    const int p = i / 5, c = i % 5;
    double acc = 0;
    for (int k = 0; k < Q2; k++) acc += b2(b, P, k % Q, k / Q, p % P, p / P) * sF[c][k];
    v[offsets[(int64_t)f * P2 + p] + c] += acc;
  }
}

// v += wdetJb * dF(q; dq) with the exterior state fixed (Freestream_Jacobian, bc_freestream.h:75-114)
// T: precision of dq and v (the state math stays FP64); FP32 serves the mixed-precision Krylov solve
template <typename T>
__global__ void k_freestream_jac(int P, int Q, const int32_t *__restrict__ offsets, const int32_t *__restrict__ faces, FaceBasis b,
                                 hb::PhysConst<double> pc, Exterior ex, const double *__restrict__ qd, const double *__restrict__ jac,
                                 const T *__restrict__ dq, T *__restrict__ v) {
  __shared__ double sN[5][kMaxP2], sF[5][kMaxQ2];
  const int f = faces[blockIdx.x], t = threadIdx.x, P2 = P * P, Q2 = Q * Q;
  for (int i = t; i < 5 * P2; i += blockDim.x) sN[i % 5][i / 5] = (double)dq[offsets[(int64_t)f * P2 + i / 5] + i % 5];
  __syncthreads();
  if (t < Q2) {
    const int q0 = t % Q, q1 = t / Q;
    double dU[5] = {0, 0, 0, 0, 0}, U[5];
    for (int p = 0; p < P2; p++) {
      const double w = b2(b, P, q0, q1, p % P, p / P);
      for (int c = 0; c < 5; c++) dU[c] += w * sN[c][p];
    }
    for (int c = 0; c < 5; c++) U[c] = jac[((int64_t)f * 5 + c) * Q2 + t];
    hb::St<double> s, ds, sx, dsx;
    hb::SAux<double> aux;
    hb::state_from_q_rt(ex.sv, pc, U, s, aux);
    hb::state_from_q_fwd_rt(ex.sv, pc, s, aux, dU, ds);
    exterior_state(ex, sx);
    memset(&dsx, 0, sizeof dsx);
    const double *qf = qd + (int64_t)f * 10 * Q2;
    const double wdetJb = qf[t], n[3] = {qf[Q2 + t], qf[2 * Q2 + t], qf[3 * Q2 + t]};
    double dF[5];
    if (ex.hllc) hb::riemann::hllc_flux_fwd(ex.gamma, ex.cv, s, ds, sx, dsx, n, dF);
    else hb::riemann::hll_flux_fwd(ex.gamma, ex.cv, s, ds, sx, dsx, n, dF);
    for (int c = 0; c < 5; c++) sF[c][t] = wdetJb * dF[c];
  }
  __syncthreads();
  for (int i = t; i < 5 * P2; i += blockDim.x) {
    const int p = i / 5, c = i % 5;
    double acc = 0;
    for (int k = 0; k < Q2; k++) acc += b2(b, P, k % Q, k / Q, p % P, p / P) * sF[c][k];
    v[offsets[(int64_t)f * P2 + p] + c] = (T)((double)v[offsets[(int64_t)f * P2 + p] + c] + acc);
  }
}

// diag += sum over the face's points of B_p^2 wdetJb dF_c/dU_c: the diagonal of the operator above, each point's
// Jacobian column c taken by the forward tangent with dU = e_c (libCEED diagonal assembly of Freestream_Jacobian).
// FULL: the whole 5 x 5 point block, out[(node * 5 + i) * 5 + j] += sum B_p^2 wdetJb dF_i/dU_j (point-block assembly).
template <bool FULL>
__global__ void k_freestream_diag(int P, int Q, const int32_t *__restrict__ offsets, const int32_t *__restrict__ faces, FaceBasis b,
                                  hb::PhysConst<double> pc, Exterior ex, const double *__restrict__ qd, const double *__restrict__ jac,
                                  double *__restrict__ diag) {
  constexpr int NC = FULL ? 25 : 5;
  __shared__ double sD[NC][kMaxQ2];
  const int f = faces[blockIdx.x], t = threadIdx.x, P2 = P * P, Q2 = Q * Q;
  if (t < Q2) {
    double U[5];
    for (int c = 0; c < 5; c++) U[c] = jac[((int64_t)f * 5 + c) * Q2 + t];
    hb::St<double> s, sx, dsx;
    hb::SAux<double> aux;
    hb::state_from_q_rt(ex.sv, pc, U, s, aux);
    exterior_state(ex, sx);
    memset(&dsx, 0, sizeof dsx);
    const double *qf = qd + (int64_t)f * 10 * Q2;
    const double wdetJb = qf[t], n[3] = {qf[Q2 + t], qf[2 * Q2 + t], qf[3 * Q2 + t]};
#pragma unroll
    for (int c = 0; c < 5; c++) {  // unrolled: c indexes registers, not a local array
      double dU[5] = {0, 0, 0, 0, 0}, dF[5];
      dU[c] = 1.0;
      hb::St<double> ds;
      hb::state_from_q_fwd_rt(ex.sv, pc, s, aux, dU, ds);
      if (ex.hllc) hb::riemann::hllc_flux_fwd(ex.gamma, ex.cv, s, ds, sx, dsx, n, dF);
      else hb::riemann::hll_flux_fwd(ex.gamma, ex.cv, s, ds, sx, dsx, n, dF);
      if (FULL) {
#pragma unroll
        for (int i = 0; i < 5; i++) sD[i * 5 + c][t] = wdetJb * dF[i];
      } else {
        sD[c][t] = wdetJb * dF[c];
      }
    }
  }
  __syncthreads();
  for (int i = t; i < NC * P2; i += blockDim.x) {
    const int p = i / NC, c = i % NC;
    double acc = 0;
    for (int k = 0; k < Q2; k++) {
      const double w = b2(b, P, k % Q, k / Q, p % P, p / P);
      acc += w * w * sD[c][k];
    }
    const int64_t o = offsets[(int64_t)f * P2 + p];
    diag[FULL ? o * 5 + c : o + c] += acc;  // FULL: c = i * 5 + j
  }
}

FaceBasis fbasis(const HbFaceOp *op) {
  FaceBasis b;
  memset(&b, 0, sizeof b);
  memcpy(b.B, op->interp1d, sizeof(double) * op->P * op->Q);
  memcpy(b.G, op->grad1d, sizeof(double) * op->P * op->Q);
  memcpy(b.w, op->qweight1d, sizeof(double) * op->Q);
  return b;
}

int nthreads(const HbFaceOp *op) {
  const int m = op->Q * op->Q > 5 * op->P * op->P ? op->Q * op->Q : 5 * op->P * op->P;
  return (m + 31) / 32 * 32 > 1024 ? 1024 : (m + 31) / 32 * 32;
}

int unpack_ctx(const void *ctx264, hb::PhysConst<double> &pc, Exterior &ex) {
  HbFreestreamContext c;
  memcpy(&c, ctx264, sizeof c);
  if (c.newt.state_var != HB_STATEVAR_CONSERVATIVE && c.newt.state_var != HB_STATEVAR_PRIMITIVE && c.newt.state_var != HB_STATEVAR_ENTROPY)
    return HB_ERROR_UNSUPPORTED;
  memset(&pc, 0, sizeof pc);
  ex.sv = c.newt.state_var;
  pc.cv = c.newt.gas.cv;
  pc.inv_cv = 1.0 / c.newt.gas.cv;
  pc.gm1 = c.newt.gas.cp / c.newt.gas.cv - 1;
  pc.Rgas = c.newt.gas.cp - c.newt.gas.cv;
  ex.cv = c.newt.gas.cv;
  ex.gamma = c.newt.gas.cp / c.newt.gas.cv;
  ex.gm1 = ex.gamma - 1;
  memcpy(ex.U, c.S_infty_U, sizeof ex.U);
  memcpy(ex.Y, c.S_infty_Y, sizeof ex.Y);
  return HB_SUCCESS;
}

template <typename T>
int freestream_jac(const HbFaceOp *op, const void *ctx264, int flux_type, const double *qdata_sur, const double *jac_data_sur, const T *dq, T *v,
                          void *stream) {
  if (!op || !ctx264 || !qdata_sur || !jac_data_sur || !dq || !v || (flux_type != 0 && flux_type != 1)) return HB_ERROR_INVALID;
  hb::PhysConst<double> pc;
  Exterior ex;
  int err = unpack_ctx(ctx264, pc, ex);
  if (err) return err;
  ex.hllc = flux_type == 1;
  const FaceBasis b = fbasis(op);
  for (int c = 0; c < op->num_colors; c++) {
    const int n = op->h_color_ptr[c + 1] - op->h_color_ptr[c];
    if (n)
      k_freestream_jac<T><<<n, nthreads(op), 0, (cudaStream_t)stream>>>(op->P, op->Q, op->d_offsets, op->d_color_elem + op->h_color_ptr[c], b, pc,
                                                                         ex, qdata_sur, jac_data_sur, dq, v);
  }
  return rc();
}

}  // namespace

extern "C" {

int hb_faceop_create(int num_faces, int P, int Q, const int32_t *offsets, int64_t l_size, const double *interp1d, const double *grad1d,
                     const double *qweight1d, HbFaceOp **out) {
  *out = NULL;
  if (num_faces < 1 || P < 2 || Q < 1 || P > HB_MAX_P || Q > HB_MAX_P || P * P > kMaxP2 || Q * Q > kMaxQ2 || !offsets) return HB_ERROR_INVALID;
  const int P2 = P * P;
  for (int64_t i = 0; i < (int64_t)num_faces * P2; i++)
    if (offsets[i] < 0 || (int64_t)offsets[i] + 4 >= l_size) return HB_ERROR_INVALID;
  HbFaceOp *op = (HbFaceOp *)calloc(1, sizeof *op);
  if (!op) return HB_ERROR_NOMEM;
  op->num_faces = num_faces;
  op->P = P;
  op->Q = Q;
  op->l_size = l_size;
  memcpy(op->interp1d, interp1d, sizeof(double) * P * Q);
  memcpy(op->grad1d, grad1d, sizeof(double) * P * Q);
  memcpy(op->qweight1d, qweight1d, sizeof(double) * Q);
  int32_t *lst = NULL;
  int err = hb_internal_color_elements(num_faces, P2, offsets, l_size, &op->h_color_ptr, &lst, &op->num_colors);
  if (err) {
    free(op);
    return err;
  }
  cudaGetDevice(&op->device);
  if (cudaMalloc((void **)&op->d_offsets, sizeof(int32_t) * (size_t)num_faces * P2) != cudaSuccess ||
      cudaMalloc((void **)&op->d_color_elem, sizeof(int32_t) * (size_t)num_faces) != cudaSuccess ||
      cudaMemcpy(op->d_offsets, offsets, sizeof(int32_t) * (size_t)num_faces * P2, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(op->d_color_elem, lst, sizeof(int32_t) * (size_t)num_faces, cudaMemcpyHostToDevice) != cudaSuccess) {
    free(lst);
    hb_faceop_destroy(op);
    return HB_ERROR_CUDA;
  }
  free(lst);
  *out = op;
  return HB_SUCCESS;
}

int hb_faceop_destroy(HbFaceOp *op) {
  if (!op) return HB_SUCCESS;
  if (op->d_offsets) cudaFree(op->d_offsets);
  if (op->d_color_elem) cudaFree(op->d_color_elem);
  free(op->h_color_ptr);
  free(op);
  return HB_SUCCESS;
}

int hb_face_setup_qdata(const HbFaceOp *op, const double *x_nodes, double *qdata_sur, void *stream) {
  if (!op) return HB_ERROR_INVALID;
  return hb_face_setup_qdata_nodes(op->num_faces, op->P, op->Q, op->interp1d, op->grad1d, op->qweight1d, x_nodes, qdata_sur, stream);
}

int hb_face_setup_qdata_nodes(int num_faces, int P, int Q, const double *interp1d, const double *grad1d, const double *qweight1d,
                              const double *x_nodes, double *qdata_sur, void *stream) {
  if (num_faces < 0 || P < 2 || Q < 1 || P > HB_MAX_P || Q > HB_MAX_P || Q * Q > kMaxQ2 || !interp1d || !grad1d || !qweight1d || !x_nodes ||
      !qdata_sur)
    return HB_ERROR_INVALID;
  if (num_faces == 0) return HB_SUCCESS;
  FaceBasis b;
  memset(&b, 0, sizeof b);
  memcpy(b.B, interp1d, sizeof(double) * P * Q);
  memcpy(b.G, grad1d, sizeof(double) * P * Q);
  memcpy(b.w, qweight1d, sizeof(double) * Q);
  k_face_setup<<<num_faces, (Q * Q + 31) / 32 * 32, 0, (cudaStream_t)stream>>>(P, Q, b, x_nodes, qdata_sur);
  return rc();
}

int hb_freestream_apply(const HbFaceOp *op, const void *ctx264, int flux_type, const double *qdata_sur, const double *q, double *jac_data_sur,
                        double *v, void *stream) {
  if (!op || !ctx264 || !qdata_sur || !q || !v || (flux_type != 0 && flux_type != 1)) return HB_ERROR_INVALID;
  hb::PhysConst<double> pc;
  Exterior ex;
  int err = unpack_ctx(ctx264, pc, ex);
  if (err) return err;
  ex.hllc = flux_type == 1;
  const FaceBasis b = fbasis(op);
  for (int c = 0; c < op->num_colors; c++) {
    const int n = op->h_color_ptr[c + 1] - op->h_color_ptr[c];
    if (n)
      k_freestream<<<n, nthreads(op), 0, (cudaStream_t)stream>>>(op->P, op->Q, op->d_offsets, op->d_color_elem + op->h_color_ptr[c], b, pc, ex,
                                                                  qdata_sur, q, jac_data_sur, v);
  }
  return rc();
}

int hb_freestream_jacobian_apply(const HbFaceOp *op, const void *ctx264, int flux_type, const double *qdata_sur, const double *jac_data_sur,
                                 const double *dq, double *v, void *stream) {
  return freestream_jac<double>(op, ctx264, flux_type, qdata_sur, jac_data_sur, dq, v, stream);
}

static int freestream_diag(const HbFaceOp *op, const void *ctx264, int flux_type, const double *qdata_sur, const double *jac_data_sur, double *diag,
                           void *stream, bool full) {
  if (!op || !ctx264 || !qdata_sur || !jac_data_sur || !diag || (flux_type != 0 && flux_type != 1)) return HB_ERROR_INVALID;
  hb::PhysConst<double> pc;
  Exterior ex;
  int err = unpack_ctx(ctx264, pc, ex);
  if (err) return err;
  ex.hllc = flux_type == 1;
  const FaceBasis b = fbasis(op);
  for (int c = 0; c < op->num_colors; c++) {
    const int n = op->h_color_ptr[c + 1] - op->h_color_ptr[c];
    if (!n) continue;
    const int nt = nthreads(op); /* >= Q^2 for the point phase; the block scatter strides over its 25 P^2 entries */
    if (full)
      k_freestream_diag<true><<<n, nt, 0, (cudaStream_t)stream>>>(op->P, op->Q, op->d_offsets, op->d_color_elem + op->h_color_ptr[c], b, pc, ex,
                                                                  qdata_sur, jac_data_sur, diag);
    else
      k_freestream_diag<false><<<n, nt, 0, (cudaStream_t)stream>>>(op->P, op->Q, op->d_offsets, op->d_color_elem + op->h_color_ptr[c], b, pc, ex,
                                                                   qdata_sur, jac_data_sur, diag);
  }
  return rc();
}

int hb_freestream_diagonal(const HbFaceOp *op, const void *ctx264, int flux_type, const double *qdata_sur, const double *jac_data_sur, double *diag,
                           void *stream) {
  return freestream_diag(op, ctx264, flux_type, qdata_sur, jac_data_sur, diag, stream, false);
}

int hb_freestream_point_block_diagonal(const HbFaceOp *op, const void *ctx264, int flux_type, const double *qdata_sur, const double *jac_data_sur,
                                       double *out, void *stream) {
  return freestream_diag(op, ctx264, flux_type, qdata_sur, jac_data_sur, out, stream, true);
}

int hb_freestream_jacobian_apply_f32(const HbFaceOp *op, const void *ctx264, int flux_type, const double *qdata_sur, const double *jac_data_sur,
                                     const float *dq, float *v, void *stream) {
  return freestream_jac<float>(op, ctx264, flux_type, qdata_sur, jac_data_sur, dq, v, stream);
}

}  // extern "C"
