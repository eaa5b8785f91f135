// k_filter.cu -- the differential filter (src/differential_filter.c, qfunctions/differential_filter.h) on the GPU, and the
// SGS training pairs computed from its output.
//
// The filter solves (M + K_alpha) u_bar = b for NC fields on the element operator's mesh, where b_c = int phi f_c with
// f = (P, u, T, u_i u_j) of the resolved state (DifferentialFilter_RHS, differential_filter.h:29-58) and the left-hand
// side per point is v = wdetJ u, Grad_v = wdetJ alpha (dXdx grad u) (DifferentialFilter_LHS_N, :66-128) with
// alpha = kernel_scaling (S Delta)(S Delta), Delta = the dimensional anisotropy tensor (grid-based width) or I, S = the
// width scaling (no wall damping).  The solve is conjugate gradients with the point Jacobi preconditioner (hb_filter.c),
// as the reference configures its KSP (differential_filter.c:174-185).
//
// Kernels here are one CTA per element, one thread per quadrature point, tensor contractions evaluated directly (P, Q
// <= 6); elements of one colour are processed per launch, so the scatter is a plain read-add-write.  This operator runs a
// few dozen times per filtered snapshot, not per time step.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include "honee_b200.h"
#include "newtonian_qf.cuh"
#include "sgs.cuh"

namespace {

constexpr int kMaxQ3 = 216;  // Q <= 6
constexpr int kMaxP3 = 216;

struct FBasis {
  double B[HB_MAX_P * HB_MAX_P], G[HB_MAX_P * HB_MAX_P];  // [Q][P]
};

struct FOpts {
  int grid_based;
  double ws[3];
  double ks;
};

inline int rc() { return cudaGetLastError() == cudaSuccess ? HB_SUCCESS : HB_ERROR_CUDA; }

// alpha = ks (S Delta)(S Delta) at a point with inverse map X (dXdx)
__device__ void filter_alpha(const FOpts &o, const double X[3][3], double al[3][3]) {
  double D[3][3];
  if (o.grid_based) {
    double kmA[6], delta;
    hb::sgs::anisotropy(X, kmA, delta);
#pragma unroll
    for (int k = 0; k < 6; k++) kmA[k] *= delta;
    hb::sgs::km_unpack(kmA, D);
  } else {
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int b = 0; b < 3; b++) D[a][b] = a == b ? 1.0 : 0.0;
  }
  double SD[3][3];
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) SD[a][b] = o.ws[a] * D[a][b];
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) {
      double s = 0;
#pragma unroll
      for (int k = 0; k < 3; k++) s += SD[a][k] * SD[k][b];
      al[a][b] = o.ks * s;
    }
}

// value and reference gradient of nodal field sN [P3] at point (i, j, k)
__device__ __forceinline__ void eval_pt(const double *sN, int P, const FBasis &b, int i, int j, int k, double &v, double g[3]) {
  v = 0;
  g[0] = g[1] = g[2] = 0;
  for (int pc = 0; pc < P; pc++) {
    const double bz = b.B[k * P + pc], gz = b.G[k * P + pc];
    for (int pb = 0; pb < P; pb++) {
      const double by = b.B[j * P + pb], gy = b.G[j * P + pb];
      for (int pa = 0; pa < P; pa++) {
        const double u = sN[(pc * P + pb) * P + pa];
        const double bx = b.B[i * P + pa], gx = b.G[i * P + pa];
        v += bx * by * bz * u;
        g[0] += gx * by * bz * u;
        g[1] += bx * gy * bz * u;
        g[2] += bx * by * gz * u;
      }
    }
  }
}

// y += (M + K_alpha) x for the elements of one colour; x, y node-interleaved [node][nc]
__global__ void k_filter_apply(int P, int Q, int nc, const int32_t *__restrict__ offsets, const int32_t *__restrict__ elems, int n_elems,
                               const double *__restrict__ qdata, FBasis b, FOpts o, const double *__restrict__ x, double *__restrict__ y) {
  __shared__ double sN[kMaxP3], sV[kMaxQ3], sGv[3][kMaxQ3], sX[9][kMaxQ3], sW[kMaxQ3];
  const int e = elems[blockIdx.x], P3 = P * P * P, Q3 = Q * Q * Q, t = threadIdx.x;
  const double *qd = qdata + (int64_t)e * 10 * Q3;
  double al[3][3] = {{0}};
  if (t < Q3) {
    sW[t] = qd[t];
    for (int k = 0; k < 9; k++) sX[k][t] = qd[(1 + k) * Q3 + t];
    double X[3][3];
    for (int k = 0; k < 9; k++) X[k / 3][k % 3] = sX[k][t];
    filter_alpha(o, X, al);
  }
  for (int c = 0; c < nc; c++) {
    __syncthreads();
    for (int p = t; p < P3; p += blockDim.x) sN[p] = x[(int64_t)(offsets[(int64_t)e * P3 + p] / 5) * nc + c];
    __syncthreads();
    if (t < Q3) {
      double v, g[3], X[3][3];
      eval_pt(sN, P, b, t % Q, (t / Q) % Q, t / (Q * Q), v, g);
      for (int k = 0; k < 9; k++) X[k / 3][k % 3] = sX[k][t];
      const double w = sW[t];
      double dq[3], dqx[3];
      for (int k = 0; k < 3; k++) dq[k] = g[0] * X[0][k] + g[1] * X[1][k] + g[2] * X[2][k];
      for (int a = 0; a < 3; a++) dqx[a] = X[a][0] * dq[0] + X[a][1] * dq[1] + X[a][2] * dq[2];
      sV[t] = w * v;
      for (int a = 0; a < 3; a++) sGv[a][t] = w * (al[a][0] * dqx[0] + al[a][1] * dqx[1] + al[a][2] * dqx[2]);
    }
    __syncthreads();
    for (int p = t; p < P3; p += blockDim.x) {
      const int pa = p % P, pb = (p / P) % P, pc = p / (P * P);
      double s = 0;
      for (int q = 0; q < Q3; q++) {
        const int i = q % Q, j = (q / Q) % Q, k = q / (Q * Q);
        const double bx = b.B[i * P + pa], by = b.B[j * P + pb], bz = b.B[k * P + pc];
        const double gx = b.G[i * P + pa], gy = b.G[j * P + pb], gz = b.G[k * P + pc];
        s += bx * by * bz * sV[q] + gx * by * bz * sGv[0][q] + bx * gy * bz * sGv[1][q] + bx * by * gz * sGv[2][q];
      }
      const int64_t idx = (int64_t)(offsets[(int64_t)e * P3 + p] / 5) * nc + c;
      y[idx] += s;
    }
  }
}

// diag += the operator's diagonal at each node (one value per node; it is the same for every field)
__global__ void k_filter_diag(int P, int Q, const int32_t *__restrict__ offsets, const int32_t *__restrict__ elems, const double *__restrict__ qdata,
                              FBasis b, FOpts o, double *__restrict__ diag) {
  __shared__ double sW[kMaxQ3], sX[9][kMaxQ3], sA[9][kMaxQ3];
  const int e = elems[blockIdx.x], P3 = P * P * P, Q3 = Q * Q * Q, t = threadIdx.x;
  const double *qd = qdata + (int64_t)e * 10 * Q3;
  if (t < Q3) {
    sW[t] = qd[t];
    double X[3][3], al[3][3];
    for (int k = 0; k < 9; k++) X[k / 3][k % 3] = sX[k][t] = qd[(1 + k) * Q3 + t];
    filter_alpha(o, X, al);
    for (int k = 0; k < 9; k++) sA[k][t] = al[k / 3][k % 3];
  }
  __syncthreads();
  for (int p = t; p < P3; p += blockDim.x) {
    const int pa = p % P, pb = (p / P) % P, pc = p / (P * P);
    double s = 0;
    for (int q = 0; q < Q3; q++) {
      const int i = q % Q, j = (q / Q) % Q, k = q / (Q * Q);
      const double bx = b.B[i * P + pa], by = b.B[j * P + pb], bz = b.B[k * P + pc];
      const double g[3] = {b.G[i * P + pa] * by * bz, bx * b.G[j * P + pb] * bz, bx * by * b.G[k * P + pc]};
      const double phi = bx * by * bz;
      double dq[3], dqx[3];
      for (int kk = 0; kk < 3; kk++) dq[kk] = g[0] * sX[0 * 3 + kk][q] + g[1] * sX[1 * 3 + kk][q] + g[2] * sX[2 * 3 + kk][q];
      for (int a = 0; a < 3; a++) dqx[a] = sX[a * 3 + 0][q] * dq[0] + sX[a * 3 + 1][q] * dq[1] + sX[a * 3 + 2][q] * dq[2];
      double gv = 0;
      for (int a = 0; a < 3; a++) gv += g[a] * (sA[a * 3 + 0][q] * dqx[0] + sA[a * 3 + 1][q] * dqx[1] + sA[a * 3 + 2][q] * dqx[2]);
      s += sW[q] * (phi * phi + gv);
    }
    diag[offsets[(int64_t)e * P3 + p] / 5] += s;
  }
}

// b += int phi f(q) with f = (P, u, T, uu_xx, uu_yy, uu_zz, uu_yz, uu_xz, uu_xy) of the state q in the variable sv, b
// node-interleaved [node][11] (DifferentialFilter_RHS_Conserv / _Prim / _Entropy, qfunctions/differential_filter.h:29-68)
__global__ void k_filter_rhs(int P, int Q, const int32_t *__restrict__ offsets, const int32_t *__restrict__ elems, const double *__restrict__ qdata,
                             FBasis b, hb::PhysConst<double> pc, int sv, const double *__restrict__ q, double *__restrict__ rhs) {
  __shared__ double sN[5][kMaxP3], sF[11][kMaxQ3];
  const int e = elems[blockIdx.x], P3 = P * P * P, Q3 = Q * Q * Q, t = threadIdx.x;
  for (int p = t; p < 5 * P3; p += blockDim.x) sN[p % 5][p / 5] = q[offsets[(int64_t)e * P3 + p / 5] + p % 5];
  __syncthreads();
  if (t < Q3) {
    const int i = t % Q, j = (t / Q) % Q, k = t / (Q * Q);
    double U[5];
    for (int c = 0; c < 5; c++) {
      double g[3];
      eval_pt(sN[c], P, b, i, j, k, U[c], g);
    }
    hb::St<double> s;
    hb::SAux<double> aux;
    hb::state_from_q_rt(sv, pc, U, s, aux);
    const double w = qdata[(int64_t)e * 10 * Q3 + t];
    const double f[11] = {s.P, s.u[0], s.u[1], s.u[2], s.T_, s.u[0] * s.u[0], s.u[1] * s.u[1], s.u[2] * s.u[2], s.u[1] * s.u[2], s.u[0] * s.u[2], s.u[0] * s.u[1]};
    for (int c = 0; c < 11; c++) sF[c][t] = w * f[c];
  }
  __syncthreads();
  for (int pp = t; pp < 11 * P3; pp += blockDim.x) {
    const int p = pp % P3, c = pp / P3;
    const int pa = p % P, pb = (p / P) % P, pcz = p / (P * P);
    double acc = 0;
    for (int qq = 0; qq < Q3; qq++) {
      const int i = qq % Q, j = (qq / Q) % Q, k = qq / (Q * Q);
      acc += b.B[i * P + pa] * b.B[j * P + pb] * b.B[k * P + pcz] * sF[c][qq];
    }
    rhs[(int64_t)(offsets[(int64_t)e * P3 + p] / 5) * 11 + c] += acc;
  }
}

// Training pairs at every quadrature point from filtered nodal fields f [node][11] = (P, u, T, uu(6)) of the filter:
// X = model inputs of the filtered velocity gradient with the anisotropy of this mesh and the width scaled by
// width_scale (the filter width relative to this mesh's elements); Y = the filtered stress uu - u u in the model's
// output frame, scaled by delta^2 |G A|^2 (not yet min-max normalised).  FP32 outputs [E * Q^3][6].
__global__ void k_sgs_pairs(int P, int Q, const int32_t *__restrict__ offsets, const double *__restrict__ qdata, FBasis b, double mu, double Rgas,
                            double width_scale, const double *__restrict__ f, float *__restrict__ X, float *__restrict__ Y) {
  __shared__ double sN[11][kMaxP3];
  const int e = blockIdx.x, P3 = P * P * P, Q3 = Q * Q * Q, t = threadIdx.x;
  for (int p = t; p < 11 * P3; p += blockDim.x) sN[p % 11][p / 11] = f[(int64_t)(offsets[(int64_t)e * P3 + p / 11] / 5) * 11 + p % 11];
  __syncthreads();
  if (t >= Q3) return;
  const int i = t % Q, j = (t / Q) % Q, k = t / (Q * Q);
  double v[11], gu[3][3];
  for (int c = 0; c < 11; c++) {
    double g[3];
    eval_pt(sN[c], P, b, i, j, k, v[c], g);
    if (c >= 1 && c <= 3)
      for (int r = 0; r < 3; r++) gu[c - 1][r] = g[r];
  }
  const double *qd = qdata + (int64_t)e * 10 * Q3;
  double Xm[3][3];
  for (int kk = 0; kk < 9; kk++) Xm[kk / 3][kk % 3] = qd[(1 + kk) * Q3 + t];
  double G[3][3];
  for (int a = 0; a < 3; a++)
    for (int c = 0; c < 3; c++) G[a][c] = gu[a][0] * Xm[0][c] + gu[a][1] * Xm[1][c] + gu[a][2] * Xm[2][c];
  double kmA[6], delta;
  hb::sgs::anisotropy(Xm, kmA, delta);
  delta *= width_scale;
  const double rho = v[0] / (Rgas * v[4]);
  double E[3][3], in[6], gmag;
  hb::sgs::inputs(G, kmA, delta, mu / rho, E, in, gmag);
  const double u0 = v[1], u1 = v[2], u2 = v[3];
  const double tau[6] = {v[5] - u0 * u0, v[6] - u1 * u1, v[7] - u2 * u2, v[8] - u1 * u2, v[9] - u0 * u2, v[10] - u0 * u1};
  double o[6];
  hb::sgs::stress_to_sframe(tau, delta, E, gmag, o);
  const int64_t s = (int64_t)e * Q3 + t;
  for (int c = 0; c < 6; c++) {
    X[s * 6 + c] = (float)in[c];
    Y[s * 6 + c] = (float)o[c];
  }
}

// conservative state (rho, rho u, E) of filtered fields (P, u, T, ...) [node][11], rho = P / (R T)
// the state of the filtered primitive fields (P, u, T) in the variable sv: conservative (StateConservativeFromPrimitive,
// newtonian_state.h:159-168), primitive as is, entropy (StateEntropyFromPrimitive, :91-103)
__global__ void k_filtered_state(const double *__restrict__ f, int64_t nodes, double cv, double R, int sv, double *__restrict__ q) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nodes; i += (int64_t)gridDim.x * blockDim.x) {
    const double *g = f + i * 11;
    const double rho = g[0] / (R * g[4]);
    const double ke = 0.5 * (g[1] * g[1] + g[2] * g[2] + g[3] * g[3]);
    if (sv == HB_STATEVAR_PRIMITIVE) {
      for (int c = 0; c < 5; c++) q[i * 5 + c] = g[c];
    } else if (sv == HB_STATEVAR_ENTROPY) {
      const double gamma = (cv + R) / cv, ent = log(g[0]) - gamma * log(rho), rho_p = rho / g[0];
      q[i * 5 + 0] = (gamma - ent) / (gamma - 1) - rho_p * ke;
      for (int c = 1; c < 4; c++) q[i * 5 + c] = rho_p * g[c];
      q[i * 5 + 4] = -rho_p;
    } else {
      q[i * 5 + 0] = rho;
      q[i * 5 + 1] = rho * g[1];
      q[i * 5 + 2] = rho * g[2];
      q[i * 5 + 3] = rho * g[3];
      q[i * 5 + 4] = rho * (cv * g[4] + ke);
    }
  }
}

__global__ void k_expand_recip(const double *__restrict__ d, int64_t nodes, int nc, double *__restrict__ dinv) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nodes * nc; i += (int64_t)gridDim.x * blockDim.x) dinv[i] = 1.0 / d[i / nc];
}

FBasis fbasis(const HbElemOp *op) {
  FBasis b;
  memset(&b, 0, sizeof b);
  memcpy(b.B, op->interp1d, sizeof(double) * op->P * op->Q);
  memcpy(b.G, op->grad1d, sizeof(double) * op->P * op->Q);
  return b;
}

FOpts fopts(const HbFilterOptions *o) {
  FOpts f;
  f.grid_based = o->grid_based_width;
  for (int i = 0; i < 3; i++) f.ws[i] = o->width_scaling[i];
  f.ks = o->kernel_scaling;
  return f;
}

int nthreads(const HbElemOp *op) {
  const int Q3 = op->Q * op->Q * op->Q, P3 = op->P * op->P * op->P;
  const int m = Q3 > P3 ? Q3 : P3;
  return (m + 31) / 32 * 32;
}

bool fits(const HbElemOp *op) { return op->Q * op->Q * op->Q <= kMaxQ3 && op->P * op->P * op->P <= kMaxP3; }

}  // namespace

extern "C" {

int hb_filter_apply(const HbElemOp *op, int nc, const HbFilterOptions *o, const double *qdata, const double *x, double *y, void *stream) {
  if (!op || !o || !qdata || !x || !y || nc < 1 || !fits(op)) return HB_ERROR_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t nodes = op->l_size / 5;
  if (cudaMemsetAsync(y, 0, sizeof(double) * nodes * nc, s) != cudaSuccess) return HB_ERROR_CUDA;
  const FBasis b = fbasis(op);
  const FOpts f = fopts(o);
  for (int c = 0; c < op->num_colors; c++) {
    const int n = op->h_color_ptr[c + 1] - op->h_color_ptr[c];
    if (n) k_filter_apply<<<n, nthreads(op), 0, s>>>(op->P, op->Q, nc, op->d_offsets, op->d_color_elem + op->h_color_ptr[c], n, qdata, b, f, x, y);
  }
  return rc();
}

int hb_filter_diagonal(const HbElemOp *op, const HbFilterOptions *o, const double *qdata, double *diag, void *stream) {
  if (!op || !o || !qdata || !diag || !fits(op)) return HB_ERROR_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemsetAsync(diag, 0, sizeof(double) * (op->l_size / 5), s) != cudaSuccess) return HB_ERROR_CUDA;
  const FBasis b = fbasis(op);
  const FOpts f = fopts(o);
  for (int c = 0; c < op->num_colors; c++) {
    const int n = op->h_color_ptr[c + 1] - op->h_color_ptr[c];
    if (n) k_filter_diag<<<n, nthreads(op), 0, s>>>(op->P, op->Q, op->d_offsets, op->d_color_elem + op->h_color_ptr[c], qdata, b, f, diag);
  }
  return rc();
}

int hb_filter_rhs(const HbElemOp *op, const void *ctx184, const double *qdata, const double *q, double *rhs, void *stream) {
  if (!op || !ctx184 || !qdata || !q || !rhs || !fits(op)) return HB_ERROR_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemsetAsync(rhs, 0, sizeof(double) * (op->l_size / 5) * 11, s) != cudaSuccess) return HB_ERROR_CUDA;
  HbNewtonianContext c;
  memcpy(&c, ctx184, sizeof c);
  if (c.state_var != HB_STATEVAR_CONSERVATIVE && c.state_var != HB_STATEVAR_PRIMITIVE && c.state_var != HB_STATEVAR_ENTROPY) return HB_ERROR_UNSUPPORTED;
  hb::PhysConst<double> pc;
  memset(&pc, 0, sizeof pc);
  pc.cv = c.gas.cv;
  pc.inv_cv = 1.0 / c.gas.cv;
  pc.gm1 = c.gas.cp / c.gas.cv - 1;
  pc.Rgas = c.gas.cp - c.gas.cv;
  const FBasis b = fbasis(op);
  for (int k = 0; k < op->num_colors; k++) {
    const int n = op->h_color_ptr[k + 1] - op->h_color_ptr[k];
    if (n) k_filter_rhs<<<n, nthreads(op), 0, s>>>(op->P, op->Q, op->d_offsets, op->d_color_elem + op->h_color_ptr[k], qdata, b, pc, c.state_var, q, rhs);
  }
  return rc();
}

int hb_filter_jacobi(const double *diag, int64_t nodes, int nc, double *dinv, void *stream) {
  if (!diag || !dinv || nodes < 0 || nc < 1) return HB_ERROR_INVALID;
  if (nodes) k_expand_recip<<<148 * 8, 256, 0, (cudaStream_t)stream>>>(diag, nodes, nc, dinv);
  return rc();
}

int hb_filtered_state(const double *filtered, int64_t nodes, const void *ctx184, double *q, void *stream) {
  if (!filtered || !ctx184 || !q || nodes < 0) return HB_ERROR_INVALID;
  HbNewtonianContext c;
  memcpy(&c, ctx184, sizeof c);
  if (c.state_var != HB_STATEVAR_CONSERVATIVE && c.state_var != HB_STATEVAR_PRIMITIVE && c.state_var != HB_STATEVAR_ENTROPY) return HB_ERROR_UNSUPPORTED;
  if (nodes) k_filtered_state<<<148 * 8, 256, 0, (cudaStream_t)stream>>>(filtered, nodes, c.gas.cv, c.gas.cp - c.gas.cv, c.state_var, q);
  return rc();
}

int hb_sgs_training_pairs(const HbElemOp *op, const void *ctx184, const double *qdata, const double *filtered, double width_scale, float *X, float *Y,
                          void *stream) {
  if (!op || !ctx184 || !qdata || !filtered || !X || !Y || !fits(op) || !(width_scale > 0)) return HB_ERROR_INVALID;
  HbNewtonianContext c;
  memcpy(&c, ctx184, sizeof c);
  k_sgs_pairs<<<op->num_elem, nthreads(op), 0, (cudaStream_t)stream>>>(op->P, op->Q, op->d_offsets, qdata, fbasis(op), c.gas.mu, c.gas.cp - c.gas.cv,
                                                                        width_scale, filtered, X, Y);
  return rc();
}

}  // extern "C"
