// sgs.cuh -- point-wise pieces of the data-driven subgrid-stress (SGS) closure, host and device.
//
// Restates, per quadrature point:
//   * the 3x3 symmetric eigen-solver the closure uses (max-pivot Jacobi rotations with the stopping rule, rotation
//     formulas and descending sort of qfunctions/utils_eigensolver_jacobi.h:26-173 -- the published jacobi_pd scheme);
//     the pivot sequence decides eigenvector signs and order, so it is kept alike on purpose
//   * the grid anisotropy tensor A_ij and width delta from the inverse metric (qfunctions/grid_anisotropy_tensor.h:14-32)
//   * the rotation-invariant model inputs in the strain-rate eigenframe (qfunctions/sgs_dd_utils.h:58-96), the
//     de-normalisation and rotation of the model outputs back to a physical stress (sgs_dd_utils.h:107-127), and the
//     inverse of that map, which turns a filtered stress into a training target
//   * the multilayer perceptron in the weight layout of the reference's SgsDDContext (sgs_dd_model.h:38-53: hidden
//     layers V = b + W x with W row-major [out][in], leaky-ReLU slope alpha, linear output), here with one or two hidden
//     layers and FP32 weights
//   * the SGS flux in the residual (sgs_dd_model.h:205-217)
// Every array index is a compile-time constant so kernel parameters are read from the constant bank, never copied.
#pragma once

#include <math.h>

#ifndef HB_HD
#define HB_HD __host__ __device__ __forceinline__
#endif

namespace hb {
namespace sgs {

template <typename T>
HB_HD T habs(T x) { return x < T(0) ? -x : x; }

// Kelvin-Mandel pack/unpack (utils.h:239-258): off-diagonals weighted by sqrt(2), order 00 11 22 12 02 01
template <typename T>
HB_HD void km_unpack(const T v[6], T A[3][3]) {
  const T w = T(1) / T(sqrt(2.));
  A[0][0] = v[0];
  A[1][1] = v[1];
  A[2][2] = v[2];
  A[1][2] = A[2][1] = w * v[3];
  A[0][2] = A[2][0] = w * v[4];
  A[0][1] = A[1][0] = w * v[5];
}
template <typename T>
HB_HD void km_pack(const T A[3][3], T v[6]) {
  const T w = T(sqrt(2.));
  v[0] = A[0][0];
  v[1] = A[1][1];
  v[2] = A[2][2];
  v[3] = A[2][1] * w;
  v[4] = A[2][0] * w;
  v[5] = A[1][0] * w;
}

// One Jacobi rotation on pivot P (0: (0,1), 1: (0,2), 2: (1,2)); returns true when the pivot is negligible (done).
// The pivot is a template constant so every operand stays in a register.
template <int P, typename T>
HB_HD bool jacobi_rotate(T &d0, T &d1, T &d2, T &u01, T &u02, T &u12, T evec[3][3]) {
  constexpr int i = P == 2 ? 1 : 0, j = P == 0 ? 1 : 2;
  T &aij = P == 0 ? u01 : (P == 1 ? u02 : u12);
  T &aii = P == 2 ? d1 : d0;
  T &ajj = P == 0 ? d1 : d2;
  // the entries coupling the third index with i and with j, in upper-triangle storage
  T &awi = P == 0 ? u02 : u01;
  T &awj = P == 2 ? u02 : u12;
  if (aii + aij == aii && ajj + aij == ajj) aij = T(0);
  if (aij == T(0)) return true;
  T t = T(1);
  const T djj_ii = ajj - aii;
  if (djj_ii != T(0)) {
    T kappa = djj_ii;
    kappa /= (T(2) * aij);
    t = T(1) / (T(sqrt(T(1) + kappa * kappa)) + habs(kappa));
    if (kappa < T(0)) t = -t;
  }
  const T c = T(1) / T(sqrt(T(1) + t * t)), s = c * t;
  aii -= t * aij;
  ajj += t * aij;
  aij = T(0);
  const T wi = awi, wj = awj;
  awi = c * wi - s * wj;
  awj = s * wi + c * wj;
#pragma unroll
  for (int v = 0; v < 3; v++) {
    const T ei = evec[i][v];
    evec[i][v] = c * ei - s * evec[j][v];
    evec[j][v] = s * ei + c * evec[j][v];
  }
  return false;
}

template <int A, int B, typename T>
HB_HD void swap_rows(T eval[3], T evec[3][3]) {
  const T te = eval[A];
  eval[A] = eval[B];
  eval[B] = te;
#pragma unroll
  for (int v = 0; v < 3; v++) {
    const T tv = evec[A][v];
    evec[A][v] = evec[B][v];
    evec[B][v] = tv;
  }
}

// Symmetric 3x3 eigen-decomposition by Jacobi rotations on the largest off-diagonal entry (ties resolved in the order
// (0,1), (0,2), (1,2)), at most 3 max_sweeps rotations.  A is read (upper triangle and diagonal); eval descending, evec
// rows are the eigenvectors.  Returns the rotation count, 0 when the sweep budget ran out.
template <typename T>
HB_HD int eig3(const T A[3][3], T eval[3], T evec[3][3], int max_sweeps) {
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) evec[a][b] = a == b ? T(1) : T(0);
  T d0 = A[0][0], d1 = A[1][1], d2 = A[2][2], u01 = A[0][1], u02 = A[0][2], u12 = A[1][2];
  const int max_iters = max_sweeps * 3;
  int it = 1;
  for (; it <= max_iters; it++) {
    int p = 0;
    T m = habs(u01);
    if (habs(u02) > m) {
      p = 1;
      m = habs(u02);
    }
    if (habs(u12) > m) p = 2;
    const bool done = p == 0 ? jacobi_rotate<0>(d0, d1, d2, u01, u02, u12, evec)
                             : (p == 1 ? jacobi_rotate<1>(d0, d1, d2, u01, u02, u12, evec) : jacobi_rotate<2>(d0, d1, d2, u01, u02, u12, evec));
    if (done) break;
  }
  eval[0] = d0;
  eval[1] = d1;
  eval[2] = d2;
  // selection sort, descending, swapping eigenvector rows along (fixed indices, so nothing leaves the registers)
  {
    int am = 0;
    T mv = eval[0];
    if (eval[1] > mv) {
      am = 1;
      mv = eval[1];
    }
    if (eval[2] > mv) am = 2;
    if (am == 1) swap_rows<0, 1>(eval, evec);
    else if (am == 2) swap_rows<0, 2>(eval, evec);
    if (eval[2] > eval[1]) swap_rows<1, 2>(eval, evec);
  }
  return it > max_iters ? 0 : it;
}

// Anisotropy tensor A_ij (normalised, symmetric) and width delta of an element from dXdx at a point
template <typename T>
HB_HD void anisotropy(const T dXdx[3][3], T km_A[6], T &delta) {
  T g[3][3], km_g[6];
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) {
      T s = T(0);
#pragma unroll
      for (int k = 0; k < 3; k++) s += dXdx[k][a] * dXdx[k][b];
      g[a][b] = s;
    }
  km_pack(g, km_g);
  km_unpack(km_g, g);
  T ev[3], E[3][3];
  eig3(g, ev, E, 15);
#pragma unroll
  for (int a = 0; a < 3; a++) ev[a] = T(1) / T(sqrt(ev[a]));
  T A[3][3];
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) {
      T s = T(0);
#pragma unroll
      for (int k = 0; k < 3; k++) s += E[k][a] * (ev[k] * E[k][b]);
      A[a][b] = s;
    }
  delta = T(sqrt(ev[0] * ev[0] + ev[1] * ev[1] + ev[2] * ev[2]));
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) A[a][b] *= T(1) / delta;
  delta *= T(2);  // physical element size, not the [-1, 1] reference size
  km_pack(A, km_A);
}

// Model inputs from the physical velocity gradient G[i][j] = du_i/dx_j, the anisotropy tensor and width, and the
// kinematic viscosity: eigenvalues of the strain rate of G A and the first two vorticity components in its eigenframe
// (oriented by the vorticity), the viscous number nu / delta^2, all divided by |G A| (+ DBL_EPSILON).
template <typename T>
HB_HD void inputs(const T G[3][3], const T km_A[6], T delta, T nu, T E[3][3], T in[6], T &gmag) {
  T A[3][3], Gi[3][3];
  km_unpack(km_A, A);
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) {
      T s = T(0);
#pragma unroll
      for (int k = 0; k < 3; k++) s += G[a][k] * A[k][b];
      Gi[a][b] = s;
    }
  T sf[3], wf[3];
  {
    const T w = T(1) / T(sqrt(2.));
    const T km_s[6] = {Gi[0][0], Gi[1][1], Gi[2][2], w * (Gi[1][2] + Gi[2][1]), w * (Gi[0][2] + Gi[2][0]), w * (Gi[0][1] + Gi[1][0])};
    T S[3][3];
    km_unpack(km_s, S);
    eig3(S, sf, E, 5);
  }
  {
    const T r12 = T(0.5) * (Gi[1][2] - Gi[2][1]), r02 = T(0.5) * (Gi[0][2] - Gi[2][0]), r01 = T(0.5) * (Gi[0][1] - Gi[1][0]);
    const T vort[3] = {-2 * r12, 2 * r02, -2 * r01};
    // orient the eigenframe with the vorticity: rows 0 and 2 towards it, row 1 completing a right-handed frame
    T al[3];
#pragma unroll
    for (int a = 0; a < 3; a++) al[a] = E[a][0] * vort[0] + E[a][1] * vort[1] + E[a][2] * vort[2];
    if (al[0] < T(0))
#pragma unroll
      for (int b = 0; b < 3; b++) E[0][b] = -E[0][b];
    if (al[2] < T(0))
#pragma unroll
      for (int b = 0; b < 3; b++) E[2][b] = -E[2][b];
    const T cr[3] = {E[2][1] * E[0][2] - E[2][2] * E[0][1], E[2][2] * E[0][0] - E[2][0] * E[0][2], E[2][0] * E[0][1] - E[2][1] * E[0][0]};
    if (cr[0] * E[1][0] + cr[1] * E[1][1] + cr[2] * E[1][2] < T(0))
#pragma unroll
      for (int b = 0; b < 3; b++) E[1][b] = -E[1][b];
#pragma unroll
    for (int a = 0; a < 3; a++) wf[a] = E[a][0] * vort[0] + E[a][1] * vort[1] + E[a][2] * vort[2];
  }
  gmag = T(sqrt(sf[0] * sf[0] + sf[1] * sf[1] + sf[2] * sf[2] + T(0.5) * (wf[0] * wf[0] + wf[1] * wf[1] + wf[2] * wf[2])));
  const T scale = T(1) / (gmag + T(2.220446049250313e-16));
  in[0] = sf[0] * scale;
  in[1] = sf[1] * scale;
  in[2] = sf[2] * scale;
  in[3] = wf[0] * scale;
  in[4] = wf[1] * scale;
  in[5] = nu / (delta * delta) * scale;
}

// Model outputs (normalised to [0, 1] by min-max bounds b[c] = {lo, hi}) -> physical SGS stress in KM notation:
// de-normalise, scale by delta^2 |G A|^2, rotate from the eigenframe: tau = E^T S E.
template <typename T, typename TB>
HB_HD void outputs_to_stress(const T out_n[6], T delta, const T E[3][3], const TB (&b)[6][2], T gmag, T km_tau[6]) {
  T o[6];
  const T sc = delta * delta * gmag * gmag;
#pragma unroll
  for (int c = 0; c < 6; c++) o[c] = ((T(b[c][1]) - T(b[c][0])) * (out_n[c] - T(1)) + T(b[c][1])) * sc;
  const T S[3][3] = {{o[0], o[3], o[4]}, {o[3], o[1], o[5]}, {o[4], o[5], o[2]}};
  T ES[3][3], tau[3][3];
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int c = 0; c < 3; c++) ES[a][c] = E[0][a] * S[0][c] + E[1][a] * S[1][c] + E[2][a] * S[2][c];
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int c = 0; c < 3; c++) tau[a][c] = ES[a][0] * E[0][c] + ES[a][1] * E[1][c] + ES[a][2] * E[2][c];
  km_pack(tau, km_tau);
}

// Inverse of outputs_to_stress before the min-max step: a physical stress tau (plain components 00 11 22 12 02 01, as
// the filtered u_i u_j - u_i u_j of the training data) -> S = E tau E^T / (delta^2 |G A|^2) in the order 00 11 22 01 02 12
// of the model outputs.
template <typename T>
HB_HD void stress_to_sframe(const T tau6[6], T delta, const T E[3][3], T gmag, T o[6]) {
  const T tau[3][3] = {{tau6[0], tau6[5], tau6[4]}, {tau6[5], tau6[1], tau6[3]}, {tau6[4], tau6[3], tau6[2]}};
  T Et[3][3], S[3][3];
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int c = 0; c < 3; c++) Et[a][c] = E[a][0] * tau[0][c] + E[a][1] * tau[1][c] + E[a][2] * tau[2][c];
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int c = 0; c < 3; c++) S[a][c] = Et[a][0] * E[c][0] + Et[a][1] * E[c][1] + Et[a][2] * E[c][2];
  const T inv = T(1) / (delta * delta * gmag * gmag + T(1e-300));
  o[0] = S[0][0] * inv;
  o[1] = S[1][1] * inv;
  o[2] = S[2][2] * inv;
  o[3] = S[0][1] * inv;
  o[4] = S[0][2] * inv;
  o[5] = S[1][2] * inv;
}

// Fully connected network 6 -> H1 [-> H2] -> 6 with FP32 weights; parameters in one flat array, per layer W [out][in]
// row-major then b [out].  H2 == 0: one hidden layer (the reference's 6-20-6 form).
template <int H1, int H2>
struct MlpShape {
  static constexpr int NI = 6, NO = 6;
  static constexpr int L2IN = H2 > 0 ? H2 : H1;  // width entering the output layer
  static constexpr int oW1 = 0, oB1 = oW1 + H1 * NI, oW2 = oB1 + H1, oB2 = oW2 + (H2 > 0 ? H2 * H1 : 0), oW3 = oB2 + (H2 > 0 ? H2 : 0),
                       oB3 = oW3 + NO * L2IN, size = oB3 + NO;
};

template <int H1, int H2, typename TW, typename T>
HB_HD void mlp_forward(const TW *__restrict__ w, float alpha, const T x[6], T y[6]) {
  using S = MlpShape<H1, H2>;
  T h1[H1];
#pragma unroll
  for (int i = 0; i < H1; i++) {
    T s = T(w[S::oB1 + i]);
#pragma unroll
    for (int j = 0; j < 6; j++) s += T(w[S::oW1 + i * 6 + j]) * x[j];
    h1[i] = s < T(0) ? s * T(alpha) : s;
  }
  if constexpr (H2 > 0) {
    T h2[H2 > 0 ? H2 : 1];
#pragma unroll
    for (int i = 0; i < H2; i++) {
      T s = T(w[S::oB2 + i]);
#pragma unroll
      for (int j = 0; j < H1; j++) s += T(w[S::oW2 + i * H1 + j]) * h1[j];
      h2[i] = s < T(0) ? s * T(alpha) : s;
    }
#pragma unroll
    for (int i = 0; i < 6; i++) {
      T s = T(w[S::oB3 + i]);
#pragma unroll
      for (int j = 0; j < H2; j++) s += T(w[S::oW3 + i * H2 + j]) * h2[j];
      y[i] = s;
    }
  } else {
#pragma unroll
    for (int i = 0; i < 6; i++) {
      T s = T(w[S::oB3 + i]);
#pragma unroll
      for (int j = 0; j < H1; j++) s += T(w[S::oW3 + i * H1 + j]) * h1[j];
      y[i] = s;
    }
  }
}

// SGS flux (sgs_dd_model.h:205-217): momentum rows tau, energy row u . tau, continuity zero; F[comp][dir]
template <typename T>
HB_HD void flux(const T u[3], const T km_tau[6], T F[5][3]) {
  T tau[3][3];
  km_unpack(km_tau, tau);
#pragma unroll
  for (int j = 0; j < 3; j++) {
    F[0][j] = T(0);
#pragma unroll
    for (int k = 0; k < 3; k++) F[k + 1][j] = tau[k][j];
    F[4][j] = u[0] * tau[0][j] + u[1] * tau[1][j] + u[2] * tau[2][j];
  }
}

}  // namespace sgs
}  // namespace hb
