// newtonian_qf.cuh -- point-wise Newtonian ideal-gas physics for the fused sm_100a kernels.
//
// Device restatement of the reference QFunctions for the three state variables (conservative, primitive, entropy; a
// template parameter, so each kernel is compiled for the one it runs):
//   IFunction_Newtonian / IFunction_Newtonian_Integrand   qfunctions/newtonian.h:205-257, newtonian_integrands.h:87-115
//   IJacobian_Newtonian / IJacobian_Newtonian_Integrand   qfunctions/newtonian.h:272-311, newtonian_integrands.h:134-166
//   Tau_diagPrim, Stabilization, StabilizationMatrix      qfunctions/stabilization.h:25-100
//   state algebra and fluxes                              qfunctions/newtonian_state.h:64-423, 425-574
// The arithmetic is reorganised for the GPU: reciprocals of density/cv are formed once and multiplied, only the rows of
// the linearised flux that are used are formed, and terms known to be zero (time derivative of Y, divergence of the
// diffusive flux when its projection is off) are dropped.  The result equals the reference to rounding (a few ulp per
// quantity); parity tests bound the operator-level difference.  Templated on the arithmetic type so the same source
// gives the FP64 residual/Jacobian and the FP32 Jacobian of the mixed-precision solver.
#pragma once

#include <cuda_runtime.h>

#include "honee_b200_types.h"

namespace hb {

// Per-launch physical constants derived once on the host from the 184-byte context.
template <typename T>
struct PhysConst {
  T mu, lambda, k, cv, inv_cv, gm1;  // gm1 = cp/cv - 1
  T Rgas;                            // cp - cv
  T g[3];
  T shift;                           // ijacobian time shift
  T Ctau_C, Ctau_M, Ctau_E, Ctau_v;
  T dts;                             // Ctau_t / dt
  int stab;                          // HbStabilizationType
  int idl_enable;
  T idl_amplitude, idl_start, idl_length, idl_pressure;
};

template <typename T>
struct St {  // state: conservative U and primitive Y
  T rho, m[3], E;
  T P, u[3], T_;
};

template <typename T>
__device__ __forceinline__ T rcp(T x) { return T(1) / x; }

// StateFromU (newtonian_state.h:64-73, 379-388); also returns 1/rho and the specific energies used by the tangents.
template <typename T>
__device__ __forceinline__ void state_from_u(const PhysConst<T> &c, const T q[5], St<T> &s, T &inv_rho, T &etot, T &eint) {
  s.rho = q[0];
  s.m[0] = q[1];
  s.m[1] = q[2];
  s.m[2] = q[3];
  s.E = q[4];
  inv_rho = rcp(s.rho);
  for (int i = 0; i < 3; i++) s.u[i] = s.m[i] * inv_rho;
  const T ke = T(.5) * (s.u[0] * s.u[0] + s.u[1] * s.u[1] + s.u[2] * s.u[2]);
  etot = s.E * inv_rho;
  eint = etot - ke;
  s.T_ = eint * c.inv_cv;
  s.P = c.gm1 * s.rho * eint;
}

// StateFromU_fwd (newtonian_state.h:75-89, 390-400): tangent of Y for a conservative tangent dU.
template <typename T>
__device__ __forceinline__ void state_from_u_fwd(const PhysConst<T> &c, const St<T> &s, T inv_rho, T etot, T eint, const T dU[5], St<T> &ds) {
  ds.rho = dU[0];
  ds.m[0] = dU[1];
  ds.m[1] = dU[2];
  ds.m[2] = dU[3];
  ds.E = dU[4];
  for (int i = 0; i < 3; i++) ds.u[i] = (ds.m[i] - s.u[i] * ds.rho) * inv_rho;
  const T dke = ds.u[0] * s.u[0] + ds.u[1] * s.u[1] + ds.u[2] * s.u[2];
  const T detot = (ds.E - etot * ds.rho) * inv_rho;
  const T deint = detot - dke;
  ds.T_ = deint * c.inv_cv;
  ds.P = c.gm1 * (ds.rho * eint + s.rho * deint);
}

// StateFromY_fwd (newtonian_state.h:170-184, 358-369): conservative tangent of a primitive tangent dY.
template <typename T>
__device__ __forceinline__ void state_from_y_fwd(const PhysConst<T> &c, const St<T> &s, T eint, const T dY[5], St<T> &ds) {
  ds.P = dY[0];
  ds.u[0] = dY[1];
  ds.u[1] = dY[2];
  ds.u[2] = dY[3];
  ds.T_ = dY[4];
  const T Tt = s.T_;
  ds.rho = (dY[0] * Tt - s.P * dY[4]) / (c.Rgas * Tt * Tt);
  for (int i = 0; i < 3; i++) ds.m[i] = ds.rho * s.u[i] + s.rho * ds.u[i];
  const T ke = T(.5) * (s.u[0] * s.u[0] + s.u[1] * s.u[1] + s.u[2] * s.u[2]);
  const T dke = ds.u[0] * s.u[0] + ds.u[1] * s.u[1] + ds.u[2] * s.u[2];
  const T e_int = c.cv * Tt;
  const T de_int = c.cv * dY[4];
  ds.E = ds.rho * (e_int + ke) + s.rho * (de_int + dke);
  (void)eint;
}

// Per-point values the tangents of each state variable reuse (1/rho and the specific energies; the entropy variables).
template <typename T>
struct SAux {
  T inv_rho, etot, eint;
  T V[5];
};

// StateFromQ (newtonian_state.h:393-407) for the state variable SV: conservative U (StateFromU), primitive Y = (P, u, T)
// (StateFromY: StateConservativeFromPrimitive, :159-168) or entropy V (StateFromV: StatePrimitiveFromEntropy and
// StateConservativeFromEntropy, :122-132, :222-238; log and exp as the reference evaluates them).
template <int SV, typename T>
__device__ __forceinline__ void state_from_q(const PhysConst<T> &c, const T q[5], St<T> &s, SAux<T> &a) {
  if constexpr (SV == HB_STATEVAR_CONSERVATIVE) {
    state_from_u(c, q, s, a.inv_rho, a.etot, a.eint);
  } else if constexpr (SV == HB_STATEVAR_PRIMITIVE) {
    s.P = q[0];
    s.u[0] = q[1];
    s.u[1] = q[2];
    s.u[2] = q[3];
    s.T_ = q[4];
    s.rho = s.P / (c.Rgas * s.T_);
    for (int i = 0; i < 3; i++) s.m[i] = s.rho * s.u[i];
    const T ke = T(.5) * (s.u[0] * s.u[0] + s.u[1] * s.u[1] + s.u[2] * s.u[2]);
    a.eint = c.cv * s.T_;
    a.etot = a.eint + ke;
    s.E = s.rho * (a.eint + ke);
    a.inv_rho = rcp(s.rho);
  } else {
    for (int i = 0; i < 5; i++) a.V[i] = q[i];
    const T inv_v4 = rcp(q[4]);
    for (int i = 0; i < 3; i++) s.u[i] = -q[1 + i] * inv_v4;
    s.T_ = T(-1) / (c.Rgas * q[4]);
    const T g = c.gm1 + T(1);
    const T ke = T(.5) * (s.u[0] * s.u[0] + s.u[1] * s.u[1] + s.u[2] * s.u[2]);
    const T ent = g - c.gm1 * (q[0] - ke * q[4]);
    const T l4 = log(-q[4]);
    s.P = exp(-(ent + g * l4) / c.gm1);
    s.rho = exp(-(ent + l4) / c.gm1);
    for (int i = 0; i < 3; i++) s.m[i] = s.rho * s.u[i];
    a.eint = -c.cv / (c.Rgas * q[4]);
    a.etot = a.eint + ke;
    s.E = s.rho * (a.eint + ke);
    a.inv_rho = rcp(s.rho);
  }
}

// StateFromQ_fwd (newtonian_state.h:409-423): the full tangent state of a tangent dq in the state variable SV
// (StateFromU_fwd; StateFromY_fwd; StateFromV_fwd = StatePrimitiveFromEntropy_fwd and StateConservativeFromEntropy_fwd,
// :134-146, :240-262).
template <int SV, typename T>
__device__ __forceinline__ void state_from_q_fwd(const PhysConst<T> &c, const St<T> &s, const SAux<T> &a, const T dq[5], St<T> &ds) {
  if constexpr (SV == HB_STATEVAR_CONSERVATIVE) {
    state_from_u_fwd(c, s, a.inv_rho, a.etot, a.eint, dq, ds);
  } else if constexpr (SV == HB_STATEVAR_PRIMITIVE) {
    state_from_y_fwd(c, s, a.eint, dq, ds);
  } else {
    const T *V = a.V;
    const T inv_v4 = rcp(V[4]);
    for (int i = 0; i < 3; i++) ds.u[i] = (-dq[1 + i] - s.u[i] * dq[4]) * inv_v4;
    const T ke = T(.5) * (s.u[0] * s.u[0] + s.u[1] * s.u[1] + s.u[2] * s.u[2]);
    const T dke = ds.u[0] * s.u[0] + ds.u[1] * s.u[1] + ds.u[2] * s.u[2];
    const T dent = -c.gm1 * (dq[0] - (dke * V[4] + ke * dq[4]));
    const T g = c.gm1 + T(1);
    ds.rho = -s.rho / c.gm1 * (dent + dq[4] * inv_v4);
    for (int i = 0; i < 3; i++) ds.m[i] = ds.rho * s.u[i] + s.rho * ds.u[i];
    const T deint = c.cv * dq[4] / (c.Rgas * V[4] * V[4]);
    ds.E = ds.rho * (a.eint + ke) + s.rho * (deint + dke);
    ds.T_ = dq[4] / (c.Rgas * V[4] * V[4]);
    ds.P = s.P * (-dent - g * dq[4] * inv_v4) / c.gm1;
  }
}

// The same with the state variable chosen at run time, for kernels off the hot path (faces, monitors, filter).
template <typename T>
__device__ __forceinline__ void state_from_q_rt(int sv, const PhysConst<T> &c, const T q[5], St<T> &s, SAux<T> &a) {
  if (sv == HB_STATEVAR_PRIMITIVE) state_from_q<HB_STATEVAR_PRIMITIVE>(c, q, s, a);
  else if (sv == HB_STATEVAR_ENTROPY) state_from_q<HB_STATEVAR_ENTROPY>(c, q, s, a);
  else state_from_q<HB_STATEVAR_CONSERVATIVE>(c, q, s, a);
}
template <typename T>
__device__ __forceinline__ void state_from_q_fwd_rt(int sv, const PhysConst<T> &c, const St<T> &s, const SAux<T> &a, const T dq[5], St<T> &ds) {
  if (sv == HB_STATEVAR_PRIMITIVE) state_from_q_fwd<HB_STATEVAR_PRIMITIVE>(c, s, a, dq, ds);
  else if (sv == HB_STATEVAR_ENTROPY) state_from_q_fwd<HB_STATEVAR_ENTROPY>(c, s, a, dq, ds);
  else state_from_q_fwd<HB_STATEVAR_CONSERVATIVE>(c, s, a, dq, ds);
}

// Row i of the linearised inviscid flux (newtonian_state.h:433-442): dF_i for components 0..4.
template <typename T>
__device__ __forceinline__ void dflux_row(const St<T> &s, const St<T> &ds, int i, T r[5]) {
  r[0] = ds.m[i];
  for (int j = 0; j < 3; j++) r[1 + j] = ds.m[i] * s.u[j] + s.m[i] * ds.u[j] + (i == j ? ds.P : T(0));
  r[4] = (ds.E + ds.P) * s.u[i] + (s.E + s.P) * ds.u[i];
}

// Diagonal tau (stabilization.h:67-100).
template <typename T>
__device__ __forceinline__ void tau_diag(const PhysConst<T> &c, const St<T> &s, const T X[3][3], T tau[3]) {
  T g[3][3];
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) g[i][j] = X[0][i] * X[0][j] + X[1][i] * X[1][j] + X[2][i] * X[2][j];
  T ugu = 0, g2 = 0;
#pragma unroll
  for (int i = 0; i < 3; i++) {
    ugu += s.u[i] * (g[i][0] * s.u[0] + g[i][1] * s.u[1] + g[i][2] * s.u[2]);
#pragma unroll
    for (int j = 0; j < 3; j++) g2 += g[i][j] * g[i][j];
  }
  const T tsum = s.rho * s.rho * (T(4) * c.dts * c.dts + ugu) + c.Ctau_v * c.mu * c.mu * g2;
  const T f = sqrt(tsum);
  // one reciprocal for both divisions: 1/f = rt / (f rt) and f / rt = f^2 / (f rt)
  const T rt = s.rho * (g[0][0] + g[1][1] + g[2][2]);
  const T r = rcp(f * rt);
  const T inv_f = rt * r;
  tau[0] = c.Ctau_C * (f * f * r) * T(0.125);
  tau[1] = c.Ctau_M * inv_f;
  tau[2] = c.Ctau_E * inv_f * c.inv_cv;
}

// SU/SUPG term stab[comp][dir] = dF_dir(StateFromY_fwd(tau . r)) with r the strong residual (stabilization.h:25-58).
template <typename T>
__device__ __forceinline__ void stabilization(const PhysConst<T> &c, const St<T> &s, T eint, const T tau[3], const St<T> gs[3],
                                              const T Udot[5], const T body[5], T stab[5][3]) {
  if (c.stab == HB_STAB_NONE) {
#pragma unroll
    for (int i = 0; i < 5; i++) stab[i][0] = stab[i][1] = stab[i][2] = 0;
    return;
  }
  T r[5] = {0, 0, 0, 0, 0};
#pragma unroll
  for (int i = 0; i < 3; i++) {
    T row[5];
    dflux_row(s, gs[i], i, row);
#pragma unroll
    for (int j = 0; j < 5; j++) r[j] += row[j];
  }
  if (c.stab == HB_STAB_SUPG) {
#pragma unroll
    for (int j = 0; j < 5; j++) r[j] += Udot[j] - body[j];
  }
  const T dY[5] = {tau[0] * r[0], tau[1] * r[1], tau[1] * r[2], tau[1] * r[3], tau[2] * r[4]};
  St<T> d;
  state_from_y_fwd(c, s, eint, dY, d);
#pragma unroll
  for (int i = 0; i < 3; i++) {
    T row[5];
    dflux_row(s, d, i, row);
#pragma unroll
    for (int j = 0; j < 5; j++) stab[j][i] = row[j];
  }
}

// KM strain rate from velocity gradients gs[j].u[i] = du_i/dx_j (newtonian_state.h:509-537).
template <typename T>
__device__ __forceinline__ void km_strain(const St<T> gs[3], T e[6]) {
  const T w = T(1.0 / 1.4142135623730951);  // 1/sqrt(2.) in the working precision (utils.h:240)
  e[0] = gs[0].u[0];
  e[1] = gs[1].u[1];
  e[2] = gs[2].u[2];
  e[3] = w * (gs[2].u[1] + gs[1].u[2]);
  e[4] = w * (gs[2].u[0] + gs[0].u[2]);
  e[5] = w * (gs[1].u[0] + gs[0].u[1]);
}

// Full stress tensor from a KM strain rate (NewtonianStress + KMUnpack, newtonian_state.h:553-558, utils.h:239-247).
template <typename T>
__device__ __forceinline__ void stress_full(const PhysConst<T> &c, const T e[6], T sig[3][3]) {
  const T w = T(1.0 / 1.4142135623730951);
  const T div = e[0] + e[1] + e[2];
  const T ld = c.lambda * div;
  sig[0][0] = c.mu * (T(2) * e[0] + ld);
  sig[1][1] = c.mu * (T(2) * e[1] + ld);
  sig[2][2] = c.mu * (T(2) * e[2] + ld);
  sig[1][2] = sig[2][1] = w * (c.mu * (T(2) * e[3]));
  sig[0][2] = sig[2][0] = w * (c.mu * (T(2) * e[4]));
  sig[0][1] = sig[1][0] = w * (c.mu * (T(2) * e[5]));
}

// Physical gradient of the state (StatePhysicalGradientFromReference, newtonian_state.h:581-593):
// gref[d][c] reference derivatives, X = dXdx; dq[c][j] = sum_k gref[k][c] X[k][j].
template <typename T>
__device__ __forceinline__ void physical_gradient(const PhysConst<T> &c, const St<T> &s, T inv_rho, T etot, T eint, const T gref[3][5],
                                                  const T X[3][3], St<T> gs[3]) {
#pragma unroll
  for (int j = 0; j < 3; j++) {
    T dq[5];
#pragma unroll
    for (int cc = 0; cc < 5; cc++) dq[cc] = gref[0][cc] * X[0][j] + gref[1][cc] * X[1][j] + gref[2][cc] * X[2][j];
    state_from_u_fwd(c, s, inv_rho, etot, eint, dq, gs[j]);
  }
}

// IDL ramp (utils.h:287-295)
template <typename T>
__device__ __forceinline__ T linear_ramp(T amplitude, T length, T start, T x) {
  if (x < start) return amplitude;
  if (x < start + length) return amplitude * ((x - start) * (T(-1) / length) + T(1));
  return T(0);
}

// IFunction at one quadrature point. Inputs: q[5], reference gradient gref[3][5], q_dot[5], qdata (wdetJ, X).
// Outputs: v[5], grad_v[3][5] in reference directions (already multiplied by wdetJ X), and the 14 stored values.
template <typename T>
__device__ __forceinline__ void ifunction_point(const PhysConst<T> &c, const T q[5], const T gref[3][5], const T qdot[5], T wdetJ, const T X[3][3],
                                                T x0, T v[5], T gv[3][5], T jd[15]) {
  St<T> s;
  T inv_rho, etot, eint;
  state_from_u(c, q, s, inv_rho, etot, eint);
  St<T> gs[3];
  physical_gradient(c, s, inv_rho, etot, eint, gref, X, gs);

  T e[6], sig[3][3];
  km_strain(gs, e);
  stress_full(c, e, sig);

  // -F_total + stab, F_total[comp][dir] (newtonian_state.h:477-484), viscous energy flux (:560-565)
  T gvi[5][3];
#pragma unroll
  for (int j = 0; j < 3; j++) {
    const T Fe = -s.u[0] * sig[0][j] - s.u[1] * sig[1][j] - s.u[2] * sig[2][j] - c.k * gs[j].T_;
    gvi[0][j] = -s.m[j];
#pragma unroll
    for (int kk = 0; kk < 3; kk++) gvi[1 + kk][j] = -(s.m[j] * s.u[kk] + (j == kk ? s.P : T(0)) - sig[kk][j]);
    gvi[4][j] = -((s.E + s.P) * s.u[j] + Fe);
  }
  const T body[5] = {T(0), s.rho * c.g[0], s.rho * c.g[1], s.rho * c.g[2], s.m[0] * c.g[0] + s.m[1] * c.g[1] + s.m[2] * c.g[2]};
  T vi[5];
#pragma unroll
  for (int j = 0; j < 5; j++) vi[j] = qdot[j] - body[j];

  T tau[3], stab[5][3];
  tau_diag(c, s, X, tau);
  stabilization(c, s, eint, tau, gs, qdot, body, stab);
#pragma unroll
  for (int j = 0; j < 5; j++)
#pragma unroll
    for (int d = 0; d < 3; d++) gvi[j][d] += stab[j][d];

  T sigma = 0;
  if (c.idl_enable) {  // newtonian_integrands.h:38-45
    sigma = linear_ramp(c.idl_amplitude, c.idl_length, c.idl_start, x0);
    const T dY[5] = {(s.P - c.idl_pressure) * sigma, T(0), T(0), T(0), T(0)};
    St<T> d;
    state_from_y_fwd(c, s, eint, dY, d);
    vi[0] += d.rho;
    vi[1] += d.m[0];
    vi[2] += d.m[1];
    vi[3] += d.m[2];
    vi[4] += d.E;
  }
#pragma unroll
  for (int j = 0; j < 5; j++) v[j] = wdetJ * vi[j];
#pragma unroll
  for (int kk = 0; kk < 3; kk++)
#pragma unroll
    for (int j = 0; j < 5; j++) gv[kk][j] = wdetJ * (gvi[j][0] * X[kk][0] + gvi[j][1] * X[kk][1] + gvi[j][2] * X[kk][2]);
#pragma unroll
  for (int j = 0; j < 5; j++) jd[j] = q[j];
#pragma unroll
  for (int j = 0; j < 6; j++) jd[5 + j] = e[j];
#pragma unroll
  for (int j = 0; j < 3; j++) jd[11 + j] = tau[j];
  jd[14] = sigma;
}

// IJacobian action at one quadrature point (jd = stored q, KM strain rate, tau [, sigma]).
template <typename T>
__device__ __forceinline__ void ijacobian_point(const PhysConst<T> &c, const T jd[15], const T dq[5], const T gref[3][5], T wdetJ, const T X[3][3],
                                                T v[5], T gv[3][5]) {
  St<T> s;
  T inv_rho, etot, eint;
  const T q[5] = {jd[0], jd[1], jd[2], jd[3], jd[4]};
  state_from_u(c, q, s, inv_rho, etot, eint);
  St<T> ds;
  state_from_u_fwd(c, s, inv_rho, etot, eint, dq, ds);
  St<T> gs[3];
  physical_gradient(c, s, inv_rho, etot, eint, gref, X, gs);

  T de[6], dsig[3][3], sig[3][3];
  km_strain(gs, de);
  stress_full(c, de, dsig);
  const T e[6] = {jd[5], jd[6], jd[7], jd[8], jd[9], jd[10]};
  stress_full(c, e, sig);

  T gvi[5][3];
#pragma unroll
  for (int j = 0; j < 3; j++) {
    T row[5];
    dflux_row(s, ds, j, row);
    const T dFe = -s.u[0] * dsig[0][j] - ds.u[0] * sig[0][j] - s.u[1] * dsig[1][j] - ds.u[1] * sig[1][j] - s.u[2] * dsig[2][j] -
                  ds.u[2] * sig[2][j] - c.k * gs[j].T_;
    gvi[0][j] = -row[0];
#pragma unroll
    for (int kk = 0; kk < 3; kk++) gvi[1 + kk][j] = -(row[1 + kk] - dsig[kk][j]);
    gvi[4][j] = -(row[4] + dFe);
  }
  const T dbody[5] = {T(0), ds.rho * c.g[0], ds.rho * c.g[1], ds.rho * c.g[2], ds.m[0] * c.g[0] + ds.m[1] * c.g[1] + ds.m[2] * c.g[2]};
  T dUdot[5], vi[5];
  const T dU[5] = {ds.rho, ds.m[0], ds.m[1], ds.m[2], ds.E};
#pragma unroll
  for (int j = 0; j < 5; j++) {
    dUdot[j] = c.shift * dU[j];
    vi[j] = dUdot[j] - dbody[j];
  }
  const T tau[3] = {jd[11], jd[12], jd[13]};
  T dstab[5][3];
  stabilization(c, s, eint, tau, gs, dUdot, dbody, dstab);
#pragma unroll
  for (int j = 0; j < 5; j++)
#pragma unroll
    for (int d = 0; d < 3; d++) gvi[j][d] += dstab[j][d];
  if (c.idl_enable) {  // newtonian_integrands.h:58-64
    const T sigma = jd[14];
    const T dY[5] = {ds.P * sigma, T(0), T(0), T(0), T(0)};
    St<T> d;
    state_from_y_fwd(c, s, eint, dY, d);
    vi[0] += d.rho;
    vi[1] += d.m[0];
    vi[2] += d.m[1];
    vi[3] += d.m[2];
    vi[4] += d.E;
  }
#pragma unroll
  for (int j = 0; j < 5; j++) v[j] = wdetJ * vi[j];
#pragma unroll
  for (int kk = 0; kk < 3; kk++)
#pragma unroll
    for (int j = 0; j < 5; j++) gv[kk][j] = wdetJ * (gvi[j][0] * X[kk][0] + gvi[j][1] * X[kk][1] + gvi[j][2] * X[kk][2]);
}

}  // namespace hb

namespace hb {

// ---------------------------------------------------------------------------------------------------------------------
// Streaming forms of the point-wise IFunction / IJacobian used by the fused kernels.  Same arithmetic as
// ifunction_point / ijacobian_point, reordered so few values are live at once: each physical-gradient direction j is
// folded into the strong residual, the velocity-gradient column and the temperature gradient as soon as it is formed,
// the fluxes are projected onto the reference directions one physical direction at a time, and stored Jacobian values
// are handed to `emit` (index, value) as soon as they are known.

// gradient direction j of the state: dq_j = sum_k gref[k][.] X[k][j] -> tangent state
template <int SV, typename T>
__device__ __forceinline__ void gradient_dir(const PhysConst<T> &c, const St<T> &s, const SAux<T> &a, const T gref[3][5], const T X[3][3], int j,
                                             St<T> &g) {
  T dq[5];
#pragma unroll
  for (int cc = 0; cc < 5; cc++) dq[cc] = gref[0][cc] * X[0][j] + gref[1][cc] * X[1][j] + gref[2][cc] * X[2][j];
  state_from_q_fwd<SV>(c, s, a, dq, g);
}

// SV: the state variable of q, q_dot and the stored q (HbStateVariable); the residual is always the conservation law in
// conservative form, with the rate dU/dt = (dU/dq) q_dot (newtonian.h:226-230).
template <typename T, int SV = HB_STATEVAR_CONSERVATIVE, typename Emit>
__device__ __forceinline__ void ifunction_point_stream(const PhysConst<T> &c, const T q[5], const T gref[3][5], const T qdot_in[5], T wdetJ,
                                                       const T X[3][3], T x0, T v[5], T gv[3][5], Emit emit) {
  St<T> s;
  SAux<T> aux;
  state_from_q<SV>(c, q, s, aux);
  const T eint = aux.eint;
  T qdot[5];
  if constexpr (SV == HB_STATEVAR_CONSERVATIVE) {
#pragma unroll
    for (int k = 0; k < 5; k++) qdot[k] = qdot_in[k];
  } else {
    St<T> sd;
    state_from_q_fwd<SV>(c, s, aux, qdot_in, sd);
    qdot[0] = sd.rho;
    qdot[1] = sd.m[0];
    qdot[2] = sd.m[1];
    qdot[3] = sd.m[2];
    qdot[4] = sd.E;
  }
  // strong convective residual, velocity gradient G[i][j] = du_i/dx_j, temperature gradient
  T r[5] = {0, 0, 0, 0, 0}, G[3][3], gT[3];
#pragma unroll
  for (int j = 0; j < 3; j++) {
    St<T> g;
    gradient_dir<SV>(c, s, aux, gref, X, j, g);
    if (c.stab != HB_STAB_NONE) {
      T row[5];
      dflux_row(s, g, j, row);
#pragma unroll
      for (int k = 0; k < 5; k++) r[k] += row[k];
    }
#pragma unroll
    for (int i = 0; i < 3; i++) G[i][j] = g.u[i];
    gT[j] = g.T_;
  }
  // KM strain rate (newtonian_state.h:523-532) and stress
  const T w = T(1.0 / 1.4142135623730951);
  T e[6];
  e[0] = G[0][0];
  e[1] = G[1][1];
  e[2] = G[2][2];
  e[3] = w * (G[1][2] + G[2][1]);
  e[4] = w * (G[0][2] + G[2][0]);
  e[5] = w * (G[0][1] + G[1][0]);
#pragma unroll
  for (int k = 0; k < 5; k++) emit(k, q[k]);
#pragma unroll
  for (int k = 0; k < 6; k++) emit(5 + k, e[k]);
  T sig[3][3];
  stress_full(c, e, sig);
  // tau and the stabilisation state perturbation
  T tau[3];
  tau_diag(c, s, X, tau);
#pragma unroll
  for (int k = 0; k < 3; k++) emit(11 + k, tau[k]);
  const T body[5] = {T(0), s.rho * c.g[0], s.rho * c.g[1], s.rho * c.g[2], s.m[0] * c.g[0] + s.m[1] * c.g[1] + s.m[2] * c.g[2]};
  St<T> d;
  const bool stab = c.stab != HB_STAB_NONE;
  if (stab) {
    if (c.stab == HB_STAB_SUPG) {
#pragma unroll
      for (int k = 0; k < 5; k++) r[k] += qdot[k] - body[k];
    }
    const T dY[5] = {tau[0] * r[0], tau[1] * r[1], tau[1] * r[2], tau[1] * r[3], tau[2] * r[4]};
    state_from_y_fwd(c, s, eint, dY, d);
  }
  T vi[5];
#pragma unroll
  for (int k = 0; k < 5; k++) vi[k] = qdot[k] - body[k];
  T sigma = 0;
  if (c.idl_enable) {
    sigma = linear_ramp(c.idl_amplitude, c.idl_length, c.idl_start, x0);
    const T dY[5] = {(s.P - c.idl_pressure) * sigma, T(0), T(0), T(0), T(0)};
    St<T> di;
    state_from_y_fwd(c, s, eint, dY, di);
    vi[0] += di.rho;
    vi[1] += di.m[0];
    vi[2] += di.m[1];
    vi[3] += di.m[2];
    vi[4] += di.E;
  }
  emit(14, sigma);
#pragma unroll
  for (int k = 0; k < 5; k++) v[k] = wdetJ * vi[k];
  // per physical direction j: gvi[.][j] = -F_total[.][j] + stab[.][j]; project onto reference directions
#pragma unroll
  for (int kk = 0; kk < 3; kk++)
#pragma unroll
    for (int k = 0; k < 5; k++) gv[kk][k] = 0;
#pragma unroll
  for (int j = 0; j < 3; j++) {
    const T Fe = -s.u[0] * sig[0][j] - s.u[1] * sig[1][j] - s.u[2] * sig[2][j] - c.k * gT[j];
    T col[5];
    col[0] = -s.m[j];
#pragma unroll
    for (int kk = 0; kk < 3; kk++) col[1 + kk] = -(s.m[j] * s.u[kk] + (j == kk ? s.P : T(0)) - sig[kk][j]);
    col[4] = -((s.E + s.P) * s.u[j] + Fe);
    if (stab) {
      T row[5];
      dflux_row(s, d, j, row);
#pragma unroll
      for (int k = 0; k < 5; k++) col[k] += row[k];
    }
#pragma unroll
    for (int kk = 0; kk < 3; kk++) {
      const T xw = wdetJ * X[kk][j];
#pragma unroll
      for (int k = 0; k < 5; k++) gv[kk][k] += col[k] * xw;
    }
  }
}

template <typename T, int SV = HB_STATEVAR_CONSERVATIVE>
__device__ __forceinline__ void ijacobian_point_stream(const PhysConst<T> &c, const T jd[15], const T dq[5], const T gref[3][5], T wdetJ,
                                                       const T X[3][3], T v[5], T gv[3][5]) {
  St<T> s;
  SAux<T> aux;
  const T q[5] = {jd[0], jd[1], jd[2], jd[3], jd[4]};
  state_from_q<SV>(c, q, s, aux);
  const T eint = aux.eint;
  St<T> ds;
  state_from_q_fwd<SV>(c, s, aux, dq, ds);
  T r[5] = {0, 0, 0, 0, 0}, G[3][3], gT[3];
#pragma unroll
  for (int j = 0; j < 3; j++) {
    St<T> g;
    gradient_dir<SV>(c, s, aux, gref, X, j, g);
    if (c.stab != HB_STAB_NONE) {
      T row[5];
      dflux_row(s, g, j, row);
#pragma unroll
      for (int k = 0; k < 5; k++) r[k] += row[k];
    }
#pragma unroll
    for (int i = 0; i < 3; i++) G[i][j] = g.u[i];
    gT[j] = g.T_;
  }
  const T w = T(1.0 / 1.4142135623730951);
  T de[6];
  de[0] = G[0][0];
  de[1] = G[1][1];
  de[2] = G[2][2];
  de[3] = w * (G[1][2] + G[2][1]);
  de[4] = w * (G[0][2] + G[2][0]);
  de[5] = w * (G[0][1] + G[1][0]);
  T dsig[3][3], sig[3][3];
  stress_full(c, de, dsig);
  const T e[6] = {jd[5], jd[6], jd[7], jd[8], jd[9], jd[10]};
  stress_full(c, e, sig);
  const T dbody[5] = {T(0), ds.rho * c.g[0], ds.rho * c.g[1], ds.rho * c.g[2], ds.m[0] * c.g[0] + ds.m[1] * c.g[1] + ds.m[2] * c.g[2]};
  T vi[5];
  const T dU[5] = {ds.rho, ds.m[0], ds.m[1], ds.m[2], ds.E};
  St<T> d;
  const bool stab = c.stab != HB_STAB_NONE;
  if (stab) {
    if (c.stab == HB_STAB_SUPG) {
#pragma unroll
      for (int k = 0; k < 5; k++) r[k] += c.shift * dU[k] - dbody[k];
    }
    const T dY[5] = {jd[11] * r[0], jd[12] * r[1], jd[12] * r[2], jd[12] * r[3], jd[13] * r[4]};
    state_from_y_fwd(c, s, eint, dY, d);
  }
#pragma unroll
  for (int k = 0; k < 5; k++) vi[k] = c.shift * dU[k] - dbody[k];
  if (c.idl_enable) {
    const T dY[5] = {ds.P * jd[14], T(0), T(0), T(0), T(0)};
    St<T> di;
    state_from_y_fwd(c, s, eint, dY, di);
    vi[0] += di.rho;
    vi[1] += di.m[0];
    vi[2] += di.m[1];
    vi[3] += di.m[2];
    vi[4] += di.E;
  }
#pragma unroll
  for (int k = 0; k < 5; k++) v[k] = wdetJ * vi[k];
#pragma unroll
  for (int kk = 0; kk < 3; kk++)
#pragma unroll
    for (int k = 0; k < 5; k++) gv[kk][k] = 0;
#pragma unroll
  for (int j = 0; j < 3; j++) {
    T row[5];
    dflux_row(s, ds, j, row);
    const T dFe = -s.u[0] * dsig[0][j] - ds.u[0] * sig[0][j] - s.u[1] * dsig[1][j] - ds.u[1] * sig[1][j] - s.u[2] * dsig[2][j] -
                  ds.u[2] * sig[2][j] - c.k * gT[j];
    T col[5];
    col[0] = -row[0];
#pragma unroll
    for (int kk = 0; kk < 3; kk++) col[1 + kk] = -(row[1 + kk] - dsig[kk][j]);
    col[4] = -(row[4] + dFe);
    if (stab) {
      T srow[5];
      dflux_row(s, d, j, srow);
#pragma unroll
      for (int k = 0; k < 5; k++) col[k] += srow[k];
    }
#pragma unroll
    for (int kk = 0; kk < 3; kk++) {
      const T xw = wdetJ * X[kk][j];
#pragma unroll
      for (int k = 0; k < 5; k++) gv[kk][k] += col[k] * xw;
    }
  }
}

}  // namespace hb

namespace hb {

// ---------------------------------------------------------------------------------------------------------------------
// Component-diagonal blocks of the linearised IJacobian point function, the point-wise input of the Jacobi diagonal
// (CeedOperatorLinearAssembleDiagonal on the IJacobian operator).  For component C the 4 x 4 block
// A[m][n] = d out(m, C) / d in(n, C), m, n in {value, reference gradient 0..2}, of ijacobian_point_stream decomposes by
// linearity:
//   A[0][0]     = v_C of the value tangent dq = e_C;   A[0][1 + d] = 0 (the value output does not see gradients)
//   A[1+k][0]   = wdetJ sum_j X[k][j] V_j              V_j    flux column j, component C, of the value tangent
//   A[1+k][1+d] = wdetJ sum_j sum_i X[k][j] R[j][i] X[d][i]
//                                                      R[j][i] flux column j, component C, of a unit physical gradient
//                                                              e_C in direction i (a reference gradient e_C in direction d
//                                                              is the physical gradient X[d][i] e_C in direction i)
// so each component costs one value tangent and three physical-gradient tangents, each folded for its unit input, instead
// of four reference-gradient evaluations of the full point function.  The set-up (state, stress, 1 / (R T^2)) is formed
// once per point.  `out(m, value)` receives the ten symmetric combinations in the order II, IGx, IGy, IGz, GxGx, GyGy,
// GzGz, GxGy, GxGz, GyGz (A[m][n] + A[n][m], one term on the diagonal).
template <int C, int SV, typename T, typename Out>
__device__ __forceinline__ void diag_point_component(const PhysConst<T> &c, const St<T> &s, const SAux<T> &aux, T inv_RT2, const T sig[3][3],
                                                     const T jd[15], T wdetJ, const T X[3][3], Out out) {
  const bool stab = c.stab != HB_STAB_NONE;
  const T tau[3] = {jd[11], jd[12], jd[13]};
  const T ke = T(.5) * (s.u[0] * s.u[0] + s.u[1] * s.u[1] + s.u[2] * s.u[2]);
  // state_from_y_fwd with the reciprocal 1 / (R T^2) formed once per point
  auto y_fwd = [&](const T dY[5], St<T> &ds) {
    ds.P = dY[0];
    ds.u[0] = dY[1];
    ds.u[1] = dY[2];
    ds.u[2] = dY[3];
    ds.T_ = dY[4];
    ds.rho = (dY[0] * s.T_ - s.P * dY[4]) * inv_RT2;
#pragma unroll
    for (int i = 0; i < 3; i++) ds.m[i] = ds.rho * s.u[i] + s.rho * ds.u[i];
    const T dke = ds.u[0] * s.u[0] + ds.u[1] * s.u[1] + ds.u[2] * s.u[2];
    ds.E = ds.rho * (c.cv * s.T_ + ke) + s.rho * (c.cv * dY[4] + dke);
  };
  // component C of flux row j of a tangent state (dflux_row)
  auto frow = [&](const St<T> &ds, int j) -> T {
    if (C == 0) return ds.m[j];
    if (C == 4) return (ds.E + ds.P) * s.u[j] + (s.E + s.P) * ds.u[j];
    return ds.m[j] * s.u[C - 1] + s.m[j] * ds.u[C - 1] + (j == C - 1 ? ds.P : T(0));
  };
  // the stabilisation state of a strong residual r: d = StateFromY_fwd(tau . r)
  auto stab_state = [&](const T r[5], St<T> &d) {
    const T dY[5] = {tau[0] * r[0], tau[1] * r[1], tau[1] * r[2], tau[1] * r[3], tau[2] * r[4]};
    y_fwd(dY, d);
  };
  St<T> dS;  // unit tangent of component C
  {
    T e[5] = {0, 0, 0, 0, 0};
    e[C] = T(1);
    state_from_q_fwd<SV>(c, s, aux, e, dS);
  }
  // value tangent
  T V[3], A00;
  {
    const T dU[5] = {dS.rho, dS.m[0], dS.m[1], dS.m[2], dS.E};
    const T dbody[5] = {T(0), dS.rho * c.g[0], dS.rho * c.g[1], dS.rho * c.g[2], dS.m[0] * c.g[0] + dS.m[1] * c.g[1] + dS.m[2] * c.g[2]};
    T vi = c.shift * dU[C] - dbody[C];
    if (c.idl_enable) {
      const T dY[5] = {dS.P * jd[14], T(0), T(0), T(0), T(0)};
      St<T> di;
      y_fwd(dY, di);
      const T dUi[5] = {di.rho, di.m[0], di.m[1], di.m[2], di.E};
      vi += dUi[C];
    }
    A00 = wdetJ * vi;
    St<T> d;
    const bool supg = c.stab == HB_STAB_SUPG;
    if (supg) {
      T r[5];
#pragma unroll
      for (int k = 0; k < 5; k++) r[k] = c.shift * dU[k] - dbody[k];
      stab_state(r, d);
    }
#pragma unroll
    for (int j = 0; j < 3; j++) {
      T col = -frow(dS, j);
      if (C == 4) col += dS.u[0] * sig[0][j] + dS.u[1] * sig[1][j] + dS.u[2] * sig[2][j];  // -dFe with dsig = 0, gT = 0
      if (supg) col += frow(d, j);
      V[j] = col;
    }
  }
  // physical-gradient tangents: R[j][i]
  T R[3][3];
  const T w = T(1.0 / 1.4142135623730951);
#pragma unroll
  for (int i = 0; i < 3; i++) {
    St<T> d;
    if (stab) {
      T r[5];
      r[0] = dS.m[i];
#pragma unroll
      for (int k = 0; k < 3; k++) r[1 + k] = dS.m[i] * s.u[k] + s.m[i] * dS.u[k] + (i == k ? dS.P : T(0));
      r[4] = (dS.E + dS.P) * s.u[i] + (s.E + s.P) * dS.u[i];
      stab_state(r, d);
    }
    // strain of a velocity gradient with only column i = dS.u
    T de[6] = {0, 0, 0, 0, 0, 0};
    de[i] = dS.u[i];
    if (i == 0) {
      de[4] = w * dS.u[2];
      de[5] = w * dS.u[1];
    } else if (i == 1) {
      de[3] = w * dS.u[2];
      de[5] = w * dS.u[0];
    } else {
      de[3] = w * dS.u[1];
      de[4] = w * dS.u[0];
    }
    T dsig[3][3];
    stress_full(c, de, dsig);
#pragma unroll
    for (int j = 0; j < 3; j++) {
      T col = 0;
      if (C >= 1 && C <= 3) col = dsig[C - 1][j];
      if (C == 4) col = s.u[0] * dsig[0][j] + s.u[1] * dsig[1][j] + s.u[2] * dsig[2][j] + (j == i ? c.k * dS.T_ : T(0));
      if (stab) col += frow(d, j);
      R[j][i] = col;
    }
  }
  // reference-direction blocks
  T XR[3][3];  // XR[k][i] = sum_j X[k][j] R[j][i]
#pragma unroll
  for (int k = 0; k < 3; k++)
#pragma unroll
    for (int i = 0; i < 3; i++) XR[k][i] = X[k][0] * R[0][i] + X[k][1] * R[1][i] + X[k][2] * R[2][i];
  auto AGG = [&](int k, int d) { return wdetJ * (XR[k][0] * X[d][0] + XR[k][1] * X[d][1] + XR[k][2] * X[d][2]); };
  out(0, A00);
#pragma unroll
  for (int k = 0; k < 3; k++) out(1 + k, wdetJ * (X[k][0] * V[0] + X[k][1] * V[1] + X[k][2] * V[2]));
  out(4, AGG(0, 0));
  out(5, AGG(1, 1));
  out(6, AGG(2, 2));
  out(7, AGG(0, 1) + AGG(1, 0));
  out(8, AGG(0, 2) + AGG(2, 0));
  out(9, AGG(1, 2) + AGG(2, 1));
}

// Shared per-point set-up of diag_point_component and the five components.
template <int SV, typename T, typename Out>
__device__ __forceinline__ void diag_point_blocks(const PhysConst<T> &c, const T jd[15], T wdetJ, const T X[3][3], Out out) {
  St<T> s;
  SAux<T> aux;
  const T q[5] = {jd[0], jd[1], jd[2], jd[3], jd[4]};
  state_from_q<SV>(c, q, s, aux);
  const T e[6] = {jd[5], jd[6], jd[7], jd[8], jd[9], jd[10]};
  T sig[3][3];
  stress_full(c, e, sig);
  const T inv_RT2 = rcp(c.Rgas * s.T_ * s.T_);
  diag_point_component<0, SV>(c, s, aux, inv_RT2, sig, jd, wdetJ, X, [&](int m, T v) { out(0, m, v); });
  diag_point_component<1, SV>(c, s, aux, inv_RT2, sig, jd, wdetJ, X, [&](int m, T v) { out(1, m, v); });
  diag_point_component<2, SV>(c, s, aux, inv_RT2, sig, jd, wdetJ, X, [&](int m, T v) { out(2, m, v); });
  diag_point_component<3, SV>(c, s, aux, inv_RT2, sig, jd, wdetJ, X, [&](int m, T v) { out(3, m, v); });
  diag_point_component<4, SV>(c, s, aux, inv_RT2, sig, jd, wdetJ, X, [&](int m, T v) { out(4, m, v); });
}

}  // namespace hb
