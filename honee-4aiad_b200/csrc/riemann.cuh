// riemann.cuh -- approximate Riemann fluxes of the free-stream boundary condition, and their forward-mode tangents.
//
// Restates qfunctions/riemann_solver.h: HLL and HLLC fluxes (Toro) with wave speeds from Roe averages of the normal
// velocity and the total specific enthalpy (ComputeHLLSpeeds_Roe, :76-133), the HLLC star-state flux (:180-245) and the
// branch selection on s_left <= 0 <= s_star <= s_right (:247-338); the inviscid flux dotted with the normal comes from
// newtonian_state.h:425-464.  The tangent routines differentiate the same expressions in the same order, with the
// exterior state allowed to vary too.  Conservative state variables only (St: rho, m, E, P, u, T).
#pragma once

#include "newtonian_qf.cuh"

namespace hb {
namespace riemann {

template <typename T>
__device__ __forceinline__ void flux_dot_n(const St<T> &s, const T n[3], T F[5]) {
  const T un = s.u[0] * n[0] + s.u[1] * n[1] + s.u[2] * n[2];
  F[0] = s.m[0] * n[0] + s.m[1] * n[1] + s.m[2] * n[2];
#pragma unroll
  for (int j = 0; j < 3; j++) F[1 + j] = (s.m[0] * n[0] + s.m[1] * n[1] + s.m[2] * n[2]) * s.u[j] + s.P * n[j];
  F[4] = (s.E + s.P) * un;
}

template <typename T>
__device__ __forceinline__ void flux_dot_n_fwd(const St<T> &s, const St<T> &ds, const T n[3], T dF[5]) {
  const T mn = s.m[0] * n[0] + s.m[1] * n[1] + s.m[2] * n[2], dmn = ds.m[0] * n[0] + ds.m[1] * n[1] + ds.m[2] * n[2];
  const T un = s.u[0] * n[0] + s.u[1] * n[1] + s.u[2] * n[2], dun = ds.u[0] * n[0] + ds.u[1] * n[1] + ds.u[2] * n[2];
  dF[0] = dmn;
#pragma unroll
  for (int j = 0; j < 3; j++) dF[1 + j] = dmn * s.u[j] + mn * ds.u[j] + ds.P * n[j];
  dF[4] = (ds.E + ds.P) * un + (s.E + s.P) * dun;
}

template <typename T>
__device__ __forceinline__ T enthalpy(T cv, const St<T> &s) {
  return cv * s.T_ + T(0.5) * (s.u[0] * s.u[0] + s.u[1] * s.u[1] + s.u[2] * s.u[2]) + s.P / s.rho;
}
template <typename T>
__device__ __forceinline__ T enthalpy_fwd(T cv, const St<T> &s, const St<T> &ds) {
  return cv * ds.T_ + (ds.u[0] * s.u[0] + ds.u[1] * s.u[1] + ds.u[2] * s.u[2]) + ds.P / s.rho - s.P / (s.rho * s.rho) * ds.rho;
}

// Roe-averaged wave speeds s_l = u_roe - a_roe, s_r = u_roe + a_roe, and their tangents
template <typename T>
__device__ __forceinline__ void roe_speeds(T gamma, T cv, const St<T> &L, T uL, const St<T> &R, T uR, T &sl, T &sr) {
  const T ql = sqrt(L.rho), qr = sqrt(R.rho);
  const T wl = ql / (ql + qr), wr = qr / (ql + qr);
  const T u = wl * uL + wr * uR;
  const T H = wl * enthalpy(cv, L) + wr * enthalpy(cv, R);
  const T a = sqrt((gamma - 1) * (H - T(0.5) * u * u));
  sl = u - a;
  sr = u + a;
}
template <typename T>
__device__ __forceinline__ void roe_speeds_fwd(T gamma, T cv, const St<T> &L, const St<T> &dL, T uL, T duL, const St<T> &R, const St<T> &dR, T uR,
                                               T duR, T &sl, T &dsl, T &sr, T &dsr) {
  const T ql = sqrt(L.rho), qr = sqrt(R.rho);
  const T wl = ql / (ql + qr), wr = qr / (ql + qr);
  const T sq = (ql + qr) * (ql + qr);
  const T dwr = (ql / (2 * qr * sq)) * dR.rho - (qr / (2 * ql * sq)) * dL.rho;
  const T dwl = (qr / (2 * ql * sq)) * dL.rho - (ql / (2 * qr * sq)) * dR.rho;
  const T u = wl * uL + wr * uR;
  const T du = uR * dwr + uL * dwl + wr * duR + wl * duL;
  const T Hl = enthalpy(cv, L), Hr = enthalpy(cv, R);
  const T H = wl * Hl + wr * Hr;
  const T dH = Hr * dwr + Hl * dwl + wr * enthalpy_fwd(cv, R, dR) + wl * enthalpy_fwd(cv, L, dL);
  const T a = sqrt((gamma - 1) * (H - T(0.5) * u * u));
  T da = T(0.5) * sqrt((gamma - 1) / (H - T(0.5) * u * u)) * dH;
  da -= T(0.5) * sqrt(gamma - 1) * u / sqrt(H - T(0.5) * u * u) * du;
  sl = u - a;
  dsl = du - da;
  sr = u + a;
  dsr = du + da;
}

template <typename T>
__device__ __forceinline__ void hll(const St<T> &L, const St<T> &R, const T Fl[5], const T Fr[5], T sl, T sr, T F[5]) {
  const T Ul[5] = {L.rho, L.m[0], L.m[1], L.m[2], L.E}, Ur[5] = {R.rho, R.m[0], R.m[1], R.m[2], R.E};
#pragma unroll
  for (int i = 0; i < 5; i++) F[i] = (sr * Fl[i] - sl * Fr[i] + sl * sr * (Ur[i] - Ul[i])) / (sr - sl);
}

// HLL flux through the face with normal n between the interior state L and the exterior state R
template <typename T>
__device__ __forceinline__ void hll_flux(T gamma, T cv, const St<T> &L, const St<T> &R, const T n[3], T F[5]) {
  T Fl[5], Fr[5], sl, sr;
  flux_dot_n(L, n, Fl);
  flux_dot_n(R, n, Fr);
  const T uL = L.u[0] * n[0] + L.u[1] * n[1] + L.u[2] * n[2], uR = R.u[0] * n[0] + R.u[1] * n[1] + R.u[2] * n[2];
  roe_speeds(gamma, cv, L, uL, R, uR, sl, sr);
  if (T(0) <= sl) {
#pragma unroll
    for (int i = 0; i < 5; i++) F[i] = Fl[i];
  } else if (sr <= T(0)) {
#pragma unroll
    for (int i = 0; i < 5; i++) F[i] = Fr[i];
  } else {
    hll(L, R, Fl, Fr, sl, sr, F);
  }
}

template <typename T>
__device__ __forceinline__ void hll_flux_fwd(T gamma, T cv, const St<T> &L, const St<T> &dL, const St<T> &R, const St<T> &dR, const T n[3], T dF[5]) {
  T Fl[5], Fr[5], dFl[5], dFr[5], sl, dsl, sr, dsr;
  flux_dot_n(L, n, Fl);
  flux_dot_n(R, n, Fr);
  flux_dot_n_fwd(L, dL, n, dFl);
  flux_dot_n_fwd(R, dR, n, dFr);
  const T uL = L.u[0] * n[0] + L.u[1] * n[1] + L.u[2] * n[2], uR = R.u[0] * n[0] + R.u[1] * n[1] + R.u[2] * n[2];
  const T duL = dL.u[0] * n[0] + dL.u[1] * n[1] + dL.u[2] * n[2], duR = dR.u[0] * n[0] + dR.u[1] * n[1] + dR.u[2] * n[2];
  roe_speeds_fwd(gamma, cv, L, dL, uL, duL, R, dR, uR, duR, sl, dsl, sr, dsr);
  if (T(0) <= sl) {
#pragma unroll
    for (int i = 0; i < 5; i++) dF[i] = dFl[i];
  } else if (sr <= T(0)) {
#pragma unroll
    for (int i = 0; i < 5; i++) dF[i] = dFr[i];
  } else {
    const T Ul[5] = {L.rho, L.m[0], L.m[1], L.m[2], L.E}, Ur[5] = {R.rho, R.m[0], R.m[1], R.m[2], R.E};
    const T dUl[5] = {dL.rho, dL.m[0], dL.m[1], dL.m[2], dL.E}, dUr[5] = {dR.rho, dR.m[0], dR.m[1], dR.m[2], dR.E};
    const T d = sr - sl;
#pragma unroll
    for (int i = 0; i < 5; i++) {
      T v = (sl * (-Fl[i] + Fr[i] + sl * Ul[i] - sl * Ur[i]) / (d * d)) * dsr;
      v += (sr * (Fl[i] - Fr[i] - sr * Ul[i] + sr * Ur[i]) / (d * d)) * dsl;
      v += (sr * dFl[i] - sl * dFr[i] + sr * sl * (dUr[i] - dUl[i])) / d;
      dF[i] = v;
    }
  }
}

// HLLC star-region flux of one side: F_side + s_side (fact U* - U_side)
template <typename T>
__device__ __forceinline__ void hllc_star(const St<T> &S, const T Fs[5], const T n[3], T us, T ss, T sst, T F[5]) {
  const T fact = S.rho * (ss - us) / (ss - sst);
  const T denom = S.rho * (ss - us);
  const T star[5] = {T(1), S.u[0] + (sst - us) * n[0], S.u[1] + (sst - us) * n[1], S.u[2] + (sst - us) * n[2],
                     S.E / S.rho + (sst - us) * (sst + S.P / denom)};
  const T U[5] = {S.rho, S.m[0], S.m[1], S.m[2], S.E};
#pragma unroll
  for (int i = 0; i < 5; i++) F[i] = Fs[i] + ss * fact * star[i] - ss * U[i];
}

template <typename T>
__device__ __forceinline__ void hllc_star_fwd(const St<T> &S, const St<T> &dS, const T Fs[5], const T dFs[5], const T n[3], T us, T dus, T ss, T dss,
                                              T sst, T dsst, T dF[5]) {
  const T fact = S.rho * (ss - us) / (ss - sst);
  const T dfact = (S.rho * (dss - dus) + dS.rho * (ss - us)) / (ss - sst) - fact / (ss - sst) * (dss - dsst);
  const T denom = S.rho * (ss - us);
  const T ddenom = S.rho * (dss - dus) + dS.rho * (ss - us);
  const T star[5] = {T(1), S.u[0] + (sst - us) * n[0], S.u[1] + (sst - us) * n[1], S.u[2] + (sst - us) * n[2],
                     S.E / S.rho + (sst - us) * (sst + S.P / denom)};
  const T dstar[5] = {T(0), dS.u[0] + (dsst - dus) * n[0], dS.u[1] + (dsst - dus) * n[1], dS.u[2] + (dsst - dus) * n[2],
                      dS.E / S.rho - S.E / (S.rho * S.rho) * dS.rho + (dsst - dus) * (sst + S.P / denom) +
                          (sst - us) * (dsst + dS.P / denom - S.P / (denom * denom) * ddenom)};
  const T U[5] = {S.rho, S.m[0], S.m[1], S.m[2], S.E}, dU[5] = {dS.rho, dS.m[0], dS.m[1], dS.m[2], dS.E};
  const T a1 = dss * fact + ss * dfact, a2 = ss * fact;
#pragma unroll
  for (int i = 0; i < 5; i++) dF[i] = dFs[i] + a1 * star[i] + a2 * dstar[i] - dss * U[i] - ss * dU[i];
}

template <typename T>
__device__ __forceinline__ T hllc_sstar(const St<T> &L, T uL, T sl, const St<T> &R, T uR, T sr) {
  const T rl = L.rho * uL, rr = R.rho * uR;
  const T numer = R.P - L.P + rl * (sl - uL) - rr * (sr - uR);
  const T denom = L.rho * (sl - uL) - R.rho * (sr - uR);
  return numer / denom;
}

template <typename T>
__device__ __forceinline__ void hllc_flux(T gamma, T cv, const St<T> &L, const St<T> &R, const T n[3], T F[5]) {
  T Fl[5], Fr[5], sl, sr;
  flux_dot_n(L, n, Fl);
  flux_dot_n(R, n, Fr);
  const T uL = L.u[0] * n[0] + L.u[1] * n[1] + L.u[2] * n[2], uR = R.u[0] * n[0] + R.u[1] * n[1] + R.u[2] * n[2];
  roe_speeds(gamma, cv, L, uL, R, uR, sl, sr);
  const T sst = hllc_sstar(L, uL, sl, R, uR, sr);
  if (T(0) <= sl) {
#pragma unroll
    for (int i = 0; i < 5; i++) F[i] = Fl[i];
  } else if (T(0) <= sst) {
    hllc_star(L, Fl, n, uL, sl, sst, F);
  } else if (T(0) <= sr) {
    hllc_star(R, Fr, n, uR, sr, sst, F);
  } else {
#pragma unroll
    for (int i = 0; i < 5; i++) F[i] = Fr[i];
  }
}

template <typename T>
__device__ __forceinline__ void hllc_flux_fwd(T gamma, T cv, const St<T> &L, const St<T> &dL, const St<T> &R, const St<T> &dR, const T n[3], T dF[5]) {
  T Fl[5], Fr[5], dFl[5], dFr[5], sl, dsl, sr, dsr;
  flux_dot_n(L, n, Fl);
  flux_dot_n(R, n, Fr);
  flux_dot_n_fwd(L, dL, n, dFl);
  flux_dot_n_fwd(R, dR, n, dFr);
  const T uL = L.u[0] * n[0] + L.u[1] * n[1] + L.u[2] * n[2], uR = R.u[0] * n[0] + R.u[1] * n[1] + R.u[2] * n[2];
  const T duL = dL.u[0] * n[0] + dL.u[1] * n[1] + dL.u[2] * n[2], duR = dR.u[0] * n[0] + dR.u[1] * n[1] + dR.u[2] * n[2];
  roe_speeds_fwd(gamma, cv, L, dL, uL, duL, R, dR, uR, duR, sl, dsl, sr, dsr);
  const T rl = L.rho * uL, drl = L.rho * duL + dL.rho * uL, rr = R.rho * uR, drr = R.rho * duR + dR.rho * uR;
  const T numer = R.P - L.P + rl * (sl - uL) - rr * (sr - uR);
  const T dnumer = dR.P - dL.P + rl * (dsl - duL) + drl * (sl - uL) - rr * (dsr - duR) - drr * (sr - uR);
  const T denom = L.rho * (sl - uL) - R.rho * (sr - uR);
  const T ddenom = L.rho * (dsl - duL) + dL.rho * (sl - uL) - R.rho * (dsr - duR) - dR.rho * (sr - uR);
  const T sst = numer / denom, dsst = dnumer / denom - numer / (denom * denom) * ddenom;
  if (T(0) <= sl) {
#pragma unroll
    for (int i = 0; i < 5; i++) dF[i] = dFl[i];
  } else if (T(0) <= sst) {
    hllc_star_fwd(L, dL, Fl, dFl, n, uL, duL, sl, dsl, sst, dsst, dF);
  } else if (T(0) <= sr) {
    hllc_star_fwd(R, dR, Fr, dFr, n, uR, duR, sr, dsr, sst, dsst, dF);
  } else {
#pragma unroll
    for (int i = 0; i < 5; i++) dF[i] = dFr[i];
  }
}

}  // namespace riemann
}  // namespace hb
