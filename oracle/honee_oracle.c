/* honee_oracle.c -- CPU oracle for the HONEE Newtonian operator (TEST INFRASTRUCTURE ONLY; see honee_oracle.h).
 *
 * Plain C99 restatement of the reference's point-wise QFunctions and of the libCEED operator semantics it relies on.
 * Every function names the reference lines it follows.  Nothing in the product library includes or links this file.
 */
#include "honee_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* The KM packing weight is evaluated as 1/sqrt(2.) (utils.h:240, newtonian_state.h:524), which rounds to one ulp
 * below M_SQRT1_2; keep the same expression so the packed strain matches the reference bit for bit. */
#define ORACLE_SQRT1_2 (1 / sqrt(2.))

/* =====================================================================================================================
 * Small helpers (qfunctions/utils.h)
 * ===================================================================================================================*/
static double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static double sq(double x) { return x * x; }

/* 3x3 inverse through the adjugate, det from the first column (utils.h:201-216). */
static void inv3(const double A[3][3], double Ainv[3][3], double *det_out) {
  Ainv[0][0] = A[1][1] * A[2][2] - A[1][2] * A[2][1];
  Ainv[0][1] = A[0][2] * A[2][1] - A[0][1] * A[2][2];
  Ainv[0][2] = A[0][1] * A[1][2] - A[0][2] * A[1][1];
  Ainv[1][0] = A[1][2] * A[2][0] - A[1][0] * A[2][2];
  Ainv[1][1] = A[0][0] * A[2][2] - A[0][2] * A[2][0];
  Ainv[1][2] = A[0][2] * A[1][0] - A[0][0] * A[1][2];
  Ainv[2][0] = A[1][0] * A[2][1] - A[1][1] * A[2][0];
  Ainv[2][1] = A[0][1] * A[2][0] - A[0][0] * A[2][1];
  Ainv[2][2] = A[0][0] * A[1][1] - A[0][1] * A[1][0];
  const double det   = A[0][0] * Ainv[0][0] + A[1][0] * Ainv[0][1] + A[2][0] * Ainv[0][2];
  const double scale = 1 / det;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) Ainv[i][j] *= scale;
  if (det_out) *det_out = det;
}

/* Kelvin-Mandel symmetric tensor (utils.h:239-247) */
static void km_to_full(const double v[6], double A[3][3]) {
  const double w = ORACLE_SQRT1_2;
  A[0][0]        = v[0];
  A[1][1]        = v[1];
  A[2][2]        = v[2];
  A[1][2] = A[2][1] = w * v[3];
  A[0][2] = A[2][0] = w * v[4];
  A[0][1] = A[1][0] = w * v[5];
}

/* =====================================================================================================================
 * State algebra (qfunctions/newtonian_state.h)
 * ===================================================================================================================*/
static double gamma_of(const HbGasProperties *g) { return g->cp / g->cv; }
static double rgas_of(const HbGasProperties *g) { return g->cp - g->cv; }

/* Y from U: newtonian_state.h:64-73 */
static void prim_from_cons(const HbGasProperties *gas, const double U[5], double Y[5]) {
  double u[3];
  for (int i = 0; i < 3; i++) u[i] = U[1 + i] / U[0];
  const double ke    = .5 * dot3(u, u);
  const double etot  = U[4] / U[0];
  const double eint  = etot - ke;
  Y[4]               = eint / gas->cv;
  Y[0]               = (gamma_of(gas) - 1) * U[0] * eint;
  for (int i = 0; i < 3; i++) Y[1 + i] = u[i];
}

/* dY from dU: newtonian_state.h:75-89 */
static void prim_from_cons_fwd(const HbGasProperties *gas, const OracleState *s, const double dU[5], double dY[5]) {
  const double *u = &s->Y[1];
  double        du[3];
  for (int i = 0; i < 3; i++) du[i] = (dU[1 + i] - u[i] * dU[0]) / s->U[0];
  const double ke    = .5 * dot3(u, u);
  const double dke   = dot3(du, u);
  const double etot  = s->U[4] / s->U[0];
  const double detot = (dU[4] - etot * dU[0]) / s->U[0];
  const double eint  = etot - ke;
  const double deint = detot - dke;
  dY[4]              = deint / gas->cv;
  dY[0]              = (gamma_of(gas) - 1) * (dU[0] * eint + s->U[0] * deint);
  for (int i = 0; i < 3; i++) dY[1 + i] = du[i];
}

/* U from Y: newtonian_state.h:159-168 */
static void cons_from_prim(const HbGasProperties *gas, const double Y[5], double U[5]) {
  const double *u = &Y[1];
  U[0]            = Y[0] / (rgas_of(gas) * Y[4]);
  for (int i = 0; i < 3; i++) U[1 + i] = U[0] * u[i];
  const double eint = gas->cv * Y[4];
  const double ke   = .5 * dot3(u, u);
  U[4]              = U[0] * (eint + ke);
}

/* dU from dY: newtonian_state.h:170-184 */
static void cons_from_prim_fwd(const HbGasProperties *gas, const OracleState *s, const double dY[5], double dU[5]) {
  const double *u  = &s->Y[1];
  const double *du = &dY[1];
  const double  T  = s->Y[4];
  dU[0]            = (dY[0] * T - s->Y[0] * dY[4]) / (rgas_of(gas) * T * T);
  for (int i = 0; i < 3; i++) dU[1 + i] = dU[0] * u[i] + s->U[0] * du[i];
  const double ke    = .5 * dot3(u, u);
  const double dke   = dot3(du, u);
  const double eint  = gas->cv * T;
  const double deint = gas->cv * dY[4];
  dU[4]              = dU[0] * (eint + ke) + s->U[0] * (deint + dke);
}

/* V from Y: newtonian_state.h:91-103 */
static void entropy_from_prim(const HbGasProperties *gas, const double Y[5], double V[5]) {
  const double g       = gamma_of(gas);
  const double rho     = Y[0] / (rgas_of(gas) * Y[4]);
  const double ent     = log(Y[0]) - g * log(rho);
  const double rho_p   = rho / Y[0];
  const double ke      = .5 * dot3(&Y[1], &Y[1]);
  V[0]                 = (g - ent) / (g - 1) - rho_p * ke;
  for (int i = 0; i < 3; i++) V[1 + i] = rho_p * Y[1 + i];
  V[4] = -rho_p;
}

/* dV from dY: newtonian_state.h:105-120 */
static void entropy_from_prim_fwd(const HbGasProperties *gas, const OracleState *s, const double dY[5], double dV[5]) {
  const double  g     = gamma_of(gas);
  const double *u     = &s->Y[1];
  const double  P = s->Y[0], T = s->Y[4], rho = s->U[0];
  const double  drho  = (dY[0] * T - P * dY[4]) / (rgas_of(gas) * T * T);
  const double  ke    = .5 * dot3(u, u);
  const double  dke   = dot3(&dY[1], u);
  const double  rho_p = rho / P;
  const double  drho_p = (drho * P - rho * dY[0]) / sq(P);
  const double  dent  = dY[0] / P - g * drho / rho;
  dV[0]               = -dent / (g - 1) - dke * rho_p - ke * drho_p;
  for (int i = 0; i < 3; i++) dV[1 + i] = rho_p * dY[1 + i] + drho_p * u[i];
  dV[4] = -drho_p;
}

/* Y from V: newtonian_state.h:122-132 */
static void prim_from_entropy(const HbGasProperties *gas, const double V[5], double Y[5]) {
  for (int i = 0; i < 3; i++) Y[1 + i] = -V[1 + i] / V[4];
  Y[4]               = -1 / (rgas_of(gas) * V[4]);
  const double g     = gamma_of(gas);
  const double ke    = .5 * dot3(&Y[1], &Y[1]);
  const double ent   = g - (g - 1) * (V[0] - ke * V[4]);
  const double log_p = -(ent + g * log(-V[4])) / (g - 1);
  Y[0]               = exp(log_p);
}

/* dY from dV: newtonian_state.h:134-146 */
static void prim_from_entropy_fwd(const HbGasProperties *gas, const OracleState *s, const double dV[5], double dY[5]) {
  double V[5];
  entropy_from_prim(gas, s->Y, V);
  for (int i = 0; i < 3; i++) dY[1 + i] = -(dV[1 + i] - V[1 + i] * dV[4] / V[4]) / V[4];
  dY[4]              = dV[4] / (rgas_of(gas) * V[4] * V[4]);
  const double g     = gamma_of(gas);
  const double ke    = .5 * dot3(&s->Y[1], &s->Y[1]);
  const double dke   = dot3(&dY[1], &s->Y[1]);
  const double dent  = (1 - g) * (dV[0] - ke * dV[4] - dke * V[4]);
  dY[0]              = s->Y[0] * (-dent - g * dV[4] / V[4]) / (g - 1);
}

/* U from V: newtonian_state.h:222-238 */
static void cons_from_entropy(const HbGasProperties *gas, const double V[5], double U[5]) {
  double u[3];
  for (int i = 0; i < 3; i++) u[i] = -V[1 + i] / V[4];
  const double g       = gamma_of(gas);
  const double ke      = .5 * dot3(u, u);
  const double ent     = g - (g - 1) * (V[0] - ke * V[4]);
  const double log_rho = -(ent + log(-V[4])) / (g - 1);
  U[0]                 = exp(log_rho);
  for (int i = 0; i < 3; i++) U[1 + i] = U[0] * u[i];
  const double eint = -gas->cv / (rgas_of(gas) * V[4]);
  U[4]              = U[0] * (eint + ke);
}

/* dU from dV: newtonian_state.h:240-262 */
static void cons_from_entropy_fwd(const HbGasProperties *gas, const OracleState *s, const double dV[5], double dU[5]) {
  double V[5], du[3];
  entropy_from_prim(gas, s->Y, V);
  const double *u = &s->Y[1];
  for (int i = 0; i < 3; i++) du[i] = (-dV[1 + i] - u[i] * dV[4]) / V[4];
  const double g       = gamma_of(gas);
  const double ke      = .5 * dot3(u, u);
  const double dke     = dot3(du, u);
  const double ent     = g - (g - 1) * (V[0] - ke * V[4]);
  const double dent    = -(g - 1) * (dV[0] - (dke * V[4] + ke * dV[4]));
  const double log_rho = -(ent + log(-V[4])) / (g - 1);
  const double rho     = exp(log_rho);
  dU[0]                = -rho / (g - 1) * (dent + dV[4] / V[4]);
  for (int i = 0; i < 3; i++) dU[1 + i] = dU[0] * u[i] + s->U[0] * du[i];
  const double eint  = -gas->cv / (rgas_of(gas) * V[4]);
  const double deint = gas->cv * dV[4] / (rgas_of(gas) * V[4] * V[4]);
  dU[4]              = dU[0] * (eint + ke) + s->U[0] * (deint + dke);
}

/* StateFromQ / StateFromQ_fwd / StateToQ / StateToQ_fwd: newtonian_state.h:299-330, 332-416 */
OracleState oracle_state_from_q(const HbGasProperties *gas, const double q[5], int state_var) {
  OracleState s;
  switch (state_var) {
    case HB_STATEVAR_PRIMITIVE:
      memcpy(s.Y, q, sizeof s.Y);
      cons_from_prim(gas, s.Y, s.U);
      break;
    case HB_STATEVAR_ENTROPY:
      cons_from_entropy(gas, q, s.U);
      prim_from_entropy(gas, q, s.Y);
      break;
    default:
      memcpy(s.U, q, sizeof s.U);
      prim_from_cons(gas, s.U, s.Y);
      break;
  }
  return s;
}

OracleState oracle_state_from_q_fwd(const HbGasProperties *gas, const OracleState *s, const double dq[5], int state_var) {
  OracleState ds;
  switch (state_var) {
    case HB_STATEVAR_PRIMITIVE:
      memcpy(ds.Y, dq, sizeof ds.Y);
      cons_from_prim_fwd(gas, s, ds.Y, ds.U);
      break;
    case HB_STATEVAR_ENTROPY:
      cons_from_entropy_fwd(gas, s, dq, ds.U);
      prim_from_entropy_fwd(gas, s, dq, ds.Y);
      break;
    default:
      memcpy(ds.U, dq, sizeof ds.U);
      prim_from_cons_fwd(gas, s, ds.U, ds.Y);
      break;
  }
  return ds;
}

void oracle_state_to_q(const HbGasProperties *gas, const OracleState *s, double q[5], int state_var) {
  switch (state_var) {
    case HB_STATEVAR_PRIMITIVE:
      memcpy(q, s->Y, 5 * sizeof(double));
      break;
    case HB_STATEVAR_ENTROPY:
      entropy_from_prim(gas, s->Y, q);
      break;
    default:
      memcpy(q, s->U, 5 * sizeof(double));
      break;
  }
}

void oracle_state_to_q_fwd(const HbGasProperties *gas, const OracleState *s, const OracleState *ds, double dq[5], int state_var) {
  if (state_var == HB_STATEVAR_ENTROPY) entropy_from_prim_fwd(gas, s, ds->Y, dq);
  else oracle_state_to_q(gas, ds, dq, state_var);
}

/* Y-perturbation to full state perturbation: StateFromY_fwd, newtonian_state.h:358-369 */
static OracleState state_from_y_fwd(const HbGasProperties *gas, const OracleState *s, const double dY[5]) {
  OracleState ds;
  memcpy(ds.Y, dY, sizeof ds.Y);
  cons_from_prim_fwd(gas, s, dY, ds.U);
  return ds;
}

/* =====================================================================================================================
 * Fluxes, stress, stabilisation (newtonian_state.h:425-567, stabilization.h)
 * ===================================================================================================================*/
/* Inviscid flux, direction-major F[i][comp] (newtonian_state.h:425-431) */
static void flux_inviscid(const OracleState *s, double F[3][5]) {
  const double *m = &s->U[1], *u = &s->Y[1], P = s->Y[0], E = s->U[4];
  for (int i = 0; i < 3; i++) {
    F[i][0] = m[i];
    for (int j = 0; j < 3; j++) F[i][1 + j] = m[i] * u[j] + P * (i == j);
    F[i][4] = (E + P) * u[i];
  }
}

/* Linearised inviscid flux (newtonian_state.h:433-442) */
static void flux_inviscid_fwd(const OracleState *s, const OracleState *ds, double dF[3][5]) {
  const double *m = &s->U[1], *u = &s->Y[1], P = s->Y[0], E = s->U[4];
  const double *dm = &ds->U[1], *du = &ds->Y[1], dP = ds->Y[0], dE = ds->U[4];
  for (int i = 0; i < 3; i++) {
    dF[i][0] = dm[i];
    for (int j = 0; j < 3; j++) dF[i][1 + j] = dm[i] * u[j] + m[i] * du[j] + dP * (i == j);
    dF[i][4] = (dE + dP) * u[i] + (E + P) * du[i];
  }
}

/* Strong-form convective residual sum_i dF_i(grad_s[i]) row i (newtonian_state.h:466-475) */
static void flux_inviscid_strong(const OracleState *s, const OracleState grad_s[3], double r[5]) {
  for (int c = 0; c < 5; c++) r[c] = 0;
  for (int i = 0; i < 3; i++) {
    double dF[3][5];
    flux_inviscid_fwd(s, &grad_s[i], dF);
    for (int c = 0; c < 5; c++) r[c] += dF[i][c];
  }
}

/* Kelvin-Mandel strain rate of grad u, G[i][j] = du_i/dx_j = grad_s[j].Y.velocity[i] (newtonian_state.h:509-537) */
static void km_strain_rate(const OracleState grad_s[3], double e[6]) {
  const double w = ORACLE_SQRT1_2;
  double       G[3][3];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) G[i][j] = grad_s[j].Y[1 + i];
  e[0] = G[0][0];
  e[1] = G[1][1];
  e[2] = G[2][2];
  e[3] = w * (G[1][2] + G[2][1]);
  e[4] = w * (G[0][2] + G[2][0]);
  e[5] = w * (G[0][1] + G[1][0]);
}

/* Newtonian stress in KM notation (newtonian_state.h:553-558) */
static void newtonian_stress(const HbGasProperties *gas, const double e[6], double sig[6]) {
  const double div_u = e[0] + e[1] + e[2];
  for (int i = 0; i < 6; i++) sig[i] = gas->mu * (2 * e[i] + gas->lambda * div_u * (i < 3));
}

/* Viscous energy flux (newtonian_state.h:560-565) */
static void viscous_energy_flux(const HbGasProperties *gas, const double Y[5], const OracleState grad_s[3], const double sig[3][3],
                                double Fe[3]) {
  for (int i = 0; i < 3; i++)
    Fe[i] = -Y[1] * sig[0][i] - Y[2] * sig[1][i] - Y[3] * sig[2][i] - gas->k * grad_s[i].Y[4];
}

/* Linearised viscous energy flux (newtonian_state.h:567-574) */
static void viscous_energy_flux_fwd(const HbGasProperties *gas, const double Y[5], const double dY[5], const OracleState grad_ds[3],
                                    const double sig[3][3], const double dsig[3][3], double dFe[3]) {
  for (int i = 0; i < 3; i++)
    dFe[i] = -Y[1] * dsig[0][i] - dY[1] * sig[0][i] - Y[2] * dsig[1][i] - dY[2] * sig[1][i] - Y[3] * dsig[2][i] - dY[3] * sig[2][i] -
             gas->k * grad_ds[i].Y[4];
}

/* Total flux Flux[comp][dir] (newtonian_state.h:477-484) */
static void flux_total(const double Fi[3][5], const double sig[3][3], const double Fe[3], double Flux[5][3]) {
  for (int j = 0; j < 3; j++) {
    Flux[0][j] = Fi[j][0];
    for (int k = 0; k < 3; k++) Flux[k + 1][j] = Fi[j][1 + k] - sig[k][j];
    Flux[4][j] = Fi[j][4] + Fe[j];
  }
}

/* Diagonal tau (stabilization.h:67-100) */
static void tau_diag_prim(const HbTauDiagCoefficients *tc, const HbGasProperties *gas, const OracleState *s, const double dXdx[3][3], double dt,
                          double tau_d[3]) {
  double gij[3][3];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      gij[i][j] = 0;
      for (int k = 0; k < 3; k++) gij[i][j] += dXdx[k][i] * dXdx[k][j];
    }
  const double dts = tc->Ctau_t / dt;
  double       gu[3] = {0, 0, 0};
  const double *u  = &s->Y[1];
  for (int i = 0; i < 3; i++) gu[i] += gij[i][0] * u[0] + gij[i][1] * u[1] + gij[i][2] * u[2];
  const double ugu = dot3(u, gu);
  double       g2  = 0;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) g2 += gij[i][j] * gij[i][j];
  const double rho  = s->U[0];
  const double tau  = sq(rho) * (4. * sq(dts) + ugu) + tc->Ctau_v * sq(gas->mu) * g2;
  const double fact = sqrt(tau);
  tau_d[0]          = tc->Ctau_C * fact / (rho * (gij[0][0] + gij[1][1] + gij[2][2])) * 0.125;
  tau_d[1]          = tc->Ctau_M / fact;
  tau_d[2]          = tc->Ctau_E / (fact * gas->cv);
}

/* SU/SUPG stabilisation term stab[comp][dir] (stabilization.h:25-58).  Note the reference scales the strong residual
 * (conservative components) by tau and feeds it to the primitive-variable tangent; that is kept. */
static void stabilization(int type, const HbGasProperties *gas, const OracleState *s, const double tau_d[3], const OracleState grad_s[3],
                          const double U_dot[5], const double body[5], const double divFdiff[5], double stab[5][3]) {
  double r[5] = {0, 0, 0, 0, 0};
  if (type == HB_STAB_SU || type == HB_STAB_SUPG) flux_inviscid_strong(s, grad_s, r);
  if (type == HB_STAB_SUPG)
    for (int c = 0; c < 5; c++) r[c] += U_dot[c] - body[c] + divFdiff[c];
  const double dY[5] = {tau_d[0] * r[0], tau_d[1] * r[1], tau_d[1] * r[2], tau_d[1] * r[3], tau_d[2] * r[4]};
  OracleState  ds    = state_from_y_fwd(gas, s, dY);
  double       dF[3][5];
  flux_inviscid_fwd(s, &ds, dF);
  for (int c = 0; c < 5; c++)
    for (int i = 0; i < 3; i++) stab[c][i] = dF[i][c];
}

/* IDL ramp (utils.h:287-295) and damping residual (newtonian_integrands.h:13-21) */
static double linear_ramp(double amplitude, double length, double start, double x) {
  if (x < start) return amplitude;
  if (x < start + length) return amplitude * ((x - start) * (-1 / length) + 1);
  return 0;
}

static void idl_residual(const HbGasProperties *gas, const OracleState *s, double sigma, const double damp_y[5], double res[5]) {
  double dy[5];
  for (int i = 0; i < 5; i++) dy[i] = damp_y[i] * sigma;
  OracleState ds = state_from_y_fwd(gas, s, dy);
  for (int i = 0; i < 5; i++) res[i] += ds.U[i];
}

/* Physical gradient of the state from the reference gradient (newtonian_state.h:581-593).
 * grad_q is [3][5][Q] reference derivatives; dq[c][j] = sum_k g[c][k] dXdx[k][j]. */
static void physical_gradient(const HbGasProperties *gas, const OracleState *s, int state_var, int Q, int i, const double *grad_q,
                              const double dXdx[3][3], OracleState grad_s[3]) {
  double g[5][3], dq[5][3];
  for (int d = 0; d < 3; d++)
    for (int c = 0; c < 5; c++) g[c][d] = grad_q[(Q * 5) * d + Q * c + i];
  for (int c = 0; c < 5; c++)
    for (int j = 0; j < 3; j++) {
      dq[c][j] = 0;
      for (int k = 0; k < 3; k++) dq[c][j] += g[c][k] * dXdx[k][j];
    }
  for (int j = 0; j < 3; j++) {
    double col[5];
    for (int c = 0; c < 5; c++) col[c] = dq[c][j];
    grad_s[j] = oracle_state_from_q_fwd(gas, s, col, state_var);
  }
}

static void unpack_qdata(int Q, int i, const double *qd, double *wdetJ, double dXdx[3][3]) {
  *wdetJ = qd[i];
  for (int k = 0; k < 9; k++) dXdx[k / 3][k % 3] = qd[(1 + k) * Q + i];
}

/* =====================================================================================================================
 * Volume QFunctions (qfunctions/newtonian.h:205-311, newtonian_integrands.h:87-166)
 * ===================================================================================================================*/
static int ifunction(void *ctx_, int Q, const double *const *in, double *const *out, int state_var) {
  const HbNewtonianContext *ctx = (const HbNewtonianContext *)ctx_;
  const HbGasProperties    *gas = &ctx->gas;
  if (ctx->divFdiff_method != HB_DIV_DIFF_FLUX_PROJ_NONE) return 1; /* projected div(F_diff) is out of scope */
  const double *q = in[0], *grad_q = in[1], *q_dot = in[2], *qdata = in[3], *x = in[4];
  double       *v = out[0], *grad_v = out[1], *jd = out[2];
  for (int i = 0; i < Q; i++) {
    double qi[5], qdi[5];
    for (int c = 0; c < 5; c++) {
      qi[c]  = q[c * Q + i];
      qdi[c] = q_dot[c * Q + i];
    }
    const OracleState s     = oracle_state_from_q(gas, qi, state_var);
    const OracleState s_dot = oracle_state_from_q_fwd(gas, &s, qdi, state_var);
    double            wdetJ, dXdx[3][3];
    unpack_qdata(Q, i, qdata, &wdetJ, dXdx);
    OracleState grad_s[3];
    physical_gradient(gas, &s, state_var, Q, i, grad_q, dXdx, grad_s);

    /* IFunction_Newtonian_Integrand, newtonian_integrands.h:87-115 */
    double strain[6], sig_km[6], sig[3][3], Fe[3], Fi[3][5], Flux[5][3], tau_d[3], stab[5][3];
    double v_i[5], gv_i[5][3];
    km_strain_rate(grad_s, strain);
    newtonian_stress(gas, strain, sig_km);
    km_to_full(sig_km, sig);
    viscous_energy_flux(gas, s.Y, grad_s, sig, Fe);
    flux_inviscid(&s, Fi);
    flux_total(Fi, sig, Fe, Flux);
    const double *gv  = ctx->g;
    const double body[5] = {0, s.U[0] * gv[0], s.U[0] * gv[1], s.U[0] * gv[2], dot3(&s.U[1], gv)};
    const double  zero[5] = {0, 0, 0, 0, 0};
    for (int c = 0; c < 5; c++) v_i[c] = s_dot.U[c] - body[c];
    tau_diag_prim(&ctx->tau_coeffs, gas, &s, dXdx, ctx->dt, tau_d);
    stabilization(ctx->stabilization, gas, &s, tau_d, grad_s, s_dot.U, body, zero, stab);
    for (int c = 0; c < 5; c++)
      for (int d = 0; d < 3; d++) gv_i[c][d] = -Flux[c][d] + stab[c][d];

    double sigma = 0;
    if (ctx->idl_enable) { /* newtonian_integrands.h:38-45 */
      sigma              = linear_ramp(ctx->idl_amplitude, ctx->idl_length, ctx->idl_start, x[0 * Q + i]);
      const double dy[5] = {s.Y[0] - ctx->idl_pressure, 0, 0, 0, 0};
      double       res[5] = {0, 0, 0, 0, 0};
      idl_residual(gas, &s, sigma, dy, res);
      for (int c = 0; c < 5; c++) v_i[c] += res[c];
    }
    for (int c = 0; c < 5; c++) v[c * Q + i] = wdetJ * v_i[c];
    for (int c = 0; c < 5; c++)
      for (int k = 0; k < 3; k++)
        grad_v[(k * 5 + c) * Q + i] = wdetJ * (gv_i[c][0] * dXdx[k][0] + gv_i[c][1] * dXdx[k][1] + gv_i[c][2] * dXdx[k][2]);
    if (jd) {
      for (int c = 0; c < 5; c++) jd[c * Q + i] = qi[c];
      for (int c = 0; c < 6; c++) jd[(5 + c) * Q + i] = strain[c];
      for (int c = 0; c < 3; c++) jd[(11 + c) * Q + i] = tau_d[c];
      if (ctx->idl_enable) jd[14 * Q + i] = sigma;
    }
  }
  return 0;
}

static int ijacobian(void *ctx_, int Q, const double *const *in, double *const *out, int state_var) {
  const HbNewtonianContext *ctx = (const HbNewtonianContext *)ctx_;
  const HbGasProperties    *gas = &ctx->gas;
  const double *dq = in[0], *grad_dq = in[1], *qdata = in[2], *jd = in[3];
  double       *v = out[0], *grad_v = out[1];
  for (int i = 0; i < Q; i++) {
    double qi[5], strain[6], tau_d[3], dqi[5];
    for (int c = 0; c < 5; c++) qi[c] = jd[c * Q + i];
    for (int c = 0; c < 6; c++) strain[c] = jd[(5 + c) * Q + i];
    for (int c = 0; c < 3; c++) tau_d[c] = jd[(11 + c) * Q + i];
    for (int c = 0; c < 5; c++) dqi[c] = dq[c * Q + i];
    const OracleState s  = oracle_state_from_q(gas, qi, state_var);
    const OracleState ds = oracle_state_from_q_fwd(gas, &s, dqi, state_var);
    double            wdetJ, dXdx[3][3];
    unpack_qdata(Q, i, qdata, &wdetJ, dXdx);
    OracleState grad_ds[3];
    physical_gradient(gas, &s, state_var, Q, i, grad_dq, dXdx, grad_ds);

    /* IJacobian_Newtonian_Integrand, newtonian_integrands.h:134-166 */
    double dstrain[6], dsig_km[6], sig_km[6], sig[3][3], dsig[3][3], dFe[3], dFi[3][5], dFlux[5][3], dstab[5][3];
    double v_i[5], gv_i[5][3];
    km_strain_rate(grad_ds, dstrain);
    newtonian_stress(gas, dstrain, dsig_km);
    newtonian_stress(gas, strain, sig_km);
    km_to_full(dsig_km, dsig);
    km_to_full(sig_km, sig);
    viscous_energy_flux_fwd(gas, s.Y, ds.Y, grad_ds, sig, dsig, dFe);
    flux_inviscid_fwd(&s, &ds, dFi);
    flux_total(dFi, dsig, dFe, dFlux);
    const double *gv       = ctx->g;
    const double  dbody[5] = {0, ds.U[0] * gv[0], ds.U[0] * gv[1], ds.U[0] * gv[2], dot3(&ds.U[1], gv)};
    double        dU_dot[5];
    const double  zero[5] = {0, 0, 0, 0, 0};
    for (int c = 0; c < 5; c++) {
      dU_dot[c] = ctx->ijacobian_time_shift * ds.U[c];
      v_i[c]    = dU_dot[c] - dbody[c];
    }
    stabilization(ctx->stabilization, gas, &s, tau_d, grad_ds, dU_dot, dbody, zero, dstab);
    for (int c = 0; c < 5; c++)
      for (int d = 0; d < 3; d++) gv_i[c][d] = -dFlux[c][d] + dstab[c][d];
    if (ctx->idl_enable) { /* newtonian_integrands.h:58-64 */
      const double sigma  = jd[14 * Q + i];
      const double dy[5]  = {ds.Y[0], 0, 0, 0, 0};
      double       res[5] = {0, 0, 0, 0, 0};
      idl_residual(gas, &s, sigma, dy, res);
      for (int c = 0; c < 5; c++) v_i[c] += res[c];
    }
    for (int c = 0; c < 5; c++) v[c * Q + i] = wdetJ * v_i[c];
    for (int c = 0; c < 5; c++)
      for (int k = 0; k < 3; k++)
        grad_v[(k * 5 + c) * Q + i] = wdetJ * (gv_i[c][0] * dXdx[k][0] + gv_i[c][1] * dXdx[k][1] + gv_i[c][2] * dXdx[k][2]);
  }
  return 0;
}

int oracle_qf_ifunction_conserv(void *c, int Q, const double *const *in, double *const *out) { return ifunction(c, Q, in, out, HB_STATEVAR_CONSERVATIVE); }
int oracle_qf_ifunction_prim(void *c, int Q, const double *const *in, double *const *out) { return ifunction(c, Q, in, out, HB_STATEVAR_PRIMITIVE); }
int oracle_qf_ifunction_entropy(void *c, int Q, const double *const *in, double *const *out) { return ifunction(c, Q, in, out, HB_STATEVAR_ENTROPY); }
int oracle_qf_ijacobian_conserv(void *c, int Q, const double *const *in, double *const *out) { return ijacobian(c, Q, in, out, HB_STATEVAR_CONSERVATIVE); }
int oracle_qf_ijacobian_prim(void *c, int Q, const double *const *in, double *const *out) { return ijacobian(c, Q, in, out, HB_STATEVAR_PRIMITIVE); }
int oracle_qf_ijacobian_entropy(void *c, int Q, const double *const *in, double *const *out) { return ijacobian(c, Q, in, out, HB_STATEVAR_ENTROPY); }

/* Geometric factors (setupgeo.h:42-56, setupgeo_helpers.h:26-32): in[0] = dx [3 ref dirs][3 comps][Q], in[1] = weights. */
int oracle_qf_setup(void *ctx, int Q, const double *const *in, double *const *out) {
  (void)ctx;
  const double *J = in[0], *w = in[1];
  double       *qd = out[0];
  for (int i = 0; i < Q; i++) {
    double dxdX[3][3], dXdx[3][3], det;
    for (int d = 0; d < 3; d++)
      for (int c = 0; c < 3; c++) dxdX[c][d] = J[(Q * 3) * d + Q * c + i];
    inv3(dxdX, dXdx, &det);
    qd[i] = w[i] * det;
    for (int k = 0; k < 9; k++) qd[(1 + k) * Q + i] = dXdx[k / 3][k % 3];
  }
  return 0;
}

/* Total kinetic energy integrands (monitor_totalkineticenergy.h:8-39), conservative variables. */
int oracle_qf_monitor_ke_conserv(void *ctx_, int Q, const double *const *in, double *const *out) {
  const HbNewtonianContext *ctx = (const HbNewtonianContext *)ctx_;
  const HbGasProperties    *gas = &ctx->gas;
  const double *q = in[0], *grad_q = in[1], *qdata = in[2];
  double       *v = out[0];
  for (int i = 0; i < Q; i++) {
    double qi[5];
    for (int c = 0; c < 5; c++) qi[c] = q[c * Q + i];
    const OracleState s = oracle_state_from_q(gas, qi, HB_STATEVAR_CONSERVATIVE);
    double            wdetJ, dXdx[3][3], e[6], S[3][3], G[3][3], w[3];
    OracleState       grad_s[3];
    unpack_qdata(Q, i, qdata, &wdetJ, dXdx);
    physical_gradient(gas, &s, HB_STATEVAR_CONSERVATIVE, Q, i, grad_q, dXdx, grad_s);
    v[0 * Q + i] = wdetJ * 0.5 * s.U[0] * dot3(&s.Y[1], &s.Y[1]);
    km_strain_rate(grad_s, e);
    const double div_u = e[0] + e[1] + e[2];
    km_to_full(e, S);
    double SS = 0;
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) SS += S[a][b] * S[a][b];
    v[1 * Q + i] = wdetJ * -2 * gas->mu * SS;
    v[2 * Q + i] = wdetJ * -gas->lambda * gas->mu * sq(div_u);
    v[3 * Q + i] = wdetJ * s.Y[0] * div_u;
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) G[a][b] = grad_s[b].Y[1 + a];
    w[0]         = G[2][1] - G[1][2];
    w[1]         = G[0][2] - G[2][0];
    w[2]         = G[1][0] - G[0][1];
    v[4 * Q + i] = wdetJ * gas->mu * dot3(w, w);
  }
  return 0;
}

/* Taylor-Green initial condition at points X (taylorgreen.h:23-51), including its cos(2z+2) and cos(z) forms. */
int oracle_qf_ics_taylorgreen(void *ctx_, int Q, const double *const *in, double *const *out) {
  const HbTaylorGreenContext *ctx = (const HbTaylorGreenContext *)ctx_;
  const HbGasProperties      *gas = &ctx->newt_ctx.gas;
  const double               *X   = in[0];
  double                     *q0  = out[0];
  const double                R    = rgas_of(gas);
  const double                V0   = sqrt(dot3(ctx->reference.velocity, ctx->reference.velocity));
  const double                rho0 = ctx->reference.pressure / (ctx->reference.temperature * R);
  const double                L[3] = {ctx->lx, ctx->ly, ctx->lz};
  for (int i = 0; i < Q; i++) {
    double x[3], Y[5], qv[5];
    for (int d = 0; d < 3; d++) x[d] = X[d * Q + i] * (2 * M_PI / L[d]);
    Y[0]          = ctx->reference.pressure + (rho0 * sq(V0) / 16) * (cos(2 * x[0]) + cos(2 * x[1])) * (cos(2 * x[2] + 2));
    Y[1]          = ctx->u[0] + V0 * sin(x[0]) * cos(x[1]) * cos(x[2]);
    Y[2]          = ctx->u[1] - V0 * cos(x[0]) * sin(x[1]) * cos(x[2]);
    Y[3]          = ctx->u[2];
    Y[4]          = ctx->reference.temperature;
    OracleState s = oracle_state_from_q(gas, Y, HB_STATEVAR_PRIMITIVE);
    oracle_state_to_q(gas, &s, qv, ctx->newt_ctx.state_var);
    for (int c = 0; c < 5; c++) q0[c * Q + i] = qv[c];
  }
  return 0;
}

/* =====================================================================================================================
 * 1D tabulation: Gauss-Legendre points, Gauss-Lobatto-Legendre nodes, Lagrange interpolation/derivative matrices.
 * (PETSc's Lagrange dual space and default tensor quadrature, src/dm-utils.c:387-485 and :691-735; PETSc itself is
 * third-party and absent here.)
 * ===================================================================================================================*/
static void legendre_eval(int n, double x, double *p, double *dp) {
  double p0 = 1, p1 = x;
  if (n == 0) {
    *p  = 1;
    *dp = 0;
    return;
  }
  for (int k = 2; k <= n; k++) {
    const double p2 = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k;
    p0              = p1;
    p1              = p2;
  }
  *p  = p1;
  *dp = n * (x * p1 - p0) / (x * x - 1);
}

void oracle_gauss_legendre(int Q, double *x, double *w) {
  for (int i = 0; i < Q; i++) {
    double z = -cos(M_PI * (i + 0.75) / (Q + 0.5)), p, dp;
    for (int it = 0; it < 100; it++) {
      legendre_eval(Q, z, &p, &dp);
      const double dz = p / dp;
      z -= dz;
      if (fabs(dz) < 1e-16) break;
    }
    legendre_eval(Q, z, &p, &dp);
    x[i] = z;
    w[i] = 2 / ((1 - z * z) * dp * dp);
  }
}

void oracle_gauss_lobatto(int P, double *x) {
  const int N = P - 1; /* polynomial degree */
  x[0]        = -1;
  x[N]        = 1;
  for (int i = 1; i < N; i++) {
    /* interior nodes are the roots of P'_N; Newton on q(z) = (1-z^2) P'_N(z) */
    double z = -cos(M_PI * i / N);
    for (int it = 0; it < 100; it++) {
      double p, dp;
      legendre_eval(N, z, &p, &dp);
      /* (1-z^2) P_N'' = 2 z P_N' - N(N+1) P_N */
      const double ddp = (2 * z * dp - N * (N + 1) * p) / (1 - z * z);
      const double dz  = dp / ddp;
      z -= dz;
      if (fabs(dz) < 1e-16) break;
    }
    x[i] = z;
  }
}

void oracle_lagrange_tabulate(int P, const double *nodes, int Q, const double *pts, double *interp, double *grad) {
  for (int q = 0; q < Q; q++) {
    const double x = pts[q];
    for (int j = 0; j < P; j++) {
      double l = 1, dl = 0;
      for (int m = 0; m < P; m++) {
        if (m == j) continue;
        const double f = (x - nodes[m]) / (nodes[j] - nodes[m]);
        dl             = dl * f + l / (nodes[j] - nodes[m]);
        l *= f;
      }
      interp[q * P + j] = l;
      grad[q * P + j]   = dl;
    }
  }
}

/* =====================================================================================================================
 * Structured box
 * ===================================================================================================================*/
static int64_t nodes_dim(int n, int P, int periodic) { return (int64_t)n * (P - 1) + (periodic ? 0 : 1); }

int64_t oracle_box_num_nodes(const int n[3], int P, const int periodic[3]) {
  return nodes_dim(n[0], P, periodic[0]) * nodes_dim(n[1], P, periodic[1]) * nodes_dim(n[2], P, periodic[2]);
}

void oracle_box_offsets(const int n[3], int P, const int periodic[3], int ncomp, int32_t *offsets) {
  const int64_t N0 = nodes_dim(n[0], P, periodic[0]), N1 = nodes_dim(n[1], P, periodic[1]), N2 = nodes_dim(n[2], P, periodic[2]);
  int64_t       e  = 0;
  for (int ez = 0; ez < n[2]; ez++)
    for (int ey = 0; ey < n[1]; ey++)
      for (int ex = 0; ex < n[0]; ex++, e++)
        for (int c = 0; c < P; c++)
          for (int b = 0; b < P; b++)
            for (int a = 0; a < P; a++) {
              const int64_t i = ((int64_t)ex * (P - 1) + a) % N0, j = ((int64_t)ey * (P - 1) + b) % N1, k = ((int64_t)ez * (P - 1) + c) % N2;
              offsets[e * P * P * P + (c * P + b) * P + a] = (int32_t)((i + N0 * (j + N1 * k)) * ncomp);
            }
}

void oracle_box_elem_coords(const int n[3], const double *xs, const double *ys, const double *zs, double *x_elem) {
  int64_t e = 0;
  for (int ez = 0; ez < n[2]; ez++)
    for (int ey = 0; ey < n[1]; ey++)
      for (int ex = 0; ex < n[0]; ex++, e++)
        for (int v = 0; v < 8; v++) {
          const int a = v & 1, b = (v >> 1) & 1, c = (v >> 2) & 1;
          x_elem[e * 24 + 0 * 8 + v] = xs[ex + a];
          x_elem[e * 24 + 1 * 8 + v] = ys[ey + b];
          x_elem[e * 24 + 2 * 8 + v] = zs[ez + c];
        }
}

/* =====================================================================================================================
 * libCEED operator semantics
 * ===================================================================================================================*/
void oracle_restrict(int num_elem, int elem_size, int ncomp, int comp_stride, const int32_t *offsets, const double *l, double *e) {
  for (int64_t el = 0; el < num_elem; el++)
    for (int c = 0; c < ncomp; c++)
      for (int p = 0; p < elem_size; p++) e[(el * ncomp + c) * elem_size + p] = l[offsets[el * elem_size + p] + (int64_t)c * comp_stride];
}

void oracle_restrict_t(int num_elem, int elem_size, int ncomp, int comp_stride, const int32_t *offsets, const double *e, double *l) {
  for (int64_t el = 0; el < num_elem; el++)
    for (int c = 0; c < ncomp; c++)
      for (int p = 0; p < elem_size; p++) l[offsets[el * elem_size + p] + (int64_t)c * comp_stride] += e[(el * ncomp + c) * elem_size + p];
}

/* out[k][j][i] = sum_{a,b,c} Mz[k][c] My[j][b] Mx[i][a] u[c][b][a]  (u: P^3, out: Q^3), by sum factorisation */
static void tensor_apply(int P, int Q, const double *Mx, const double *My, const double *Mz, const double *u, double *out) {
  double t1[8 * 8 * 8], t2[8 * 8 * 8];
  for (int c = 0; c < P; c++)
    for (int b = 0; b < P; b++)
      for (int i = 0; i < Q; i++) {
        double s = 0;
        for (int a = 0; a < P; a++) s += Mx[i * P + a] * u[(c * P + b) * P + a];
        t1[(c * P + b) * Q + i] = s;
      }
  for (int c = 0; c < P; c++)
    for (int j = 0; j < Q; j++)
      for (int i = 0; i < Q; i++) {
        double s = 0;
        for (int b = 0; b < P; b++) s += My[j * P + b] * t1[(c * P + b) * Q + i];
        t2[(c * Q + j) * Q + i] = s;
      }
  for (int k = 0; k < Q; k++)
    for (int j = 0; j < Q; j++)
      for (int i = 0; i < Q; i++) {
        double s = 0;
        for (int c = 0; c < P; c++) s += Mz[k * P + c] * t2[(c * Q + j) * Q + i];
        out[(k * Q + j) * Q + i] = s;
      }
}

/* u[c][b][a] += sum_{i,j,k} Mz[k][c] My[j][b] Mx[i][a] w[k][j][i]  (transpose of tensor_apply) */
static void tensor_apply_t(int P, int Q, const double *Mx, const double *My, const double *Mz, const double *w, double *u) {
  double t1[8 * 8 * 8], t2[8 * 8 * 8];
  for (int k = 0; k < Q; k++)
    for (int j = 0; j < Q; j++)
      for (int a = 0; a < P; a++) {
        double s = 0;
        for (int i = 0; i < Q; i++) s += Mx[i * P + a] * w[(k * Q + j) * Q + i];
        t1[(k * Q + j) * P + a] = s;
      }
  for (int k = 0; k < Q; k++)
    for (int b = 0; b < P; b++)
      for (int a = 0; a < P; a++) {
        double s = 0;
        for (int j = 0; j < Q; j++) s += My[j * P + b] * t1[(k * Q + j) * P + a];
        t2[(k * P + b) * P + a] = s;
      }
  for (int c = 0; c < P; c++)
    for (int b = 0; b < P; b++)
      for (int a = 0; a < P; a++) {
        double s = 0;
        for (int k = 0; k < Q; k++) s += Mz[k * P + c] * t2[(k * P + b) * P + a];
        u[(c * P + b) * P + a] += s;
      }
}

typedef struct {
  const OracleMesh *m;
  int               P3, Q3;
} OpShape;

/* E-vector gather of 5 interleaved components, then interp [5][Q3] and reference gradient [3][5][Q3] */
static void elem_eval(const OracleMesh *m, int64_t e, const double *l, double *ue, double *interp, double *grad) {
  const int P = m->P, Q = m->Q, P3 = P * P * P, Q3 = Q * Q * Q;
  for (int c = 0; c < 5; c++)
    for (int p = 0; p < P3; p++) ue[c * P3 + p] = l[m->offsets[e * P3 + p] + c];
  const double *B = m->interp1d, *G = m->grad1d;
  for (int c = 0; c < 5; c++) {
    if (interp) tensor_apply(P, Q, B, B, B, &ue[c * P3], &interp[c * Q3]);
    if (grad) {
      tensor_apply(P, Q, G, B, B, &ue[c * P3], &grad[(0 * 5 + c) * Q3]);
      tensor_apply(P, Q, B, G, B, &ue[c * P3], &grad[(1 * 5 + c) * Q3]);
      tensor_apply(P, Q, B, B, G, &ue[c * P3], &grad[(2 * 5 + c) * Q3]);
    }
  }
}

/* Transpose basis of (v [5][Q3], grad_v [3][5][Q3]) and scatter-add into the L-vector */
static void elem_scatter(const OracleMesh *m, int64_t e, const double *v, const double *gv, double *ve, double *l) {
  const int     P = m->P, Q = m->Q, P3 = P * P * P, Q3 = Q * Q * Q;
  const double *B = m->interp1d, *G = m->grad1d;
  memset(ve, 0, sizeof(double) * 5 * P3);
  for (int c = 0; c < 5; c++) {
    tensor_apply_t(P, Q, B, B, B, &v[c * Q3], &ve[c * P3]);
    tensor_apply_t(P, Q, G, B, B, &gv[(0 * 5 + c) * Q3], &ve[c * P3]);
    tensor_apply_t(P, Q, B, G, B, &gv[(1 * 5 + c) * Q3], &ve[c * P3]);
    tensor_apply_t(P, Q, B, B, G, &gv[(2 * 5 + c) * Q3], &ve[c * P3]);
  }
  for (int c = 0; c < 5; c++)
    for (int p = 0; p < P3; p++) l[m->offsets[e * P3 + p] + c] += ve[c * P3 + p];
}

typedef void (*ElemKernel)(const OracleMesh *m, int64_t e, void *user, double *scratch, int *err);

/* Run kern over all elements; colouring (if given) makes concurrent scatters race free, otherwise serial. */
static void for_each_elem(const OracleMesh *m, ElemKernel kern, void *user, size_t scratch_doubles, int *err) {
  if (m->color_ptr && m->num_colors > 0) {
#ifdef _OPENMP
    const int nt = m->num_threads > 0 ? m->num_threads : omp_get_max_threads();
#endif
    for (int col = 0; col < m->num_colors; col++) {
      const int64_t lo = m->color_ptr[col], hi = m->color_ptr[col + 1];
#ifdef _OPENMP
#pragma omp parallel num_threads(nt)
#endif
      {
        double *scratch = (double *)malloc(sizeof(double) * scratch_doubles);
        int     lerr    = 0;
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
        for (int64_t i = lo; i < hi; i++) kern(m, m->color_elem[i], user, scratch, &lerr);
        if (lerr) {
#ifdef _OPENMP
#pragma omp atomic write
#endif
          *err = lerr;
        }
        free(scratch);
      }
    }
  } else {
    double *scratch = (double *)malloc(sizeof(double) * scratch_doubles);
    for (int64_t e = 0; e < m->num_elem; e++) kern(m, e, user, scratch, err);
    free(scratch);
  }
}

typedef struct {
  OracleQF      qf;
  void         *ctx;
  const double *q, *q_dot, *qdata, *x_q, *jd_in;
  double       *jd_out, *v;
  int           num_jd;
} ApplyArgs;

static size_t apply_scratch(const OracleMesh *m) {
  const size_t P3 = (size_t)m->P * m->P * m->P, Q3 = (size_t)m->Q * m->Q * m->Q;
  return 5 * P3 + 5 * Q3 + 15 * Q3 + 5 * Q3 + 5 * Q3 + 15 * Q3 + 5 * P3 + 3 * Q3;
}

static void ifunction_elem(const OracleMesh *m, int64_t e, void *user, double *s, int *err) {
  ApplyArgs *a  = (ApplyArgs *)user;
  const int  P3 = m->P * m->P * m->P, Q3 = m->Q * m->Q * m->Q;
  double *ue = s, *qi = ue + 5 * P3, *gq = qi + 5 * Q3, *qdi = gq + 15 * Q3, *v = qdi + 5 * Q3, *gv = v + 5 * Q3, *ve = gv + 15 * Q3;
  double *xz = ve + 5 * P3; /* the reference QFunction always reads the "x" input (newtonian.h:225); zeros without IDL */
  elem_eval(m, e, a->q, ue, qi, gq);
  elem_eval(m, e, a->q_dot, ue, qdi, NULL);
  if (!a->x_q) memset(xz, 0, sizeof(double) * 3 * Q3);
  const double *in[5]  = {qi, gq, qdi, a->qdata + e * 10 * Q3, a->x_q ? a->x_q + e * 3 * Q3 : xz};
  double       *out[3] = {v, gv, a->jd_out ? a->jd_out + e * (int64_t)a->num_jd * Q3 : NULL};
  if (a->qf(a->ctx, Q3, in, out)) *err = 1;
  elem_scatter(m, e, v, gv, ve, a->v);
}

static void ijacobian_elem(const OracleMesh *m, int64_t e, void *user, double *s, int *err) {
  ApplyArgs *a  = (ApplyArgs *)user;
  const int  P3 = m->P * m->P * m->P, Q3 = m->Q * m->Q * m->Q;
  double *ue = s, *qi = ue + 5 * P3, *gq = qi + 5 * Q3, *v = gq + 15 * Q3 + 5 * Q3, *gv = v + 5 * Q3, *ve = gv + 15 * Q3;
  elem_eval(m, e, a->q, ue, qi, gq);
  const double *in[4]  = {qi, gq, a->qdata + e * 10 * Q3, a->jd_in + e * (int64_t)a->num_jd * Q3};
  double       *out[2] = {v, gv};
  if (a->qf(a->ctx, Q3, in, out)) *err = 1;
  elem_scatter(m, e, v, gv, ve, a->v);
}

int oracle_apply_ifunction(const OracleMesh *m, OracleQF qf, void *ctx, const double *q, const double *q_dot, const double *qdata,
                           const double *x_q, double *jac_data, int num_jd, double *v, int64_t l_size) {
  ApplyArgs a = {qf, ctx, q, q_dot, qdata, x_q, NULL, jac_data, v, num_jd};
  int       err = 0;
  memset(v, 0, sizeof(double) * l_size);
  for_each_elem(m, ifunction_elem, &a, apply_scratch(m), &err);
  return err;
}

int oracle_apply_ijacobian(const OracleMesh *m, OracleQF qf, void *ctx, const double *dq, const double *qdata, const double *jac_data, int num_jd,
                           double *v, int64_t l_size) {
  ApplyArgs a = {qf, ctx, dq, NULL, qdata, NULL, jac_data, NULL, v, num_jd};
  int       err = 0;
  memset(v, 0, sizeof(double) * l_size);
  for_each_elem(m, ijacobian_elem, &a, apply_scratch(m), &err);
  return err;
}

/* ---- diagonal (libCEED CeedOperatorLinearAssembleDiagonal semantics) ---- */
static void diagonal_elem(const OracleMesh *m, int64_t e, void *user, double *s, int *err) {
  ApplyArgs    *a  = (ApplyArgs *)user;
  const int     P = m->P, Q = m->Q, P3 = P * P * P, Q3 = Q * Q * Q;
  const double *B = m->interp1d, *G = m->grad1d;
  double       *de = s; /* [5][P3] */
  memset(de, 0, sizeof(double) * 5 * P3);
  for (int qp = 0; qp < Q3; qp++) {
    const int qi = qp % Q, qj = (qp / Q) % Q, qk = qp / (Q * Q);
    /* linearised QFunction at this point: A[out 20][in 20], field order (interp comps 0-4, grad [dim][comp]) */
    double A[20][20], qd[10], jd[HB_JAC_DATA_COMPS_IDL];
    for (int c = 0; c < 10; c++) qd[c] = a->qdata[(e * 10 + c) * Q3 + qp];
    for (int c = 0; c < a->num_jd; c++) jd[c] = a->jd_in[(e * a->num_jd + c) * Q3 + qp];
    for (int j = 0; j < 20; j++) {
      double dq[5] = {0}, gdq[15] = {0}, v[5], gv[15];
      if (j < 5) dq[j] = 1;
      else gdq[j - 5] = 1;
      const double *in[4]  = {dq, gdq, qd, jd};
      double       *out[2] = {v, gv};
      if (a->qf(a->ctx, 1, in, out)) *err = 1;
      for (int i = 0; i < 5; i++) A[i][j] = v[i];
      for (int i = 0; i < 15; i++) A[5 + i][j] = gv[i];
    }
    for (int p = 0; p < P3; p++) {
      const int pa = p % P, pb = (p / P) % P, pc = p / (P * P);
      const double bx = B[qi * P + pa], by = B[qj * P + pb], bz = B[qk * P + pc];
      const double gx = G[qi * P + pa], gy = G[qj * P + pb], gz = G[qk * P + pc];
      const double phi[4] = {bx * by * bz, gx * by * bz, bx * gy * bz, bx * by * gz};
      for (int c = 0; c < 5; c++) {
        double acc = 0;
        for (int mo = 0; mo < 4; mo++) {
          const int io = mo == 0 ? c : 5 + (mo - 1) * 5 + c;
          for (int mi = 0; mi < 4; mi++) {
            const int ii = mi == 0 ? c : 5 + (mi - 1) * 5 + c;
            acc += phi[mo] * A[io][ii] * phi[mi];
          }
        }
        de[c * P3 + p] += acc;
      }
    }
  }
  for (int c = 0; c < 5; c++)
    for (int p = 0; p < P3; p++) a->v[m->offsets[e * P3 + p] + c] += de[c * P3 + p];
}

int oracle_assemble_diagonal(const OracleMesh *m, OracleQF qf, void *ctx, const double *qdata, const double *jac_data, int num_jd, double *diag,
                             int64_t l_size) {
  ApplyArgs a = {qf, ctx, NULL, NULL, qdata, NULL, jac_data, NULL, diag, num_jd};
  int       err = 0;
  memset(diag, 0, sizeof(double) * l_size);
  for_each_elem(m, diagonal_elem, &a, (size_t)5 * m->P * m->P * m->P, &err);
  return err;
}

/* ---- point-block diagonal (libCEED CeedOperatorLinearAssemblePointBlockDiagonal semantics): per node a row-major
 * 5 x 5 block [component out][component in], out[(node * 5 + i) * 5 + j], from the same linearised QFunction ---- */
static void point_block_elem(const OracleMesh *m, int64_t e, void *user, double *s, int *err) {
  ApplyArgs    *a  = (ApplyArgs *)user;
  const int     P = m->P, Q = m->Q, P3 = P * P * P, Q3 = Q * Q * Q;
  const double *B = m->interp1d, *G = m->grad1d;
  double       *be = s; /* [P3][5][5] */
  memset(be, 0, sizeof(double) * 25 * P3);
  for (int qp = 0; qp < Q3; qp++) {
    const int qi = qp % Q, qj = (qp / Q) % Q, qk = qp / (Q * Q);
    double A[20][20], qd[10], jd[HB_JAC_DATA_COMPS_IDL];
    for (int c = 0; c < 10; c++) qd[c] = a->qdata[(e * 10 + c) * Q3 + qp];
    for (int c = 0; c < a->num_jd; c++) jd[c] = a->jd_in[(e * a->num_jd + c) * Q3 + qp];
    for (int j = 0; j < 20; j++) {
      double dq[5] = {0}, gdq[15] = {0}, v[5], gv[15];
      if (j < 5) dq[j] = 1;
      else gdq[j - 5] = 1;
      const double *in[4]  = {dq, gdq, qd, jd};
      double       *out[2] = {v, gv};
      if (a->qf(a->ctx, 1, in, out)) *err = 1;
      for (int i = 0; i < 5; i++) A[i][j] = v[i];
      for (int i = 0; i < 15; i++) A[5 + i][j] = gv[i];
    }
    for (int p = 0; p < P3; p++) {
      const int pa = p % P, pb = (p / P) % P, pc = p / (P * P);
      const double bx = B[qi * P + pa], by = B[qj * P + pb], bz = B[qk * P + pc];
      const double gx = G[qi * P + pa], gy = G[qj * P + pb], gz = G[qk * P + pc];
      const double phi[4] = {bx * by * bz, gx * by * bz, bx * gy * bz, bx * by * gz};
      for (int ci = 0; ci < 5; ci++)
        for (int cj = 0; cj < 5; cj++) {
          double acc = 0;
          for (int mo = 0; mo < 4; mo++) {
            const int io = mo == 0 ? ci : 5 + (mo - 1) * 5 + ci;
            for (int mi = 0; mi < 4; mi++) {
              const int ii = mi == 0 ? cj : 5 + (mi - 1) * 5 + cj;
              acc += phi[mo] * A[io][ii] * phi[mi];
            }
          }
          be[(p * 5 + ci) * 5 + cj] += acc;
        }
    }
  }
  for (int p = 0; p < P3; p++)
    for (int k = 0; k < 25; k++) a->v[(int64_t)m->offsets[e * P3 + p] * 5 + k] += be[p * 25 + k];
}

int oracle_assemble_point_block(const OracleMesh *m, OracleQF qf, void *ctx, const double *qdata, const double *jac_data, int num_jd, double *out,
                                int64_t l_size) {
  ApplyArgs a = {qf, ctx, NULL, NULL, qdata, NULL, jac_data, NULL, out, num_jd};
  int       err = 0;
  memset(out, 0, sizeof(double) * 5 * l_size);
  for_each_elem(m, point_block_elem, &a, (size_t)25 * m->P * m->P * m->P, &err);
  return err;
}

/* ---- geometric factors ---- */
static void linear_basis(int Q, double *Bx, double *Gx, double *w) {
  double x[16];
  oracle_gauss_legendre(Q, x, w);
  for (int q = 0; q < Q; q++) {
    Bx[q * 2 + 0] = 0.5 * (1 - x[q]);
    Bx[q * 2 + 1] = 0.5 * (1 + x[q]);
    Gx[q * 2 + 0] = -0.5;
    Gx[q * 2 + 1] = 0.5;
  }
}

/* ---- explicit path: RHSFunction_Newtonian (qfunctions/newtonian.h:133-202) and Mass_N (qfunctions/mass.h:19-26) ---- */
/* The IFunction integrand (newtonian.h:205-257) at q_dot = 0 is v = -wdetJ body (+ the damping-layer residual) and
 * grad v = wdetJ dXdx (-F_total + stab) with the SUPG strong residual evaluated at U_dot = 0, which is exactly the negative
 * of the RHS integrand (v = wdetJ body - damping, grad v = wdetJ dXdx (F_total - stab), U_dot = 0). */
int oracle_qf_rhs_conserv(void *ctx, int Q, const double *const *in, double *const *out) {
  double *zero = (double *)calloc((size_t)5 * Q, sizeof(double)), *jd = (double *)malloc(sizeof(double) * HB_JAC_DATA_COMPS_IDL * Q);
  if (!zero || !jd) {
    free(zero);
    free(jd);
    return 1;
  }
  const double *in_if[5]  = {in[0], in[1], zero, in[2], in[3]};
  double       *out_if[3] = {out[0], out[1], jd};
  const int     err       = oracle_qf_ifunction_conserv(ctx, Q, in_if, out_if);
  for (int i = 0; i < 5 * Q; i++) out[0][i] = -out[0][i];
  for (int i = 0; i < 15 * Q; i++) out[1][i] = -out[1][i];
  free(zero);
  free(jd);
  return err;
}

static void rhs_elem(const OracleMesh *m, int64_t e, void *user, double *s, int *err) {
  ApplyArgs *a  = (ApplyArgs *)user;
  const int  P3 = m->P * m->P * m->P, Q3 = m->Q * m->Q * m->Q;
  double *ue = s, *qi = ue + 5 * P3, *gq = qi + 5 * Q3, *v = gq + 15 * Q3 + 5 * Q3, *gv = v + 5 * Q3, *ve = gv + 15 * Q3;
  double *xz = ve + 5 * P3;
  elem_eval(m, e, a->q, ue, qi, gq);
  if (!a->x_q) memset(xz, 0, sizeof(double) * 3 * Q3);
  const double *in[4]  = {qi, gq, a->qdata + e * 10 * Q3, a->x_q ? a->x_q + e * 3 * Q3 : xz};
  double       *out[2] = {v, gv};
  if (a->qf(a->ctx, Q3, in, out)) *err = 1;
  elem_scatter(m, e, v, gv, ve, a->v);
}

int oracle_apply_rhs(const OracleMesh *m, OracleQF qf, void *ctx, const double *q, const double *qdata, const double *x_q, double *v,
                     int64_t l_size) {
  ApplyArgs a = {qf, ctx, q, NULL, qdata, x_q, NULL, NULL, v, 14};
  int       err = 0;
  memset(v, 0, sizeof(double) * l_size);
  for_each_elem(m, rhs_elem, &a, apply_scratch(m), &err);
  return err;
}

int oracle_qf_mass(void *ctx, int Q, const double *const *in, double *const *out) {
  (void)ctx;
  for (int j = 0; j < 5; j++)
    for (int i = 0; i < Q; i++) out[0][j * Q + i] = in[1][i] * in[0][j * Q + i];
  return 0;
}

static void mass_elem(const OracleMesh *m, int64_t e, void *user, double *s, int *err) {
  ApplyArgs    *a = (ApplyArgs *)user;
  const int     P = m->P, Q = m->Q, P3 = P * P * P, Q3 = Q * Q * Q;
  const double *B = m->interp1d;
  double *ue = s, *ui = ue + 5 * P3, *v = ui + 5 * Q3, *ve = v + 5 * Q3;
  elem_eval(m, e, a->q, ue, ui, NULL);
  const double *in[2]  = {ui, a->qdata + e * 10 * Q3};
  double       *out[1] = {v};
  if (a->qf(NULL, Q3, in, out)) *err = 1;
  memset(ve, 0, sizeof(double) * 5 * P3);
  for (int c = 0; c < 5; c++) tensor_apply_t(P, Q, B, B, B, &v[c * Q3], &ve[c * P3]);
  for (int c = 0; c < 5; c++)
    for (int p = 0; p < P3; p++) a->v[m->offsets[e * P3 + p] + c] += ve[c * P3 + p];
}

int oracle_apply_mass(const OracleMesh *m, OracleQF qf, const double *u, const double *qdata, double *v, int64_t l_size) {
  ApplyArgs a = {qf, NULL, u, NULL, qdata, NULL, NULL, NULL, v, 0};
  int       err = 0;
  memset(v, 0, sizeof(double) * l_size);
  for_each_elem(m, mass_elem, &a, apply_scratch(m), &err);
  return err;
}

/* Restatement of MassFunction_Newtonian for conservative variables (qfunctions/newtonian.h:44-86): v = wdetJ q_dot and
 * Grad_v = wdetJ dXdx stab, stab from the stabilization with zero state gradient, zero body force and the rate as U_dot (for
 * SUPG the strong residual is U_dot; for SU and none the term vanishes). */
int oracle_qf_mass_stab_conserv(void *ctx_, int Q, const double *const *in, double *const *out) {
  const HbNewtonianContext *ctx = (const HbNewtonianContext *)ctx_;
  const HbGasProperties    *gas = &ctx->gas;
  const double             *qd = in[0], *q = in[1], *qdata = in[2];
  double                   *v = out[0], *gv = out[1];
  for (int i = 0; i < Q; i++) {
    double qi[5], U_dot[5];
    for (int c = 0; c < 5; c++) {
      qi[c]    = q[c * Q + i];
      U_dot[c] = qd[c * Q + i];
    }
    const OracleState s = oracle_state_from_q(gas, qi, HB_STATEVAR_CONSERVATIVE);
    double            wdetJ, dXdx[3][3];
    unpack_qdata(Q, i, qdata, &wdetJ, dXdx);
    for (int c = 0; c < 5; c++) v[c * Q + i] = wdetJ * U_dot[c];
    OracleState grad_s[3];
    memset(grad_s, 0, sizeof grad_s);
    const double zero[5] = {0, 0, 0, 0, 0};
    double       tau_d[3], stab[5][3];
    tau_diag_prim(&ctx->tau_coeffs, gas, &s, dXdx, ctx->dt, tau_d);
    stabilization(ctx->stabilization, gas, &s, tau_d, grad_s, U_dot, zero, zero, stab);
    for (int c = 0; c < 5; c++)
      for (int k = 0; k < 3; k++) gv[(k * 5 + c) * Q + i] = wdetJ * (stab[c][0] * dXdx[k][0] + stab[c][1] * dXdx[k][1] + stab[c][2] * dXdx[k][2]);
  }
  return 0;
}

/* The SUPG-stabilized mass operator of the explicit path (MassFunction_Newtonian, qfunctions/newtonian.h:44-86; built by
 * CreateKSPMassOperator_NewtonianStabilized, problems/newtonian.c:212-265, when stab = supg and the run is explicit):
 * inputs q_dot (active, INTERP), q (passive, INTERP), qdata; outputs v (INTERP) and Grad_v (GRAD). */
static void mass_stab_elem(const OracleMesh *m, int64_t e, void *user, double *s, int *err) {
  ApplyArgs *a  = (ApplyArgs *)user;
  const int  P3 = m->P * m->P * m->P, Q3 = m->Q * m->Q * m->Q;
  double *ue = s, *qdi = ue + 5 * P3, *qi = qdi + 5 * Q3, *v = qi + 15 * Q3 + 5 * Q3, *gv = v + 5 * Q3, *ve = gv + 15 * Q3;
  elem_eval(m, e, a->q_dot, ue, qdi, NULL);
  elem_eval(m, e, a->q, ue, qi, NULL);
  const double *in[3]  = {qdi, qi, a->qdata + e * 10 * Q3};
  double       *out[2] = {v, gv};
  if (a->qf(a->ctx, Q3, in, out)) *err = 1;
  elem_scatter(m, e, v, gv, ve, a->v);
}

int oracle_apply_mass_stab(const OracleMesh *m, OracleQF qf, void *ctx, const double *q_dot, const double *q, const double *qdata, double *v,
                           int64_t l_size) {
  ApplyArgs a = {qf, ctx, q, q_dot, qdata, NULL, NULL, NULL, v, 14};
  int       err = 0;
  memset(v, 0, sizeof(double) * l_size);
  for_each_elem(m, mass_stab_elem, &a, apply_scratch(m), &err);
  return err;
}

/* Diagonal of the stabilized mass at the state q: the QFunction linearised in the rate at each point (unit rates), tested
 * with the value and the reference gradient of the same basis function (libCEED diagonal assembly semantics). */
static void mass_stab_diag_elem(const OracleMesh *m, int64_t e, void *user, double *s, int *err) {
  ApplyArgs    *a = (ApplyArgs *)user;
  const int     P = m->P, Q = m->Q, P3 = P * P * P, Q3 = Q * Q * Q;
  const double *B = m->interp1d, *G = m->grad1d;
  double       *ue = s, *qi = ue + 5 * P3, *de = qi + 5 * Q3;
  elem_eval(m, e, a->q, ue, qi, NULL);
  memset(de, 0, sizeof(double) * 5 * P3);
  for (int qp = 0; qp < Q3; qp++) {
    const int qx = qp % Q, qy = (qp / Q) % Q, qz = qp / (Q * Q);
    double    qd[10], qv[5], A[20][5];
    for (int c = 0; c < 10; c++) qd[c] = a->qdata[(e * 10 + c) * Q3 + qp];
    for (int c = 0; c < 5; c++) qv[c] = qi[c * Q3 + qp];
    for (int j = 0; j < 5; j++) {
      double u[5] = {0}, v[5], gv[15];
      u[j]                 = 1;
      const double *in[3]  = {u, qv, qd};
      double       *out[2] = {v, gv};
      if (a->qf(a->ctx, 1, in, out)) *err = 1;
      for (int i = 0; i < 5; i++) A[i][j] = v[i];
      for (int i = 0; i < 15; i++) A[5 + i][j] = gv[i];
    }
    for (int p = 0; p < P3; p++) {
      const int    pa = p % P, pb = (p / P) % P, pc = p / (P * P);
      const double bx = B[qx * P + pa], by = B[qy * P + pb], bz = B[qz * P + pc];
      const double gx = G[qx * P + pa], gy = G[qy * P + pb], gz = G[qz * P + pc];
      const double phi[4] = {bx * by * bz, gx * by * bz, bx * gy * bz, bx * by * gz};
      for (int c = 0; c < 5; c++) {
        double acc = 0;
        for (int mo = 0; mo < 4; mo++) acc += phi[mo] * A[mo == 0 ? c : 5 + (mo - 1) * 5 + c][c] * phi[0];
        de[c * P3 + p] += acc;
      }
    }
  }
  for (int c = 0; c < 5; c++)
    for (int p = 0; p < P3; p++) a->v[m->offsets[e * P3 + p] + c] += de[c * P3 + p];
}

int oracle_assemble_mass_stab_diagonal(const OracleMesh *m, OracleQF qf, void *ctx, const double *q, const double *qdata, double *diag,
                                       int64_t l_size) {
  ApplyArgs a = {qf, ctx, q, NULL, qdata, NULL, NULL, NULL, diag, 14};
  int       err = 0;
  memset(diag, 0, sizeof(double) * l_size);
  const size_t P3 = (size_t)m->P * m->P * m->P, Q3 = (size_t)m->Q * m->Q * m->Q;
  for_each_elem(m, mass_stab_diag_elem, &a, 10 * P3 + 5 * Q3, &err);
  return err;
}

int oracle_setup_qdata(int num_elem, int Q, const double *x_elem, double *qdata) {
  const int Q3 = Q * Q * Q;
  double    B[32], G[32], w1[16];
  linear_basis(Q, B, G, w1);
  double *J = (double *)malloc(sizeof(double) * 9 * Q3), *w = (double *)malloc(sizeof(double) * Q3);
  for (int k = 0; k < Q; k++)
    for (int j = 0; j < Q; j++)
      for (int i = 0; i < Q; i++) w[(k * Q + j) * Q + i] = w1[i] * w1[j] * w1[k];
  for (int64_t e = 0; e < num_elem; e++) {
    for (int c = 0; c < 3; c++) {
      const double *xe = &x_elem[e * 24 + c * 8];
      tensor_apply(2, Q, G, B, B, xe, &J[(0 * 3 + c) * Q3]);
      tensor_apply(2, Q, B, G, B, xe, &J[(1 * 3 + c) * Q3]);
      tensor_apply(2, Q, B, B, G, xe, &J[(2 * 3 + c) * Q3]);
    }
    const double *in[2]  = {J, w};
    double       *out[1] = {qdata + e * 10 * Q3};
    oracle_qf_setup(NULL, Q3, in, out);
  }
  free(J);
  free(w);
  return 0;
}

int oracle_coords_at_qpts(int num_elem, int Q, const double *x_elem, double *x_q) {
  const int Q3 = Q * Q * Q;
  double    B[32], G[32], w1[16];
  linear_basis(Q, B, G, w1);
  for (int64_t e = 0; e < num_elem; e++)
    for (int c = 0; c < 3; c++) tensor_apply(2, Q, B, B, B, &x_elem[e * 24 + c * 8], &x_q[(e * 3 + c) * Q3]);
  return 0;
}

int oracle_monitor_ke(const OracleMesh *m, void *ctx, const double *q, const double *qdata, double sums[5]) {
  const int P3 = m->P * m->P * m->P, Q3 = m->Q * m->Q * m->Q;
  double   *ue = (double *)malloc(sizeof(double) * 5 * P3), *qi = (double *)malloc(sizeof(double) * 5 * Q3);
  double   *gq = (double *)malloc(sizeof(double) * 15 * Q3), *v = (double *)malloc(sizeof(double) * 5 * Q3);
  for (int c = 0; c < 5; c++) sums[c] = 0;
  for (int64_t e = 0; e < m->num_elem; e++) {
    elem_eval(m, e, q, ue, qi, gq);
    const double *in[3]  = {qi, gq, qdata + e * 10 * Q3};
    double       *out[1] = {v};
    oracle_qf_monitor_ke_conserv(ctx, Q3, in, out);
    for (int c = 0; c < 5; c++)
      for (int i = 0; i < Q3; i++) sums[c] += v[c * Q3 + i];
  }
  free(ue);
  free(qi);
  free(gq);
  free(v);
  return 0;
}
