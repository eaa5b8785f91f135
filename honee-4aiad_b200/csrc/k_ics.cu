// k_ics.cu -- initial-condition operators of HONEE's set-up (SetupLibceed's op_ics, src/setuplibceed.c:143-175) for sm_100a.
//
// HONEE evaluates the initial state at the nodes of the solution basis: the coordinate field (restriction elem_restr_x,
// trilinear basis) is projected onto the solution nodes by CeedBasisCreateProjection(basis_x, basis_q), the IC QFunction
// runs at those nodes, and its output (EVAL_NONE through the state restriction) is summed into the local vector;
// ICs_FixMultiplicity (src/misc.c:16-45) then divides by the node multiplicity.  Here one thread evaluates one node of
// one element: the node coordinates from the element's vertex coordinates through the 1D projection matrix, then the
// IC QFunction, written to the E-vector [elem][5][P^3] that the restriction transpose sums.
//
// QFunctions restated (arithmetic in the reference's order; cos, sin, exp and log are CUDA's):
//   ICsNewtonianIG_{Conserv,Prim,Entropy}   qfunctions/newtonian.h:17-42       uniform reference state
//   ICsTaylorGreen                          qfunctions/taylorgreen.h:23-51     (keeps the reference's cos(2 z + 2))
//   ICsChannel                              qfunctions/channel.h:24-73         (Pr as the reference forms it: mu / (cp k))
//   IC_GaussianWave_{Conserv,Prim,Entropy}  qfunctions/gaussianwave.h:20-71
// State conversions: StateFromPrimitive / StateFromU / StateToQ (qfunctions/newtonian_state.h:64-73, 159-168, 282-304),
// the entropy variables by StateEntropyFromPrimitive (:91-103).
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include "honee_b200.h"

namespace {

struct FullState {
  double rho, m[3], E;  // conservative
  double P, u[3], T;    // primitive
};

__device__ __forceinline__ double gas_R(const HbGasProperties &g) { return g.cp - g.cv; }
__device__ __forceinline__ double gas_gamma(const HbGasProperties &g) { return g.cp / g.cv; }

// StateConservativeFromPrimitive (newtonian_state.h:159-168)
__device__ FullState state_from_Y(const HbGasProperties &g, const double Y[5]) {
  FullState s;
  s.P = Y[0];
  s.u[0] = Y[1];
  s.u[1] = Y[2];
  s.u[2] = Y[3];
  s.T = Y[4];
  s.rho = s.P / (gas_R(g) * s.T);
  for (int i = 0; i < 3; i++) s.m[i] = s.rho * s.u[i];
  const double e_internal = g.cv * s.T;
  const double e_kinetic = .5 * (s.u[0] * s.u[0] + s.u[1] * s.u[1] + s.u[2] * s.u[2]);
  s.E = s.rho * (e_internal + e_kinetic);
  return s;
}

// StatePrimitiveFromConservative (newtonian_state.h:64-73)
__device__ FullState state_from_U(const HbGasProperties &g, const double U[5]) {
  FullState s;
  s.rho = U[0];
  s.m[0] = U[1];
  s.m[1] = U[2];
  s.m[2] = U[3];
  s.E = U[4];
  for (int i = 0; i < 3; i++) s.u[i] = s.m[i] / s.rho;
  const double e_kinetic = .5 * (s.u[0] * s.u[0] + s.u[1] * s.u[1] + s.u[2] * s.u[2]);
  const double e_total = s.E / s.rho;
  const double e_internal = e_total - e_kinetic;
  s.T = e_internal / g.cv;
  s.P = (gas_gamma(g) - 1) * s.rho * e_internal;
  return s;
}

// StateToQ (newtonian_state.h:282-304); entropy variables from the primitive state (StateEntropyFromPrimitive, :91-103)
__device__ void state_to_q(const HbGasProperties &g, const FullState &s, int state_var, double q[5]) {
  if (state_var == HB_STATEVAR_PRIMITIVE) {
    q[0] = s.P;
    q[1] = s.u[0];
    q[2] = s.u[1];
    q[3] = s.u[2];
    q[4] = s.T;
  } else if (state_var == HB_STATEVAR_ENTROPY) {
    const double gamma = gas_gamma(g);
    const double rho = s.P / (gas_R(g) * s.T);
    const double entropy = log(s.P) - gamma * log(rho);
    const double rho_div_p = rho / s.P;
    const double e_kinetic = 0.5 * (s.u[0] * s.u[0] + s.u[1] * s.u[1] + s.u[2] * s.u[2]);
    q[0] = (gamma - entropy) / (gamma - 1) - rho_div_p * e_kinetic;
    for (int i = 0; i < 3; i++) q[1 + i] = rho_div_p * s.u[i];
    q[4] = -rho_div_p;
  } else {
    q[0] = s.rho;
    q[1] = s.m[0];
    q[2] = s.m[1];
    q[3] = s.m[2];
    q[4] = s.E;
  }
}

struct IcsArgs {
  int kind, state_var, num_elem, P_to;
  double B[HB_MAX_P * 2];  // projection of the trilinear coordinate nodes onto the solution nodes [P_to][2]
  const double *x_e;       // [elem][3][8] vertex coordinates (E-vector of the coordinate restriction)
  double *q0_e;            // [elem][5][P_to^3]
  unsigned char ctx[320];  // the IC QFunction's context bytes
};

__global__ void k_ics(const IcsArgs a) {
  const int P3 = a.P_to * a.P_to * a.P_to;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)a.num_elem * P3) return;
  const int64_t e = t / P3;
  const int p = (int)(t % P3), i = p % a.P_to, j = (p / a.P_to) % a.P_to, k = p / (a.P_to * a.P_to);
  // node coordinates: tensor product of the 1D projection rows (vertex index = x + 2 y + 4 z)
  double X[3];
  for (int c = 0; c < 3; c++) {
    const double *xv = a.x_e + (e * 3 + c) * 8;
    double s = 0;
    for (int v = 0; v < 8; v++) s += a.B[k * 2 + (v >> 2)] * a.B[j * 2 + ((v >> 1) & 1)] * a.B[i * 2 + (v & 1)] * xv[v];
    X[c] = s;
  }
  double q[5];
  if (a.kind == HB_IC_NEWTONIAN) {  // ICsNewtonianIG: the reference state everywhere
    HbSetupContext ctx;
    memcpy(&ctx, a.ctx, sizeof ctx);
    const double Y[5] = {ctx.reference.pressure, ctx.reference.velocity[0], ctx.reference.velocity[1], ctx.reference.velocity[2],
                         ctx.reference.temperature};
    state_to_q(ctx.newt_ctx.gas, state_from_Y(ctx.newt_ctx.gas, Y), a.state_var, q);
  } else if (a.kind == HB_IC_TAYLOR_GREEN) {
    HbTaylorGreenContext ctx;
    memcpy(&ctx, a.ctx, sizeof ctx);
    const HbGasProperties &g = ctx.newt_ctx.gas;
    const HbStatePrimitive &ref = ctx.reference;
    const double R = gas_R(g);
    const double V0 = sqrt(ref.velocity[0] * ref.velocity[0] + ref.velocity[1] * ref.velocity[1] + ref.velocity[2] * ref.velocity[2]);
    const double density0 = ref.pressure / (ref.temperature * R);
    double x[3] = {X[0], X[1], X[2]};
    const double scale = 2 * M_PI / ctx.lx;
    for (int c = 0; c < 3; c++) x[c] *= scale;
    double Y[5];
    Y[0] = ref.pressure + (density0 * (V0 * V0) / 16) * (cos(2 * x[0]) + cos(2 * x[1])) * (cos(2 * x[2] + 2));
    Y[1] = ctx.u[0] + V0 * sin(x[0]) * cos(x[1]) * cos(x[2]);
    Y[2] = ctx.u[1] - V0 * cos(x[0]) * sin(x[1]) * cos(x[2]);
    Y[3] = ctx.u[2];
    Y[4] = ref.temperature;
    state_to_q(g, state_from_Y(g, Y), ctx.newt_ctx.state_var, q);
  } else if (a.kind == HB_IC_CHANNEL) {
    HbChannelContext ctx;
    memcpy(&ctx, a.ctx, sizeof ctx);
    const HbGasProperties &g = ctx.newt_ctx.gas;
    const double Pr = g.mu / (g.cp * g.k);
    const double Ec = (ctx.umax * ctx.umax) / (g.cp * ctx.theta0);
    const double yc = (X[1] - ctx.center) / ctx.H, yc2 = yc * yc;
    const double theta = ctx.theta0 * (1 + (Pr * Ec / 3) * (1 - yc2 * yc2));
    const double Y[5] = {ctx.P0, ctx.umax * (1 - yc2), 0., 0., theta};
    state_to_q(g, state_from_Y(g, Y), ctx.newt_ctx.state_var, q);
  } else {  // IC_GaussianWave
    HbGaussianWaveContext ctx;
    memcpy(&ctx, a.ctx, sizeof ctx);
    const HbGasProperties &g = ctx.newt_ctx.gas;
    const HbState &S = ctx.S_infty;
    const double gamma = gas_gamma(g);
    const double x0 = X[0] - ctx.epicenter[0], y0 = X[1] - ctx.epicenter[1];
    const double e_kinetic = 0.5 * S.density * (S.Y.velocity[0] * S.Y.velocity[0] + S.Y.velocity[1] * S.Y.velocity[1] + S.Y.velocity[2] * S.Y.velocity[2]);
    const double perturbation = 1 + ctx.amplitude * exp(-((x0 * x0) + (y0 * y0)) / (2 * (ctx.width * ctx.width)));
    double U[5];
    U[0] = S.density * perturbation;
    U[1] = S.Y.velocity[0] * U[0];
    U[2] = S.Y.velocity[1] * U[0];
    U[3] = S.Y.velocity[2] * U[0];
    U[4] = S.Y.pressure / (gamma - 1) * perturbation + e_kinetic;
    state_to_q(g, state_from_U(g, U), a.state_var, q);
  }
  for (int c = 0; c < 5; c++) a.q0_e[(e * 5 + c) * P3 + p] = q[c];
}

}  // namespace

extern "C" int hb_ics_apply(int kind, int state_var, const void *ctx, size_t ctx_size, int num_elem, int P_to, const double *proj1d, const double *x_e,
                            double *q0_e, void *stream) {
  static const size_t sizes[4] = {sizeof(HbSetupContext), sizeof(HbTaylorGreenContext), sizeof(HbChannelContext), sizeof(HbGaussianWaveContext)};
  if (kind < 0 || kind > 3 || ctx_size != sizes[kind] || P_to < 2 || P_to > HB_MAX_P || num_elem < 0) return HB_ERROR_INVALID;
  if (state_var != HB_STATEVAR_CONSERVATIVE && state_var != HB_STATEVAR_PRIMITIVE && state_var != HB_STATEVAR_ENTROPY) return HB_ERROR_UNSUPPORTED;
  if (num_elem == 0) return HB_SUCCESS;
  IcsArgs a;
  memset(&a, 0, sizeof a);
  a.kind = kind;
  a.state_var = state_var;
  a.num_elem = num_elem;
  a.P_to = P_to;
  memcpy(a.B, proj1d, sizeof(double) * 2 * P_to);
  a.x_e = x_e;
  a.q0_e = q0_e;
  memcpy(a.ctx, ctx, ctx_size);
  const int64_t n = (int64_t)num_elem * P_to * P_to * P_to;
  const int bs = 128;
  k_ics<<<(unsigned)((n + bs - 1) / bs), bs, 0, (cudaStream_t)stream>>>(a);
  return cudaGetLastError() == cudaSuccess ? HB_SUCCESS : HB_ERROR_CUDA;
}
