/* ref_qfunctions.c -- exports the reference's own QFunctions, compiled unchanged, for the oracle checks
 * (TEST INFRASTRUCTURE ONLY).
 *
 * Built by oracle/Makefile with -I pointing at the reference's qfunctions/ directory and at oracle/ref_shim, into
 * oracle/_ref/libhonee_ref.so.  Nothing of the reference is copied: this file only includes its headers and gives
 * each QFunction / state helper an exported name so the tests can call it through ctypes and compare it with the
 * oracle restatement (oracle/honee_oracle.c) and with the CUDA kernels.
 */
#include <ceed/types.h>

#include "bc_freestream.h"
#include "channel.h"
#include "gaussianwave.h"
#include "differential_filter.h"
#include "grid_anisotropy_tensor.h"
#include "mass.h"
#include "monitor_cfl.h"
#include "monitor_totalkineticenergy.h"
#include "newtonian.h"
#include "setupgeo.h"
#include "sgs_dd_model.h"
#include "spanstats/turbulence.h"
#include "taylorgreen.h"
#include "velocity_gradient_projection.h"
#include "inverse_multiplicity.h"

#include <stddef.h>

#define EXPORT __attribute__((visibility("default")))
typedef const CeedScalar *const *In;
typedef CeedScalar *const       *Out;

EXPORT int ref_IFunction_Newtonian_Conserv(void *c, CeedInt Q, In in, Out out) { return IFunction_Newtonian_Conserv(c, Q, in, out); }
EXPORT int ref_IFunction_Newtonian_Prim(void *c, CeedInt Q, In in, Out out) { return IFunction_Newtonian_Prim(c, Q, in, out); }
EXPORT int ref_IFunction_Newtonian_Entropy(void *c, CeedInt Q, In in, Out out) { return IFunction_Newtonian_Entropy(c, Q, in, out); }
EXPORT int ref_IJacobian_Newtonian_Conserv(void *c, CeedInt Q, In in, Out out) { return IJacobian_Newtonian_Conserv(c, Q, in, out); }
EXPORT int ref_IJacobian_Newtonian_Prim(void *c, CeedInt Q, In in, Out out) { return IJacobian_Newtonian_Prim(c, Q, in, out); }
EXPORT int ref_IJacobian_Newtonian_Entropy(void *c, CeedInt Q, In in, Out out) { return IJacobian_Newtonian_Entropy(c, Q, in, out); }
EXPORT int ref_Setup(void *c, CeedInt Q, In in, Out out) { return Setup(c, Q, in, out); }
EXPORT int ref_RHSFunction_Newtonian(void *c, CeedInt Q, In in, Out out) { return RHSFunction_Newtonian(c, Q, in, out); }
EXPORT int ref_Mass_5(void *c, CeedInt Q, In in, Out out) { return Mass_5(c, Q, in, out); }
EXPORT int ref_MassFunction_Newtonian_Conserv(void *c, CeedInt Q, In in, Out out) { return MassFunction_Newtonian_Conserv(c, Q, in, out); }
EXPORT int ref_MonitorTotalKineticEnergy_Conserv(void *c, CeedInt Q, In in, Out out) { return MonitorTotalKineticEnergy_Conserv(c, Q, in, out); }
EXPORT int ref_ICsTaylorGreen(void *c, CeedInt Q, In in, Out out) { return ICsTaylorGreen(c, Q, in, out); }
EXPORT int ref_ICsNewtonianIG_Conserv(void *c, CeedInt Q, In in, Out out) { return ICsNewtonianIG_Conserv(c, Q, in, out); }
EXPORT int ref_ICsNewtonianIG_Prim(void *c, CeedInt Q, In in, Out out) { return ICsNewtonianIG_Prim(c, Q, in, out); }
EXPORT int ref_ICsNewtonianIG_Entropy(void *c, CeedInt Q, In in, Out out) { return ICsNewtonianIG_Entropy(c, Q, in, out); }
EXPORT int ref_IC_GaussianWave_Prim(void *c, CeedInt Q, In in, Out out) { return IC_GaussianWave_Prim(c, Q, in, out); }
EXPORT int ref_IC_GaussianWave_Entropy(void *c, CeedInt Q, In in, Out out) { return IC_GaussianWave_Entropy(c, Q, in, out); }
EXPORT int ref_MonitorCFL_3D_Conserv(void *c, CeedInt Q, In in, Out out) { return MonitorCFL_3D_Conserv(c, Q, in, out); }
EXPORT int ref_MonitorCFL_3D_Prim(void *c, CeedInt Q, In in, Out out) { return MonitorCFL_3D_Prim(c, Q, in, out); }
EXPORT int ref_MonitorCFL_3D_Entropy(void *c, CeedInt Q, In in, Out out) { return MonitorCFL_3D_Entropy(c, Q, in, out); }
EXPORT int ref_MonitorTotalKineticEnergy_Prim(void *c, CeedInt Q, In in, Out out) { return MonitorTotalKineticEnergy_Prim(c, Q, in, out); }
EXPORT int ref_MonitorTotalKineticEnergy_Entropy(void *c, CeedInt Q, In in, Out out) { return MonitorTotalKineticEnergy_Entropy(c, Q, in, out); }
EXPORT int ref_ICsChannel(void *c, CeedInt Q, In in, Out out) { return ICsChannel(c, Q, in, out); }
EXPORT size_t ref_channel_ctx_size(void) { return sizeof(struct ChannelContext_); }
EXPORT int ref_IC_GaussianWave_Conserv(void *c, CeedInt Q, In in, Out out) { return IC_GaussianWave_Conserv(c, Q, in, out); }
EXPORT size_t ref_gaussianwave_ctx_size(void) { return sizeof(struct GaussianWaveContext_); }
EXPORT int ref_ChildStatsCollection_Conserv(void *c, CeedInt Q, In in, Out out) { return ChildStatsCollection_Conserv(c, Q, in, out); }
EXPORT int ref_ChildStatsCollection_Prim(void *c, CeedInt Q, In in, Out out) { return ChildStatsCollection_Prim(c, Q, in, out); }
EXPORT int ref_ChildStatsCollection_Entropy(void *c, CeedInt Q, In in, Out out) { return ChildStatsCollection_Entropy(c, Q, in, out); }
EXPORT size_t ref_turb_spanstats_ctx_size(void) { return sizeof(struct Turbulence_SpanStatsContext_); }

/* State helpers: q (5) in state_var -> U (5) and Y (5); forward-mode tangents. */
EXPORT void ref_StateFromQ(const NewtonianIGProperties *gas, const CeedScalar q[5], int state_var, CeedScalar U[5], CeedScalar Y[5]) {
  State s = StateFromQ(*gas, q, (StateVariable)state_var);
  UnpackState_U(s.U, U);
  UnpackState_Y(s.Y, Y);
}
EXPORT void ref_StateFromQ_fwd(const NewtonianIGProperties *gas, const CeedScalar q[5], const CeedScalar dq[5], int state_var, CeedScalar dU[5],
                               CeedScalar dY[5]) {
  State s  = StateFromQ(*gas, q, (StateVariable)state_var);
  State ds = StateFromQ_fwd(*gas, s, dq, (StateVariable)state_var);
  UnpackState_U(ds.U, dU);
  UnpackState_Y(ds.Y, dY);
}
EXPORT void ref_StateToQ(const NewtonianIGProperties *gas, const CeedScalar qa[5], int var_a, int var_b, CeedScalar qb[5]) {
  State s = StateFromQ(*gas, qa, (StateVariable)var_a);
  StateToQ(*gas, s, qb, (StateVariable)var_b);
}
EXPORT void ref_StateToQ_fwd(const NewtonianIGProperties *gas, const CeedScalar qa[5], const CeedScalar dqa[5], int var_a, int var_b,
                             CeedScalar dqb[5]) {
  State s  = StateFromQ(*gas, qa, (StateVariable)var_a);
  State ds = StateFromQ_fwd(*gas, s, dqa, (StateVariable)var_a);
  StateToQ_fwd(*gas, s, ds, dqb, (StateVariable)var_b);
}
EXPORT int ref_context_size(void) { return (int)sizeof(struct NewtonianIdealGasContext_); }
EXPORT int ref_setup_context_size(void) { return (int)sizeof(struct SetupContext_); }

/* Data-driven SGS closure and its training data (sgs_dd_model.h, sgs_dd_training.h, grid_anisotropy_tensor.h) and the
 * differential filter (differential_filter.h). */
EXPORT int ref_ComputeSgsDDNodal_Conserv(void *c, CeedInt Q, In in, Out out) { return ComputeSgsDDNodal_Conserv(c, Q, in, out); }
EXPORT int ref_AnisotropyTensorCollocate(void *c, CeedInt Q, In in, Out out) { return AnisotropyTensorCollocate(c, Q, in, out); }
EXPORT int ref_IFunction_NodalSgs_Conserv(void *c, CeedInt Q, In in, Out out) { return IFunction_NodalSgs_Conserv(c, Q, in, out); }
EXPORT int ref_IFunction_NodalSgs_Prim(void *c, CeedInt Q, In in, Out out) { return IFunction_NodalSgs_Prim(c, Q, in, out); }
EXPORT int ref_IFunction_NodalSgs_Entropy(void *c, CeedInt Q, In in, Out out) { return IFunction_NodalSgs_Entropy(c, Q, in, out); }
EXPORT int ref_ComputeSgsDDNodal_Prim(void *c, CeedInt Q, In in, Out out) { return ComputeSgsDDNodal_Prim(c, Q, in, out); }
EXPORT int ref_ComputeSgsDDNodal_Entropy(void *c, CeedInt Q, In in, Out out) { return ComputeSgsDDNodal_Entropy(c, Q, in, out); }
EXPORT int ref_AnisotropyTensorProjection(void *c, CeedInt Q, In in, Out out) { return AnisotropyTensorProjection(c, Q, in, out); }
EXPORT int ref_InverseMultiplicity(void *c, CeedInt Q, In in, Out out) { return InverseMultiplicity(c, Q, in, out); }
EXPORT int ref_VelocityGradientProjectionRHS_Conserv(void *c, CeedInt Q, In in, Out out) { return VelocityGradientProjectionRHS_Conserv(c, Q, in, out); }
EXPORT int ref_VelocityGradientProjectionRHS_Prim(void *c, CeedInt Q, In in, Out out) { return VelocityGradientProjectionRHS_Prim(c, Q, in, out); }
EXPORT int ref_VelocityGradientProjectionRHS_Entropy(void *c, CeedInt Q, In in, Out out) { return VelocityGradientProjectionRHS_Entropy(c, Q, in, out); }
EXPORT int ref_Mass_7(void *c, CeedInt Q, In in, Out out) { return Mass_7(c, Q, in, out); }
EXPORT int ref_Mass_9(void *c, CeedInt Q, In in, Out out) { return Mass_9(c, Q, in, out); }
EXPORT int ref_DifferentialFilter_RHS_Conserv(void *c, CeedInt Q, In in, Out out) { return DifferentialFilter_RHS_Conserv(c, Q, in, out); }
EXPORT int ref_DifferentialFilter_RHS_Prim(void *c, CeedInt Q, In in, Out out) { return DifferentialFilter_RHS_Prim(c, Q, in, out); }
EXPORT int ref_DifferentialFilter_RHS_Entropy(void *c, CeedInt Q, In in, Out out) { return DifferentialFilter_RHS_Entropy(c, Q, in, out); }
EXPORT int ref_DifferentialFilter_LHS_11(void *c, CeedInt Q, In in, Out out) { return DifferentialFilter_LHS_11(c, Q, in, out); }
EXPORT int ref_DifferentialFilter_LHS_1(void *c, CeedInt Q, In in, Out out) { return DifferentialFilter_LHS_1(c, Q, in, out); }
/* ComputeSgsDDInputs / ComputeSgsDDOutputs / DataDrivenInference on single points */
EXPORT void ref_ComputeSgsDDInputs(const CeedScalar grad_velo[3][3], const CeedScalar km_A_ij[6], CeedScalar delta, CeedScalar nu,
                                   CeedScalar evec[3][3], CeedScalar inputs[6], CeedScalar *gmag) {
  ComputeSgsDDInputs(grad_velo, km_A_ij, delta, nu, evec, inputs, gmag);
}
EXPORT void ref_ComputeSgsDDOutputs(CeedScalar outputs[6], CeedScalar delta, const CeedScalar evec[3][3], const CeedScalar bounds[6][2],
                                    CeedScalar gmag, CeedScalar km_sgs[6]) {
  ComputeSgsDDOutputs(outputs, delta, evec, bounds, gmag, km_sgs);
}
EXPORT void ref_DataDrivenInference(const CeedScalar *inputs, CeedScalar *outputs, void *ctx) { DataDrivenInference(inputs, outputs, ctx); }
EXPORT int  ref_Diagonalize3(CeedScalar A[3][3], CeedScalar eval[3], CeedScalar evec[3][3], int sweeps) {
  CeedInt work[3] = {0};
  return Diagonalize3(A, eval, evec, work, SORT_DECREASING_EVALS, true, sweeps);
}
/* struct layouts the tests build contexts with: {sizeof, offsetof(newt_ctx), offsetof(offsets), offsetof(data)} */
EXPORT void ref_sgs_dd_ctx_layout(size_t out[4]) {
  out[0] = sizeof(struct SgsDDContext_);
  out[1] = offsetof(struct SgsDDContext_, newt_ctx);
  out[2] = offsetof(struct SgsDDContext_, offsets);
  out[3] = offsetof(struct SgsDDContext_, data);
}
EXPORT void ref_diff_filter_ctx_layout(size_t out[4]) {
  out[0] = sizeof(struct DifferentialFilterContext_);
  out[1] = offsetof(struct DifferentialFilterContext_, newt_ctx);
  out[2] = offsetof(struct DifferentialFilterContext_, kernel_scaling);
  out[3] = offsetof(struct DifferentialFilterContext_, damping_function);
}

/* Free-stream boundary condition (bc_freestream.h) and face geometric factors (setupgeo.h:SetupBoundary). */
EXPORT int ref_Freestream_Conserv_HLL(void *c, CeedInt Q, In in, Out out) { return Freestream_Conserv_HLL(c, Q, in, out); }
EXPORT int ref_Freestream_Conserv_HLLC(void *c, CeedInt Q, In in, Out out) { return Freestream_Conserv_HLLC(c, Q, in, out); }
EXPORT int ref_Freestream_Jacobian_Conserv_HLL(void *c, CeedInt Q, In in, Out out) { return Freestream_Jacobian_Conserv_HLL(c, Q, in, out); }
EXPORT int ref_Freestream_Jacobian_Conserv_HLLC(void *c, CeedInt Q, In in, Out out) { return Freestream_Jacobian_Conserv_HLLC(c, Q, in, out); }
EXPORT int ref_Freestream_Prim_HLLC(void *c, CeedInt Q, In in, Out out) { return Freestream_Prim_HLLC(c, Q, in, out); }
EXPORT int ref_Freestream_Entropy_HLL(void *c, CeedInt Q, In in, Out out) { return Freestream_Entropy_HLL(c, Q, in, out); }
EXPORT int ref_Freestream_Jacobian_Prim_HLLC(void *c, CeedInt Q, In in, Out out) { return Freestream_Jacobian_Prim_HLLC(c, Q, in, out); }
EXPORT int ref_Freestream_Jacobian_Entropy_HLL(void *c, CeedInt Q, In in, Out out) { return Freestream_Jacobian_Entropy_HLL(c, Q, in, out); }
EXPORT int ref_SetupBoundary(void *c, CeedInt Q, In in, Out out) { return SetupBoundary(c, Q, in, out); }
EXPORT int ref_freestream_ctx_size(void) { return (int)sizeof(struct FreestreamContext_); }
