/* ref_qfunctions.c -- exports the reference's own QFunctions, compiled unchanged, for the oracle checks
 * (TEST INFRASTRUCTURE ONLY).
 *
 * Built by oracle/Makefile with -I pointing at the reference's qfunctions/ directory and at oracle/ref_shim, into
 * oracle/_ref/libhonee_ref.so.  Nothing of the reference is copied: this file only includes its headers and gives
 * each QFunction / state helper an exported name so the tests can call it through ctypes and compare it with the
 * oracle restatement (oracle/honee_oracle.c) and with the CUDA kernels.
 */
#include <ceed/types.h>

#include "monitor_totalkineticenergy.h"
#include "newtonian.h"
#include "setupgeo.h"
#include "taylorgreen.h"

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
EXPORT int ref_MonitorTotalKineticEnergy_Conserv(void *c, CeedInt Q, In in, Out out) { return MonitorTotalKineticEnergy_Conserv(c, Q, in, out); }
EXPORT int ref_ICsTaylorGreen(void *c, CeedInt Q, In in, Out out) { return ICsTaylorGreen(c, Q, in, out); }

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
