/* honee_b200_types.h -- QFunction context structs shared by the host library, the CUDA kernels and the oracle.
 *
 * The byte layout of every struct here must equal the reference's, because HONEE hands the context to libCEED as an
 * opaque blob (CeedQFunctionContextSetData with sizeof(*ctx), problems/newtonian.c:744-745) and updates fields by
 * byte offset (CeedQFunctionContextRegisterDouble with offsetof(...), problems/newtonian.c:747-753).  The static
 * asserts at the bottom pin the sizes and the registered offsets.
 *
 * Field names and order follow qfunctions/newtonian_types.h:20-75 and qfunctions/stabilization_types.h:6-38.
 */
#ifndef HONEE_B200_TYPES_H
#define HONEE_B200_TYPES_H

#ifdef __cplusplus
#include <cstddef>
#include <cstdint>
#else
#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* qfunctions/newtonian_types.h:11-15 */
typedef enum {
  HB_STATEVAR_CONSERVATIVE = 0,
  HB_STATEVAR_PRIMITIVE    = 1,
  HB_STATEVAR_ENTROPY      = 2,
} HbStateVariable;

/* qfunctions/stabilization_types.h:6-10 */
typedef enum {
  HB_STAB_NONE = 0,
  HB_STAB_SU   = 1,
  HB_STAB_SUPG = 2,
} HbStabilizationType;

/* qfunctions/stabilization_types.h:24-28 */
typedef enum {
  HB_DIV_DIFF_FLUX_PROJ_NONE     = 0,
  HB_DIV_DIFF_FLUX_PROJ_DIRECT   = 1,
  HB_DIV_DIFF_FLUX_PROJ_INDIRECT = 2,
} HbDivDiffFluxProjectionMethod;

/* qfunctions/stabilization_types.h:32-38 */
typedef struct {
  double Ctau_t;
  double Ctau_v;
  double Ctau_C;
  double Ctau_M;
  double Ctau_E;
} HbTauDiagCoefficients;

/* qfunctions/newtonian_types.h:20-26 */
typedef struct {
  double lambda;
  double mu;
  double k;
  double cv;
  double cp;
} HbGasProperties;

/* qfunctions/newtonian_types.h:28-47 (struct NewtonianIdealGasContext_, 184 bytes) */
typedef struct HbNewtonianContext {
  HbGasProperties               gas;
  double                        g[3];
  double                        time;
  double                        ijacobian_time_shift;
  bool                          is_implicit;
  HbStateVariable               state_var;
  HbStabilizationType           stabilization;
  bool                          idl_enable;
  double                        idl_pressure;
  double                        idl_amplitude;
  double                        idl_start;
  double                        idl_length;
  HbTauDiagCoefficients         tau_coeffs;
  double                        dt;
  HbDivDiffFluxProjectionMethod divFdiff_method;
} HbNewtonianContext;

/* qfunctions/newtonian_types.h:49-54 */
typedef struct {
  double pressure;
  double velocity[3];
  double temperature;
} HbStatePrimitive;

/* qfunctions/newtonian_types.h:61-64 */
typedef struct {
  HbStatePrimitive wall;
  double           height;
} HbICBoundaryLayer;

/* qfunctions/newtonian_types.h:66-75 (struct SetupContext_, 304 bytes) */
typedef struct {
  HbStatePrimitive   reference;
  HbICBoundaryLayer  ic_boundary_layer;
  HbNewtonianContext newt_ctx;
  double             lx, ly, lz;
  double             time;
} HbSetupContext;

/* qfunctions/taylorgreen.h:12-20 */
typedef struct {
  HbStatePrimitive   reference;
  HbNewtonianContext newt_ctx;
  double             lx, ly, lz;
  double             u[3];
} HbTaylorGreenContext;

/* qfunctions/newtonian_state.h:11-22 (State: conservative then primitive values, 80 bytes) */
typedef struct {
  double density, momentum[3], E_total;
  HbStatePrimitive Y;
} HbState;

/* qfunctions/channel.h:12-21 (struct ChannelContext_, 240 bytes) */
typedef struct {
  bool               implicit;
  double             theta0, P0, umax, center, H, B;
  HbNewtonianContext newt_ctx;
} HbChannelContext;

/* qfunctions/gaussianwave.h:11-18 (struct GaussianWaveContext_, 304 bytes) */
typedef struct {
  double             epicenter[3];
  double             width;
  double             amplitude;
  HbState            S_infty;
  HbNewtonianContext newt_ctx;
} HbGaussianWaveContext;

/* qfunctions/sgs_dd_model.h:16-31 (struct SgsDDContext_, 264 bytes with one data entry): the network's shape, the leaky
 * ReLU slope, the Newtonian context, the offsets (in doubles) of the biases, weights and output bounds inside data[],
 * the total size in bytes of the context with its data (problems/sgs_dd_model.c:605-620). */
typedef struct {
  int32_t            num_inputs, num_outputs;
  int32_t            num_layers;
  int32_t            num_neurons;
  double             alpha;
  HbNewtonianContext newt_ctx;
  struct {
    size_t bias1, bias2;
    size_t weight1, weight2;
    size_t out_scaling;
  } offsets;
  size_t total_bytes;
  double data[1];
} HbSgsDDContext;

/* Number of stored Jacobian components per quadrature point: q (5), Kelvin-Mandel strain rate (6), diagonal tau (3),
 * plus the IDL ramp coefficient when enabled (problems/newtonian.c:756-757; qfunctions/newtonian.h:251-254). */
#define HB_JAC_DATA_COMPS 14
#define HB_JAC_DATA_COMPS_IDL 15
/* Volume qdata per quadrature point: w*detJ and the 3x3 inverse mapping Jacobian (qfunctions/setupgeo.h:42-56). */
#define HB_QDATA_COMPS 10

#ifdef __cplusplus
}
#define HB_STATIC_ASSERT static_assert
#else
#define HB_STATIC_ASSERT _Static_assert
#endif

HB_STATIC_ASSERT(sizeof(HbNewtonianContext) == 184, "NewtonianIdealGasContext_ layout");
HB_STATIC_ASSERT(offsetof(HbNewtonianContext, time) == 64, "solution time offset");
HB_STATIC_ASSERT(offsetof(HbNewtonianContext, ijacobian_time_shift) == 72, "ijacobian time shift offset");
HB_STATIC_ASSERT(offsetof(HbNewtonianContext, dt) == 168, "timestep size offset");
HB_STATIC_ASSERT(sizeof(HbSetupContext) == 304, "SetupContext_ layout");
HB_STATIC_ASSERT(sizeof(HbTaylorGreenContext) == 272, "TaylorGreenContext_ layout");
HB_STATIC_ASSERT(sizeof(HbState) == 80, "State layout");
HB_STATIC_ASSERT(sizeof(HbChannelContext) == 240, "ChannelContext_ layout");
HB_STATIC_ASSERT(offsetof(HbChannelContext, newt_ctx) == 56, "ChannelContext_ newt_ctx offset");
HB_STATIC_ASSERT(sizeof(HbGaussianWaveContext) == 304, "GaussianWaveContext_ layout");
HB_STATIC_ASSERT(offsetof(HbGaussianWaveContext, newt_ctx) == 120, "GaussianWaveContext_ newt_ctx offset");
HB_STATIC_ASSERT(sizeof(HbSgsDDContext) == 264, "SgsDDContext_ layout");
HB_STATIC_ASSERT(offsetof(HbSgsDDContext, newt_ctx) == 24, "SgsDDContext_ newt_ctx offset");
HB_STATIC_ASSERT(offsetof(HbSgsDDContext, offsets) == 208, "SgsDDContext_ offsets offset");
HB_STATIC_ASSERT(offsetof(HbSgsDDContext, data) == 256, "SgsDDContext_ data offset");

#endif
