/* honee_b200.h -- kernel-level C ABI of the B200 Newtonian operator backend.
 *
 * Plain pointers and sizes, no CUDA or torch types: device pointers are `double *` / `float *` allocated by the caller
 * (or by the libCEED-compatible layer in ceed_b200.c), streams are passed as `void *` (a cudaStream_t, NULL = legacy
 * default stream).  Every call is asynchronous on that stream.
 *
 * This is the layer the libCEED API of include/ceed/ceed.h dispatches to once it has recognised the HONEE operators;
 * it is also exported so a caller that manages its own device memory (a solver, a test, the benchmark) can drive the
 * fused kernels directly.  Each entry names the reference call it serves.
 */
#ifndef HONEE_B200_H
#define HONEE_B200_H

#include <stddef.h>
#include <stdint.h>

#include "honee_b200_types.h"

#ifdef __cplusplus
extern "C" {
#endif

#define HB_EXPORT __attribute__((visibility("default")))

/* Status codes (0 = success; the values match libCEED's CEED_ERROR_* where they overlap). */
enum {
  HB_SUCCESS           = 0,
  HB_ERROR_MINOR       = 1,
  HB_ERROR_DIMENSION   = 2,
  HB_ERROR_INCOMPLETE  = 3,
  HB_ERROR_INCOMPATIBLE = 4,
  HB_ERROR_ACCESS      = 5,
  HB_ERROR_MAJOR       = -1,
  HB_ERROR_BACKEND     = -2,
  HB_ERROR_UNSUPPORTED = -3,
  HB_ERROR_INVALID     = -4,
  HB_ERROR_CUDA        = -5,
  HB_ERROR_NOMEM       = -6,
};

#define HB_MAX_P 8

/* Device-resident description of one H1 element operator on a hex mesh: restriction offsets (int32, one per element
 * node, pointing at component 0 of a node-interleaved 5-component L-vector, comp_stride 1), an element colouring in
 * which no two elements of one colour share an L-vector entry, and the 1D tensor basis.
 * Replaces what libCEED builds from CeedElemRestrictionCreate (src/dm-utils.c:83-137) and CeedBasisCreateTensorH1
 * (src/dm-utils.c:766-879). */
typedef struct HbElemOp {
  int            num_elem, P, Q;
  int64_t        l_size;        /* entries of the L-vector (5 * nodes) */
  int32_t       *d_offsets;     /* device [num_elem][P^3] */
  int            num_colors;
  int32_t       *h_color_ptr;   /* host CSR pointer [num_colors + 1] */
  int32_t       *d_color_elem;  /* device element ids grouped by colour */
  double         interp1d[HB_MAX_P * HB_MAX_P];   /* [Q][P] */
  double         grad1d[HB_MAX_P * HB_MAX_P];     /* [Q][P] */
  double         colo_grad1d[HB_MAX_P * HB_MAX_P];/* [Q][Q] derivative on the quadrature points: grad1d = colo * interp1d */
  double         qref1d[HB_MAX_P], qweight1d[HB_MAX_P];
  double        *d_x_elem;      /* device [num_elem][3][8] vertex coordinates (only needed with the IDL), may be NULL */
  int            num_sms;
  int            device;
  int           *d_status;      /* device error word written by the kernels (bit 0: a bounded wait gave up) */
} HbElemOp;

/* Build the device description from host arrays.  Validates every offset against l_size (bounds are checked on the
 * host once, so the kernels need no per-access checks), colours the elements greedily and uploads. */
HB_EXPORT int hb_elemop_create(int num_elem, int P, int Q, const int32_t *offsets, int64_t l_size, const double *interp1d, const double *grad1d,
                     const double *qref1d, const double *qweight1d, HbElemOp **op);
/* Attach trilinear vertex coordinates [num_elem][3][8] (host pointer) used by the internal damping layer. */
HB_EXPORT int hb_elemop_set_vertex_coords(HbElemOp *op, const double *x_elem);
HB_EXPORT int hb_elemop_destroy(HbElemOp *op);
/* Read (synchronising the device) and optionally clear the kernels' error word.  The fused kernels never trap: a wait
 * that gives up records bit 0 here and the kernel returns early, leaving its output incomplete. */
HB_EXPORT int hb_elemop_status(HbElemOp *op, int *status, int clear);

/* Inputs/outputs of one IFunction apply (device pointers). */
typedef struct {
  const double *q, *q_dot; /* L-vectors */
  const double *qdata;     /* [num_elem][10][Q^3] */
  double       *jac_data;  /* [num_elem][14 or 15][Q^3] FP64 stored values, may be NULL */
  float        *jac_data_f32; /* same layout in FP32 for the mixed-precision Jacobian, may be NULL */
  double       *v;         /* L-vector output */
  int           add;       /* 0: v = F(q), 1: v += F(q) */
} HbIFunctionIO;

/* Fused IFunction_Newtonian_Conserv / _Prim / _Entropy operator, the variable taken from the context's state_var
 * (qfunctions/newtonian.h:205-269 inside the volume operator of src/setuplibceed.c:209-243), called where HONEE calls
 * CeedOperatorApply(op_ifunction) (src/setupts.c:109).  Primitive and entropy variables for degree 1-3. */
HB_EXPORT int hb_ifunction_apply(const HbElemOp *op, const void *ctx184, const HbIFunctionIO *io, void *stream);

/* Fused IJacobian_Newtonian_Conserv / _Prim / _Entropy action (qfunctions/newtonian.h:272-323, operator src/setuplibceed.c:245-269),
 * called where MatMult_Ceed calls CeedOperatorApplyAdd (src/mat-ceed.c:1669).  FP64 and FP32 variants; the FP32 one
 * reads the FP32 shadow of jac_data and FP32 L-vectors, qdata stays FP64 and is rounded on load. */
HB_EXPORT int hb_ijacobian_apply_f64(const HbElemOp *op, const void *ctx184, const double *qdata, const double *jac_data, const double *dq, double *v,
                           int add, void *stream);
HB_EXPORT int hb_ijacobian_apply_f32(const HbElemOp *op, const void *ctx184, const double *qdata, const float *jac_data, const float *dq, float *v,
                           int add, void *stream);

/* Point-wise diagonal of the IJacobian operator, where MatGetDiagonal_Ceed calls CeedOperatorLinearAssembleDiagonal
 * (src/mat-ceed.c:1603-1630). */
HB_EXPORT int hb_diagonal_assemble_f64(const HbElemOp *op, const void *ctx184, const double *qdata, const double *jac_data, double *diag, int add,
                             void *stream);
HB_EXPORT int hb_diagonal_assemble_f32(const HbElemOp *op, const void *ctx184, const double *qdata, const float *jac_data, float *diag, int add,
                             void *stream);
/* Point-block diagonal of the IJacobian operator (CeedOperatorLinearAssemblePointBlockDiagonal, what MatCEED assembles for
 * -pc_type vpbjacobi, src/mat-ceed.c:76-153): out[(node * 5 + i) * 5 + j] (+)= dv_(node,i) / ddq_(node,j), a row-major
 * 5 x 5 block per node of the node-interleaved L-vector; out holds 5 * l_size values. */
HB_EXPORT int hb_point_block_diagonal_f64(const HbElemOp *op, const void *ctx184, const double *qdata, const double *jac_data, double *out, int add,
                                          void *stream);
HB_EXPORT int hb_point_block_diagonal_f32(const HbElemOp *op, const void *ctx184, const double *qdata, const float *jac_data, float *out, int add,
                                          void *stream);

/* Geometric factors of the Setup QFunction (qfunctions/setupgeo.h:42-56; driven by QDataGet, src/qdata.c:133-190) from
 * trilinear vertex coordinates x_elem [num_elem][3][8] (device) with the Gauss rule qref1d/qweight1d (host). */
HB_EXPORT int hb_setup_qdata(int num_elem, int Q, const double *qref1d, const double *qweight1d, const double *x_elem, double *qdata, void *stream);

/* Device vector helpers used by the libCEED layer and the Newton-Krylov driver (asynchronous on `s`, except the
 * reductions, which synchronise `s` and return the value on the host; `scratch` is a device buffer of >= 1024 doubles;
 * reduce type 0: sum|x|, 1: sum x^2, 2: max|x|, 3: dot(x, y)). */
HB_EXPORT int hb_vec_set_f64(double *x, int64_t n, double v, void *s);
HB_EXPORT int hb_vec_set_f32(float *x, int64_t n, float v, void *s);
HB_EXPORT int hb_vec_scale_f64(double *x, int64_t n, double a, void *s);
HB_EXPORT int hb_vec_scale_f32(float *x, int64_t n, float a, void *s);
HB_EXPORT int hb_vec_axpy_f64(double *y, double a, const double *x, int64_t n, void *s);
HB_EXPORT int hb_vec_axpy_f32(float *y, float a, const float *x, int64_t n, void *s);
HB_EXPORT int hb_vec_axpby_f64(double *y, double a, double b, const double *x, int64_t n, void *s);
HB_EXPORT int hb_vec_axpby_f32(float *y, float a, float b, const float *x, int64_t n, void *s);
HB_EXPORT int hb_vec_pointwise_mult_f64(double *w, const double *x, const double *y, int64_t n, void *s);
HB_EXPORT int hb_vec_pointwise_mult_f32(float *w, const float *x, const float *y, int64_t n, void *s);
HB_EXPORT int hb_vec_reciprocal_f64(double *x, int64_t n, void *s);
HB_EXPORT int hb_vec_f64_to_f32(const double *x, float *y, int64_t n, int add, void *s);
HB_EXPORT int hb_vec_f32_to_f64(const float *x, double *y, int64_t n, int add, void *s);
/* type 0: sum|x|, 1: sum x^2, 2: max|x|, 3: dot(x, y); scratch: device buffer of >= 1024 doubles; synchronises s */
HB_EXPORT int hb_vec_reduce_f64(const double *x, const double *y, int64_t n, int type, double *scratch, double *result, void *s);
HB_EXPORT int hb_vec_reduce_f32(const float *x, const float *y, int64_t n, int type, double *scratch, double *result, void *s);

HB_EXPORT int hb_restrict_apply(int num_elem, int esize, int ncomp, int cstride, const int32_t *d_off, const int32_t *d_strides, const double *l, double *e,
                      void *s);
HB_EXPORT int hb_restrict_apply_t_csr(int64_t l_size, const int64_t *d_ptr, const int64_t *d_eidx, const double *e, double *l, void *s);
HB_EXPORT int hb_restrict_apply_t_strided(int num_elem, int esize, int ncomp, const int32_t *d_strides, const double *e, double *l, void *s);
HB_EXPORT int hb_basis_apply_generic(int num_elem, int ncomp, int dim, int P, int Q, int tmode, int emode, const double *d_B, const double *d_G,
                           const double *d_w, const double *u, double *v, void *s);

/* ---- Implicit time loop (the caller of the hot path; PETSc TSBDF + SNES + KSP GMRES + PCJacobi in HONEE,
 *      src/setupts.c:78-157, :333-480; src/mat-ceed.c:1603-1700) ---- */
#define HB_GMRES_MAX_BASIS 32

typedef struct {
  double dt;              /* time step */
  int    bdf_order;       /* 1 or 2 (the first step of BDF2 is BDF1, as TSBDF starts) */
  double newton_rtol, newton_atol;
  int    newton_max_it;
  double ksp_rtol;        /* GMRES relative tolerance */
  int    ksp_max_it, gmres_restart;
  int    pc_jacobi;       /* 1: Jacobi from the assembled diagonal (-pc_type jacobi), 2: point-block Jacobi on the 5 x 5 node
                             blocks (-pc_type vpbjacobi), 0: none */
  int    pc_every_newton; /* 0: diagonal once per time step (lagged), 1: every Newton iteration */
  int    jacobian_fp32;   /* mixed precision: FP32 Krylov basis, Jacobian action and diagonal; FP64 residual and update */
  int    cgs_refine;      /* 0: classical Gram-Schmidt once (PETSc default), 1: a second pass every iteration (CGS2) */
  int    sgs_lagged;      /* with a closure attached: 1 (default) evaluate it at the previous state, explicitly, so Newton
                             converges with the Newtonian Jacobian; 0 implicit (the Jacobian then omits its derivative) */
  int    jfnk;            /* 1: Krylov products by a forward difference of the full residual (closure included, implicit);
                             FP64 only; the Jacobi preconditioner stays the Newtonian diagonal */
} HbSolverOptions;

typedef struct {
  int    newton_its, ksp_its, converged_reason; /* 1 converged, -1 non-finite residual, -2 iteration limit,
                                                   -3 preconditioner set-up failed (a singular point block) */
  double res0, res_final, seconds;
} HbStepStats;

typedef struct HbTimeStepper HbTimeStepper;

HB_EXPORT void hb_solver_default_options(HbSolverOptions *o);
/* ctx184 is copied; its dt / ijacobian_time_shift / time fields are set every step like HONEE's context labels. */
HB_EXPORT int hb_ts_create(const HbElemOp *op, const void *ctx184, const double *d_qdata, const HbSolverOptions *opts, void *stream,
                           HbTimeStepper **ts);
HB_EXPORT int hb_ts_set_state(HbTimeStepper *ts, const double *d_q, double t);
HB_EXPORT int hb_ts_get_state(HbTimeStepper *ts, double *d_q, double *t);
HB_EXPORT int hb_ts_step(HbTimeStepper *ts, HbStepStats *stats);
HB_EXPORT const void *hb_ts_context(HbTimeStepper *ts);
HB_EXPORT int hb_ts_destroy(HbTimeStepper *ts);

/* ---- Explicit time loop (HONEE's -ts_type rk path: RHS_NS, src/setupts.c:31-75, with the mass-matrix KSP of
 *      CreateKSPMass, src/setuplibceed.c:15-93; PETSc TSRK and KSP restated here) ---- */

/* Mass operator (Mass_N, N = 5: qfunctions/mass.h:19-26) on the state restriction and basis: v (+)= M u, and its
 * diagonal (what MatGetDiagonal_Ceed gives PCJacobi "diagonal"; the row sums of PCJacobi "rowsum" are M applied to ones). */
HB_EXPORT int hb_mass_apply(const HbElemOp *op, const double *qdata, const double *u, double *v, int add, void *stream);
HB_EXPORT int hb_mass_diagonal(const HbElemOp *op, const double *qdata, double *diag, int add, void *stream);
/* The SUPG-stabilized mass HONEE uses instead when stab = supg and the run is explicit (MassFunction_Newtonian,
 * qfunctions/newtonian.h:44-86; problems/newtonian.c:212-265, 795), at the state q_state: v (+)= M_stab u, with
 * v = wdetJ u and grad v = wdetJ dXdx stab(u) (the SUPG term of the rate, tau from q_state); and its diagonal. */
HB_EXPORT int hb_mass_stab_apply(const HbElemOp *op, const void *ctx184, const double *qdata, const double *q_state, const double *u, double *v,
                                 int add, void *stream);
HB_EXPORT int hb_mass_stab_diagonal(const HbElemOp *op, const void *ctx184, const double *qdata, const double *q_state, double *diag, int add,
                                    void *stream);
/* its point blocks (5 * l_size values, row-major 5 x 5 per node): the diagonal on each block's diagonal, zeros elsewhere */
HB_EXPORT int hb_mass_point_block_diagonal(const HbElemOp *op, const double *qdata, double *out, int add, void *stream);

#define HB_RK_MAX_STAGES 6
typedef struct {
  double dt;
  /* explicit Butcher tableau (TSRK): stages s <= HB_RK_MAX_STAGES, a row-major s x s (strictly lower), b, c */
  int    rk_stages;
  double rk_a[HB_RK_MAX_STAGES * HB_RK_MAX_STAGES], rk_b[HB_RK_MAX_STAGES], rk_c[HB_RK_MAX_STAGES];
  /* mass solve: 0 = "lumped" (KSPPREONLY + PCJacobi row sum, HONEE's default, src/setuplibceed.c:81-87),
   *             1 = KSPGMRES, left-preconditioned by PCJacobi, preconditioned residual norm (PETSc's GMRES defaults) */
  int    mass_ksp;
  int    mass_pc_rowsum; /* Jacobi from the row sums (1) or from the diagonal (0, -mass_pc_jacobi_type diagonal) */
  double mass_rtol, mass_atol;
  int    mass_max_it, mass_restart;
  int    mass_type; /* 0: as HONEE (the SUPG-stabilized mass MassFunction_Newtonian when stab = supg, else Mass_5), 1: Mass_5 */
} HbExplicitOptions;

typedef struct {
  int    mass_its;        /* Krylov iterations of the step's mass solves (0 when lumped) */
  int    converged_reason; /* 1 every mass solve converged, -1 non-finite, -2 iteration limit */
  double seconds;
} HbExplicitStats;

typedef struct HbExplicitStepper HbExplicitStepper;
struct HbFaceOp; /* boundary faces, declared below */

/* Classical 4-stage RK (TSRK4), lumped mass, PETSc's KSP defaults (rtol 1e-5, atol 1e-50, 10000 its, restart 30).  The
 * Jacobi preconditioner of the mass solve is set up at the first solve and kept, as PETSc keeps it (the MatCEED object never
 * changes state, so PCSetUp runs once): for the stabilized mass that is the state of the first right-hand side. */
HB_EXPORT void hb_explicit_default_options(HbExplicitOptions *o);
/* ctx184 is copied; "timestep size" and "solution time" are set per stage like RHS_NS does (src/setupts.c:40-46). */
HB_EXPORT int hb_explicit_create(const HbElemOp *op, const void *ctx184, const double *d_qdata, const HbExplicitOptions *opts, void *stream,
                                 HbExplicitStepper **ex);
HB_EXPORT int hb_explicit_set_state(HbExplicitStepper *ex, const double *d_q, double t);
HB_EXPORT int hb_explicit_get_state(HbExplicitStepper *ex, double *d_q, double *t);
/* G = M^-1 RHS(q) with RHS = RHSFunction_Newtonian (qfunctions/newtonian.h:133-202), the explicit right-hand side of
 * one call of RHS_NS; *its receives the mass-solve iterations and *converged_reason 1, -1 or -2 (either may be NULL). */
HB_EXPORT int hb_explicit_rhs(HbExplicitStepper *ex, const double *d_q, double t, double *d_g, int *its, int *converged_reason);
HB_EXPORT int hb_explicit_step(HbExplicitStepper *ex, HbExplicitStats *stats);
/* Essential DOFs (as hb_ts_set_essential): the state keeps their values, the right-hand side and the mass solve act on the
 * free DOFs only (RHS_NS after DMLocalToGlobal). */
HB_EXPORT int hb_explicit_set_essential(HbExplicitStepper *ex, const int32_t *h_idx, const double *h_val, int64_t n);
/* Free-stream faces in the explicit right-hand side (the reference's explicit Freestream QFunction contributes -wdetJb F,
 * bc_freestream.h:45-48); faces == NULL removes them. */
HB_EXPORT int hb_explicit_set_freestream(HbExplicitStepper *ex, const struct HbFaceOp *faces, const void *ctx264, int flux_type, const double *qdata_sur);
HB_EXPORT int hb_explicit_destroy(HbExplicitStepper *ex);

/* Krylov block operations (FP64 accumulation): out[i] = V_i . w for i < k (d_partial: 512*HB_GMRES_MAX_BASIS doubles),
 * w += sum_i c_i V_i */
HB_EXPORT int hb_krylov_multidot_f64(const double *V, int64_t ldv, int k, const double *w, int64_t n, double *d_partial, double *d_out, void *s);
HB_EXPORT int hb_krylov_multidot_f32(const float *V, int64_t ldv, int k, const float *w, int64_t n, double *d_partial, double *d_out, void *s);
/* hb_krylov_multidot_f64 that allocates nothing and takes no work buffer: the partial sums live in a fixed 128 KiB device
 * array inside this library (room for k <= HB_GMRES_MAX_BASIS; larger k returns HB_ERROR_INVALID, nothing launched).
 * No counterpart in the reference (PETSc's VecMDot owns its work space); it exists for callers that cannot hand over a
 * device buffer, such as a vector-library inner-product callback.  The first call on each device looks the array up (and
 * reads the block kernels' occupancy, which sizes their grids)
 * and belongs before any stream capture; calls that overlap on one device (different streams or host threads) race on
 * the shared array and must be serialised by the caller.  The looked-up address is kept per device ordinal for the life
 * of the process: after cudaDeviceReset (or any teardown of the device's primary context) the module is loaded anew and
 * the array may move, so this entry point must not be called on a device after its context was reset. */
HB_EXPORT int hb_krylov_multidot_f64_static(const double *V, int64_t ldv, int k, const double *w, int64_t n, double *d_out, void *s);
HB_EXPORT int hb_krylov_multiaxpy_f64(double *w, const double *V, int64_t ldv, int k, const double *c, int64_t n, void *s);
HB_EXPORT int hb_krylov_multiaxpy_f32(float *w, const float *V, int64_t ldv, int k, const double *c, int64_t n, void *s);
HB_EXPORT int hb_krylov_multiaxpy_f32_to_f64(double *w, const float *V, int64_t ldv, int k, const double *c, int64_t n, void *s);
/* w += sign * sum_{i<k} d_c[i] V_i with the k coefficients in device memory (e.g. a multi-dot's d_out, sign -1 for the
 * Gram-Schmidt step), so no host synchronisation separates the multi-dot and the update; FP64 sums as above. */
HB_EXPORT int hb_krylov_multiaxpy_dev_f64(double *w, const double *V, int64_t ldv, int k, const double *d_c, double sign, int64_t n, void *s);
HB_EXPORT int hb_krylov_multiaxpy_dev_f32(float *w, const float *V, int64_t ldv, int k, const double *d_c, double sign, int64_t n, void *s);
/* Point-block Jacobi (PCVPBJACOBI on 5 x 5 node blocks, row-major, as hb_point_block_diagonal_* writes them): invert every
 * block in FP64 with partial pivoting (inv may equal blocks for the FP64 form); blocks with a vanishing pivot become the
 * identity and are counted in *d_singular (a device int), copied to *h_singular when that is not NULL (synchronises s).
 * Apply: y = B^-1 x per node (x and y must differ). */
HB_EXPORT int hb_pb_invert_f64(const double *blocks, double *inv, int64_t nodes, int *d_singular, int *h_singular, void *s);
HB_EXPORT int hb_pb_invert_f64_to_f32(const double *blocks, float *inv, int64_t nodes, int *d_singular, int *h_singular, void *s);
HB_EXPORT int hb_pb_apply_f64(const double *inv, const double *x, double *y, int64_t nodes, void *s);
HB_EXPORT int hb_pb_apply_f32(const float *inv, const float *x, float *y, int64_t nodes, void *s);
/* Essential (Dirichlet) DOFs, given as indices idx[n] into the node-interleaved L-vector (node * 5 + component): x[idx[i]] =
 * val[i] (0 when val is NULL); hb_pb_constrain turns the constrained rows and columns of the 5 x 5 node blocks into those
 * of the identity, so a block preconditioner leaves constrained entries at zero. */
HB_EXPORT int hb_constrain_set_f64(double *x, const int32_t *idx, const double *val, int64_t n, void *s);
HB_EXPORT int hb_constrain_set_f32(float *x, const int32_t *idx, const double *val, int64_t n, void *s);
HB_EXPORT int hb_pb_constrain(double *blocks, const int32_t *idx, int64_t n, void *s);
HB_EXPORT int hb_bdf_qdot(const double *q, const double *z, double alpha, double *qdot, int64_t n, void *s);
HB_EXPORT int hb_vec_combine_f64(const double *q1, const double *q2, double a, double b, double *z, int64_t n, void *s);

/* Monitors (src/monitor_totalkineticenergy.c:134-163, src/monitor_cfl.c:140-164): kinetic-energy integrand sums (not divided
 * by the volume; d_scratch >= 5*num_elem doubles) and dt * min/max CFL (d_scratch >= 2*num_elem doubles).  Synchronise. */
HB_EXPORT int hb_monitor_ke(const HbElemOp *op, const void *ctx184, const double *q, const double *qdata, double *d_scratch, double sums[5], void *s);
/* The same integrands at every quadrature point, E-vector e_out [elem][5][Q^3] (the Ceed-bound MonitorTotalKineticEnergy_*
 * operator, src/monitor_totalkineticenergy.c:80-103, before VecStrideSum); and sqrt(u . g u) at every point, e_out
 * [elem][Q^3] (MonitorCFL_3D_*, src/monitor_cfl.c:100-110, before the min / max and the time-step factor).  Asynchronous. */
HB_EXPORT int hb_monitor_ke_points(const HbElemOp *op, const void *ctx184, const double *q, const double *qdata, double *e_out, void *s);
HB_EXPORT int hb_monitor_cfl_points(const HbElemOp *op, const void *ctx184, const double *q, const double *qdata, double *e_out, void *s);

/* ---- Nodal data-driven SGS pipeline (problems/sgs_dd_model.c:98-200, 508-560, 645-737; src/velocity_gradient_projection.c;
 *      src/grid_anisotropy_tensor.c; src/inverse_multiplicity.c).  Element operators take an HbElemOp whose offsets are
 *      node * 5 (the node numbering every field of the pipeline shares); node-interleaved L-vectors of nc fields are
 *      addressed [node][nc].  All outputs are added to. ---- */
/* v [node][9] += int phi wdetJ du_i/dx_j (row-major i, j) of the state q in state_var (VelocityGradientProjectionRHS_*,
 * qfunctions/velocity_gradient_projection.h:9-37). */
HB_EXPORT int hb_velocity_gradient_rhs(const HbElemOp *op, const void *ctx184, int state_var, const double *qdata, const double *q, double *v, void *s);
/* v [node][7] += int phi wdetJ (KM anisotropy tensor (6), delta) (AnisotropyTensorProjection, grid_anisotropy_tensor.h:35-55). */
HB_EXPORT int hb_anisotropy_rhs(const HbElemOp *op, const double *qdata, double *v, void *s);
/* v [node][nc] += M u, the mass matrix on nc fields (Mass_N, src/honee-mass.c:20-60); its diagonal, the same in every field. */
HB_EXPORT int hb_mass_n_apply(const HbElemOp *op, int nc, const double *qdata, const double *u, double *v, void *s);
HB_EXPORT int hb_mass_n_diagonal(const HbElemOp *op, int nc, const double *qdata, double *diag, void *s);
/* e_out[i] = 1 / mult[offsets[i]] for the n entries of an element vector (InverseMultiplicity, qfunctions/inverse_multiplicity.h). */
HB_EXPORT int hb_inverse_multiplicity(int64_t n, const int32_t *offsets, const double *mult, double *e_out, void *s);
/* w [node] += the entries of the element vector e_vec [elem][P^3] at that node (transposed restriction of one field). */
HB_EXPORT int hb_node_weight_sum(const HbElemOp *op, const double *e_vec, double *w, void *s);
/* km_sgs [node][6] += w [node] tau(node): the data-driven closure at every node with w != 0 (ComputeSgsDDNodal_*,
 * qfunctions/sgs_dd_model.h:69-96) from q [node][5] in state_var, the velocity gradient G [node][9] and the anisotropy
 * tensor with width A [node][7]; sgs_ctx is the SgsDDContext_ blob of ctx_bytes bytes (6-20-6 network, FP64 weights). */
HB_EXPORT int hb_sgs_nodal_closure(int64_t nodes, const void *sgs_ctx, size_t ctx_bytes, int state_var, const double *q, const double *G, const double *A,
                                   const double *w, double *km_sgs, void *s);
/* v [node][5] += int grad phi . (-wdetJ dXdx F_sgs), F_sgs the flux of the interpolated nodal stress km_sgs [node][6]
 * (IFunction_NodalSgs_*, qfunctions/sgs_dd_model.h:205-243). */
HB_EXPORT int hb_sgs_nodal_ifunction(const HbElemOp *op, const void *ctx184, int state_var, const double *qdata, const double *q, const double *km_sgs,
                                     double *v, void *s);
HB_EXPORT int hb_monitor_cfl(const HbElemOp *op, const void *ctx184, const double *q, const double *qdata, double dt, double *d_scratch,
                             double minmax[2], void *s);

/* ---- Learned subgrid-stress closure (the data-driven SGS model of qfunctions/sgs_dd_model.h, sgs_dd_utils.h,
 *      grid_anisotropy_tensor.h; problems/sgs_dd_model.c:561-737).  The reference evaluates a trained network; here the
 *      network is also trained on the GPU from filtered fine-grid data. ---- */
typedef struct {
  int   hidden1, hidden2;   /* hidden widths: 20, 20 (two layers) or 20, 0 (one layer, the reference's 6-20-6 form) */
  float leaky_alpha;        /* negative slope of the activation; 0 = ReLU (the reference default) */
  float out_bounds[6][2];   /* min-max bounds {lo, hi} that de-normalise the 6 outputs (OutScaling.dat) */
  int   clamp_outputs;      /* inference in the residual: 1 limits the normalised outputs to [0, 1] (the training range) */
  int   no_backscatter;     /* inference in the residual: 1 drops the deviatoric stress where it would feed energy to the
                               resolved scales (tau : S > 0); both 0 = the reference's evaluation */
} HbMlpDesc;

/* Parameter count of the network (W1, b1, [W2, b2,] W3, b3; W row-major [out][in]); negative: unsupported shape. */
HB_EXPORT int hb_mlp_num_params(const HbMlpDesc *d);
/* One training step, FP32: MSE over `batch` samples of X/Y ([n][6] each, device), drawn with replacement by a hash of
 * (seed, step) or taken from idx[batch] when idx is not NULL; then Adam (beta 0.9/0.999, eps 1e-8) at learning rate lr
 * on w with moments m, v (step is 1-based).  lr == 0: gradient only (d_grad receives it, w/m/v untouched).
 * d_work >= ceil(batch/256) * (num_params + 1) floats; d_loss[0] = the batch loss; d_grad (optional) = the gradient. */
HB_EXPORT int hb_mlp_train_step(const HbMlpDesc *d, float *w, float *m, float *v, const float *X, const float *Y, int64_t n, const int32_t *idx,
                                int batch, uint64_t seed, int step, float lr, float *d_work, float *d_loss, float *d_grad, void *s);
/* IFunction with the closure fused in at every quadrature point: hb_ifunction_apply plus the SGS flux of the network
 * (weights: host array of hb_mlp_num_params floats, copied into the launch; bounds and activation from d).  Built for
 * P, Q = (3, 3), (3, 4), (4, 5); the Jacobian operators do not include the closure (nor does the reference's). */
HB_EXPORT int hb_ifunction_apply_sgs(const HbElemOp *op, const void *ctx184, const HbIFunctionIO *io, const HbMlpDesc *d, const float *h_weights,
                                     void *stream);
/* Attach (or with d == NULL detach) the closure to a time stepper: its residual becomes hb_ifunction_apply_sgs with these
 * weights (copied); the Krylov Jacobian stays the Newtonian one. */
HB_EXPORT int hb_ts_set_sgs(HbTimeStepper *ts, const HbMlpDesc *d, const float *h_weights);
/* Batch inference Y = net(X), [n][6] FP32 on the device. */
HB_EXPORT int hb_mlp_forward(const HbMlpDesc *d, const float *w, const float *X, float *Y, int64_t n, void *s);
/* Point-wise maps (FP64, arrays of n points on the device): the anisotropy tensor (KM) and width from dXdx [n][9]; the
 * model inputs, eigenframe E [n][9] and |G A| from the velocity gradient G [n][9] (G[i][j] = du_i/dx_j), A, delta and
 * the kinematic viscosity; the physical stress (KM) from normalised outputs. */
HB_EXPORT int hb_sgs_anisotropy(int64_t n, const double *dXdx, double *kmA, double *delta, void *s);
HB_EXPORT int hb_sgs_inputs(int64_t n, const double *G, const double *kmA, const double *delta, const double *nu, double *inputs, double *E,
                            double *gmag, void *s);
HB_EXPORT int hb_sgs_stress(int64_t n, const double *out_n, const double *delta, const double *E, const double *gmag, const float bounds[12],
                            double *km_tau, void *s);
/* Column-wise min/max of training targets Y [n][6] (d_work >= 3072 floats; synchronises), and the min-max map to [0, 1]. */
HB_EXPORT int hb_sgs_target_bounds(const float *Y, int64_t n, float *d_work, float bounds[12], void *s);
HB_EXPORT int hb_sgs_normalize_targets(float *Y, int64_t n, const float bounds[12], void *s);

/* ---- Differential filter (src/differential_filter.c, qfunctions/differential_filter.h) and SGS training pairs ---- */
typedef struct {
  int    grid_based_width;  /* 1: width tensor from the element anisotropy tensor (-diff_filter_grid_based_width), 0: identity */
  double width_scaling[3];  /* -diff_filter_width_scaling (default 1, 1, 1) */
  double kernel_scaling;    /* -diff_filter_kernel_scaling (default 0.1) */
} HbFilterOptions;

/* y = (M + K_alpha) x for nc node-interleaved fields on the element operator's mesh (DifferentialFilter_LHS_N). */
HB_EXPORT int hb_filter_apply(const HbElemOp *op, int nc, const HbFilterOptions *o, const double *qdata, const double *x, double *y, void *s);
/* The operator's diagonal, one value per node (the same for every field), and its reciprocal expanded to nc fields. */
HB_EXPORT int hb_filter_diagonal(const HbElemOp *op, const HbFilterOptions *o, const double *qdata, double *diag, void *s);
HB_EXPORT int hb_filter_jacobi(const double *diag, int64_t nodes, int nc, double *dinv, void *s);
/* rhs [node][11] = int phi (P, u, T, uu_xx, uu_yy, uu_zz, uu_yz, uu_xz, uu_xy) of the conservative state q
 * (DifferentialFilter_RHS_Conserv). */
HB_EXPORT int hb_filter_rhs(const HbElemOp *op, const void *ctx184, const double *qdata, const double *q, double *rhs, void *s);
/* CG + point Jacobi to relative natural-norm tolerance rtol; work >= hb_filter_work_doubles(op, nc) doubles.  Returns
 * HB_ERROR_INCOMPLETE when max_it was reached. */
HB_EXPORT size_t hb_filter_work_doubles(const HbElemOp *op, int nc);
HB_EXPORT int hb_filter_solve(const HbElemOp *op, int nc, const HbFilterOptions *o, const double *qdata, const double *b, double *x, double rtol,
                              int max_it, double *work, int *its, double *rel_norm, void *s);
/* Conservative state [node][5] of filtered fields [node][11] (rho = P / (R T)), e.g. to monitor the filtered solution. */
HB_EXPORT int hb_filtered_state(const double *filtered, int64_t nodes, const void *ctx184, double *q, void *s);
/* Training pairs at every quadrature point (X: model inputs, Y: filtered stress in the model's output frame scaled by
 * delta^2 |G A|^2, [num_elem * Q^3][6] FP32) from filtered fields [node][11] (qfunctions/sgs_dd_training.h:22-56 with
 * the stress taken into the model frame); width_scale = filter width / this mesh's element width. */
HB_EXPORT int hb_sgs_training_pairs(const HbElemOp *op, const void *ctx184, const double *qdata, const double *filtered, double width_scale, float *X,
                                    float *Y, void *s);

/* ---- Free-stream boundary condition (qfunctions/bc_freestream.h, riemann_solver.h; problems/bc_freestream.c): the
 *      face sub-operators of the composite IFunction / IJacobian on the boundary faces of the mesh ---- */
typedef struct HbFaceOp {
  int      num_faces, P, Q;
  int64_t  l_size;
  int32_t *d_offsets;      /* device [num_faces][P^2], node * 5 of the volume L-vector, face-tensor order */
  int      num_colors;
  int32_t *h_color_ptr;    /* host [num_colors + 1] */
  int32_t *d_color_elem;   /* device face ids grouped by colour */
  double   interp1d[HB_MAX_P * HB_MAX_P], grad1d[HB_MAX_P * HB_MAX_P], qweight1d[HB_MAX_P];
  int      device;
} HbFaceOp;

/* FreestreamContext_ (qfunctions/bc_freestream_type.h): the Newtonian context and the exterior State (U then Y). */
typedef struct {
  HbNewtonianContext newt;
  double             S_infty_U[5]; /* rho, rho u (3), E */
  double             S_infty_Y[5]; /* P, u (3), T */
} HbFreestreamContext;

HB_EXPORT int hb_faceop_create(int num_faces, int P, int Q, const int32_t *offsets, int64_t l_size, const double *interp1d, const double *grad1d,
                               const double *qweight1d, HbFaceOp **op);
HB_EXPORT int hb_faceop_destroy(HbFaceOp *op);
/* Face geometric factors (SetupBoundary, setupgeo.h:100-117) [F][10][Q^2] from the face nodes' coordinates x_nodes
 * [F][3][P^2] (device): w detJb, unit normal, dX/dx (2 x 3).  The normal is the cross product of the two face tangents
 * in face-tensor order; the face node order decides its orientation (outward for the box faces of problem.py). */
HB_EXPORT int hb_face_setup_qdata(const HbFaceOp *op, const double *x_nodes, double *qdata_sur, void *s);
/* The same geometric factors for any face coordinate basis (P coordinate nodes per direction, e.g. the bilinear P = 2
 * field DMPlexCeedCoordinateCreateField gives HONEE's surface Setup operator, src/qdata.c:228-261): x_nodes [F][3][P^2]. */
HB_EXPORT int hb_face_setup_qdata_nodes(int num_faces, int P, int Q, const double *interp1d, const double *grad1d, const double *qweight1d,
                                        const double *x_nodes, double *qdata_sur, void *s);
/* v += int phi wdetJb F(q, S_infty, n), F = HLL (flux_type 0) or HLLC (1); jac_data_sur [F][5][Q^2] (may be NULL) = q at
 * the points (Freestream, bc_freestream.h:14-48). */
HB_EXPORT int hb_freestream_apply(const HbFaceOp *op, const void *ctx264, int flux_type, const double *qdata_sur, const double *q, double *jac_data_sur,
                                  double *v, void *s);
/* v += int phi wdetJb dF(q; dq) with the exterior state fixed (Freestream_Jacobian, bc_freestream.h:75-114). */
HB_EXPORT int hb_freestream_jacobian_apply(const HbFaceOp *op, const void *ctx264, int flux_type, const double *qdata_sur, const double *jac_data_sur,
                                           const double *dq, double *v, void *s);
/* diag += the diagonal of that Jacobian (what CeedOperatorLinearAssembleAddDiagonal gives for the Freestream_Jacobian
 * sub-operator): per face node p and component c, sum over points of B_p^2 wdetJb dF_c/dU_c. */
HB_EXPORT int hb_freestream_diagonal(const HbFaceOp *op, const void *ctx264, int flux_type, const double *qdata_sur, const double *jac_data_sur,
                                     double *diag, void *s);
/* out[(node * 5 + i) * 5 + j] += the 5 x 5 point block of that Jacobian (sum over points of B_p^2 wdetJb dF_i/dU_j) */
HB_EXPORT int hb_freestream_point_block_diagonal(const HbFaceOp *op, const void *ctx264, int flux_type, const double *qdata_sur,
                                                 const double *jac_data_sur, double *out, void *s);
/* the same with FP32 dq and v (state and flux math in FP64), for the mixed-precision Krylov solve */
HB_EXPORT int hb_freestream_jacobian_apply_f32(const HbFaceOp *op, const void *ctx264, int flux_type, const double *qdata_sur,
                                               const double *jac_data_sur, const float *dq, float *v, void *s);

/* Essential boundary conditions (strong Dirichlet values, as HONEE's bc_*_essential_comps / essential_values insert them
 * through DMPlexInsertBoundaryValues, src/setupts.c:16-25, with the DOFs removed from the global system): h_idx[n] L-vector
 * indices (node * 5 + component) and their values (NULL: zero).  The state takes the values, the rate is zero there, and
 * the residual, the Jacobian rows and the preconditioner act only on the free DOFs.  n = 0 removes them. */
HB_EXPORT int hb_ts_set_essential(HbTimeStepper *ts, const int32_t *h_idx, const double *h_val, int64_t n);
/* Attach (faces != NULL) or detach the free-stream boundary to a time stepper: its flux joins every residual, its
 * tangent every Krylov product (FP32 in mixed precision) and its diagonal the Jacobi preconditioner (FP64). */
HB_EXPORT int hb_ts_set_freestream(HbTimeStepper *ts, const HbFaceOp *faces, const void *ctx264, int flux_type, const double *qdata_sur);

/* ---- spanwise statistics of turbulence quantities ------------------------------------------------------------------
 * HONEE's -ts_monitor_spanstats_turbulence (src/spanstats/turbulence.c:152-278, src/spanstats/spanstats.c:343-470):
 * every step the 22 statistics of qfunctions/spanstats/turbulence.h:8-32 (mean density, pressure, pressure squared,
 * pressure-velocity, density-temperature and its fluxes, momentum, momentum fluxes, velocity), weighted by w detJ and by
 * the step's time increment, are summed over the span onto the quadrature points of the 2D parent plane; processing
 * divides by the duration and the span width, projects onto the parent nodes (B^T) and solves with the parent mass
 * matrix (CG, point Jacobi, natural norm), giving the time- and span-averaged fields [parent node][22]. */
#define HB_TURB_NUM_COMPONENTS 22

/* The parent plane: a 2D tensor-product mesh of P^2-node elements whose quadrature points carry the (x, y) of the
 * child elements' points (DMPlexFilter of the spanwise face, spanstats.c:42-112, with the same P and Q).  Offsets are
 * node indices into [num_nodes][22] vectors; colours as in HbElemOp. */
typedef struct HbPlaneOp {
  int            num_elem, P, Q;
  int64_t        num_nodes;
  int32_t       *d_offsets;     /* device [num_elem][P^2] */
  int            num_colors;
  int32_t       *h_color_ptr;
  int32_t       *d_color_elem;
  double         interp1d[HB_MAX_P * HB_MAX_P];
  double         qref1d[HB_MAX_P], qweight1d[HB_MAX_P];
  double        *d_wdetJ;       /* device [num_elem][Q^2] */
} HbPlaneOp;

/* Parent-point sums of one collection (ChildStatsCollection_Conserv applied and reduced over the span,
 * turbulence.c:19-108 + spanstats.c:425-443): sums[col][Q^2][22] += sum over the elements d_column_elems[col][*] and their
 * quadrature planes of w detJ * dt * stats(q).  Each column lists the 3D elements whose first two reference axes
 * coincide with those of parent element `col`.  q in the context's state variable (ChildStatsCollection_Conserv/_Prim/_Entropy). */
HB_EXPORT int hb_stats_collect(const HbElemOp *op, const void *ctx184, const double *q, const double *qdata, double dt, int num_columns,
                               int column_length, const int32_t *d_column_elems, double *sums, void *stream);
/* Parent mass matrix M (HoneeMassQFunctionCreate on the parent basis, spanstats.c:313-320), 22 components: v (+)= M u */
HB_EXPORT int hb_plane_mass_apply(const HbPlaneOp *pl, const double *u, double *v, int add, void *stream);
/* Its diagonal, one value per node (the same for all 22 components). */
HB_EXPORT int hb_plane_mass_diagonal(const HbPlaneOp *pl, double *diag, int add, void *stream);
/* Projection right-hand side v (+)= B^T (scale * sums) (the identity QFunction of spanstats.c:302-309). */
HB_EXPORT int hb_plane_project_rhs(const HbPlaneOp *pl, const double *sums, double scale, double *v, int add, void *stream);
/* w detJ of the parent points from the bilinear vertex coordinates x_plane [num_elem][3][4] (vertex a + 2b), as
 * Setup2D_3Dcoords (qfunctions/setupgeo2d.h:136-152) computes it: weight times |dx/dX0 x dx/dX1|.  Device pointers. */
HB_EXPORT int hb_plane_setup_qdata(int num_elem, int Q, const double *qref1d, const double *qweight1d, const double *x_plane, double *wdetJ,
                                   void *stream);

/* The statistics monitor: owns the parent plane, the columns, the sums and the projection work space. */
typedef struct HbSpanStats HbSpanStats;
/* op: the 3D operator (its P, Q and basis are the parent's); column_elems [num_columns][column_length] host element ids;
 * parent_offsets [num_columns][P^2] host parent-node indices (< num_parent_nodes); parent_x [num_columns][3][4] host
 * vertex coordinates; span_width the spanwise extent of the domain (spanstats.c:52-54). */
HB_EXPORT int hb_spanstats_create(const HbElemOp *op, int num_columns, int column_length, const int32_t *column_elems,
                                  const int32_t *parent_offsets, int64_t num_parent_nodes, const double *parent_x, double span_width,
                                  HbSpanStats **st);
/* Zero the sums and start a new averaging window at initial_time (SpanwiseStatisticsSetupFinalize, spanstats.c:371-389). */
HB_EXPORT int hb_spanstats_reset(HbSpanStats *st, double initial_time, void *stream);
/* One collection at solution_time (SpanwiseStatisticsCollect, spanstats.c:392-411): dt = solution_time - previous time. */
HB_EXPORT int hb_spanstats_collect(HbSpanStats *st, const void *ctx184, const double *q, const double *qdata, double solution_time, void *stream);
/* Device pointer to the parent-point sums [num_columns][Q^2][22] and the parent plane. */
HB_EXPORT int hb_spanstats_view(const HbSpanStats *st, const double **d_sums, const HbPlaneOp **plane);
/* Copy the sums into dst (host or device; synchronous). */
HB_EXPORT int hb_spanstats_copy_sums(const HbSpanStats *st, double *dst);
/* Processing at solution_time (SpanwiseStatisticsProcess, spanstats.c:414-458): stats [num_parent_nodes][22] (device)
 * solves M stats = B^T sums / ((solution_time - initial_time) * span_width); rtol as -ts_monitor_spanstats_turbulence_ksp_rtol
 * (default 1e-10).  HB_ERROR_INCOMPLETE when max_it iterations do not reach it. */
HB_EXPORT int hb_spanstats_process(HbSpanStats *st, double solution_time, double rtol, int max_it, double *stats, int *its, double *rel_norm,
                                   void *stream);
HB_EXPORT int hb_spanstats_destroy(HbSpanStats *st);

/* Initial condition at the solution nodes (SetupLibceed's op_ics, src/setuplibceed.c:143-175): one thread per node of
 * each element evaluates the coordinates through proj1d ([P_to][2], the 1D CeedBasisCreateProjection of the trilinear
 * coordinate basis onto the solution basis) from x_e ([elem][3][8] vertex coordinates) and the IC QFunction `kind` with
 * its context bytes (HbSetupContext, HbTaylorGreenContext, HbChannelContext or HbGaussianWaveContext; ctx_size checked),
 * writing q0_e [elem][5][P_to^3].  state_var: the QFunction's state variable for ICsNewtonianIG_* and IC_GaussianWave_*
 * (the Taylor-Green and channel ICs use their context's). */
#define HB_IC_NEWTONIAN 0     /* ICsNewtonianIG_{Conserv,Prim,Entropy}, qfunctions/newtonian.h:17-42 */
#define HB_IC_TAYLOR_GREEN 1  /* ICsTaylorGreen, qfunctions/taylorgreen.h:23-51 */
#define HB_IC_CHANNEL 2       /* ICsChannel, qfunctions/channel.h:58-73 */
#define HB_IC_GAUSSIAN_WAVE 3 /* IC_GaussianWave_{Conserv,Prim,Entropy}, qfunctions/gaussianwave.h:20-71 */
HB_EXPORT int hb_ics_apply(int kind, int state_var, const void *ctx, size_t ctx_size, int num_elem, int P_to, const double *proj1d, const double *x_e,
                           double *q0_e, void *stream);

/* Arithmetic-pipe throughput probe (no reference counterpart; the pipe-side denominator of the operator roofline): one
 * launch of 8 x SMs CTAs of 256 threads, each thread running eight independent FMA chains of `iters` steps in FP64
 * (fp64 != 0) or FP32.  d_sink: device scratch of at least 2048 x SMs elements of that type (written only on an
 * impossible value); *fma_per_launch receives the FMA count, to be divided by the caller's event time on `stream`. */
HB_EXPORT int hb_fma_peak_probe(int fp64, int iters, void *d_sink, int64_t sink_elems, int64_t *fma_per_launch, void *stream);

/* Basis-contraction mechanism A/B probe (no reference counterpart): `reps` rounds of u <- D_x u + D_y u, the in-plane
 * collocated derivatives of five FP64 components at the Q = 5 points of each element (d_u, d_out: [num_elem][5][125],
 * x fastest; D: host 5 x 5 row-major), by shared-memory fibre passes (variant 0, the operator kernels' mechanism, 128
 * threads per element) or warp shuffles (variant 1, one z-plane per warp, 160 threads per element).  Results are
 * bit-identical between the variants.  ctas_per_sm = 0: each variant at its own occupancy limit.  *fma_per_launch
 * receives the FMA count (num_elem x reps x 6250). */
HB_EXPORT int hb_contraction_probe(int variant, const double *D, const double *d_u, double *d_out, int num_elem, int reps, int ctas_per_sm,
                                   int64_t *fma_per_launch, void *stream);

/* Library identification */
const char *hb_version(void);

#ifdef __cplusplus
}
#endif
#endif
