/* hb_solver.c -- implicit time loop on the GPU: BDF1/BDF2 + Newton + right-preconditioned GMRES with a Jacobi
 * preconditioner, in FP64 or mixed precision.
 *
 * This is the caller side of the hot path.  HONEE drives the same operators through PETSc: TSBDF (src/setupts.c:343) calls
 * IFunction_NS (src/setupts.c:78-125) for the residual F(t, q, alpha q + z), FormIJacobian_NS (src/setupts.c:131-157) sets the
 * "ijacobian time shift" alpha, KSP (GMRES) applies MatMult_Ceed (src/mat-ceed.c:1643-1700) and PCJacobi uses
 * MatGetDiagonal_Ceed (src/mat-ceed.c:1603-1634).  PETSc is not part of this project, so the loop is restated here in C on
 * device buffers with the fused kernels of include/honee_b200.h.
 *
 * Mixed precision (the `jacobian_fp32` option): the Newton residual, the Newton update and its norm stay FP64; the IFunction
 * also writes the stored Jacobian data in FP32, and the Krylov basis, the Jacobian actions and the Jacobi diagonal are FP32
 * with FP64 accumulation of every inner product.  The Newton iteration converges to the same FP64 residual tolerance; only
 * the Krylov solve is less exact per step.
 */
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "honee_b200.h"

#define MAXK HB_GMRES_MAX_BASIS

struct HbTimeStepper {
  const HbElemOp    *op;
  HbNewtonianContext ctx;
  const double      *qdata;
  HbSolverOptions    o;
  int64_t            n, ldv; /* ldv: row stride of the Krylov basis, n rounded up so every row starts 16-byte aligned */
  int                njd, steps_taken;
  double             t;
  cudaStream_t       s;
  /* FP64 state */
  double *q, *q_prev, *q_prev2, *z, *qdot, *res, *jd64, *d_partial, *d_dots, *d_dots2, *scratch;
  double *h_dots; /* pinned host copies of the Gram-Schmidt coefficients: [0, MAXK) first pass, [MAXK, 2 MAXK) refinement */
  /* Krylov (FP32 or FP64) */
  void  *V, *w, *zvec, *diag, *jd32, *y_work;
  float *res32;
  double *delta;
  /* optional learned closure fused into the residual (host copy of the weights); with sgs_lagged its contribution is
   * evaluated once per step at the previous state and added to every Newton residual */
  HbMlpDesc sgs_desc;
  float    *sgs_w;
  double   *sgs_res;
  /* matrix-free (finite-difference) Jacobian action: perturbed state, rate and residual */
  double *qp, *qdp, *rp;
  /* optional free-stream boundary faces: residual and Jacobian sub-operators of the composite */
  /* essential DOFs: L-vector indices and values (device) */
  int32_t *ess_idx;
  double  *ess_val, *ess_one;
  int64_t  ess_n;
  /* point-block Jacobi (pc_jacobi 2): FP64 blocks, inverted in place (FP64) or into pb32 (mixed precision) */
  double *pb64;
  float  *pb32;
  int    *d_sing;
  const HbFaceOp *bc;
  unsigned char   bc_ctx[sizeof(HbFreestreamContext)];
  int             bc_flux;
  const double   *bc_qdata;
  double         *bc_jac;
};

#define CUCK(x)                                \
  do {                                         \
    if ((x) != cudaSuccess) return HB_ERROR_CUDA; \
  } while (0)
#define HBCK(x)          \
  do {                   \
    int e_ = (x);        \
    if (e_) return e_;   \
  } while (0)

void hb_solver_default_options(HbSolverOptions *o) {
  memset(o, 0, sizeof *o);
  o->dt            = 1e-5;
  o->bdf_order     = 2;
  o->newton_rtol   = 1e-8;
  o->newton_atol   = 1e-30;
  o->newton_max_it = 20;
  o->ksp_rtol      = 1e-5;  /* PETSc's KSP defaults: rtol 1e-5, at most 10000 iterations */
  o->ksp_max_it    = 10000;
  o->gmres_restart = 30;
  o->pc_jacobi     = 1;
  o->jacobian_fp32 = 0;
  o->cgs_refine    = 0; /* KSPGMRESSetCGSRefinementType default: never */
  o->sgs_lagged    = 1;
  o->jfnk          = 0;
}

static size_t ksz(const HbTimeStepper *ts) { return ts->o.jacobian_fp32 ? sizeof(float) : sizeof(double); }

int hb_ts_create(const HbElemOp *op, const void *ctx184, const double *d_qdata, const HbSolverOptions *opts, void *stream, HbTimeStepper **out) {
  *out = NULL;
  if (!op || !ctx184 || !d_qdata || !opts) return HB_ERROR_INVALID;
  if (opts->gmres_restart < 1 || opts->gmres_restart + 1 > MAXK || opts->dt <= 0 || (opts->bdf_order != 1 && opts->bdf_order != 2))
    return HB_ERROR_INVALID;
  if (opts->jfnk && opts->jacobian_fp32) return HB_ERROR_INVALID; /* the difference quotient needs FP64 Krylov vectors */
  if (opts->pc_jacobi < 0 || opts->pc_jacobi > 2) return HB_ERROR_INVALID;
  HbTimeStepper *ts = (HbTimeStepper *)calloc(1, sizeof *ts);
  if (!ts) return HB_ERROR_NOMEM;
  ts->op = op;
  memcpy(&ts->ctx, ctx184, sizeof ts->ctx);
  ts->qdata = d_qdata;
  ts->o     = *opts;
  ts->n     = op->l_size;
  ts->ldv   = (op->l_size + 3) & ~(int64_t)3;
  ts->njd   = ts->ctx.idl_enable ? 15 : 14;
  ts->s     = (cudaStream_t)stream;
  const size_t nb = sizeof(double) * (size_t)ts->n, Q3 = (size_t)op->Q * op->Q * op->Q, njd = (size_t)ts->njd * op->num_elem * Q3;
  const int m = ts->o.gmres_restart;
  int err = 0;
  err |= cudaMalloc((void **)&ts->q, nb) | cudaMalloc((void **)&ts->q_prev, nb) | cudaMalloc((void **)&ts->q_prev2, nb);
  err |= cudaMalloc((void **)&ts->z, nb) | cudaMalloc((void **)&ts->qdot, nb) | cudaMalloc((void **)&ts->res, nb) | cudaMalloc((void **)&ts->delta, nb);
  err |= cudaMalloc((void **)&ts->d_partial, sizeof(double) * 512 * MAXK) | cudaMalloc((void **)&ts->d_dots, sizeof(double) * MAXK);
  err |= cudaMalloc((void **)&ts->d_dots2, sizeof(double) * MAXK) | cudaMallocHost((void **)&ts->h_dots, sizeof(double) * 2 * MAXK);
  err |= cudaMalloc((void **)&ts->scratch, sizeof(double) * 1024);
  err |= cudaMalloc(&ts->V, ksz(ts) * (size_t)ts->ldv * (m + 1)) | cudaMalloc(&ts->w, ksz(ts) * (size_t)ts->n);
  err |= cudaMalloc(&ts->zvec, ksz(ts) * (size_t)ts->n) | cudaMalloc(&ts->diag, ksz(ts) * (size_t)ts->n);
  if (ts->o.jacobian_fp32) err |= cudaMalloc(&ts->jd32, sizeof(float) * njd) | cudaMalloc((void **)&ts->res32, sizeof(float) * (size_t)ts->n);
  else err |= cudaMalloc((void **)&ts->jd64, sizeof(double) * njd);
  if (ts->o.jfnk) err |= cudaMalloc((void **)&ts->qp, nb) | cudaMalloc((void **)&ts->qdp, nb) | cudaMalloc((void **)&ts->rp, nb);
  if (ts->o.pc_jacobi == 2) {
    err |= cudaMalloc((void **)&ts->pb64, 5 * nb) | cudaMalloc((void **)&ts->d_sing, sizeof(int));
    if (ts->o.jacobian_fp32) err |= cudaMalloc((void **)&ts->pb32, 5 * sizeof(float) * (size_t)ts->n);
  }
  if (err) {
    hb_ts_destroy(ts);
    return HB_ERROR_NOMEM;
  }
  *out = ts;
  return HB_SUCCESS;
}

int hb_ts_destroy(HbTimeStepper *ts) {
  if (!ts) return HB_SUCCESS;
  void *p[] = {ts->q, ts->q_prev, ts->q_prev2, ts->z, ts->qdot, ts->res, ts->delta, ts->d_partial, ts->d_dots, ts->d_dots2, ts->scratch,
               ts->V, ts->w, ts->zvec, ts->diag, ts->jd32, ts->res32, ts->jd64, ts->qp, ts->qdp, ts->rp, ts->pb64, ts->pb32, ts->d_sing};
  for (size_t i = 0; i < sizeof p / sizeof p[0]; i++)
    if (p[i]) cudaFree(p[i]);
  if (ts->h_dots) cudaFreeHost(ts->h_dots);
  free(ts->sgs_w);
  if (ts->sgs_res) cudaFree(ts->sgs_res);
  if (ts->bc_jac) cudaFree(ts->bc_jac);
  if (ts->ess_idx) cudaFree(ts->ess_idx);
  if (ts->ess_val) cudaFree(ts->ess_val);
  if (ts->ess_one) cudaFree(ts->ess_one);
  free(ts);
  return HB_SUCCESS;
}

int hb_ts_set_state(HbTimeStepper *ts, const double *d_q, double t) {
  CUCK(cudaMemcpyAsync(ts->q, d_q, sizeof(double) * (size_t)ts->n, cudaMemcpyDeviceToDevice, ts->s));
  if (ts->ess_n) HBCK(hb_constrain_set_f64(ts->q, ts->ess_idx, ts->ess_val, ts->ess_n, ts->s)); /* boundary values inserted */
  ts->t           = t;
  ts->steps_taken = 0;
  return HB_SUCCESS;
}

int hb_ts_get_state(HbTimeStepper *ts, double *d_q, double *t) {
  CUCK(cudaMemcpyAsync(d_q, ts->q, sizeof(double) * (size_t)ts->n, cudaMemcpyDeviceToDevice, ts->s));
  if (t) *t = ts->t;
  return HB_SUCCESS;
}

const void *hb_ts_context(HbTimeStepper *ts) { return &ts->ctx; }

int hb_ts_set_freestream(HbTimeStepper *ts, const HbFaceOp *faces, const void *ctx264, int flux_type, const double *qdata_sur) {
  if (!ts) return HB_ERROR_INVALID;
  if (ts->bc_jac) cudaFree(ts->bc_jac);
  ts->bc_jac = NULL;
  ts->bc     = NULL;
  if (!faces) return HB_SUCCESS; /* boundary off */
  if (!ctx264 || !qdata_sur || (flux_type != 0 && flux_type != 1) || faces->l_size != ts->n) return HB_ERROR_INVALID;
  if (cudaMalloc((void **)&ts->bc_jac, sizeof(double) * 5 * (size_t)faces->num_faces * faces->Q * faces->Q) != cudaSuccess) return HB_ERROR_NOMEM;
  memcpy(ts->bc_ctx, ctx264, sizeof ts->bc_ctx);
  ts->bc       = faces;
  ts->bc_flux  = flux_type;
  ts->bc_qdata = qdata_sur;
  return HB_SUCCESS;
}

int hb_ts_set_essential(HbTimeStepper *ts, const int32_t *h_idx, const double *h_val, int64_t n) {
  if (!ts || n < 0 || (n && !h_idx)) return HB_ERROR_INVALID;
  for (int64_t i = 0; i < n; i++)
    if (h_idx[i] < 0 || h_idx[i] >= ts->n) return HB_ERROR_INVALID;
  if (ts->ess_idx) cudaFree(ts->ess_idx);
  if (ts->ess_val) cudaFree(ts->ess_val);
  if (ts->ess_one) cudaFree(ts->ess_one);
  ts->ess_idx = NULL;
  ts->ess_val = ts->ess_one = NULL;
  ts->ess_n   = 0;
  if (!n) return HB_SUCCESS;
  if (cudaMalloc((void **)&ts->ess_idx, sizeof(int32_t) * (size_t)n) != cudaSuccess ||
      cudaMalloc((void **)&ts->ess_val, sizeof(double) * (size_t)n) != cudaSuccess ||
      cudaMalloc((void **)&ts->ess_one, sizeof(double) * (size_t)n) != cudaSuccess)
    return HB_ERROR_NOMEM;
  HBCK(hb_vec_set_f64(ts->ess_one, n, 1.0, ts->s));
  CUCK(cudaMemcpy(ts->ess_idx, h_idx, sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice));
  if (h_val) CUCK(cudaMemcpy(ts->ess_val, h_val, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice));
  else CUCK(cudaMemset(ts->ess_val, 0, sizeof(double) * (size_t)n));
  ts->ess_n = n;
  /* the current state takes the boundary values */
  return hb_constrain_set_f64(ts->q, ts->ess_idx, ts->ess_val, n, ts->s);
}

int hb_ts_set_sgs(HbTimeStepper *ts, const HbMlpDesc *d, const float *h_weights) {
  if (!ts) return HB_ERROR_INVALID;
  free(ts->sgs_w);
  ts->sgs_w = NULL;
  if (!d || !h_weights) return HB_SUCCESS; /* closure off */
  const int np = hb_mlp_num_params(d);
  if (np < 0) return np;
  ts->sgs_w = (float *)malloc(sizeof(float) * (size_t)np);
  if (!ts->sgs_w) return HB_ERROR_NOMEM;
  if (!ts->sgs_res && cudaMalloc((void **)&ts->sgs_res, sizeof(double) * (size_t)ts->n) != cudaSuccess) return HB_ERROR_NOMEM;
  memcpy(ts->sgs_w, h_weights, sizeof(float) * (size_t)np);
  ts->sgs_desc = *d;
  return HB_SUCCESS;
}

/* ---- small helpers on the Krylov precision ---- */
static int kv_norm2(HbTimeStepper *ts, const void *x, double *nrm) {
  double r;
  if (ts->o.jacobian_fp32) HBCK(hb_vec_reduce_f32((const float *)x, NULL, ts->n, 1, ts->scratch, &r, ts->s));
  else HBCK(hb_vec_reduce_f64((const double *)x, NULL, ts->n, 1, ts->scratch, &r, ts->s));
  *nrm = sqrt(r);
  return HB_SUCCESS;
}
static void *kv_col(HbTimeStepper *ts, int j) { return (char *)ts->V + ksz(ts) * (size_t)ts->ldv * j; }
static int kv_scale(HbTimeStepper *ts, void *x, double a) {
  return ts->o.jacobian_fp32 ? hb_vec_scale_f32((float *)x, ts->n, (float)a, ts->s) : hb_vec_scale_f64((double *)x, ts->n, a, ts->s);
}
static int kv_copy(HbTimeStepper *ts, void *dst, const void *src) {
  return cudaMemcpyAsync(dst, src, ksz(ts) * (size_t)ts->n, cudaMemcpyDeviceToDevice, ts->s) == cudaSuccess ? HB_SUCCESS : HB_ERROR_CUDA;
}
/* y = J x (the IJacobian operator at the current linearisation point) */
/* residual F(q, q_dot) of the current model (with the closure when attached and not lagged), without Jacobian data */
static int residual(HbTimeStepper *ts, const double *q, const double *qdot, double *out, double *jd64, float *jd32) {
  /* constrained DOFs: the rate is zero there (PETSc never writes them into the local rate vector) */
  if (ts->ess_n) HBCK(hb_constrain_set_f64((double *)qdot, ts->ess_idx, NULL, ts->ess_n, ts->s));
  HbIFunctionIO io = {q, qdot, ts->qdata, jd64, jd32, out, 0};
  if (ts->sgs_w && !(ts->o.sgs_lagged && !ts->o.jfnk)) HBCK(hb_ifunction_apply_sgs(ts->op, &ts->ctx, &io, &ts->sgs_desc, ts->sgs_w, ts->s));
  else HBCK(hb_ifunction_apply(ts->op, &ts->ctx, &io, ts->s));
  /* boundary faces add their flux; the state at the face points is kept only for the Newton iterate's Jacobian */
  if (ts->bc) HBCK(hb_freestream_apply(ts->bc, ts->bc_ctx, ts->bc_flux, ts->bc_qdata, q, (jd64 || jd32) ? ts->bc_jac : NULL, out, ts->s));
  /* constrained rows are not part of the system (DMLocalToGlobal drops them) */
  if (ts->ess_n) HBCK(hb_constrain_set_f64(out, ts->ess_idx, NULL, ts->ess_n, ts->s));
  return HB_SUCCESS;
}

/* y = J x by a forward difference of the full residual (PETSc's -snes_mf_operator form): the state moves by eps x and its
 * rate by shift * eps x; eps = sqrt(DBL_EPSILON) (1 + |q|) / |x|.  ts->res holds F at the current Newton iterate. */
static int jac_fd(HbTimeStepper *ts, const double *x, double *y) {
  double xx, qq;
  HBCK(hb_vec_reduce_f64(x, NULL, ts->n, 1, ts->scratch, &xx, ts->s));
  if (xx == 0) return hb_vec_set_f64(y, ts->n, 0.0, ts->s);
  HBCK(hb_vec_reduce_f64(ts->q, NULL, ts->n, 1, ts->scratch, &qq, ts->s));
  const double eps = 1.4901161193847656e-08 * (1 + sqrt(qq)) / sqrt(xx);
  CUCK(cudaMemcpyAsync(ts->qp, ts->q, sizeof(double) * (size_t)ts->n, cudaMemcpyDeviceToDevice, ts->s));
  CUCK(cudaMemcpyAsync(ts->qdp, ts->qdot, sizeof(double) * (size_t)ts->n, cudaMemcpyDeviceToDevice, ts->s));
  HBCK(hb_vec_axpy_f64(ts->qp, eps, x, ts->n, ts->s));
  HBCK(hb_vec_axpy_f64(ts->qdp, ts->ctx.ijacobian_time_shift * eps, x, ts->n, ts->s));
  HBCK(residual(ts, ts->qp, ts->qdp, ts->rp, NULL, NULL));
  CUCK(cudaMemcpyAsync(y, ts->rp, sizeof(double) * (size_t)ts->n, cudaMemcpyDeviceToDevice, ts->s));
  HBCK(hb_vec_axpby_f64(y, -1.0 / eps, 1.0 / eps, ts->res, ts->n, ts->s)); /* y = (F(q + eps x) - F(q)) / eps */
  return HB_SUCCESS;
}

static int kv_jac(HbTimeStepper *ts, const void *x, void *y) {
  if (ts->o.jfnk) return jac_fd(ts, (const double *)x, (double *)y);
  if (ts->o.jacobian_fp32) {
    HBCK(hb_ijacobian_apply_f32(ts->op, &ts->ctx, ts->qdata, (const float *)ts->jd32, (const float *)x, (float *)y, 0, ts->s));
    if (ts->bc) HBCK(hb_freestream_jacobian_apply_f32(ts->bc, ts->bc_ctx, ts->bc_flux, ts->bc_qdata, ts->bc_jac, (const float *)x, (float *)y, ts->s));
    if (ts->ess_n) HBCK(hb_constrain_set_f32((float *)y, ts->ess_idx, NULL, ts->ess_n, ts->s));
    return HB_SUCCESS;
  }
  HBCK(hb_ijacobian_apply_f64(ts->op, &ts->ctx, ts->qdata, ts->jd64, (const double *)x, (double *)y, 0, ts->s));
  if (ts->bc) HBCK(hb_freestream_jacobian_apply(ts->bc, ts->bc_ctx, ts->bc_flux, ts->bc_qdata, ts->bc_jac, (const double *)x, (double *)y, ts->s));
  if (ts->ess_n) HBCK(hb_constrain_set_f64((double *)y, ts->ess_idx, NULL, ts->ess_n, ts->s));
  return HB_SUCCESS;
}
/* z = M^-1 x (Jacobi) or copy */
static int kv_pc(HbTimeStepper *ts, const void *x, void *z) {
  if (!ts->o.pc_jacobi) return kv_copy(ts, z, x);
  if (ts->o.pc_jacobi == 2) {
    if (ts->o.jacobian_fp32) return hb_pb_apply_f32(ts->pb32, (const float *)x, (float *)z, ts->n / 5, ts->s);
    return hb_pb_apply_f64(ts->pb64, (const double *)x, (double *)z, ts->n / 5, ts->s);
  }
  if (ts->o.jacobian_fp32) return hb_vec_pointwise_mult_f32((float *)z, (const float *)ts->diag, (const float *)x, ts->n, ts->s);
  return hb_vec_pointwise_mult_f64((double *)z, (const double *)ts->diag, (const double *)x, ts->n, ts->s);
}
/* d_h = V[:, :k]^T w, left on the device */
static int kv_multidot_dev(HbTimeStepper *ts, int k, const void *w, double *d_h) {
  if (ts->o.jacobian_fp32) HBCK(hb_krylov_multidot_f32((const float *)ts->V, ts->ldv, k, (const float *)w, ts->n, ts->d_partial, d_h, ts->s));
  else HBCK(hb_krylov_multidot_f64((const double *)ts->V, ts->ldv, k, (const double *)w, ts->n, ts->d_partial, d_h, ts->s));
  return HB_SUCCESS;
}
/* w -= V[:, :k] d_h with the coefficients read on the device */
static int kv_multiaxpy_dev(HbTimeStepper *ts, void *w, int k, const double *d_h) {
  if (ts->o.jacobian_fp32) return hb_krylov_multiaxpy_dev_f32((float *)w, (const float *)ts->V, ts->ldv, k, d_h, -1.0, ts->n, ts->s);
  return hb_krylov_multiaxpy_dev_f64((double *)w, (const double *)ts->V, ts->ldv, k, d_h, -1.0, ts->n, ts->s);
}

/* Jacobi diagonal (or point blocks) at the current linearisation point, stored inverted; *failed: a point block had no
 * pivot (PETSc reports the same as a failed preconditioner set-up) */
static int assemble_pc(HbTimeStepper *ts, int *failed) {
  *failed = 0;
  if (!ts->o.pc_jacobi) return HB_SUCCESS;
  if (ts->o.pc_jacobi == 2) {
    const int64_t nodes = ts->n / 5;
    int           sing  = 0;
    if (ts->o.jacobian_fp32) {
      HBCK(hb_point_block_diagonal_f32(ts->op, &ts->ctx, ts->qdata, (const float *)ts->jd32, ts->pb32, 0, ts->s));
      HBCK(hb_vec_f32_to_f64(ts->pb32, ts->pb64, 5 * ts->n, 0, ts->s));
    } else {
      HBCK(hb_point_block_diagonal_f64(ts->op, &ts->ctx, ts->qdata, ts->jd64, ts->pb64, 0, ts->s));
    }
    if (ts->bc) HBCK(hb_freestream_point_block_diagonal(ts->bc, ts->bc_ctx, ts->bc_flux, ts->bc_qdata, ts->bc_jac, ts->pb64, ts->s));
    if (ts->ess_n) HBCK(hb_pb_constrain(ts->pb64, ts->ess_idx, ts->ess_n, ts->s));
    if (ts->o.jacobian_fp32) HBCK(hb_pb_invert_f64_to_f32(ts->pb64, ts->pb32, nodes, ts->d_sing, &sing, ts->s));
    else HBCK(hb_pb_invert_f64(ts->pb64, ts->pb64, nodes, ts->d_sing, &sing, ts->s));
    *failed = sing > 0;
    return HB_SUCCESS;
  }
  if (ts->o.jacobian_fp32) {
    HBCK(hb_diagonal_assemble_f32(ts->op, &ts->ctx, ts->qdata, (const float *)ts->jd32, (float *)ts->diag, 0, ts->s));
    /* invert in FP64 (delta is free before the Krylov solve), store FP32 */
    HBCK(hb_vec_f32_to_f64((const float *)ts->diag, ts->delta, ts->n, 0, ts->s));
    if (ts->bc) HBCK(hb_freestream_diagonal(ts->bc, ts->bc_ctx, ts->bc_flux, ts->bc_qdata, ts->bc_jac, ts->delta, ts->s));
    if (ts->ess_n) HBCK(hb_constrain_set_f64(ts->delta, ts->ess_idx, ts->ess_one, ts->ess_n, ts->s)); /* identity rows */
    HBCK(hb_vec_reciprocal_f64(ts->delta, ts->n, ts->s));
    return hb_vec_f64_to_f32(ts->delta, (float *)ts->diag, ts->n, 0, ts->s);
  }
  HBCK(hb_diagonal_assemble_f64(ts->op, &ts->ctx, ts->qdata, ts->jd64, (double *)ts->diag, 0, ts->s));
  if (ts->bc) HBCK(hb_freestream_diagonal(ts->bc, ts->bc_ctx, ts->bc_flux, ts->bc_qdata, ts->bc_jac, (double *)ts->diag, ts->s));
  if (ts->ess_n) HBCK(hb_constrain_set_f64((double *)ts->diag, ts->ess_idx, ts->ess_one, ts->ess_n, ts->s)); /* identity rows */
  return hb_vec_reciprocal_f64((double *)ts->diag, ts->n, ts->s);
}

/* GMRES(m), right preconditioned, classical Gram-Schmidt (PETSc's KSPGMRES default, refinement "never") or CGS2 with
 * `cgs_refine`; solves J delta = -res
 * (res FP64) to relative tolerance ksp_rtol.  delta (FP64) receives the solution. */
static int gmres(HbTimeStepper *ts, int *its_out, double *rnorm_out) {
  const int m = ts->o.gmres_restart;
  double    H[MAXK + 1][MAXK], cs[MAXK], sn[MAXK], g[MAXK + 1], y[MAXK];
  int       its = 0;
  HBCK(hb_vec_set_f64(ts->delta, ts->n, 0.0, ts->s));
  /* r0 = -res (x0 = 0) */
  void *v0 = kv_col(ts, 0);
  if (ts->o.jacobian_fp32) HBCK(hb_vec_f64_to_f32(ts->res, (float *)v0, ts->n, 0, ts->s));
  else HBCK(cudaMemcpyAsync(v0, ts->res, sizeof(double) * (size_t)ts->n, cudaMemcpyDeviceToDevice, ts->s) == cudaSuccess ? 0 : HB_ERROR_CUDA);
  HBCK(kv_scale(ts, v0, -1.0));
  double beta0;
  HBCK(kv_norm2(ts, v0, &beta0));
  double beta = beta0;
  if (beta0 == 0) {
    *its_out   = 0;
    *rnorm_out = 0;
    return HB_SUCCESS;
  }
  const double target = ts->o.ksp_rtol * beta0;
  while (its < ts->o.ksp_max_it) {
    HBCK(kv_scale(ts, kv_col(ts, 0), 1.0 / beta));
    memset(g, 0, sizeof g);
    g[0]  = beta;
    int k = 0;
    for (; k < m && its < ts->o.ksp_max_it; k++, its++) {
      /* the operator writes the next basis vector in place; it is orthogonalised and normalised there */
      void *wk = kv_col(ts, k + 1);
      HBCK(kv_pc(ts, kv_col(ts, k), ts->zvec));
      HBCK(kv_jac(ts, ts->zvec, wk));
      /* classical Gram-Schmidt, optionally with one refinement pass (CGS2).  The coefficients stay on the device for the
       * update and reach the host by asynchronous copies into pinned memory, complete once the norm has synchronised the
       * stream: one host round trip per iteration */
      HBCK(kv_multidot_dev(ts, k + 1, wk, ts->d_dots));
      HBCK(kv_multiaxpy_dev(ts, wk, k + 1, ts->d_dots));
      CUCK(cudaMemcpyAsync(ts->h_dots, ts->d_dots, sizeof(double) * (size_t)(k + 1), cudaMemcpyDeviceToHost, ts->s));
      if (ts->o.cgs_refine) {
        HBCK(kv_multidot_dev(ts, k + 1, wk, ts->d_dots2));
        HBCK(kv_multiaxpy_dev(ts, wk, k + 1, ts->d_dots2));
        CUCK(cudaMemcpyAsync(ts->h_dots + MAXK, ts->d_dots2, sizeof(double) * (size_t)(k + 1), cudaMemcpyDeviceToHost, ts->s));
      }
      double hn;
      HBCK(kv_norm2(ts, wk, &hn));
      for (int i = 0; i <= k; i++) H[i][k] = ts->o.cgs_refine ? ts->h_dots[i] + ts->h_dots[MAXK + i] : ts->h_dots[i];
      H[k + 1][k] = hn;
      if (hn > 0) HBCK(kv_scale(ts, wk, 1.0 / hn));
      /* apply the previous Givens rotations, then a new one */
      for (int i = 0; i < k; i++) {
        const double a = H[i][k], b = H[i + 1][k];
        H[i][k]         = cs[i] * a + sn[i] * b;
        H[i + 1][k]     = -sn[i] * a + cs[i] * b;
      }
      const double a = H[k][k], b = H[k + 1][k], r = hypot(a, b);
      cs[k]    = r > 0 ? a / r : 1;
      sn[k]    = r > 0 ? b / r : 0;
      H[k][k]  = r;
      H[k + 1][k] = 0;
      g[k + 1] = -sn[k] * g[k];
      g[k]     = cs[k] * g[k];
      if (fabs(g[k + 1]) <= target || hn == 0) {
        k++;
        its++;
        break;
      }
    }
    /* y = H^-1 g (upper triangular k x k) ; delta += M^-1 V y */
    for (int i = k - 1; i >= 0; i--) {
      double s = g[i];
      for (int j = i + 1; j < k; j++) s -= H[i][j] * y[j];
      y[i] = s / H[i][i];
    }
    if (ts->o.jacobian_fp32) {
      HBCK(hb_vec_set_f32((float *)ts->w, ts->n, 0.0f, ts->s));
      HBCK(hb_krylov_multiaxpy_f32((float *)ts->w, (const float *)ts->V, ts->ldv, k, y, ts->n, ts->s));
      HBCK(kv_pc(ts, ts->w, ts->zvec));
      HBCK(hb_vec_f32_to_f64((const float *)ts->zvec, ts->delta, ts->n, 1, ts->s));
    } else {
      HBCK(hb_vec_set_f64((double *)ts->w, ts->n, 0.0, ts->s));
      HBCK(hb_krylov_multiaxpy_f64((double *)ts->w, (const double *)ts->V, ts->ldv, k, y, ts->n, ts->s));
      HBCK(kv_pc(ts, ts->w, ts->zvec));
      HBCK(hb_vec_axpy_f64(ts->delta, 1.0, (const double *)ts->zvec, ts->n, ts->s));
    }
    beta = fabs(g[k]);
    if (beta <= target || its >= ts->o.ksp_max_it) break;
    /* restart: r = -res - J delta, in the Krylov precision */
    void *r = kv_col(ts, 0);
    if (ts->o.jacobian_fp32) {
      HBCK(hb_vec_f64_to_f32(ts->delta, (float *)ts->zvec, ts->n, 0, ts->s));
      HBCK(kv_jac(ts, ts->zvec, r));
      HBCK(hb_vec_f64_to_f32(ts->res, (float *)ts->w, ts->n, 0, ts->s));
      HBCK(hb_vec_axpby_f32((float *)r, -1.0f, -1.0f, (const float *)ts->w, ts->n, ts->s)); /* r = -res - J delta */
    } else {
      HBCK(kv_jac(ts, ts->delta, r));
      HBCK(hb_vec_axpby_f64((double *)r, -1.0, -1.0, ts->res, ts->n, ts->s));
    }
    HBCK(kv_norm2(ts, r, &beta));
  }
  *its_out   = its;
  *rnorm_out = beta / beta0;
  return HB_SUCCESS;
}

int hb_ts_step(HbTimeStepper *ts, HbStepStats *st) {
  memset(st, 0, sizeof *st);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, ts->s);
  const double dt  = ts->o.dt;
  const int    bdf = (ts->o.bdf_order == 2 && ts->steps_taken >= 1) ? 2 : 1;
  double       alpha;
  /* history: q_prev2 <- q_prev, q_prev <- q (the initial Newton guess is the previous state) */
  if (bdf == 2) CUCK(cudaMemcpyAsync(ts->q_prev2, ts->q_prev, sizeof(double) * (size_t)ts->n, cudaMemcpyDeviceToDevice, ts->s));
  CUCK(cudaMemcpyAsync(ts->q_prev, ts->q, sizeof(double) * (size_t)ts->n, cudaMemcpyDeviceToDevice, ts->s));
  if (bdf == 1) { /* q_dot = (q - q_n)/dt */
    alpha = 1.0 / dt;
    HBCK(hb_vec_combine_f64(ts->q_prev, NULL, -1.0 / dt, 0.0, ts->z, ts->n, ts->s));
  } else { /* q_dot = (3 q - 4 q_n + q_{n-1}) / (2 dt) */
    alpha = 1.5 / dt;
    HBCK(hb_vec_combine_f64(ts->q_prev, ts->q_prev2, -2.0 / dt, 0.5 / dt, ts->z, ts->n, ts->s));
  }
  ts->ctx.dt                   = dt;
  ts->ctx.ijacobian_time_shift = alpha;
  ts->ctx.time                 = ts->t + dt;
  const int sgs_lag = ts->sgs_w && ts->o.sgs_lagged && !ts->o.jfnk;
  if (sgs_lag) { /* closure contribution at the previous state: F_sgs(q_n) - F(q_n), independent of q_dot */
    HBCK(hb_vec_set_f64(ts->qdot, ts->n, 0.0, ts->s)); /* any finite q_dot; it cancels in the difference */
    HbIFunctionIO io_a = {ts->q, ts->qdot, ts->qdata, NULL, NULL, ts->sgs_res, 0};
    HbIFunctionIO io_b = {ts->q, ts->qdot, ts->qdata, NULL, NULL, ts->delta, 0};
    HBCK(hb_ifunction_apply_sgs(ts->op, &ts->ctx, &io_a, &ts->sgs_desc, ts->sgs_w, ts->s));
    HBCK(hb_ifunction_apply(ts->op, &ts->ctx, &io_b, ts->s));
    HBCK(hb_vec_axpy_f64(ts->sgs_res, -1.0, ts->delta, ts->n, ts->s));
  }
  double r0 = 0, rn = 0;
  int    it = 0, ksp_total = 0, converged = 0;
  for (; it <= ts->o.newton_max_it; it++) {
    HBCK(hb_bdf_qdot(ts->q, ts->z, alpha, ts->qdot, ts->n, ts->s));
    HbIFunctionIO io = {ts->q, ts->qdot, ts->qdata, ts->o.jacobian_fp32 ? NULL : ts->jd64, ts->o.jacobian_fp32 ? (float *)ts->jd32 : NULL, ts->res, 0};
    HBCK(residual(ts, io.q, io.q_dot, io.v, io.jac_data, io.jac_data_f32));
    if (sgs_lag) HBCK(hb_vec_axpy_f64(ts->res, 1.0, ts->sgs_res, ts->n, ts->s));
    if (sgs_lag && ts->ess_n) HBCK(hb_constrain_set_f64(ts->res, ts->ess_idx, NULL, ts->ess_n, ts->s));
    double r2;
    HBCK(hb_vec_reduce_f64(ts->res, NULL, ts->n, 1, ts->scratch, &r2, ts->s));
    rn = sqrt(r2);
    if (it == 0) r0 = rn;
    if (!isfinite(rn)) {
      st->converged_reason = -1; /* diverged: non-finite residual (src/setupts.c:232-249 checks for NaN the same way) */
      break;
    }
    if (rn <= ts->o.newton_rtol * r0 || rn <= ts->o.newton_atol) {
      converged = 1;
      break;
    }
    if (it == ts->o.newton_max_it) break;
    if (it == 0 || ts->o.pc_every_newton) {
      int pc_failed;
      HBCK(assemble_pc(ts, &pc_failed));
      if (pc_failed) {
        st->converged_reason = -3;
        break;
      }
    }
    int    kits;
    double krel;
    HBCK(gmres(ts, &kits, &krel));
    ksp_total += kits;
    HBCK(hb_vec_axpy_f64(ts->q, 1.0, ts->delta, ts->n, ts->s));
  }
  cudaEventRecord(e1, ts->s);
  cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  st->newton_its = it;
  st->ksp_its    = ksp_total;
  st->res0       = r0;
  st->res_final  = rn;
  st->seconds    = ms * 1e-3;
  if (st->converged_reason == 0) st->converged_reason = converged ? 1 : -2;
  ts->t += dt;
  ts->steps_taken++;
  int status = 0;
  HBCK(hb_elemop_status((HbElemOp *)ts->op, &status, 1));
  return status ? HB_ERROR_BACKEND : HB_SUCCESS;
}
