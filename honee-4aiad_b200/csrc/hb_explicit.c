/* hb_explicit.c -- explicit time loop on the GPU: an explicit Runge-Kutta tableau whose right-hand side is the Newtonian
 * residual with the mass matrix inverted, lumped or by left-preconditioned GMRES.
 *
 * HONEE's explicit path (-ts_type rk): RHS_NS (src/setupts.c:31-75) applies the RHSFunction_Newtonian operator
 * (qfunctions/newtonian.h:133-202) and solves with the "mass_" KSP that CreateKSPMass builds (src/setuplibceed.c:15-93):
 * KSPPREONLY + PCJacobi row sum by default ("lumped"), or e.g. GMRES + PCJacobi diagonal from the options file
 * (examples/taylor_green_vortex.yaml).  With stab = supg the mass operator is the SUPG-stabilized one
 * (MassFunction_Newtonian, problems/newtonian.c:212-265, 795), linearised at the state of each right-hand side; the Jacobi
 * preconditioner is set up at the first solve and kept (the MatCEED object PETSc sees never changes state).  PETSc's TSRK and KSPGMRES are not part of this project, so the loop is restated
 * here on device buffers.
 *
 * The right-hand side is the IFunction kernel at q_dot = 0 with the sign reversed: the IFunction integrand
 * (newtonian.h:205-257) at zero rate is v = -wdetJ body (+ the damping layer), grad v = wdetJ dXdx (-F + stab), where the
 * SUPG strong residual sees U_dot = 0 as in the RHS QFunction, so RHS = -F(q, 0).  The stages therefore hold
 * f_i = M^-1 F(Y_i, 0) and the update subtracts them.
 *
 * GMRES follows PETSc's defaults: left preconditioning, convergence on the preconditioned residual norm estimate
 * |g_{k+1}| <= max(rtol ||D^-1 b||, atol) with a zero initial guess, classical Gram-Schmidt without refinement, restart
 * after mass_restart iterations with the residual recomputed.
 */
#include <cuda_runtime.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "honee_b200.h"

#define MAXK HB_GMRES_MAX_BASIS
#define MAXS HB_RK_MAX_STAGES

struct HbExplicitStepper {
  const HbElemOp    *op;
  HbNewtonianContext ctx;
  const double      *qdata;
  HbExplicitOptions  o;
  int64_t            n, ldv;
  double             t;
  int                steps_taken;
  cudaStream_t       s;
  double *q, *y, *f, *zero, *dinv, *K; /* K: stage block [stages][ldv] */
  double *V, *r, *scratch, *d_partial, *d_dots;
  double *h_dots; /* pinned host copy of the Gram-Schmidt coefficients */
  /* stabilized mass (stab = supg): the state it is linearised at, and whether the Jacobi set-up has run */
  int           mass_stab, pc_ready;
  const double *qstate;
  /* essential DOFs (device indices and values) */
  int32_t *ess_idx;
  double  *ess_val, *ess_one;
  int64_t  ess_n;
  /* free-stream faces: their flux joins the right-hand side */
  const HbFaceOp *bc;
  unsigned char   bc_ctx[sizeof(HbFreestreamContext)];
  int             bc_flux;
  const double   *bc_qdata;
};

#define CUCK(x)                                   \
  do {                                            \
    if ((x) != cudaSuccess) return HB_ERROR_CUDA; \
  } while (0)
#define HBCK(x)        \
  do {                 \
    int e_ = (x);      \
    if (e_) return e_; \
  } while (0)

void hb_explicit_default_options(HbExplicitOptions *o) {
  memset(o, 0, sizeof *o);
  o->dt        = 1e-5;
  o->rk_stages = 4; /* TSRK4: classical fourth order */
  o->rk_a[1 * MAXS + 0] = 0.5;
  o->rk_a[2 * MAXS + 1] = 0.5;
  o->rk_a[3 * MAXS + 2] = 1.0;
  o->rk_b[0] = 1.0 / 6, o->rk_b[1] = 1.0 / 3, o->rk_b[2] = 1.0 / 3, o->rk_b[3] = 1.0 / 6;
  o->rk_c[1] = 0.5, o->rk_c[2] = 0.5, o->rk_c[3] = 1.0;
  o->mass_ksp       = 0;
  o->mass_pc_rowsum = 1;
  o->mass_rtol      = 1e-5;
  o->mass_atol      = 1e-50;
  o->mass_max_it    = 10000;
  o->mass_restart   = 30;
}

static double *col(double *B, int64_t ldv, int j) { return B + ldv * j; }

static int norm2(HbExplicitStepper *ex, const double *x, double *nrm) {
  double r;
  HBCK(hb_vec_reduce_f64(x, NULL, ex->n, 1, ex->scratch, &r, ex->s));
  *nrm = sqrt(r);
  return HB_SUCCESS;
}

/* constrained entries leave the system (DMLocalToGlobal drops them): zero them */
static int mask(HbExplicitStepper *ex, double *x) { return ex->ess_n ? hb_constrain_set_f64(x, ex->ess_idx, NULL, ex->ess_n, ex->s) : HB_SUCCESS; }

/* w = M x: Mass_5, or the stabilized mass at the current right-hand side's state */
static int mass(HbExplicitStepper *ex, const double *x, double *w) {
  if (ex->mass_stab) return hb_mass_stab_apply(ex->op, &ex->ctx, ex->qdata, ex->qstate, x, w, 0, ex->s);
  return hb_mass_apply(ex->op, ex->qdata, x, w, 0, ex->s);
}

/* w = D^-1 M x */
static int pmass(HbExplicitStepper *ex, const double *x, double *w) {
  HBCK(mass(ex, x, w));
  HBCK(mask(ex, w));
  return hb_vec_pointwise_mult_f64(w, w, ex->dinv, ex->n, ex->s);
}

/* Jacobi from the mass diagonal or its row sums, stored inverted.  The row sums are those of the free-DOF system (PETSc's
 * MatGetRowSum multiplies the global, constrained-free matrix by ones); constrained rows get 1 (their residual is zero). */
static int setup_jacobi(HbExplicitStepper *ex) {
  if (ex->o.mass_pc_rowsum) {
    HBCK(hb_vec_set_f64(ex->r, ex->n, 1.0, ex->s));
    HBCK(mask(ex, ex->r));
    HBCK(mass(ex, ex->r, ex->dinv));
  } else if (ex->mass_stab) {
    HBCK(hb_mass_stab_diagonal(ex->op, &ex->ctx, ex->qdata, ex->qstate, ex->dinv, 0, ex->s));
  } else {
    HBCK(hb_mass_diagonal(ex->op, ex->qdata, ex->dinv, 0, ex->s));
  }
  ex->pc_ready = 1;
  if (ex->ess_n) HBCK(hb_constrain_set_f64(ex->dinv, ex->ess_idx, ex->ess_one, ex->ess_n, ex->s));
  return hb_vec_reciprocal_f64(ex->dinv, ex->n, ex->s);
}

/* x = M^-1 b by left-preconditioned GMRES(m); x must not alias b */
static int mass_gmres(HbExplicitStepper *ex, const double *b, double *x, int *its_out, int *reason) {
  const int m = ex->o.mass_restart;
  double    H[MAXK + 1][MAXK], cs[MAXK], sn[MAXK], g[MAXK + 1], y[MAXK];
  int       its = 0;
  *reason       = -2;
  HBCK(hb_vec_set_f64(x, ex->n, 0.0, ex->s));
  double *v0 = col(ex->V, ex->ldv, 0);
  HBCK(hb_vec_pointwise_mult_f64(v0, b, ex->dinv, ex->n, ex->s));
  double beta;
  HBCK(norm2(ex, v0, &beta));
  if (!isfinite(beta)) {
    *reason = -1;
    *its_out = 0;
    return HB_SUCCESS;
  }
  const double ttol = fmax(ex->o.mass_rtol * beta, ex->o.mass_atol);
  if (beta <= ttol || beta == 0) {
    *reason  = 1;
    *its_out = 0;
    return HB_SUCCESS;
  }
  for (;;) {
    HBCK(hb_vec_scale_f64(v0, ex->n, 1.0 / beta, ex->s));
    memset(g, 0, sizeof g);
    g[0]      = beta;
    int k     = 0;
    int done  = 0;
    while (k < m && its < ex->o.mass_max_it) {
      /* the operator writes the next basis vector in place; classical Gram-Schmidt with the coefficients kept on the
       * device, their host copy (pinned, asynchronous) complete once the norm has synchronised the stream */
      double *wk = col(ex->V, ex->ldv, k + 1);
      HBCK(pmass(ex, col(ex->V, ex->ldv, k), wk));
      HBCK(hb_krylov_multidot_f64(ex->V, ex->ldv, k + 1, wk, ex->n, ex->d_partial, ex->d_dots, ex->s));
      HBCK(hb_krylov_multiaxpy_dev_f64(wk, ex->V, ex->ldv, k + 1, ex->d_dots, -1.0, ex->n, ex->s));
      CUCK(cudaMemcpyAsync(ex->h_dots, ex->d_dots, sizeof(double) * (size_t)(k + 1), cudaMemcpyDeviceToHost, ex->s));
      double hn;
      HBCK(norm2(ex, wk, &hn));
      for (int i = 0; i <= k; i++) H[i][k] = ex->h_dots[i];
      H[k + 1][k] = hn;
      if (hn > 0) HBCK(hb_vec_scale_f64(wk, ex->n, 1.0 / hn, ex->s));
      for (int i = 0; i < k; i++) {
        const double a = H[i][k], c = H[i + 1][k];
        H[i][k]     = cs[i] * a + sn[i] * c;
        H[i + 1][k] = -sn[i] * a + cs[i] * c;
      }
      const double a = H[k][k], c = H[k + 1][k], rr = hypot(a, c);
      cs[k]       = rr > 0 ? a / rr : 1;
      sn[k]       = rr > 0 ? c / rr : 0;
      H[k][k]     = rr;
      H[k + 1][k] = 0;
      g[k + 1]    = -sn[k] * g[k];
      g[k]        = cs[k] * g[k];
      k++;
      its++;
      if (!isfinite(g[k])) {
        *reason = -1;
        done    = 1;
        break;
      }
      if (fabs(g[k]) <= ttol || hn == 0) {
        *reason = 1;
        done    = 1;
        break;
      }
    }
    /* x += V y with H y = g (upper triangular k x k) */
    for (int i = k - 1; i >= 0; i--) {
      double sum = g[i];
      for (int j = i + 1; j < k; j++) sum -= H[i][j] * y[j];
      y[i] = sum / H[i][i];
    }
    HBCK(hb_krylov_multiaxpy_f64(x, ex->V, ex->ldv, k, y, ex->n, ex->s));
    if (done || its >= ex->o.mass_max_it) break;
    /* restart: r = D^-1 (b - M x) */
    HBCK(mass(ex, x, ex->r));
    HBCK(mask(ex, ex->r));
    HBCK(hb_vec_axpby_f64(ex->r, -1.0, 1.0, b, ex->n, ex->s)); /* r = b - M x */
    HBCK(hb_vec_pointwise_mult_f64(v0, ex->r, ex->dinv, ex->n, ex->s));
    HBCK(norm2(ex, v0, &beta));
    if (!isfinite(beta)) {
      *reason = -1;
      break;
    }
    if (beta <= ttol) {
      *reason = 1;
      break;
    }
  }
  *its_out = its;
  return HB_SUCCESS;
}

/* out = M^-1 F(q, 0): the negated explicit right-hand side */
static int neg_rhs(HbExplicitStepper *ex, const double *q, double t, double *out, int *its, int *reason) {
  ex->ctx.dt   = ex->o.dt;
  ex->ctx.time = t;
  HbIFunctionIO io = {q, ex->zero, ex->qdata, NULL, NULL, ex->f, 0};
  HBCK(hb_ifunction_apply(ex->op, &ex->ctx, &io, ex->s));
  /* the face flux: the reference's explicit Freestream QFunction returns -wdetJb F (bc_freestream.h:45-48) into the RHS,
   * so the negated right-hand side gains +wdetJb F */
  if (ex->bc) {
    HbFreestreamContext fc;
    memcpy(&fc, ex->bc_ctx, sizeof fc);
    fc.newt.time = t;
    HBCK(hb_freestream_apply(ex->bc, &fc, ex->bc_flux, ex->bc_qdata, q, NULL, ex->f, ex->s));
  }
  HBCK(mask(ex, ex->f));
  ex->qstate = q;
  if (!ex->pc_ready) HBCK(setup_jacobi(ex)); /* first solve: PCSetUp */
  *its    = 0;
  *reason = 1;
  if (ex->o.mass_ksp == 0) return hb_vec_pointwise_mult_f64(out, ex->f, ex->dinv, ex->n, ex->s);
  return mass_gmres(ex, ex->f, out, its, reason);
}

int hb_explicit_create(const HbElemOp *op, const void *ctx184, const double *d_qdata, const HbExplicitOptions *opts, void *stream,
                       HbExplicitStepper **out) {
  *out = NULL;
  if (!op || !ctx184 || !d_qdata || !opts) return HB_ERROR_INVALID;
  if (opts->dt <= 0 || opts->rk_stages < 1 || opts->rk_stages > MAXS || (opts->mass_ksp != 0 && opts->mass_ksp != 1)) return HB_ERROR_INVALID;
  if (opts->mass_ksp == 1 && (opts->mass_restart < 1 || opts->mass_restart + 1 > MAXK || opts->mass_max_it < 1)) return HB_ERROR_INVALID;
  if (opts->mass_type != 0 && opts->mass_type != 1) return HB_ERROR_INVALID;
  for (int i = 0; i < opts->rk_stages; i++)
    for (int j = i; j < opts->rk_stages; j++)
      if (opts->rk_a[i * MAXS + j] != 0) return HB_ERROR_INVALID; /* explicit tableaux only */
  HbExplicitStepper *ex = (HbExplicitStepper *)calloc(1, sizeof *ex);
  if (!ex) return HB_ERROR_NOMEM;
  ex->op = op;
  memcpy(&ex->ctx, ctx184, sizeof ex->ctx);
  ex->qdata = d_qdata;
  ex->o     = *opts;
  ex->n     = op->l_size;
  ex->ldv   = (op->l_size + 3) & ~(int64_t)3;
  ex->s     = (cudaStream_t)stream;
  const size_t nb = sizeof(double) * (size_t)ex->n, lb = sizeof(double) * (size_t)ex->ldv;
  int          err = 0;
  err |= cudaMalloc((void **)&ex->q, nb) | cudaMalloc((void **)&ex->y, nb) | cudaMalloc((void **)&ex->f, nb);
  err |= cudaMalloc((void **)&ex->zero, nb) | cudaMalloc((void **)&ex->dinv, nb) | cudaMalloc((void **)&ex->r, nb);
  err |= cudaMalloc((void **)&ex->K, lb * opts->rk_stages) | cudaMalloc((void **)&ex->scratch, sizeof(double) * 1024);
  if (opts->mass_ksp == 1) {
    err |= cudaMalloc((void **)&ex->V, lb * (opts->mass_restart + 1));
    err |= cudaMalloc((void **)&ex->d_partial, sizeof(double) * 512 * MAXK) | cudaMalloc((void **)&ex->d_dots, sizeof(double) * MAXK);
    err |= cudaMallocHost((void **)&ex->h_dots, sizeof(double) * MAXK);
  }
  if (err) {
    hb_explicit_destroy(ex);
    return HB_ERROR_NOMEM;
  }
  ex->mass_stab = opts->mass_type == 0 && ex->ctx.stabilization == HB_STAB_SUPG;
  ex->pc_ready  = 0; /* the Jacobi set-up runs at the first solve */
  int rc = hb_vec_set_f64(ex->zero, ex->n, 0.0, ex->s);
  if (rc) {
    hb_explicit_destroy(ex);
    return rc;
  }
  *out = ex;
  return HB_SUCCESS;
}

int hb_explicit_set_essential(HbExplicitStepper *ex, const int32_t *h_idx, const double *h_val, int64_t n) {
  if (!ex || n < 0 || (n && !h_idx)) return HB_ERROR_INVALID;
  for (int64_t i = 0; i < n; i++)
    if (h_idx[i] < 0 || h_idx[i] >= ex->n) return HB_ERROR_INVALID;
  if (ex->ess_idx) cudaFree(ex->ess_idx);
  if (ex->ess_val) cudaFree(ex->ess_val);
  if (ex->ess_one) cudaFree(ex->ess_one);
  ex->ess_idx = NULL;
  ex->ess_val = ex->ess_one = NULL;
  ex->ess_n   = 0;
  if (n) {
    if (cudaMalloc((void **)&ex->ess_idx, sizeof(int32_t) * (size_t)n) != cudaSuccess ||
        cudaMalloc((void **)&ex->ess_val, sizeof(double) * (size_t)n) != cudaSuccess ||
        cudaMalloc((void **)&ex->ess_one, sizeof(double) * (size_t)n) != cudaSuccess)
      return HB_ERROR_NOMEM;
    CUCK(cudaMemcpy(ex->ess_idx, h_idx, sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice));
    if (h_val) CUCK(cudaMemcpy(ex->ess_val, h_val, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice));
    else CUCK(cudaMemset(ex->ess_val, 0, sizeof(double) * (size_t)n));
    HBCK(hb_vec_set_f64(ex->ess_one, n, 1.0, ex->s));
    ex->ess_n = n;
    HBCK(hb_constrain_set_f64(ex->q, ex->ess_idx, ex->ess_val, n, ex->s));
  }
  ex->pc_ready = 0; /* the free-DOF mass system changed: set the preconditioner up again at the next solve */
  return HB_SUCCESS;
}

int hb_explicit_set_freestream(HbExplicitStepper *ex, const HbFaceOp *faces, const void *ctx264, int flux_type, const double *qdata_sur) {
  if (!ex) return HB_ERROR_INVALID;
  ex->bc = NULL;
  if (!faces) return HB_SUCCESS;
  if (!ctx264 || !qdata_sur || (flux_type != 0 && flux_type != 1) || faces->l_size != ex->n) return HB_ERROR_INVALID;
  memcpy(ex->bc_ctx, ctx264, sizeof ex->bc_ctx);
  ex->bc       = faces;
  ex->bc_flux  = flux_type;
  ex->bc_qdata = qdata_sur;
  return HB_SUCCESS;
}

int hb_explicit_destroy(HbExplicitStepper *ex) {
  if (!ex) return HB_SUCCESS;
  if (ex->ess_idx) cudaFree(ex->ess_idx);
  if (ex->ess_val) cudaFree(ex->ess_val);
  if (ex->ess_one) cudaFree(ex->ess_one);
  void *p[] = {ex->q, ex->y, ex->f, ex->zero, ex->dinv, ex->K, ex->V, ex->r, ex->scratch, ex->d_partial, ex->d_dots};
  for (size_t i = 0; i < sizeof p / sizeof p[0]; i++)
    if (p[i]) cudaFree(p[i]);
  if (ex->h_dots) cudaFreeHost(ex->h_dots);
  free(ex);
  return HB_SUCCESS;
}

int hb_explicit_set_state(HbExplicitStepper *ex, const double *d_q, double t) {
  if (!ex || !d_q) return HB_ERROR_INVALID;
  CUCK(cudaMemcpyAsync(ex->q, d_q, sizeof(double) * (size_t)ex->n, cudaMemcpyDeviceToDevice, ex->s));
  if (ex->ess_n) HBCK(hb_constrain_set_f64(ex->q, ex->ess_idx, ex->ess_val, ex->ess_n, ex->s)); /* boundary values inserted */
  ex->t           = t;
  ex->steps_taken = 0;
  return HB_SUCCESS;
}

int hb_explicit_get_state(HbExplicitStepper *ex, double *d_q, double *t) {
  if (!ex) return HB_ERROR_INVALID;
  if (d_q) CUCK(cudaMemcpyAsync(d_q, ex->q, sizeof(double) * (size_t)ex->n, cudaMemcpyDeviceToDevice, ex->s));
  if (t) *t = ex->t;
  return HB_SUCCESS;
}

int hb_explicit_rhs(HbExplicitStepper *ex, const double *d_q, double t, double *d_g, int *its, int *converged_reason) {
  if (!ex || !d_q || !d_g || d_g == d_q) return HB_ERROR_INVALID;
  int it, reason;
  HBCK(neg_rhs(ex, d_q, t, d_g, &it, &reason));
  if (its) *its = it;
  if (converged_reason) *converged_reason = reason;
  HBCK(hb_vec_scale_f64(d_g, ex->n, -1.0, ex->s));
  CUCK(cudaStreamSynchronize(ex->s));
  return HB_SUCCESS;
}

int hb_explicit_step(HbExplicitStepper *ex, HbExplicitStats *st) {
  if (!ex || !st) return HB_ERROR_INVALID;
  memset(st, 0, sizeof *st);
  st->converged_reason = 1;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, ex->s);
  const int    S  = ex->o.rk_stages;
  const double dt = ex->o.dt;
  double       c[MAXS];
  for (int i = 0; i < S; i++) {
    /* Y_i = q_n - dt sum_j a_ij f_j */
    const double *Yi = ex->q;
    int           nz = 0;
    for (int j = 0; j < i; j++) {
      c[j] = -dt * ex->o.rk_a[i * MAXS + j];
      nz |= c[j] != 0;
    }
    if (nz) {
      CUCK(cudaMemcpyAsync(ex->y, ex->q, sizeof(double) * (size_t)ex->n, cudaMemcpyDeviceToDevice, ex->s));
      HBCK(hb_krylov_multiaxpy_f64(ex->y, ex->K, ex->ldv, i, c, ex->n, ex->s));
      Yi = ex->y;
    }
    int its, reason;
    HBCK(neg_rhs(ex, Yi, ex->t + ex->o.rk_c[i] * dt, col(ex->K, ex->ldv, i), &its, &reason));
    st->mass_its += its;
    if (reason != 1 && st->converged_reason == 1) st->converged_reason = reason;
  }
  for (int i = 0; i < S; i++) c[i] = -dt * ex->o.rk_b[i];
  HBCK(hb_krylov_multiaxpy_f64(ex->q, ex->K, ex->ldv, S, c, ex->n, ex->s));
  ex->t += dt;
  ex->steps_taken++;
  cudaEventRecord(e1, ex->s);
  CUCK(cudaEventSynchronize(e1));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  st->seconds = ms * 1e-3;
  if (st->converged_reason == 1) {
    double nq;
    HBCK(norm2(ex, ex->q, &nq));
    if (!isfinite(nq)) st->converged_reason = -1;
  }
  return HB_SUCCESS;
}
