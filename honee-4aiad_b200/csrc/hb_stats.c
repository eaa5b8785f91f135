/* hb_stats.c -- host side of the spanwise turbulence statistics (include/honee_b200.h, kernels in k_stats.cu).
 *
 * Mirrors HONEE's statistics monitor (src/spanstats/spanstats.c, src/spanstats/turbulence.c): set-up builds the parent
 * plane (geometric factors, colouring, mass diagonal), each collection adds one step's weighted statistics into the
 * parent-point sums, and processing scales them by 1 / (duration * span width), projects them onto the parent nodes and
 * solves with the parent mass matrix by conjugate gradients with point Jacobi in the natural norm, as the reference's
 * statistics KSP is configured (spanstats.c:322-333: KSPCG, PCJACOBI diagonal, KSP_NORM_NATURAL, rtol 1e-10). */
#include <cuda_runtime.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "hb_internal.h"

#define HBCK(x)        \
  do {                 \
    int e_ = (x);      \
    if (e_) return e_; \
  } while (0)

struct HbSpanStats {
  const HbElemOp *op;
  HbPlaneOp       plane;
  int             num_columns, column_length;
  int32_t        *d_column_elems;
  double         *d_sums;    /* [num_columns][Q^2][22] */
  double         *d_work;    /* r, z, p, Ap [nodes * 22] each, dinv [nodes * 22], diag [nodes], scratch [1024] */
  double          span_width, initial_time, previous_time;
};

static void plane_free(HbPlaneOp *pl) {
  if (pl->d_offsets) cudaFree(pl->d_offsets);
  if (pl->d_color_elem) cudaFree(pl->d_color_elem);
  if (pl->d_wdetJ) cudaFree(pl->d_wdetJ);
  free(pl->h_color_ptr);
  memset(pl, 0, sizeof *pl);
}

int hb_spanstats_destroy(HbSpanStats *st) {
  if (!st) return HB_SUCCESS;
  plane_free(&st->plane);
  if (st->d_column_elems) cudaFree(st->d_column_elems);
  if (st->d_sums) cudaFree(st->d_sums);
  if (st->d_work) cudaFree(st->d_work);
  free(st);
  return HB_SUCCESS;
}

static size_t work_doubles(const HbSpanStats *st) {
  const size_t n = (size_t)st->plane.num_nodes * HB_TURB_NUM_COMPONENTS;
  return 5 * n + (size_t)st->plane.num_nodes + 1024;
}

int hb_spanstats_create(const HbElemOp *op, int num_columns, int column_length, const int32_t *column_elems, const int32_t *parent_offsets,
                        int64_t num_parent_nodes, const double *parent_x, double span_width, HbSpanStats **out) {
  if (!out) return HB_ERROR_INVALID;
  *out = NULL;
  if (!op || num_columns < 1 || column_length < 1 || !column_elems || !parent_offsets || num_parent_nodes < 1 || !parent_x || !(span_width > 0))
    return HB_ERROR_INVALID;
  const int P = op->P, Q = op->Q, P2 = P * P;
  for (int64_t i = 0; i < (int64_t)num_columns * column_length; i++)
    if (column_elems[i] < 0 || column_elems[i] >= op->num_elem) return HB_ERROR_INVALID;
  for (int64_t i = 0; i < (int64_t)num_columns * P2; i++)
    if (parent_offsets[i] < 0 || parent_offsets[i] >= num_parent_nodes) return HB_ERROR_INVALID;
  HbSpanStats *st = (HbSpanStats *)calloc(1, sizeof *st);
  if (!st) return HB_ERROR_NOMEM;
  st->op            = op;
  st->num_columns   = num_columns;
  st->column_length = column_length;
  st->span_width    = span_width;
  HbPlaneOp *pl     = &st->plane;
  pl->num_elem      = num_columns;
  pl->P             = P;
  pl->Q             = Q;
  pl->num_nodes     = num_parent_nodes;
  memcpy(pl->interp1d, op->interp1d, sizeof(double) * P * Q);
  memcpy(pl->qref1d, op->qref1d, sizeof(double) * Q);
  memcpy(pl->qweight1d, op->qweight1d, sizeof(double) * Q);
  int32_t *color_elem = NULL;
  double  *d_x        = NULL;
  int      err        = hb_internal_color_elements(num_columns, P2, parent_offsets, num_parent_nodes, &pl->h_color_ptr, &color_elem, &pl->num_colors);
  const size_t nb_col = sizeof(int32_t) * (size_t)num_columns * column_length, nb_off = sizeof(int32_t) * (size_t)num_columns * P2;
  const size_t nb_sums = sizeof(double) * (size_t)num_columns * Q * Q * HB_TURB_NUM_COMPONENTS;
  if (!err && (cudaMalloc((void **)&st->d_column_elems, nb_col) != cudaSuccess || cudaMalloc((void **)&pl->d_offsets, nb_off) != cudaSuccess ||
               cudaMalloc((void **)&pl->d_color_elem, sizeof(int32_t) * (size_t)num_columns) != cudaSuccess ||
               cudaMalloc((void **)&pl->d_wdetJ, sizeof(double) * (size_t)num_columns * Q * Q) != cudaSuccess ||
               cudaMalloc((void **)&st->d_sums, nb_sums) != cudaSuccess ||
               cudaMalloc((void **)&st->d_work, sizeof(double) * work_doubles(st)) != cudaSuccess ||
               cudaMalloc((void **)&d_x, sizeof(double) * 12 * (size_t)num_columns) != cudaSuccess))
    err = HB_ERROR_NOMEM;
  if (!err && (cudaMemcpy(st->d_column_elems, column_elems, nb_col, cudaMemcpyHostToDevice) != cudaSuccess ||
               cudaMemcpy(pl->d_offsets, parent_offsets, nb_off, cudaMemcpyHostToDevice) != cudaSuccess ||
               cudaMemcpy(pl->d_color_elem, color_elem, sizeof(int32_t) * (size_t)num_columns, cudaMemcpyHostToDevice) != cudaSuccess ||
               cudaMemcpy(d_x, parent_x, sizeof(double) * 12 * (size_t)num_columns, cudaMemcpyHostToDevice) != cudaSuccess))
    err = HB_ERROR_CUDA;
  if (!err) err = hb_plane_setup_qdata(num_columns, Q, pl->qref1d, pl->qweight1d, d_x, pl->d_wdetJ, NULL);
  if (!err) {  /* Jacobi: 1 / diag(M), the same for every component */
    const int64_t n = pl->num_nodes * HB_TURB_NUM_COMPONENTS;
    double *dinv = st->d_work + 4 * n, *diag = dinv + n;
    err = hb_plane_mass_diagonal(pl, diag, 0, NULL);
    if (!err) err = hb_filter_jacobi(diag, pl->num_nodes, HB_TURB_NUM_COMPONENTS, dinv, NULL);
  }
  if (!err) err = hb_spanstats_reset(st, 0.0, NULL);
  if (!err && cudaDeviceSynchronize() != cudaSuccess) err = HB_ERROR_CUDA;
  if (d_x) cudaFree(d_x);
  free(color_elem);
  if (err) {
    hb_spanstats_destroy(st);
    return err;
  }
  *out = st;
  return HB_SUCCESS;
}

int hb_spanstats_reset(HbSpanStats *st, double initial_time, void *stream) {
  if (!st) return HB_ERROR_INVALID;
  st->initial_time  = initial_time;
  st->previous_time = initial_time;
  const size_t nb   = sizeof(double) * (size_t)st->num_columns * st->plane.Q * st->plane.Q * HB_TURB_NUM_COMPONENTS;
  return cudaMemsetAsync(st->d_sums, 0, nb, (cudaStream_t)stream) == cudaSuccess ? HB_SUCCESS : HB_ERROR_CUDA;
}

int hb_spanstats_collect(HbSpanStats *st, const void *ctx184, const double *q, const double *qdata, double solution_time, void *stream) {
  if (!st) return HB_ERROR_INVALID;
  HBCK(hb_stats_collect(st->op, ctx184, q, qdata, solution_time - st->previous_time, st->num_columns, st->column_length, st->d_column_elems,
                        st->d_sums, stream));
  st->previous_time = solution_time;
  return HB_SUCCESS;
}

int hb_spanstats_view(const HbSpanStats *st, const double **d_sums, const HbPlaneOp **plane) {
  if (!st) return HB_ERROR_INVALID;
  if (d_sums) *d_sums = st->d_sums;
  if (plane) *plane = &st->plane;
  return HB_SUCCESS;
}

int hb_spanstats_copy_sums(const HbSpanStats *st, double *dst) {
  if (!st || !dst) return HB_ERROR_INVALID;
  const size_t nb = sizeof(double) * (size_t)st->num_columns * st->plane.Q * st->plane.Q * HB_TURB_NUM_COMPONENTS;
  return cudaMemcpy(dst, st->d_sums, nb, cudaMemcpyDefault) == cudaSuccess ? HB_SUCCESS : HB_ERROR_CUDA;
}

int hb_spanstats_process(HbSpanStats *st, double solution_time, double rtol, int max_it, double *x, int *its, double *rel_norm, void *s) {
  if (!st || !x || max_it < 1 || !(rtol > 0)) return HB_ERROR_INVALID;
  const double duration = solution_time - st->initial_time;
  if (!(duration > 0)) return HB_ERROR_INVALID;
  const HbPlaneOp *pl = &st->plane;
  const int64_t    n  = pl->num_nodes * HB_TURB_NUM_COMPONENTS;
  double *r = st->d_work, *z = r + n, *p = z + n, *Ap = p + n, *dinv = Ap + n, *scratch = dinv + n + pl->num_nodes;
  HBCK(hb_plane_project_rhs(pl, st->d_sums, 1.0 / (duration * st->span_width), r, 0, s));
  HBCK(hb_vec_set_f64(x, n, 0.0, s));
  HBCK(hb_vec_pointwise_mult_f64(z, dinv, r, n, s));
  if (cudaMemcpyAsync(p, z, sizeof(double) * n, cudaMemcpyDeviceToDevice, (cudaStream_t)s) != cudaSuccess) return HB_ERROR_CUDA;
  double rz, rz0;
  HBCK(hb_vec_reduce_f64(r, z, n, 3, scratch, &rz, s));
  rz0   = rz;
  int k = 0;
  if (rz0 > 0) {
    for (k = 1; k <= max_it; k++) {
      double pAp, rz_new;
      HBCK(hb_plane_mass_apply(pl, p, Ap, 0, s));
      HBCK(hb_vec_reduce_f64(p, Ap, n, 3, scratch, &pAp, s));
      if (!(pAp > 0)) return HB_ERROR_BACKEND; /* the mass matrix is SPD; anything else is a broken plane */
      const double alpha = rz / pAp;
      HBCK(hb_vec_axpy_f64(x, alpha, p, n, s));
      HBCK(hb_vec_axpy_f64(r, -alpha, Ap, n, s));
      HBCK(hb_vec_pointwise_mult_f64(z, dinv, r, n, s));
      HBCK(hb_vec_reduce_f64(r, z, n, 3, scratch, &rz_new, s));
      const double beta = rz_new / rz;
      rz                = rz_new;
      if (sqrt(fabs(rz_new)) <= rtol * sqrt(rz0)) break;
      HBCK(hb_vec_axpby_f64(p, 1.0, beta, z, n, s)); /* p = z + beta p */
    }
  }
  if (its) *its = k > max_it ? max_it : k;
  if (rel_norm) *rel_norm = rz0 > 0 ? sqrt(fabs(rz) / rz0) : 0.0;
  return (k > max_it) ? HB_ERROR_INCOMPLETE : HB_SUCCESS;
}
