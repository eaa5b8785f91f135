/* hb_filter.c -- the differential filter solve: conjugate gradients with the point Jacobi preconditioner on the operator
 * of k_filter.cu, as HONEE configures its filter KSP (src/differential_filter.c:174-185: KSPCG, PCJACOBI diagonal,
 * natural norm, rtol 1e-10).  Device vectors are node-interleaved [node][nc]. */
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include "honee_b200.h"

#define HBCK(x)        \
  do {                 \
    int e_ = (x);      \
    if (e_) return e_; \
  } while (0)

size_t hb_filter_work_doubles(const HbElemOp *op, int nc) {
  const size_t nodes = (size_t)(op->l_size / 5), n = nodes * (size_t)nc;
  return 5 * n + nodes + 1024;
}

int hb_filter_solve(const HbElemOp *op, int nc, const HbFilterOptions *o, const double *qdata, const double *b, double *x, double rtol, int max_it,
                    double *work, int *its, double *rel_norm, void *s) {
  if (!op || !o || !qdata || !b || !x || !work || nc < 1 || max_it < 1) return HB_ERROR_INVALID;
  const int64_t nodes = op->l_size / 5, n = nodes * nc;
  double *r = work, *z = r + n, *p = z + n, *Ap = p + n, *dinv = Ap + n, *diag = dinv + n, *scratch = diag + nodes;
  HBCK(hb_filter_diagonal(op, o, qdata, diag, s));
  HBCK(hb_filter_jacobi(diag, nodes, nc, dinv, s));
  HBCK(hb_vec_set_f64(x, n, 0.0, s));
  if (cudaMemcpyAsync(r, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, (cudaStream_t)s) != cudaSuccess) return HB_ERROR_CUDA;
  HBCK(hb_vec_pointwise_mult_f64(z, dinv, r, n, s));
  if (cudaMemcpyAsync(p, z, sizeof(double) * n, cudaMemcpyDeviceToDevice, (cudaStream_t)s) != cudaSuccess) return HB_ERROR_CUDA;
  double rz, rz0;
  HBCK(hb_vec_reduce_f64(r, z, n, 3, scratch, &rz, s));
  rz0 = rz;
  int k = 0;
  if (rz0 > 0) {
    for (k = 1; k <= max_it; k++) {
      double pAp, rz_new;
      HBCK(hb_filter_apply(op, nc, o, qdata, p, Ap, s));
      HBCK(hb_vec_reduce_f64(p, Ap, n, 3, scratch, &pAp, s));
      if (!(pAp > 0)) return HB_ERROR_BACKEND; /* the operator is SPD; anything else is a broken input */
      const double alpha = rz / pAp;
      HBCK(hb_vec_axpy_f64(x, alpha, p, n, s));
      HBCK(hb_vec_axpy_f64(r, -alpha, Ap, n, s));
      HBCK(hb_vec_pointwise_mult_f64(z, dinv, r, n, s));
      HBCK(hb_vec_reduce_f64(r, z, n, 3, scratch, &rz_new, s));
      if (sqrt(fabs(rz_new)) <= rtol * sqrt(rz0)) {
        rz = rz_new;
        break;
      }
      HBCK(hb_vec_axpby_f64(p, 1.0, rz_new / rz, z, n, s)); /* p = z + beta p */
      rz = rz_new;
    }
  }
  if (its) *its = k > max_it ? max_it : k;
  if (rel_norm) *rel_norm = rz0 > 0 ? sqrt(fabs(rz) / rz0) : 0.0;
  return (k > max_it) ? HB_ERROR_INCOMPLETE : HB_SUCCESS;
}
