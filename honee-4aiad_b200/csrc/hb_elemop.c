/* hb_elemop.c -- host set-up of the device element-operator description (include/honee_b200.h).
 *
 * Validates the restriction offsets once on the host (so the kernels can index without per-access checks), builds an
 * element colouring for the atomic-free scatter, forms the collocated derivative matrix of the tensor basis and
 * uploads everything to the current CUDA device.
 */
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "honee_b200.h"

const char *hb_version(void) { return "honee-b200 0.1 (sm_100a)"; }

/* Greedy first-fit colouring: element e takes the lowest colour not used by any element sharing one of its offsets.
 * For lexicographically numbered boxes this yields the 2x2x2 parity colouring (8 colours). */
int hb_internal_color_elements(int num_elem, int elem_size, const int32_t *offsets, int64_t l_size, int32_t **color_ptr_out, int32_t **color_elem_out,
                          int *num_colors_out) {
  uint64_t *mask  = (uint64_t *)calloc((size_t)l_size, sizeof(uint64_t));
  uint8_t  *color = (uint8_t *)malloc((size_t)num_elem);
  if (!mask || !color) {
    free(mask);
    free(color);
    return HB_ERROR_NOMEM;
  }
  int ncol = 0;
  for (int64_t e = 0; e < num_elem; e++) {
    uint64_t used = 0;
    const int32_t *o = offsets + e * elem_size;
    for (int p = 0; p < elem_size; p++) used |= mask[o[p]];
    int c = 0;
    while (c < 64 && (used >> c) & 1) c++;
    if (c == 64) {
      free(mask);
      free(color);
      return HB_ERROR_UNSUPPORTED;
    }
    color[e] = (uint8_t)c;
    if (c + 1 > ncol) ncol = c + 1;
    for (int p = 0; p < elem_size; p++) {
      /* colour c was free on all of e's nodes, so a bit already set here means e lists this node twice (a periodic
       * direction with one element); its scatter would then race with itself */
      if (mask[o[p]] & ((uint64_t)1 << c)) {
        free(mask);
        free(color);
        return HB_ERROR_UNSUPPORTED;
      }
      mask[o[p]] |= (uint64_t)1 << c;
    }
  }
  free(mask);
  int32_t *ptr = (int32_t *)calloc((size_t)ncol + 1, sizeof(int32_t));
  int32_t *lst = (int32_t *)malloc(sizeof(int32_t) * (size_t)num_elem);
  for (int64_t e = 0; e < num_elem; e++) ptr[color[e] + 1]++;
  for (int c = 0; c < ncol; c++) ptr[c + 1] += ptr[c];
  int32_t *fill = (int32_t *)malloc(sizeof(int32_t) * (size_t)ncol);
  memcpy(fill, ptr, sizeof(int32_t) * (size_t)ncol);
  for (int64_t e = 0; e < num_elem; e++) lst[fill[color[e]]++] = (int32_t)e;
  free(fill);
  free(color);
  *color_ptr_out  = ptr;
  *color_elem_out = lst;
  *num_colors_out = ncol;
  return HB_SUCCESS;
}

/* D = G B^+ with B^+ = (B^T B)^{-1} B^T (Cholesky in long double): the derivative on the quadrature grid such that
 * D (B u) = G u for every nodal u.  Exact for tensor H1 bases with Q >= P, which the caller's tabulation satisfies. */
static int collocated_derivative(int P, int Q, const double *B, const double *G, double *D) {
  long double M[HB_MAX_P][HB_MAX_P], L[HB_MAX_P][HB_MAX_P];
  for (int a = 0; a < P; a++)
    for (int b = 0; b < P; b++) {
      long double s = 0;
      for (int q = 0; q < Q; q++) s += (long double)B[q * P + a] * B[q * P + b];
      M[a][b] = s;
    }
  for (int i = 0; i < P; i++)
    for (int j = 0; j <= i; j++) {
      long double s = M[i][j];
      for (int k = 0; k < j; k++) s -= L[i][k] * L[j][k];
      if (i == j) {
        if (s <= 0) return HB_ERROR_INVALID;
        L[i][i] = sqrtl(s);
      } else L[i][j] = s / L[j][j];
    }
  /* Bp = M^{-1} B^T, column by column (each column q solves M x = B[q,:]^T) */
  long double Bp[HB_MAX_P][HB_MAX_P];
  for (int q = 0; q < Q; q++) {
    long double y[HB_MAX_P], x[HB_MAX_P];
    for (int i = 0; i < P; i++) {
      long double s = B[q * P + i];
      for (int k = 0; k < i; k++) s -= L[i][k] * y[k];
      y[i] = s / L[i][i];
    }
    for (int i = P - 1; i >= 0; i--) {
      long double s = y[i];
      for (int k = i + 1; k < P; k++) s -= L[k][i] * x[k];
      x[i] = s / L[i][i];
    }
    for (int i = 0; i < P; i++) Bp[i][q] = x[i];
  }
  for (int i = 0; i < Q; i++)
    for (int l = 0; l < Q; l++) {
      long double s = 0;
      for (int a = 0; a < P; a++) s += (long double)G[i * P + a] * Bp[a][l];
      D[i * Q + l] = (double)s;
    }
  return HB_SUCCESS;
}

int hb_elemop_create(int num_elem, int P, int Q, const int32_t *offsets, int64_t l_size, const double *interp1d, const double *grad1d,
                     const double *qref1d, const double *qweight1d, HbElemOp **op_out) {
  *op_out = NULL;
  if (num_elem <= 0 || P < 2 || P > HB_MAX_P || Q < P || Q > HB_MAX_P || l_size <= 0) return HB_ERROR_UNSUPPORTED;
  const int P3 = P * P * P;
  for (int64_t i = 0; i < (int64_t)num_elem * P3; i++)
    if (offsets[i] < 0 || (int64_t)offsets[i] + 5 > l_size) return HB_ERROR_INVALID;
  HbElemOp *op = (HbElemOp *)calloc(1, sizeof(HbElemOp));
  if (!op) return HB_ERROR_NOMEM;
  op->num_elem = num_elem;
  op->P        = P;
  op->Q        = Q;
  op->l_size   = l_size;
  memcpy(op->interp1d, interp1d, sizeof(double) * P * Q);
  memcpy(op->grad1d, grad1d, sizeof(double) * P * Q);
  if (qref1d) memcpy(op->qref1d, qref1d, sizeof(double) * Q);
  if (qweight1d) memcpy(op->qweight1d, qweight1d, sizeof(double) * Q);
  int err = collocated_derivative(P, Q, interp1d, grad1d, op->colo_grad1d);
  int32_t *color_elem = NULL;
  if (!err) err = hb_internal_color_elements(num_elem, P3, offsets, l_size, &op->h_color_ptr, &color_elem, &op->num_colors);
  if (!err) {
    cudaGetDevice(&op->device);
    cudaDeviceGetAttribute(&op->num_sms, cudaDevAttrMultiProcessorCount, op->device);
    if (op->num_sms <= 0) op->num_sms = 148;
    const size_t nb_off = sizeof(int32_t) * (size_t)num_elem * P3, nb_col = sizeof(int32_t) * (size_t)num_elem;
    if (cudaMalloc((void **)&op->d_offsets, nb_off) != cudaSuccess || cudaMalloc((void **)&op->d_color_elem, nb_col) != cudaSuccess ||
        cudaMalloc((void **)&op->d_status, sizeof(int)) != cudaSuccess)
      err = HB_ERROR_NOMEM;
    else if (cudaMemset(op->d_status, 0, sizeof(int)) != cudaSuccess)
      err = HB_ERROR_CUDA;
    else if (cudaMemcpy(op->d_offsets, offsets, nb_off, cudaMemcpyHostToDevice) != cudaSuccess ||
             cudaMemcpy(op->d_color_elem, color_elem, nb_col, cudaMemcpyHostToDevice) != cudaSuccess)
      err = HB_ERROR_CUDA;
  }
  free(color_elem);
  if (err) {
    hb_elemop_destroy(op);
    return err;
  }
  *op_out = op;
  return HB_SUCCESS;
}

int hb_elemop_set_vertex_coords(HbElemOp *op, const double *x_elem) {
  if (!op || !x_elem) return HB_ERROR_INVALID;
  const size_t nb = sizeof(double) * 24 * (size_t)op->num_elem;
  if (!op->d_x_elem && cudaMalloc((void **)&op->d_x_elem, nb) != cudaSuccess) return HB_ERROR_NOMEM;
  return cudaMemcpy(op->d_x_elem, x_elem, nb, cudaMemcpyHostToDevice) == cudaSuccess ? HB_SUCCESS : HB_ERROR_CUDA;
}

int hb_elemop_status(HbElemOp *op, int *status, int clear) {
  if (!op || !status) return HB_ERROR_INVALID;
  if (cudaDeviceSynchronize() != cudaSuccess) return HB_ERROR_CUDA;
  if (cudaMemcpy(status, op->d_status, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return HB_ERROR_CUDA;
  if (clear && *status && cudaMemset(op->d_status, 0, sizeof(int)) != cudaSuccess) return HB_ERROR_CUDA;
  return HB_SUCCESS;
}

int hb_elemop_destroy(HbElemOp *op) {
  if (!op) return HB_SUCCESS;
  if (op->d_status) cudaFree(op->d_status);
  if (op->d_offsets) cudaFree(op->d_offsets);
  if (op->d_color_elem) cudaFree(op->d_color_elem);
  if (op->d_x_elem) cudaFree(op->d_x_elem);
  free(op->h_color_ptr);
  free(op);
  return HB_SUCCESS;
}
