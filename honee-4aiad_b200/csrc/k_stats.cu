// k_stats.cu -- spanwise statistics of turbulence quantities for sm_100a.
//
// Reference semantics (src/spanstats/spanstats.c, src/spanstats/turbulence.c, qfunctions/spanstats/turbulence.h):
//   collect   every step, at every quadrature point of the 3D ("child") mesh, the 22 statistics of the state times
//             w detJ * (t - t_prev) are added into a child array (ChildStatsCollection_Conserv, turbulence.h:41-79)
//   process   a star forest sums the child points onto the 2D ("parent") quadrature points with the same (x, y)
//             (spanstats.c:253-289, 425-443), the sums are scaled by 1 / (duration * span width) (:445-448), projected
//             onto the parent nodes by B^T (an identity QFunction, :302-309) and solved with the parent mass matrix by
//             CG with point Jacobi, natural norm, rtol 1e-10 (:315-337, 450-455).
// B200 form: the child array is never stored.  The 3D elements are grouped into columns along the span (all elements
// whose quadrature points share the (x, y) of one parent element's points); one CTA owns a column, walks its elements,
// interpolates the state to the quadrature points by sum factorisation, evaluates the statistics and sums them over
// the span in a fixed order into the parent-point sums [E2][Q^2][22] (the reference's collocated parent layout).  No
// atomics, deterministic, and one read of the state, of w detJ and of the 0.2 % of the data the sums occupy per step.
// The parent operators are small (E2 = nx * ny elements): one CTA per element, coloured scatter.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include "honee_b200.h"
#include "newtonian_qf.cuh"

namespace hbs {

constexpr int kThreads = 256;
constexpr int kMaxP = HB_MAX_P;
constexpr int NS = HB_TURB_NUM_COMPONENTS;

struct Interp1D {
  double B[kMaxP * kMaxP];  // [Q][P]
};

struct CollectArgs {
  const int32_t *offsets;       // [E][P^3] node * 5
  const int32_t *column_elems;  // [num_columns][column_length]
  int num_columns, column_length;
  const double *q;              // L-vector, node-interleaved 5 components
  const double *qdata;          // [E][10][Q^3], component 0 = w detJ
  double dt;                    // solution_time - previous_time
  double cv, gm1;               // cv and cp / cv - 1
  hb::PhysConst<double> pc;     // gas constants for primitive / entropy states (state_from_q)
  double *sums;                 // [num_columns][Q^2][22]
};

template <int P, int Q>
struct CollectPlan {
  static constexpr int P3 = P * P * P, Q2 = Q * Q, Q3 = Q2 * Q;
  static constexpr int oB = 0, oX = oB + Q * P, oY = oX + 5 * Q3, oS = oY + 5 * Q3, oAcc = oS + NS * Q3, doubles = oAcc + NS * Q2;
  static constexpr size_t bytes = sizeof(double) * doubles;
};

// The 22 statistics of one point (turbulence.h:51-77 with StateFromU, newtonian_state.h:64-73), already multiplied by
// w = w detJ * dt; products are associated left to right as the reference writes them.
__device__ __forceinline__ void turb_stats(const double U[5], double w, double cv, double gm1, double v[NS]) {
  const double rho = U[0];
  const double u[3] = {U[1] / rho, U[2] / rho, U[3] / rho};
  const double e_kinetic = .5 * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
  const double e_total = U[4] / rho;
  const double e_internal = e_total - e_kinetic;
  const double T = e_internal / cv;
  const double p = gm1 * rho * e_internal;
  v[0] = w * rho;
  v[1] = w * p;
  v[2] = w * (p * p);
  for (int i = 0; i < 3; i++) v[3 + i] = w * p * u[i];
  v[6] = w * rho * T;
  for (int i = 0; i < 3; i++) v[7 + i] = w * rho * T * u[i];
  for (int i = 0; i < 3; i++) v[10 + i] = w * U[1 + i];
  v[13] = w * U[1] * u[0];
  v[14] = w * U[2] * u[1];
  v[15] = w * U[3] * u[2];
  v[16] = w * U[2] * u[2];
  v[17] = w * U[1] * u[2];
  v[18] = w * U[1] * u[1];
  for (int i = 0; i < 3; i++) v[19 + i] = w * u[i];
}

// The same statistics from a state given in any of the three variables (ChildStatsCollection_Prim / _Entropy,
// turbulence.h:85-91: StateFromQ first), products in the reference's order.
__device__ __forceinline__ void turb_stats_state(const hb::St<double> &s, double w, double v[NS]) {
  v[0] = w * s.rho;
  v[1] = w * s.P;
  v[2] = w * (s.P * s.P);
  for (int i = 0; i < 3; i++) v[3 + i] = w * s.P * s.u[i];
  v[6] = w * s.rho * s.T_;
  for (int i = 0; i < 3; i++) v[7 + i] = w * s.rho * s.T_ * s.u[i];
  for (int i = 0; i < 3; i++) v[10 + i] = w * s.m[i];
  v[13] = w * s.m[0] * s.u[0];
  v[14] = w * s.m[1] * s.u[1];
  v[15] = w * s.m[2] * s.u[2];
  v[16] = w * s.m[1] * s.u[2];
  v[17] = w * s.m[0] * s.u[2];
  v[18] = w * s.m[0] * s.u[1];
  for (int i = 0; i < 3; i++) v[19 + i] = w * s.u[i];
}

template <int P, int Q, int SV = HB_STATEVAR_CONSERVATIVE>
__global__ void __launch_bounds__(kThreads) k_stats_collect(const CollectArgs a, const Interp1D bas) {
  using L = CollectPlan<P, Q>;
  constexpr int NT = kThreads, P2 = P * P, P3 = L::P3, Q2 = L::Q2, Q3 = L::Q3, P2Q = P2 * Q, PQ2 = P * Q2;
  extern __shared__ double smem[];
  double *sB = smem + L::oB, *sX = smem + L::oX, *sY = smem + L::oY, *sS = smem + L::oS, *sAcc = smem + L::oAcc;
  for (int t = threadIdx.x; t < Q * P; t += NT) sB[t] = bas.B[t];
  for (int col = blockIdx.x; col < a.num_columns; col += gridDim.x) {
    for (int t = threadIdx.x; t < NS * Q2; t += NT) sAcc[t] = 0;
    for (int k = 0; k < a.column_length; k++) {
      const int e = __ldg(a.column_elems + (int64_t)col * a.column_length + k);
      const int32_t *off = a.offsets + (int64_t)e * P3;
      for (int i = threadIdx.x; i < 5 * P3; i += NT) sX[(i % 5) * P3 + i / 5] = __ldg(a.q + __ldg(off + i / 5) + i % 5);
      __syncthreads();
      for (int f = threadIdx.x; f < 5 * P2Q; f += NT) {  // x: [c][pc][pb][qi]
        const int qi = f % Q, pcb = (f / Q) % P2, c = f / P2Q;
        double s = 0;
#pragma unroll
        for (int i = 0; i < P; i++) s += sB[qi * P + i] * sX[c * P3 + pcb * P + i];
        sY[f] = s;
      }
      __syncthreads();
      for (int f = threadIdx.x; f < 5 * PQ2; f += NT) {  // y: [c][pc][qj][qi]
        const int qi = f % Q, qj = (f / Q) % Q, pc = (f / Q2) % P, c = f / PQ2;
        double s = 0;
#pragma unroll
        for (int j = 0; j < P; j++) s += sB[qj * P + j] * sY[c * P2Q + (pc * P + j) * Q + qi];
        sX[f] = s;
      }
      __syncthreads();
      for (int f = threadIdx.x; f < 5 * Q3; f += NT) {  // z: [c][qk][qj][qi]
        const int qji = f % Q2, qk = (f / Q2) % Q, c = f / Q3;
        double s = 0;
#pragma unroll
        for (int kk = 0; kk < P; kk++) s += sB[qk * P + kk] * sX[c * PQ2 + kk * Q2 + qji];
        sY[f] = s;
      }
      __syncthreads();
      const double *wq = a.qdata + (int64_t)e * 10 * Q3;
      for (int qp = threadIdx.x; qp < Q3; qp += NT) {
        double U[5], v[NS];
#pragma unroll
        for (int c = 0; c < 5; c++) U[c] = sY[c * Q3 + qp];
        if constexpr (SV == HB_STATEVAR_CONSERVATIVE) {
          turb_stats(U, __ldg(wq + qp) * a.dt, a.cv, a.gm1, v);
        } else {
          hb::St<double> st;
          hb::SAux<double> aux;
          hb::state_from_q<SV>(a.pc, U, st, aux);
          turb_stats_state(st, __ldg(wq + qp) * a.dt, v);
        }
#pragma unroll
        for (int s = 0; s < NS; s++) sS[s * Q3 + qp] = v[s];
      }
      __syncthreads();
      for (int t = threadIdx.x; t < NS * Q2; t += NT) {  // span sum over the element's quadrature planes, in order
        const int s = t / Q2, qxy = t % Q2;
        double acc = 0;
#pragma unroll
        for (int qk = 0; qk < Q; qk++) acc += sS[s * Q3 + qk * Q2 + qxy];
        sAcc[t] += acc;
      }
      // the next gather writes sX (last read by the z pass), the next x pass sY (last read by the point-wise phase) and
      // the next point-wise phase sS (last read just above): each behind at least one barrier
    }
    __syncthreads();
    double *out = a.sums + (int64_t)col * Q2 * NS;
    for (int t = threadIdx.x; t < NS * Q2; t += NT) {  // [qxy][stat], stats fastest
      const int qxy = t / NS, s = t % NS;
      out[t] += sAcc[s * Q2 + qxy];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------------------------------------------------
// parent plane: 2D tensor element of P^2 nodes / Q^2 points, 22 components node-interleaved [node][22]

struct PlaneArgs {
  const int32_t *offsets;  // [E2][P^2] parent node index
  const int32_t *elems;    // element ids of this colour
  int n_elems;
  const double *wdetJ;     // [E2][Q^2]
};

template <int P, int Q>
struct PlanePlan {
  static constexpr int Q2 = Q * Q, oB = 0, oU = oB + Q * P, oT = oU + NS * Q2, doubles = oT + NS * Q2;
  static constexpr size_t bytes = sizeof(double) * doubles;
};

// y^T then x^T of sU [c][qj][qi] and the scatter-add into v
template <int P, int Q>
__device__ __forceinline__ void plane_transpose_scatter(const double *sB, const double *sU, double *sT, const int32_t *off, double *v) {
  constexpr int NT = kThreads, PQ = P * Q, Q2 = Q * Q, P2 = P * P;
  for (int f = threadIdx.x; f < NS * PQ; f += NT) {  // y^T: [c][pb][qi]
    const int qi = f % Q, pb = (f / Q) % P, c = f / PQ;
    double s = 0;
#pragma unroll
    for (int j = 0; j < Q; j++) s += sB[j * P + pb] * sU[c * Q2 + j * Q + qi];
    sT[f] = s;
  }
  __syncthreads();
  for (int f = threadIdx.x; f < NS * P2; f += NT) {  // x^T and the scatter, components fastest
    const int c = f % NS, p = f / NS, pa = p % P, pb = p / P;
    double s = 0;
#pragma unroll
    for (int i = 0; i < Q; i++) s += sB[i * P + pa] * sT[c * PQ + pb * Q + i];
    v[(int64_t)__ldg(off + p) * NS + c] += s;
  }
}

template <int P, int Q>
__global__ void __launch_bounds__(kThreads) k_plane_mass(const PlaneArgs a, const Interp1D bas, const double *__restrict__ u, double *__restrict__ v) {
  using L = PlanePlan<P, Q>;
  constexpr int NT = kThreads, P2 = P * P, PQ = P * Q, Q2 = Q * Q;
  extern __shared__ double smem[];
  double *sB = smem + L::oB, *sU = smem + L::oU, *sT = smem + L::oT;
  for (int t = threadIdx.x; t < Q * P; t += NT) sB[t] = bas.B[t];
  for (int idx = blockIdx.x; idx < a.n_elems; idx += gridDim.x) {
    const int e = a.elems[idx];
    const int32_t *off = a.offsets + (int64_t)e * P2;
    for (int i = threadIdx.x; i < NS * P2; i += NT) sU[(i % NS) * P2 + i / NS] = u[(int64_t)__ldg(off + i / NS) * NS + i % NS];
    __syncthreads();
    for (int f = threadIdx.x; f < NS * PQ; f += NT) {  // x: [c][pb][qi]
      const int qi = f % Q, pb = (f / Q) % P, c = f / PQ;
      double s = 0;
#pragma unroll
      for (int i = 0; i < P; i++) s += sB[qi * P + i] * sU[c * P2 + pb * P + i];
      sT[f] = s;
    }
    __syncthreads();
    const double *w = a.wdetJ + (int64_t)e * Q2;
    for (int f = threadIdx.x; f < NS * Q2; f += NT) {  // y, times w detJ: [c][qj][qi]
      const int qi = f % Q, qj = (f / Q) % Q, c = f / Q2;
      double s = 0;
#pragma unroll
      for (int j = 0; j < P; j++) s += sB[qj * P + j] * sT[c * PQ + j * Q + qi];
      sU[f] = s * __ldg(w + qj * Q + qi);
    }
    __syncthreads();
    plane_transpose_scatter<P, Q>(sB, sU, sT, off, v);
    // the next gather writes sU, last read by the y^T pass behind the barrier inside plane_transpose_scatter; the next
    // x pass writes sT after the gather's barrier, which every thread reaches only after its x^T reads
  }
}

template <int P, int Q>
__global__ void __launch_bounds__(kThreads) k_plane_rhs(const PlaneArgs a, const Interp1D bas, const double *__restrict__ sums, double scale,
                                                        double *__restrict__ v) {
  using L = PlanePlan<P, Q>;
  constexpr int NT = kThreads, P2 = P * P, Q2 = Q * Q;
  extern __shared__ double smem[];
  double *sB = smem + L::oB, *sU = smem + L::oU, *sT = smem + L::oT;
  for (int t = threadIdx.x; t < Q * P; t += NT) sB[t] = bas.B[t];
  for (int idx = blockIdx.x; idx < a.n_elems; idx += gridDim.x) {
    const int e = a.elems[idx];
    const double *src = sums + (int64_t)e * Q2 * NS;
    for (int i = threadIdx.x; i < NS * Q2; i += NT) sU[(i % NS) * Q2 + i / NS] = scale * __ldg(src + i);
    __syncthreads();
    plane_transpose_scatter<P, Q>(sB, sU, sT, a.offsets + (int64_t)e * P2, v);
  }
}

template <int P, int Q>
__global__ void __launch_bounds__(kThreads) k_plane_mass_diag(const PlaneArgs a, const Interp1D bas, double *__restrict__ diag) {
  constexpr int P2 = P * P, Q2 = Q * Q;
  for (int idx = blockIdx.x; idx < a.n_elems; idx += gridDim.x) {
    const int e = a.elems[idx];
    const double *w = a.wdetJ + (int64_t)e * Q2;
    for (int p = threadIdx.x; p < P2; p += kThreads) {
      const int pa = p % P, pb = p / P;
      double d = 0;
      for (int qj = 0; qj < Q; qj++)
        for (int qi = 0; qi < Q; qi++) {
          const double b = bas.B[qi * P + pa] * bas.B[qj * P + pb];
          d += b * b * __ldg(w + qj * Q + qi);
        }
      diag[__ldg(a.offsets + (int64_t)e * P2 + p)] += d;
    }
  }
}

// w detJ of the parent plane (Setup2D_3Dcoords, qfunctions/setupgeo2d.h:136-152): |dx/dX0 x dx/dX1| of the bilinear
// coordinate field through the element's 4 vertices x_plane [E2][3][4] (vertex a + 2b), times the tensor weight.
struct QRef1D {
  double x[kMaxP], w[kMaxP];
};

__global__ void k_plane_qdata(int num_elem, int Q, const double *__restrict__ xp, QRef1D qr, double *__restrict__ wdetJ) {
  const int Q2 = Q * Q;
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (int64_t)num_elem * Q2) return;
  const int64_t e = gid / Q2;
  const int qi = (int)(gid % Q2) % Q, qj = (int)(gid % Q2) / Q;
  const double xi = qr.x[qi], eta = qr.x[qj];
  double J[3][2];
  for (int c = 0; c < 3; c++) {
    const double *v = xp + e * 12 + c * 4;
    J[c][0] = 0.25 * ((1 - eta) * (v[1] - v[0]) + (1 + eta) * (v[3] - v[2]));
    J[c][1] = 0.25 * ((1 - xi) * (v[2] - v[0]) + (1 + xi) * (v[3] - v[1]));
  }
  const double n0 = J[1][0] * J[2][1] - J[2][0] * J[1][1], n1 = J[2][0] * J[0][1] - J[0][0] * J[2][1], n2 = J[0][0] * J[1][1] - J[1][0] * J[0][1];
  wdetJ[gid] = qr.w[qi] * qr.w[qj] * sqrt(n0 * n0 + n1 * n1 + n2 * n2);
}

static int grid_for(int n_items, const void *fn, size_t smem) {
  int dev = 0, sms = 148, per = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, kThreads, smem) != cudaSuccess || per < 1) per = 1;
  const int g = sms * per;
  return n_items < g ? (n_items > 0 ? n_items : 1) : g;
}

template <int P, int Q, int SV>
static int launch_collect_sv(const CollectArgs &a, const Interp1D &b, cudaStream_t s) {
  const size_t sm = CollectPlan<P, Q>::bytes;
  if (cudaFuncSetAttribute(k_stats_collect<P, Q, SV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess) return HB_ERROR_CUDA;
  k_stats_collect<P, Q, SV><<<grid_for(a.num_columns, (const void *)k_stats_collect<P, Q, SV>, sm), kThreads, sm, s>>>(a, b);
  return cudaGetLastError() == cudaSuccess ? HB_SUCCESS : HB_ERROR_CUDA;
}
template <int P, int Q>
static int launch_collect(const CollectArgs &a, const Interp1D &b, int sv, cudaStream_t s) {
  if (sv == HB_STATEVAR_PRIMITIVE) return launch_collect_sv<P, Q, HB_STATEVAR_PRIMITIVE>(a, b, s);
  if (sv == HB_STATEVAR_ENTROPY) return launch_collect_sv<P, Q, HB_STATEVAR_ENTROPY>(a, b, s);
  return launch_collect_sv<P, Q, HB_STATEVAR_CONSERVATIVE>(a, b, s);
}

// kind 0: mass apply (u -> v), 1: projection right-hand side (sums -> v), 2: mass diagonal (-> v[node])
template <int P, int Q>
static int launch_plane(int kind, const HbPlaneOp *pl, const Interp1D &b, const double *in, double scale, double *out, cudaStream_t s) {
  const size_t sm = PlanePlan<P, Q>::bytes;
  if (kind == 0 && cudaFuncSetAttribute(k_plane_mass<P, Q>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess) return HB_ERROR_CUDA;
  if (kind == 1 && cudaFuncSetAttribute(k_plane_rhs<P, Q>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess) return HB_ERROR_CUDA;
  for (int c = 0; c < pl->num_colors; c++) {
    PlaneArgs a;
    a.offsets = pl->d_offsets;
    a.elems = pl->d_color_elem + pl->h_color_ptr[c];
    a.n_elems = pl->h_color_ptr[c + 1] - pl->h_color_ptr[c];
    a.wdetJ = pl->d_wdetJ;
    if (a.n_elems == 0) continue;
    if (kind == 0)
      k_plane_mass<P, Q><<<grid_for(a.n_elems, (const void *)k_plane_mass<P, Q>, sm), kThreads, sm, s>>>(a, b, in, out);
    else if (kind == 1)
      k_plane_rhs<P, Q><<<grid_for(a.n_elems, (const void *)k_plane_rhs<P, Q>, sm), kThreads, sm, s>>>(a, b, in, scale, out);
    else
      k_plane_mass_diag<P, Q><<<grid_for(a.n_elems, (const void *)k_plane_mass_diag<P, Q>, 0), kThreads, 0, s>>>(a, b, out);
  }
  return cudaGetLastError() == cudaSuccess ? HB_SUCCESS : HB_ERROR_CUDA;
}

#define HB_STATS_PQ_LIST(X) X(2, 2) X(2, 3) X(2, 4) X(3, 3) X(3, 4) X(3, 5) X(4, 4) X(4, 5) X(5, 5) X(5, 6) X(6, 6) X(6, 7)

}  // namespace hbs

using namespace hbs;

static Interp1D interp_of(const double *interp1d, int P, int Q) {
  Interp1D b;
  memset(&b, 0, sizeof b);
  memcpy(b.B, interp1d, sizeof(double) * P * Q);
  return b;
}

extern "C" int hb_stats_collect(const HbElemOp *op, const void *ctx184, const double *q, const double *qdata, double dt, int num_columns,
                                int column_length, const int32_t *d_column_elems, double *sums, void *stream) {
  if (!op || !ctx184 || !q || !qdata || !d_column_elems || !sums || num_columns < 0 || column_length < 1) return HB_ERROR_INVALID;
  if (num_columns == 0) return HB_SUCCESS;
  HbNewtonianContext ctx;
  memcpy(&ctx, ctx184, sizeof ctx);
  if (ctx.state_var != HB_STATEVAR_CONSERVATIVE && ctx.state_var != HB_STATEVAR_PRIMITIVE && ctx.state_var != HB_STATEVAR_ENTROPY)
    return HB_ERROR_UNSUPPORTED;
  CollectArgs a;
  memset(&a, 0, sizeof a);
  a.offsets = op->d_offsets;
  a.column_elems = d_column_elems;
  a.num_columns = num_columns;
  a.column_length = column_length;
  a.q = q;
  a.qdata = qdata;
  a.dt = dt;
  a.cv = ctx.gas.cv;
  a.gm1 = ctx.gas.cp / ctx.gas.cv - 1;
  a.pc.cv = ctx.gas.cv;
  a.pc.inv_cv = 1.0 / ctx.gas.cv;
  a.pc.gm1 = a.gm1;
  a.pc.Rgas = ctx.gas.cp - ctx.gas.cv;
  a.sums = sums;
  const Interp1D b = interp_of(op->interp1d, op->P, op->Q);
  cudaStream_t s = (cudaStream_t)stream;
#define HB_CASE(PP, QQ) \
  if (op->P == PP && op->Q == QQ) return launch_collect<PP, QQ>(a, b, ctx.state_var, s);
  HB_STATS_PQ_LIST(HB_CASE)
#undef HB_CASE
  return HB_ERROR_UNSUPPORTED;
}

static int plane_dispatch(int kind, const HbPlaneOp *pl, const double *in, double scale, double *out, void *stream) {
  if (!pl || !out || (kind != 2 && !in)) return HB_ERROR_INVALID;
  const Interp1D b = interp_of(pl->interp1d, pl->P, pl->Q);
  cudaStream_t s = (cudaStream_t)stream;
#define HB_CASE(PP, QQ) \
  if (pl->P == PP && pl->Q == QQ) return launch_plane<PP, QQ>(kind, pl, b, in, scale, out, s);
  HB_STATS_PQ_LIST(HB_CASE)
#undef HB_CASE
  return HB_ERROR_UNSUPPORTED;
}

extern "C" int hb_plane_mass_apply(const HbPlaneOp *pl, const double *u, double *v, int add, void *stream) {
  if (!pl || !v) return HB_ERROR_INVALID;
  if (!add && cudaMemsetAsync(v, 0, sizeof(double) * pl->num_nodes * NS, (cudaStream_t)stream) != cudaSuccess) return HB_ERROR_CUDA;
  return plane_dispatch(0, pl, u, 1.0, v, stream);
}

extern "C" int hb_plane_project_rhs(const HbPlaneOp *pl, const double *sums, double scale, double *v, int add, void *stream) {
  if (!pl || !v) return HB_ERROR_INVALID;
  if (!add && cudaMemsetAsync(v, 0, sizeof(double) * pl->num_nodes * NS, (cudaStream_t)stream) != cudaSuccess) return HB_ERROR_CUDA;
  return plane_dispatch(1, pl, sums, scale, v, stream);
}

extern "C" int hb_plane_mass_diagonal(const HbPlaneOp *pl, double *diag, int add, void *stream) {
  if (!pl || !diag) return HB_ERROR_INVALID;
  if (!add && cudaMemsetAsync(diag, 0, sizeof(double) * pl->num_nodes, (cudaStream_t)stream) != cudaSuccess) return HB_ERROR_CUDA;
  return plane_dispatch(2, pl, NULL, 1.0, diag, stream);
}

extern "C" int hb_plane_setup_qdata(int num_elem, int Q, const double *qref1d, const double *qweight1d, const double *x_plane, double *wdetJ,
                                    void *stream) {
  if (num_elem < 0 || Q < 1 || Q > kMaxP || !qref1d || !qweight1d || !x_plane || !wdetJ) return HB_ERROR_INVALID;
  if (num_elem == 0) return HB_SUCCESS;
  QRef1D qr;
  memset(&qr, 0, sizeof qr);
  memcpy(qr.x, qref1d, sizeof(double) * Q);
  memcpy(qr.w, qweight1d, sizeof(double) * Q);
  const int64_t n = (int64_t)num_elem * Q * Q;
  k_plane_qdata<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(num_elem, Q, x_plane, qr, wdetJ);
  return cudaGetLastError() == cudaSuccess ? HB_SUCCESS : HB_ERROR_CUDA;
}
