// k_newtonian.cu -- fused element kernels of the Newtonian operator for sm_100a.
//
// One kernel launch per element colour.  Each CTA walks a strided slice of that colour's element list and, per
// element, does the whole libCEED operator chain in shared memory:
//   restriction gather (L-vector -> E-vector, int32 offsets, node-interleaved 5 components)
//   -> tensor interpolation and gradient by sum factorisation (x, y, z fibre passes; the gradient uses the collocated
//      derivative D = G B^+ on the quadrature grid, exact for tensor H1 bases with Q >= P)
//   -> point-wise IFunction / IJacobian / linearised diagonal (newtonian_qf.cuh), one thread per quadrature point, with
//      qdata read and jac_data written coalesced in the [elem][comp][qpt] layout
//   -> transpose gradient + interpolation back to the element nodes
//   -> scatter-add into the L-vector through element colouring: elements of one colour share no node and colours run in
//      stream order, so every entry receives one uncontended addition per launch (issued as a reduction without return,
//      performed in L2; deterministic, the same sum as a load-add-store).
// Reference semantics: libCEED CeedOperatorApply / CeedOperatorLinearAssembleDiagonal as called from src/setupts.c:109,
// src/mat-ceed.c:1618,1669 on the operators built in src/setuplibceed.c:209-269.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "honee_b200.h"
#include "newtonian_qf.cuh"
#include "pair_f32.cuh"
#include "pipeline.cuh"
#include "sgs.cuh"

// Optional per-phase cycle accounting of the fused kernels (debug builds with -DHB_PHASE_TIMING only): thread 0 of
// every CTA adds the clock64() deltas of each phase to hb_phase_cycles[].
#ifdef HB_PHASE_TIMING
__device__ unsigned long long hb_phase_cycles[16];
#define HB_PT_DECL unsigned long long hb_t0 = clock64(), hb_acc[16] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
#define HB_PT(k)                             \
  if (threadIdx.x == 0) {                    \
    const unsigned long long t1 = clock64(); \
    hb_acc[k] += t1 - hb_t0;                 \
    hb_t0 = t1;                              \
  }
#define HB_PT_FLUSH(base) \
  if (threadIdx.x == 0)   \
    for (int k = 0; k < 16; k++) atomicAdd(&hb_phase_cycles[(base) + k], hb_acc[k]);
#else
#define HB_PT_DECL
#define HB_PT(k)
#define HB_PT_FLUSH(base)
#endif

namespace hb {

constexpr int kMaxP = 8;

template <typename T>
struct Basis1D {
  T B[kMaxP * kMaxP];  // interp  [Q][P]
  T D[kMaxP * kMaxP];  // collocated derivative on the quadrature points [Q][Q]
  T Gx[4];             // unused padding keeps the struct size a multiple of 16 bytes
};

template <typename T>
__host__ __device__ constexpr int nthreads_for(int Q) {
  return ((Q * Q * Q + 31) / 32) * 32;
}
// resident CTAs per SM the register budget is tuned for (65536 registers / (threads * CTAs), and at most 16384 per SM
// sub-partition for the warps placed on it); the FP32 Jacobian holds half the point-wise state in registers and fits four
// CTAs (121 registers, no spills at P=4, Q=5).  At Q = 6 a CTA is seven warps: two CTAs put four warps on a sub-partition,
// 128 registers, which spills the FP64 point-wise phase (188-260 bytes); one CTA per SM without spills measured faster
// (IFunction 1.19 -> 1.10 ms, IJacobian 1.10 -> 1.04 ms per 32^3 apply at P = 5), while the FP32 Jacobian keeps two.
#ifndef HB_F32_MIN_BLOCKS
#define HB_F32_MIN_BLOCKS 4
#endif
__host__ __device__ constexpr int min_blocks_for(int Q, bool staged = true, int elem_bytes = 8) {
  return Q <= 5 ? (elem_bytes == 4 ? HB_F32_MIN_BLOCKS : (staged ? 3 : 4)) : (Q == 6 && elem_bytes == 4 ? 2 : 1);
}

// ---------------------------------------------------------------------------------------------------------------------
// fibre passes over shared-memory tensors.  All arrays are [comp][n2][n1][n0] with n0 fastest.
// M is row-major [rows][cols]; forward passes use out[i] = sum_a M[i][a] in[a], transposed passes out[a] = sum_i M[i][a] in[i].

// along n0: in [NF][NIN] contiguous rows -> out [NF][NOUT]
template <int NF, int NIN, int NOUT, bool TR, int NT, typename T>
__device__ __forceinline__ void pass0(const T *__restrict__ in, T *__restrict__ out, const T *__restrict__ M, int ldm) {
  for (int f = threadIdx.x; f < NF; f += NT) {
    T x[NIN];
#pragma unroll
    for (int a = 0; a < NIN; a++) x[a] = in[f * NIN + a];
#pragma unroll
    for (int i = 0; i < NOUT; i++) {
      T s = 0;
#pragma unroll
      for (int a = 0; a < NIN; a++) s += (TR ? M[a * ldm + i] : M[i * ldm + a]) * x[a];
      out[f * NOUT + i] = s;
    }
  }
}

// along n1: in [NC][N2][NIN][N0] -> out [NC][N2][NOUT][N0].  Each thread takes two fibres (f and f + NT) per round, loads
// both before computing either, so the two dot-product chains overlap; a missing second fibre recomputes the first and
// skips its store.
template <int NC, int N2, int N0, int NIN, int NOUT, bool TR, int NT, typename T>
__device__ __forceinline__ void pass1(const T *__restrict__ in, T *__restrict__ out, const T *__restrict__ M, int ldm) {
  constexpr int NF = NC * N2 * N0;
  constexpr bool TWO = NF > NT;  // one round of one fibre per thread covers the pass otherwise
#pragma unroll 1
  for (int f0 = threadIdx.x; f0 < NF; f0 += (TWO ? 2 : 1) * NT) {
    const bool h1 = TWO && f0 + NT < NF;
    const int f1 = h1 ? f0 + NT : f0;
    const int x0 = f0 % N0, cz0 = f0 / N0, x1 = f1 % N0, cz1 = f1 / N0;
    const T *src0 = in + cz0 * NIN * N0 + x0, *src1 = in + cz1 * NIN * N0 + x1;
    T v0[NIN], v1[NIN];
#pragma unroll
    for (int a = 0; a < NIN; a++) {
      v0[a] = src0[a * N0];
      if constexpr (TWO) v1[a] = src1[a * N0];
    }
    T *dst0 = out + cz0 * NOUT * N0 + x0, *dst1 = out + cz1 * NOUT * N0 + x1;
#pragma unroll
    for (int i = 0; i < NOUT; i++) {
      T s0 = 0, s1 = 0;
#pragma unroll
      for (int a = 0; a < NIN; a++) {
        const T m = TR ? M[a * ldm + i] : M[i * ldm + a];
        s0 += m * v0[a];
        if constexpr (TWO) s1 += m * v1[a];
      }
      dst0[i * N0] = s0;
      if (TWO && h1) dst1[i * N0] = s1;
    }
  }
}

// ---------------------------------------------------------------------------------------------------------------------
// kernel arguments

template <typename T>
struct ElemArgs {
  const int32_t *offsets;  // [E][P^3] node*5
  const int32_t *elems;    // element ids of this colour
  int n_elems;
  Basis1D<T> basis;
  PhysConst<T> pc;
  const double *qdata;     // [E][10][Q^3]
  const double *x_elem;    // [E][3][8] vertex coordinates (IDL only), may be null
  int num_jd;              // 14 or 15
  int *status;             // device error word: bit 0 = a bounded wait gave up
};

template <typename T>
__device__ __forceinline__ void load_qdata(const double *__restrict__ qd, int Q3, int q, T &wdetJ, T X[3][3]) {
  wdetJ = T(__ldg(qd + q));
#pragma unroll
  for (int k = 0; k < 9; k++) X[k / 3][k % 3] = T(__ldg(qd + (1 + k) * Q3 + q));
}

// x coordinate of quadrature point (i,j,k) from the element's vertex coordinates (trilinear coordinate field); scalar
// code only, so nothing is placed in local memory.
template <int Q>
__device__ __forceinline__ double qpt_x0(const double *__restrict__ xe, const double *qref, int i, int j, int k) {
  const double lx = 0.5 * (1 - qref[i]), hx = 0.5 * (1 + qref[i]), ly = 0.5 * (1 - qref[j]), hy = 0.5 * (1 + qref[j]);
  const double lz = 0.5 * (1 - qref[k]), hz = 0.5 * (1 + qref[k]);
  return lz * (ly * (lx * __ldg(xe + 0) + hx * __ldg(xe + 1)) + hy * (lx * __ldg(xe + 2) + hx * __ldg(xe + 3))) +
         hz * (ly * (lx * __ldg(xe + 4) + hx * __ldg(xe + 5)) + hy * (lx * __ldg(xe + 6) + hx * __ldg(xe + 7)));
}

struct QRef {
  double x[kMaxP];
};

// ---------------------------------------------------------------------------------------------------------------------
// Element pipeline.  Per CTA, elements are processed one after another; while element e is computed, the data of the
// next element e' of the same colour is already being copied into shared memory:
//   * its node values (state, time derivative) by cp.async, issued once the first fibre pass has consumed e's values
//   * its per-point blocks (qdata, stored Jacobian data) by TMA bulk copies on an mbarrier, issued after e's point-wise
//     phase has consumed e's blocks
// so each element starts with all its inputs resident.  The element's contribution is added to the output L-vector by
// reductions without return (scatter_add): elements of one colour share no node, so each entry receives one addition per
// launch and the result equals a load-add-store, with no output values staged and no thread waiting on them.

// Offsets of the entries a thread handles in a 5-component node gather/scatter: entries t = threadIdx.x + j*NT
// (node t/5, component t%5).  They are loaded into registers one element ahead (so no gather waits on them) and kept in
// shared memory for the scatter and the output gather, so they are not live across the point-wise phase.  load() only
// issues the loads: the registers hold the node offsets as loaded and the component is added where they are used, so no
// instruction waits for the load until the next element starts.  L-vector indices fit in int32 (checked on the host).
template <int P, int NT>
struct EntryOffsets {
  static constexpr int P3 = P * P * P, NJ = (5 * P3 + NT - 1) / NT;
  int32_t o[NJ];  // node offset (node * 5) of entry threadIdx.x + j*NT
  __device__ __forceinline__ void load(const int32_t *__restrict__ offsets, int e) {
    const int32_t *off = offsets + (int64_t)e * P3;
#pragma unroll
    for (int j = 0; j < NJ; j++) {
      const int t = threadIdx.x + j * NT;
      if (t < 5 * P3) o[j] = __ldg(off + t / 5);
    }
  }
  __device__ __forceinline__ int32_t entry(int j) const { return o[j] + (int)((threadIdx.x + j * NT) % 5); }
  __device__ __forceinline__ void store(int32_t *sO) const {
#pragma unroll
    for (int j = 0; j < NJ; j++) {
      const int t = threadIdx.x + j * NT;
      if (t < 5 * P3) sO[t] = entry(j);
    }
  }
};

// Row stride of the staged node values: P rounded up to an odd number so the x pass reads without bank conflicts.
template <int P>
__host__ __device__ constexpr int padded_row() { return P | 1; }

// Gather NV L-vectors at one element's nodes into comp-major sN [NV*5][P][P][PX] (x rows padded to PX).
template <int P, int NV, int NT, typename T>
__device__ __forceinline__ void gather_async(const EntryOffsets<P, NT> &eo, const T *l0, const T *l1, T *sN) {
  constexpr int P3 = P * P * P, PX = padded_row<P>(), PS = P * P * PX;
#pragma unroll
  for (int j = 0; j < EntryOffsets<P, NT>::NJ; j++) {
    const int t = threadIdx.x + j * NT;
    if (t < 5 * P3) {
      const int p = t / 5, c = t % 5, srow = (p / P) * PX + p % P;
      const int32_t o = eo.o[j] + c;
      if (sizeof(T) == 8) cp_async8(&sN[c * PS + srow], l0 + o);
      else cp_async4(&sN[c * PS + srow], l0 + o);
      if (NV > 1) {
        if (sizeof(T) == 8) cp_async8(&sN[(5 + c) * PS + srow], l1 + o);
        else cp_async4(&sN[(5 + c) * PS + srow], l1 + o);
      }
    }
  }
}

// x pass from the padded staging rows: sN [NC][P*P][PX] -> s1 [NC][P*P][Q] (two fibres per thread and round)
template <int P, int Q, int NC, int NT, typename T>
__device__ __forceinline__ void pass_x_staged(const Basis1D<T> &bas, const T *sN, T *s1) {
  constexpr int PX = padded_row<P>(), NF = NC * P * P;
  constexpr bool TWO = NF > NT;
#pragma unroll 1
  for (int f0 = threadIdx.x; f0 < NF; f0 += (TWO ? 2 : 1) * NT) {
    const bool h1 = TWO && f0 + NT < NF;
    const int f1 = h1 ? f0 + NT : f0;
    T x0[P], x1[P];
#pragma unroll
    for (int a = 0; a < P; a++) {
      x0[a] = sN[f0 * PX + a];
      if constexpr (TWO) x1[a] = sN[f1 * PX + a];
    }
#pragma unroll
    for (int i = 0; i < Q; i++) {
      T s0 = 0, s1v = 0;
#pragma unroll
      for (int a = 0; a < P; a++) {
        s0 += bas.B[i * P + a] * x0[a];
        if constexpr (TWO) s1v += bas.B[i * P + a] * x1[a];
      }
      s1[f0 * Q + i] = s0;
      if (TWO && h1) s1[f1 * Q + i] = s1v;
    }
  }
}

// The x/y-derivative fibres of one element: 2 x 5 x Q2 of them (direction x or y, component, position on the other two
// directions), each as (direction << 16) | (component * Q3 + first point); the stride along the fibre is 1 (x) or Q (y).
// A kernel that keeps this table in shared memory (FT below) reads one int per fibre where the others divide and take
// remainders per fibre and element.  At Q <= 5 the IFunction, the IJacobian and the FP32 pair kernel use it (per 64^3
// apply at P = 4, in the natural order: IFunction 3.60 -> 3.47 ms, pair 1.88 -> 1.80 ms, FP64 IJacobian 3.08 -> 3.10;
// in the order below: 3.42, 1.78 and 3.04 ms).  At Q = 6 only the FP64 IJacobian uses it (1.038 -> 1.031 ms per 32^3
// apply at P = 5; the IFunction measured the same and the FP32 Jacobian 0.582 -> 0.587 ms).
//
// The table also fixes which thread takes which fibre (thread t takes entries t and t + NT), and that order sets the
// shared-memory bank conflicts of the pass: an 8-byte access of 16 threads is one wavefront when their 16 offsets differ
// modulo 16.  The x fibres start Q apart, which is conflict-free for odd Q.  The y fibres start at c Q3 + z Q2 + x; in
// that natural order, at Q = 5, groups of 16 repeat offsets modulo 16 (0-4, 25-29, 50-54, ...) and take two wavefronts.
// So the x fibres keep their order and each y fibre goes, first fit, to the next slot whose 16-slot group holds no
// offset equal to it modulo 16 (the first one left when none fits).  At Q = 5 every group is then conflict-free.
template <int Q>
struct FibreOrder {
  int v[2 * 5 * Q * Q];
};

template <int Q>
constexpr FibreOrder<Q> make_fibre_order() {
  constexpr int Q2 = Q * Q, Q3 = Q2 * Q, NX = 5 * Q2;
  FibreOrder<Q> o{};
  bool taken[NX] = {};
  for (int f = 0; f < NX; f++) o.v[f] = (f / Q2) * Q3 + (f % Q2) * Q;
  for (int p = NX; p < 2 * NX; p++) {
    const int g0 = p - p % 16;
    int pick = -1, first = -1;
    for (int r = 0; r < NX && pick < 0; r++) {
      if (taken[r]) continue;
      if (first < 0) first = r;
      const int cb = (r / Q2) * Q3 + ((r % Q2) / Q) * Q2 + (r % Q2) % Q;
      bool clash = false;
      for (int i = g0; i < p; i++) clash = clash || ((o.v[i] & 0xffff) - cb) % 16 == 0;
      if (!clash) pick = r;
    }
    if (pick < 0) pick = first;
    taken[pick] = true;
    o.v[p] = (1 << 16) | ((pick / Q2) * Q3 + ((pick % Q2) / Q) * Q2 + (pick % Q2) % Q);
  }
  return o;
}

template <int Q>
__constant__ FibreOrder<Q> c_fibre_order = make_fibre_order<Q>();

template <int Q, int NT>
__device__ __forceinline__ void fill_fibres(int *tab) {
  for (int f = threadIdx.x; f < 2 * 5 * Q * Q; f += NT) tab[f] = c_fibre_order<Q>.v[f];
}

// Forward passes after the x pass: s1 -> (y) s2 -> (z) interp sU [NC][Q3] and, for the first vector, the z
// derivative; then x/y derivatives of the first vector on the quadrature grid.  Two fibres per thread and round.
template <int P, int Q, int NC, int NT, typename T, bool FT = false>
__device__ __forceinline__ void forward_yz(const Basis1D<T> &bas, const T *s1, T *s2, T *sU, T *sG, const int *fib = nullptr) {
  constexpr int Q2 = Q * Q, Q3 = Q2 * Q;
  pass1<NC, P, Q, P, Q, false, NT>(s1, s2, bas.B, P);
  __syncthreads();
  constexpr bool TWO = NC * Q2 > NT;
  constexpr bool D1 = TWO && NT / Q2 < 5;  // a second fibre can belong to the first vector (needs its z derivative)
#pragma unroll 1
  for (int f0 = threadIdx.x; f0 < NC * Q2; f0 += (TWO ? 2 : 1) * NT) {
    const bool h1 = TWO && f0 + NT < NC * Q2;
    const int f1 = h1 ? f0 + NT : f0;
    const int yx0 = f0 % Q2, c0 = f0 / Q2, yx1 = f1 % Q2, c1 = f1 / Q2;
    T in0[P], in1[P], val0[Q], val1[Q];
#pragma unroll
    for (int cz = 0; cz < P; cz++) {
      in0[cz] = s2[(c0 * P + cz) * Q2 + yx0];
      if constexpr (TWO) in1[cz] = s2[(c1 * P + cz) * Q2 + yx1];
    }
#pragma unroll
    for (int k = 0; k < Q; k++) {
      T a0 = 0, a1 = 0;
#pragma unroll
      for (int cz = 0; cz < P; cz++) {
        a0 += bas.B[k * P + cz] * in0[cz];
        if constexpr (TWO) a1 += bas.B[k * P + cz] * in1[cz];
      }
      val0[k] = a0;
      val1[k] = a1;
      sU[c0 * Q3 + k * Q2 + yx0] = a0;
      if (TWO && h1) sU[c1 * Q3 + k * Q2 + yx1] = a1;
    }
    // z derivative of the first vector (components 0-4)
    if (c0 < 5) {
#pragma unroll
      for (int k = 0; k < Q; k++) {
        T d0 = 0;
#pragma unroll
        for (int l = 0; l < Q; l++) d0 += bas.D[k * Q + l] * val0[l];
        sG[(2 * 5 + c0) * Q3 + k * Q2 + yx0] = d0;
      }
    }
    if (D1 && h1 && c1 < 5) {
#pragma unroll
      for (int k = 0; k < Q; k++) {
        T d1 = 0;
#pragma unroll
        for (int l = 0; l < Q; l++) d1 += bas.D[k * Q + l] * val1[l];
        sG[(2 * 5 + c1) * Q3 + k * Q2 + yx1] = d1;
      }
    }
  }
  __syncthreads();
  constexpr int NXY = 2 * 5 * Q2;
  constexpr bool TWO_XY = NXY > NT;
#pragma unroll 1
  for (int f0 = threadIdx.x; f0 < NXY; f0 += (TWO_XY ? 2 : 1) * NT) {
    const bool h1 = TWO_XY && f0 + NT < NXY;
    const int f1 = h1 ? f0 + NT : f0;
    const T *src0, *src1;
    T *dst0, *dst1;
    int st0, st1;
    if constexpr (FT) {
      const int t0 = fib[f0], t1 = fib[f1], dir0 = t0 >> 16, cb0 = t0 & 0xffff, dir1 = t1 >> 16, cb1 = t1 & 0xffff;
      st0 = dir0 == 0 ? 1 : Q;
      st1 = dir1 == 0 ? 1 : Q;
      src0 = sU + cb0;
      src1 = sU + cb1;
      dst0 = sG + dir0 * 5 * Q3 + cb0;
      dst1 = sG + dir1 * 5 * Q3 + cb1;
    } else {
      const int dir0 = f0 / (5 * Q2), r0 = f0 % (5 * Q2), cc0 = r0 / Q2, rem0 = r0 % Q2;
      const int dir1 = f1 / (5 * Q2), r1 = f1 % (5 * Q2), cc1 = r1 / Q2, rem1 = r1 % Q2;
      const int base0 = dir0 == 0 ? rem0 * Q : (rem0 / Q) * Q2 + (rem0 % Q), base1 = dir1 == 0 ? rem1 * Q : (rem1 / Q) * Q2 + (rem1 % Q);
      st0 = dir0 == 0 ? 1 : Q;
      st1 = dir1 == 0 ? 1 : Q;
      src0 = sU + cc0 * Q3 + base0;
      src1 = sU + cc1 * Q3 + base1;
      dst0 = sG + (dir0 * 5 + cc0) * Q3 + base0;
      dst1 = sG + (dir1 * 5 + cc1) * Q3 + base1;
    }
    T v0[Q], v1[Q];
#pragma unroll
    for (int l = 0; l < Q; l++) {
      v0[l] = src0[l * st0];
      if constexpr (TWO_XY) v1[l] = src1[l * st1];
    }
#pragma unroll
    for (int k = 0; k < Q; k++) {
      T d0 = 0, d1 = 0;
#pragma unroll
      for (int l = 0; l < Q; l++) {
        d0 += bas.D[k * Q + l] * v0[l];
        if constexpr (TWO_XY) d1 += bas.D[k * Q + l] * v1[l];
      }
      dst0[k * st0] = d0;
      if (TWO_XY && h1) dst1[k * st1] = d1;
    }
  }
  __syncthreads();
}

// Transpose of the point values v [5][Q3] (sU) and reference-direction fluxes [3][5][Q3] (sG) back to the element
// nodes, node-major sF [P3][5].  Scratch: sW1 [5][Q3], sW2 [5][Q3], sT2 [5][P][Q][Q], sT1 [5][P][P][Q]; sT1 may alias
// sG (free once the z pass is done), sF may alias sW2.  Two fibres per thread and round where a pass has more fibres
// than threads.
template <int P, int Q, int NT, typename T, bool FT = false>
__device__ __forceinline__ void transpose_passes(const Basis1D<T> &bas, const T *sU, const T *sG, T *sW1, T *sW2, T *sT2, T *sT1, T *sF,
                                                 const int *fib = nullptr) {
  constexpr int Q2 = Q * Q, Q3 = Q2 * Q, NXY = 2 * 5 * Q2;
  constexpr bool TWO = NXY > NT;
#pragma unroll 1
  for (int f0 = threadIdx.x; f0 < NXY; f0 += (TWO ? 2 : 1) * NT) {
    const bool h1 = TWO && f0 + NT < NXY;
    const int f1 = h1 ? f0 + NT : f0;
    // x direction adds the point values (w1 = v + D^T g_x); y direction starts from zero (w2 = D^T g_y)
    const T *g0, *g1, *v0, *v1;
    T *w0, *w1;
    int dir0, dir1, st0, st1;
    if constexpr (FT) {
      const int t0 = fib[f0], t1 = fib[f1], cb0 = t0 & 0xffff, cb1 = t1 & 0xffff;
      dir0 = t0 >> 16;
      dir1 = t1 >> 16;
      g0 = sG + dir0 * 5 * Q3 + cb0;
      g1 = sG + dir1 * 5 * Q3 + cb1;
      v0 = sU + cb0;
      v1 = sU + cb1;
      w0 = (dir0 == 0 ? sW1 : sW2) + cb0;
      w1 = (dir1 == 0 ? sW1 : sW2) + cb1;
    } else {
      dir0 = f0 / (5 * Q2);
      dir1 = f1 / (5 * Q2);
      const int r0 = f0 % (5 * Q2), c0 = r0 / Q2, rem0 = r0 % Q2;
      const int r1 = f1 % (5 * Q2), c1 = r1 / Q2, rem1 = r1 % Q2;
      const int base0 = dir0 == 0 ? rem0 * Q : (rem0 / Q) * Q2 + (rem0 % Q), base1 = dir1 == 0 ? rem1 * Q : (rem1 / Q) * Q2 + (rem1 % Q);
      g0 = sG + (dir0 * 5 + c0) * Q3 + base0;
      g1 = sG + (dir1 * 5 + c1) * Q3 + base1;
      v0 = sU + c0 * Q3 + base0;
      v1 = sU + c1 * Q3 + base1;
      w0 = (dir0 == 0 ? sW1 : sW2) + c0 * Q3 + base0;
      w1 = (dir1 == 0 ? sW1 : sW2) + c1 * Q3 + base1;
    }
    st0 = dir0 == 0 ? 1 : Q;
    st1 = dir1 == 0 ? 1 : Q;
    T gv0[Q], gv1[Q], b0[Q], b1[Q];
#pragma unroll
    for (int l = 0; l < Q; l++) {
      gv0[l] = g0[l * st0];
      b0[l] = dir0 == 0 ? v0[l] : T(0);
      if constexpr (TWO) {
        gv1[l] = g1[l * st1];
        b1[l] = dir1 == 0 ? v1[l] : T(0);
      }
    }
#pragma unroll
    for (int i = 0; i < Q; i++) {
      T s0 = b0[i], s1 = TWO ? b1[i] : T(0);
#pragma unroll
      for (int l = 0; l < Q; l++) {
        s0 += bas.D[l * Q + i] * gv0[l];
        if constexpr (TWO) s1 += bas.D[l * Q + i] * gv1[l];
      }
      w0[i * st0] = s0;
      if (TWO && h1) w1[i * st1] = s1;
    }
  }
  __syncthreads();
  for (int f = threadIdx.x; f < 5 * Q2; f += NT) {
    const int yx = f % Q2, c = f / Q2;
    T w[Q], gz[Q];
#pragma unroll
    for (int l = 0; l < Q; l++) gz[l] = sG[(2 * 5 + c) * Q3 + l * Q2 + yx];
#pragma unroll
    for (int k = 0; k < Q; k++) {
      T s = sW1[c * Q3 + k * Q2 + yx] + sW2[c * Q3 + k * Q2 + yx];
#pragma unroll
      for (int l = 0; l < Q; l++) s += bas.D[l * Q + k] * gz[l];
      w[k] = s;
    }
#pragma unroll
    for (int cz = 0; cz < P; cz++) {
      T s = 0;
#pragma unroll
      for (int k = 0; k < Q; k++) s += bas.B[k * P + cz] * w[k];
      sT2[(c * P + cz) * Q2 + yx] = s;
    }
  }
  __syncthreads();
  pass1<5, P, Q, Q, P, true, NT>(sT2, sT1, bas.B, P);
  __syncthreads();
  for (int f = threadIdx.x; f < 5 * P * P; f += NT) {
    const int c = f / (P * P), zb = f % (P * P);
    T in[Q];
#pragma unroll
    for (int i = 0; i < Q; i++) in[i] = sT1[f * Q + i];
#pragma unroll
    for (int pa = 0; pa < P; pa++) {
      T s = 0;
#pragma unroll
      for (int i = 0; i < Q; i++) s += bas.B[i * P + pa] * in[i];
      sF[(zb * P + pa) * 5 + c] = s;
    }
  }
  __syncthreads();
}

// out[o] += contribution, node-major sF [P3][5] at the element's entry offsets sO.  Elements of one colour share no node,
// so every entry receives exactly one addition per launch: a reduction without return (red.global.add, performed at L2)
// gives the same sum as a load-add-store, in any order, and leaves no thread waiting for the old value.
template <int P, int NT, typename T>
__device__ __forceinline__ void scatter_add(const int32_t *sO, const T *sF, T *l_out) {
  constexpr int P3 = P * P * P;
  for (int t = threadIdx.x; t < 5 * P3; t += NT) atomicAdd(l_out + sO[t], sF[t]);
}

// Shared-memory plan (in units of T unless noted):
//   sN  [NV*5][P][P][PX] staged node values (x rows padded to odd PX) of the element being computed / the next one
//   s1  [NV*5][P][P][Q] x-pass output; later sT2 (transpose scratch)
//   s2  [NV*5][P][Q][Q] y-pass output; later w2 and the final node values
//   sU  [10][Q3]        interpolated values (q, then q_dot or w1); point-wise outputs v in place
//   sG  [15][Q3]        reference gradients; point-wise fluxes in place; later sT1
//   sJD [15][Q3]        staged stored Jacobian data (IJacobian only)
//   sQD [10][Q3] double staged qdata (IJacobian only; the residual reads qdata at the point)
template <int P, int Q, int NV, typename T, bool JD, bool ST = true>
struct Plan {
  static constexpr int P3 = P * P * P, Q2 = Q * Q, Q3 = Q2 * Q;
  static constexpr int cmax(int x, int y) { return x > y ? x : y; }
  static constexpr int nN = NV * 5 * P * P * padded_row<P>(), nU = 10 * Q3, nG = 15 * Q3;
  static constexpr int n1 = cmax(NV * 5 * P * P * Q, 5 * P * Q2);          // x-pass output, then sT2
  static constexpr int n2 = cmax(cmax(NV * 5 * P * Q2, 5 * Q3), 5 * P3);   // y-pass output, then w2 and node values
  static constexpr int nJD = (JD && ST) ? 15 * Q3 : 0;
  static constexpr int kAl = 16 / (int)sizeof(T);
  static constexpr int pad(int n) { return (n + kAl - 1) / kAl * kAl; }  // every buffer 16-byte aligned (bulk copies)
  static constexpr int oN = 0, o1 = pad(oN + nN), o2 = pad(o1 + n1), oU = pad(o2 + n2), oG = pad(oU + nU),
                       oJD = pad(oG + nG), end_T = pad(oJD + nJD);
  static constexpr size_t qd_offset_bytes = ((size_t)end_T * sizeof(T) + 15) & ~(size_t)15;
  static constexpr size_t mbar_offset = qd_offset_bytes + (ST ? sizeof(double) * 10 * Q3 : 0);  // staged qdata, then the mbarrier
  static constexpr size_t bytes = mbar_offset + 16;
  static_assert(5 * P * Q2 <= n1, "sT2 fits in s1");
  static_assert(5 * Q3 <= n2, "w2 fits in s2");
  static_assert(5 * P3 <= n2, "final node values fit in s2");
  static_assert(5 * P * P * Q <= nG, "sT1 fits in sG");
};

// ---------------------------------------------------------------------------------------------------------------------
// Learned SGS closure fused into the residual (qfunctions/sgs_dd_model.h:65-98 and :205-241 evaluated at the quadrature
// points instead of through a nodal projection): velocity gradient -> anisotropy-frame features -> FP32 network (weights
// in the kernel's parameter space, read through the constant cache) -> de-normalised SGS stress -> its flux, added to the
// reference-direction fluxes.  SGS = 1: one hidden layer of 20 (the reference's model), 2: two hidden layers of 20.

template <int SGS>
struct SgsArg {
  int unused;
};
template <>
struct SgsArg<1> {
  float w[sgs::MlpShape<20, 0>::size];
  float alpha;
  float b[6][2];
  int clamp, no_backscatter;
};
template <>
struct SgsArg<2> {
  float w[sgs::MlpShape<20, 20>::size];
  float alpha;
  float b[6][2];
  int clamp, no_backscatter;
};

template <int SGS, int SV = HB_STATEVAR_CONSERVATIVE>
__device__ __forceinline__ void sgs_add(const PhysConst<double> &c, const double q[5], const double gref[3][5], double wdetJ, const double X[3][3],
                                        const SgsArg<SGS> &sg, double gv[3][5]) {
  St<double> st;
  SAux<double> aux;
  state_from_q<SV>(c, q, st, aux);
  const double inv_rho = aux.inv_rho;
  St<double> gs[3];
#pragma unroll
  for (int j = 0; j < 3; j++) gradient_dir<SV>(c, st, aux, gref, X, j, gs[j]);
  double G[3][3];
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) G[i][j] = gs[j].u[i];
  double kmA[6], delta, E[3][3], in[6], gmag;
  sgs::anisotropy(X, kmA, delta);
  sgs::inputs(G, kmA, delta, c.mu * inv_rho, E, in, gmag);
  float xf[6], yf[6];
#pragma unroll
  for (int k = 0; k < 6; k++) xf[k] = (float)in[k];
  sgs::mlp_forward<20, SGS == 2 ? 20 : 0>(sg.w, sg.alpha, xf, yf);
  double y[6], km[6], F[5][3];
#pragma unroll
  for (int k = 0; k < 6; k++) y[k] = sg.clamp ? fmin(fmax((double)yf[k], 0.0), 1.0) : (double)yf[k];
  sgs::outputs_to_stress(y, delta, E, sg.b, gmag, km);
  if (sg.no_backscatter) {  // tau : S > 0 feeds energy to the resolved scales: keep only the isotropic part there
    double tau[3][3], ts = 0;
    sgs::km_unpack(km, tau);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = 0; j < 3; j++) ts += tau[i][j] * 0.5 * (G[i][j] + G[j][i]);
    if (ts > 0) {
      const double iso = (km[0] + km[1] + km[2]) / 3;
      km[0] = km[1] = km[2] = iso;
      km[3] = km[4] = km[5] = 0;
    }
  }
  sgs::flux(st.u, km, F);
#pragma unroll
  for (int d = 0; d < 3; d++)
#pragma unroll
    for (int k = 0; k < 5; k++) gv[d][k] -= wdetJ * (X[d][0] * F[k][0] + X[d][1] * F[k][1] + X[d][2] * F[k][2]);
}

// ---------------------------------------------------------------------------------------------------------------------
// IFunction

struct IfunctionPtrs {
  const double *q, *q_dot;
  double *jac_data;   // [E][num_jd][Q3], may be null
  float *jac_f32;     // [E][num_jd][Q3] single-precision shadow for the mixed-precision Jacobian, may be null
  double *v;
  QRef qref;
};

// qdata is read at the point (coalesced: thread q reads entry q of each of the element's ten [Q3] rows) after an L2
// prefetch two elements ahead; staging it in shared memory by TMA measured slower (3.75 against 3.64 ms per 64^3 apply
// at P = 4, Q = 5; 1.25 against 1.21 ms per 32^3 apply at P = 5, Q = 6), so the kernel has no bulk copies and no waits.
template <int P, int Q, int SGS = 0, int SV = HB_STATEVAR_CONSERVATIVE>
__global__ void __launch_bounds__(nthreads_for<double>(Q), min_blocks_for(Q)) k_ifunction(const ElemArgs<double> a, const IfunctionPtrs p,
                                                                                           const SgsArg<SGS> sg) {
  constexpr int NT = nthreads_for<double>(Q);
  using L = Plan<P, Q, 2, double, false, false>;
  constexpr int Q3 = L::Q3;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *sm = reinterpret_cast<double *>(smem_raw);
  double *sN = sm + L::oN, *s1 = sm + L::o1, *s2 = sm + L::o2, *sU = sm + L::oU, *sG = sm + L::oG;
  double *sD = sU + 5 * Q3;
  __shared__ double s_qref[kMaxP];
  __shared__ int32_t sO[2][5 * L::P3];  // entry offsets of the current / next element
  constexpr bool FT = Q <= 5;           // x/y-derivative fibre table
  __shared__ int sFib[FT ? 2 * 5 * Q * Q : 1];
  const unsigned qd_bytes = sizeof(double) * 10 * Q3;
  if constexpr (FT) fill_fibres<Q, NT>(sFib);

  if (threadIdx.x == 0) {  // constant indices: indexing the parameter array with threadIdx would copy it to local memory
#pragma unroll
    for (int i = 0; i < kMaxP; i++) s_qref[i] = p.qref.x[i];
  }
  __syncthreads();
  int idx = blockIdx.x;
  if (idx >= a.n_elems) return;
  int buf = 0;
  {  // prologue: stage the first element
    const int e0 = a.elems[idx];
    EntryOffsets<P, NT> eo;
    eo.load(a.offsets, e0);
    eo.store(sO[0]);
    gather_async<P, 2, NT, double>(eo, p.q, p.q_dot, sN);
    if (threadIdx.x == 0) {
      prefetch_l2_bulk(a.qdata + (int64_t)e0 * 10 * Q3, qd_bytes);
      if (idx + (int)gridDim.x < a.n_elems) prefetch_l2_bulk(a.qdata + (int64_t)a.elems[idx + gridDim.x] * 10 * Q3, qd_bytes);
    }
    cp_async_commit();
  }
  // element ids and entry offsets are read two elements ahead so no global load latency sits on the critical path
  const int G = gridDim.x;
  int ecur = a.elems[idx];
  int en = idx + G < a.n_elems ? a.elems[idx + G] : -1;
  int en2 = idx + 2 * G < a.n_elems ? a.elems[idx + 2 * G] : -1;
  EntryOffsets<P, NT> nxt, nxt2;
  if (en >= 0) nxt.load(a.offsets, en);
  HB_PT_DECL
  for (; idx < a.n_elems; idx += gridDim.x) {
    const int e = ecur;
    int en3 = -1;  // used one iteration later: a predicated load, so nothing waits for it here
    if (idx + 3 * G < a.n_elems) en3 = __ldg(a.elems + idx + 3 * G);
    if (en2 >= 0) nxt2.load(a.offsets, en2);
    HB_PT(7)
    cp_async_wait_group<0>();  // this element's node values have landed
    HB_PT(8)
    __syncthreads();
    HB_PT(0)
    if (en2 >= 0 && threadIdx.x == 0) prefetch_l2_bulk(a.qdata + (int64_t)en2 * 10 * Q3, qd_bytes);
    pass_x_staged<P, Q, 10, NT, double>(a.basis, sN, s1);
    __syncthreads();
    HB_PT(1)
    if (en >= 0) {  // sN consumed: stage the next element's node values
      gather_async<P, 2, NT, double>(nxt, p.q, p.q_dot, sN);
      cp_async_commit();
      nxt.store(sO[buf ^ 1]);
    }
    forward_yz<P, Q, 10, NT, double, FT>(a.basis, s1, s2, sU, sG, sFib);
    HB_PT(2)
    const int q = threadIdx.x;
    if (q < Q3) {
      double qi[5], qd[5], gref[3][5], wdetJ, X[3][3], v[5], gv[3][5];
#pragma unroll
      for (int c = 0; c < 5; c++) {
        qi[c] = sU[c * Q3 + q];
        qd[c] = sD[c * Q3 + q];
#pragma unroll
        for (int d = 0; d < 3; d++) gref[d][c] = sG[(d * 5 + c) * Q3 + q];
      }
      const double *qdp = a.qdata + (int64_t)e * 10 * Q3;
      wdetJ = qdp[q];
#pragma unroll
      for (int k = 0; k < 9; k++) X[k / 3][k % 3] = qdp[(1 + k) * Q3 + q];
      double x0 = 0;
      if (a.pc.idl_enable) x0 = qpt_x0<Q>(a.x_elem + (int64_t)e * 24, s_qref, q % Q, (q / Q) % Q, q / (Q * Q));
      // stored Jacobian values go to global memory as soon as they are known (FP64 and/or the FP32 shadow)
      double *jd64 = p.jac_data ? p.jac_data + (int64_t)e * a.num_jd * Q3 + q : nullptr;
      float *jd32 = p.jac_f32 ? p.jac_f32 + (int64_t)e * a.num_jd * Q3 + q : nullptr;
      const int njd = a.num_jd;
      auto emit = [=](int k, double val) {
        if (k < njd) {
          if (jd64) jd64[k * Q3] = val;
          if (jd32) jd32[k * Q3] = float(val);
        }
      };
      ifunction_point_stream<double, SV>(a.pc, qi, gref, qd, wdetJ, X, x0, v, gv, emit);
      if constexpr (SGS > 0) sgs_add<SGS, SV>(a.pc, qi, gref, wdetJ, X, sg, gv);
#pragma unroll
      for (int c = 0; c < 5; c++) {
        sU[c * Q3 + q] = v[c];
#pragma unroll
        for (int d = 0; d < 3; d++) sG[(d * 5 + c) * Q3 + q] = gv[d][c];
      }
    }
    __syncthreads();
    HB_PT(3)
    if (en2 >= 0) {  // warm L2 for the element after next: its node rows of q, q_dot and v (its qdata follows below)
#pragma unroll
      for (int j = 0; j < EntryOffsets<P, NT>::NJ; j++) {
        const int t = threadIdx.x + j * NT;
        if (t < 5 * L::P3 && t % 5 == 0) {
          prefetch_l2(p.q + nxt2.o[j]);
          prefetch_l2(p.q_dot + nxt2.o[j]);
          prefetch_l2(p.v + nxt2.o[j]);
        }
      }
    }
    // transpose scratch: w1 in the q_dot slot, w2 and the node values in s2, sT2 in s1, sT1 in sG
    HB_PT(4)
    transpose_passes<P, Q, NT, double, FT>(a.basis, sU, sG, sD, s2, s1, sG, s2, sFib);
    HB_PT(5)
    scatter_add<P, NT, double>(sO[buf], s2, p.v);  // no barrier after it: nothing writes shared memory before the next
    HB_PT(12)                                       // iteration's top barrier
    buf ^= 1;
    ecur = en;
    en = en2;
    en2 = en3;
    nxt = nxt2;
    HB_PT(6)
  }
  HB_PT_FLUSH(0)
  cp_async_wait_all();
}

// ---------------------------------------------------------------------------------------------------------------------
// IJacobian action (FP64 or FP32 arithmetic; jac_data and L-vectors in the same precision, qdata FP64)

template <typename T>
struct IjacobianPtrs {
  const T *dq;
  const T *jac_data;  // [E][num_jd][Q3]
  T *v;
  int qdata_tma, jd_tma;
};

template <int P, int Q, typename T, bool ST, int SV = HB_STATEVAR_CONSERVATIVE>
__global__ void __launch_bounds__(nthreads_for<T>(Q), min_blocks_for(Q, ST, (int)sizeof(T))) k_ijacobian(const ElemArgs<T> a, const IjacobianPtrs<T> p) {
  constexpr int NT = nthreads_for<T>(Q);
  using L = Plan<P, Q, 1, T, true, ST>;
  constexpr int Q3 = L::Q3;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *sm = reinterpret_cast<T *>(smem_raw);
  T *sN = sm + L::oN, *s1 = sm + L::o1, *s2 = sm + L::o2, *sU = sm + L::oU, *sG = sm + L::oG, *sJD = sm + L::oJD;
  T *sW1 = sU + 5 * Q3;
  double *sQD = reinterpret_cast<double *>(smem_raw + L::qd_offset_bytes);
  uint64_t *mbar = reinterpret_cast<uint64_t *>(smem_raw + L::mbar_offset);
  __shared__ int s_bail;
  __shared__ int32_t sO[2][5 * L::P3];  // entry offsets of the current / next element
  constexpr bool FT = Q <= 5 || (Q == 6 && sizeof(T) == 8);  // x/y-derivative fibre table (FP32 at Q = 6: slower with it)
  __shared__ int sFib[FT ? 2 * 5 * Q * Q : 1];
  if constexpr (FT) fill_fibres<Q, NT>(sFib);
  const unsigned qd_bytes = sizeof(double) * 10 * Q3;
  const int njd = a.num_jd;
  const unsigned jd_bytes = (unsigned)(sizeof(T) * njd * Q3);
  const unsigned tx = (p.qdata_tma ? qd_bytes : 0) + (p.jd_tma ? jd_bytes : 0);

  if (threadIdx.x == 0) {
    mbar_init(mbar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_bail = 0;
  }
  __syncthreads();
  int idx = blockIdx.x;
  if (idx >= a.n_elems) return;
  int buf = 0;
  {
    const int e0 = a.elems[idx];
    EntryOffsets<P, NT> eo;
    eo.load(a.offsets, e0);
    eo.store(sO[0]);
    gather_async<P, 1, NT, T>(eo, p.dq, p.dq, sN);
    if constexpr (ST) {
      if (threadIdx.x == 0) mbar_arrive_expect_tx(mbar, tx);
      stage_block<double, NT>(sQD, a.qdata + (int64_t)e0 * 10 * Q3, 10 * Q3, p.qdata_tma, mbar);
      stage_block<T, NT>(sJD, p.jac_data + (int64_t)e0 * njd * Q3, njd * Q3, p.jd_tma, mbar);
    } else if (threadIdx.x == 0) {
      prefetch_l2_bulk(a.qdata + (int64_t)e0 * 10 * Q3, qd_bytes);
      prefetch_l2_bulk(p.jac_data + (int64_t)e0 * njd * Q3, jd_bytes);
    }
    cp_async_commit();
  }
  unsigned phase = 0;
  // element ids and entry offsets are read two elements ahead so no global load latency sits on the critical path
  const int G = gridDim.x;
  int ecur = a.elems[idx];
  int en = idx + G < a.n_elems ? a.elems[idx + G] : -1;
  int en2 = idx + 2 * G < a.n_elems ? a.elems[idx + 2 * G] : -1;
  EntryOffsets<P, NT> nxt, nxt2;
  if (en >= 0) nxt.load(a.offsets, en);
  for (; idx < a.n_elems; idx += gridDim.x) {
    const int e = ecur;
    int en3 = -1;  // used one iteration later: a predicated load, so nothing waits for it here
    if (idx + 3 * G < a.n_elems) en3 = __ldg(a.elems + idx + 3 * G);
    if (en2 >= 0) nxt2.load(a.offsets, en2);
    cp_async_wait_group<0>();  // this element's node values (and point data staged by cp.async) have landed
    if (ST && threadIdx.x == 0 && !mbar_wait_bounded(mbar, phase)) {
      s_bail = 1;
      atomicOr(a.status, 1);
    }
    __syncthreads();
    if (s_bail) break;
    phase ^= 1;
    if (en2 >= 0 && threadIdx.x == 0) {  // warm L2 for the element after next (its own staging follows the next point phase)
      prefetch_l2_bulk(a.qdata + (int64_t)en2 * 10 * Q3, qd_bytes);
      prefetch_l2_bulk(p.jac_data + (int64_t)en2 * njd * Q3, jd_bytes);
    }
    pass_x_staged<P, Q, 5, NT, T>(a.basis, sN, s1);
    __syncthreads();
    if (en >= 0) {
      gather_async<P, 1, NT, T>(nxt, p.dq, p.dq, sN);
      cp_async_commit();
      nxt.store(sO[buf ^ 1]);
    }
    forward_yz<P, Q, 5, NT, T, FT>(a.basis, s1, s2, sU, sG, sFib);
    const int q = threadIdx.x;
    if (q < Q3) {
      T dq[5], gref[3][5], wdetJ, X[3][3], v[5], gv[3][5], jd[15];
#pragma unroll
      for (int c = 0; c < 5; c++) {
        dq[c] = sU[c * Q3 + q];
#pragma unroll
        for (int d = 0; d < 3; d++) gref[d][c] = sG[(d * 5 + c) * Q3 + q];
      }
      const T *jdp = ST ? sJD : p.jac_data + (int64_t)e * njd * Q3;
      const double *qdp = ST ? sQD : a.qdata + (int64_t)e * 10 * Q3;
#pragma unroll
      for (int c = 0; c < 14; c++) jd[c] = jdp[c * Q3 + q];
      jd[14] = njd > 14 ? jdp[14 * Q3 + q] : T(0);
      wdetJ = T(qdp[q]);
#pragma unroll
      for (int k = 0; k < 9; k++) X[k / 3][k % 3] = T(qdp[(1 + k) * Q3 + q]);
      ijacobian_point_stream<T, SV>(a.pc, jd, dq, gref, wdetJ, X, v, gv);
#pragma unroll
      for (int c = 0; c < 5; c++) {
        sU[c * Q3 + q] = v[c];
#pragma unroll
        for (int d = 0; d < 3; d++) sG[(d * 5 + c) * Q3 + q] = gv[d][c];
      }
    }
    __syncthreads();
    if (en2 >= 0) {  // and the node rows of dq and v of the element after next
#pragma unroll
      for (int j = 0; j < EntryOffsets<P, NT>::NJ; j++) {
        const int t = threadIdx.x + j * NT;
        if (t < 5 * L::P3 && t % 5 == 0) {
          prefetch_l2(p.dq + nxt2.o[j]);
          prefetch_l2(p.v + nxt2.o[j]);
        }
      }
    }
    if (en >= 0) {
      if constexpr (ST) {
        if (threadIdx.x == 0) {
          fence_proxy_async_smem();
          mbar_arrive_expect_tx(mbar, tx);
        }
        stage_block<double, NT>(sQD, a.qdata + (int64_t)en * 10 * Q3, 10 * Q3, p.qdata_tma, mbar);
        stage_block<T, NT>(sJD, p.jac_data + (int64_t)en * njd * Q3, njd * Q3, p.jd_tma, mbar);
      }
      cp_async_commit();
    }
    transpose_passes<P, Q, NT, T, FT>(a.basis, sU, sG, sW1, s2, s1, sG, s2, sFib);
    scatter_add<P, NT, T>(sO[buf], s2, p.v);  // the next iteration's top barrier orders it before any shared-memory write
    buf ^= 1;
    ecur = en;
    en = en2;
    en2 = en3;
    nxt = nxt2;
  }
  cp_async_wait_all();
  if (ST && s_bail && threadIdx.x == 0) mbar_wait_bounded(mbar, phase);
}

// ---------------------------------------------------------------------------------------------------------------------
// Mixed-precision Jacobian action on element pairs with packed FP32 arithmetic (pair_f32.cuh).  Each CTA pass takes two
// elements of the colour (list positions 2i and 2i + 1; an odd count leaves the last pair with one element, whose second
// lane recomputes the first and is not stored): the node values of both are gathered into the two lanes of one 8-byte
// slot, every basis pass and the point-wise tangent run once for both lanes, and the scatter stores each lane at its own
// element's nodes.  Same arithmetic per lane as k_ijacobian<float> (FP32 values and Jacobian data, FP64 qdata rounded to
// FP32 at the point), half the instructions.  qdata of both elements is staged by TMA; their Jacobian data are read at
// the point from global memory (coalesced per component, warmed in L2 one pair ahead), which keeps three CTAs per SM.

struct IjacobianPairPtrs {
  const float *dq;
  const float *jac_data;  // [E][num_jd][Q3]
  float *v;
};

// node gathers into one lane (byte offset 0 or 4) of the pair slots: sN [5][P][P][PX]
template <int P, int NT>
__device__ __forceinline__ void gather_lane_async(const EntryOffsets<P, NT> &eo, const float *l, f2 *sN, int lane) {
  constexpr int P3 = P * P * P, PX = padded_row<P>(), PS = P * P * PX;
#pragma unroll
  for (int j = 0; j < EntryOffsets<P, NT>::NJ; j++) {
    const int t = threadIdx.x + j * NT;
    if (t < 5 * P3) {
      const int pp = t / 5, c = t % 5, srow = (pp / P) * PX + pp % P;
      cp_async4(reinterpret_cast<float *>(&sN[c * PS + srow]) + lane, l + eo.o[j] + c);
    }
  }
}

template <int P, int Q, int SV = HB_STATEVAR_CONSERVATIVE>
__global__ void __launch_bounds__(nthreads_for<float>(Q), (Q <= 5 ? 3 : 1)) k_ijacobian_pair(const ElemArgs<f2> a, const IjacobianPairPtrs p) {
  constexpr int NT = nthreads_for<float>(Q);
  using L = Plan<P, Q, 1, f2, false, false>;
  constexpr int Q3 = L::Q3, P3 = L::P3;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  f2 *sm = reinterpret_cast<f2 *>(smem_raw);
  f2 *sN = sm + L::oN, *s1 = sm + L::o1, *s2 = sm + L::o2, *sU = sm + L::oU, *sG = sm + L::oG;
  f2 *sW1 = sU + 5 * Q3;
  double *sQD = reinterpret_cast<double *>(smem_raw + L::qd_offset_bytes);  // [2][10][Q3]: the pair's qdata
  uint64_t *mbar = reinterpret_cast<uint64_t *>(smem_raw + L::qd_offset_bytes + 2 * sizeof(double) * 10 * Q3);
  __shared__ int s_bail;
  __shared__ int32_t sO[2][2][5 * P3];  // entry offsets of the current / next pair, per lane
  __shared__ int sFib[2 * 5 * Q * Q];   // x/y-derivative fibre table
  fill_fibres<Q, NT>(sFib);
  const unsigned qd_bytes = sizeof(double) * 10 * Q3;
  const int njd = a.num_jd;
  const int npairs = (a.n_elems + 1) / 2;
  // element ids of pair i: list positions 2i and 2i + 1 (the second repeats the first when the count is odd)
  auto pair_elems = [&](int i, int &eA, int &eB, int &hasB) {
    eA = a.elems[2 * i];
    hasB = 2 * i + 1 < a.n_elems;
    eB = hasB ? a.elems[2 * i + 1] : eA;
  };
  auto stage_qdata = [&](int eA, int eB) {  // thread 0: both elements' qdata by TMA on one mbarrier phase
    mbar_arrive_expect_tx(mbar, 2 * qd_bytes);
    tma_load_1d(sQD, a.qdata + (int64_t)eA * 10 * Q3, qd_bytes, mbar);
    tma_load_1d(sQD + 10 * Q3, a.qdata + (int64_t)eB * 10 * Q3, qd_bytes, mbar);
  };
  auto warm_jd = [&](int eA, int eB) {
    prefetch_l2_bulk(p.jac_data + (int64_t)eA * njd * Q3, sizeof(float) * njd * Q3);
    prefetch_l2_bulk(p.jac_data + (int64_t)eB * njd * Q3, sizeof(float) * njd * Q3);
  };

  if (threadIdx.x == 0) {
    mbar_init(mbar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_bail = 0;
  }
  __syncthreads();
  int idx = blockIdx.x;
  if (idx >= npairs) return;
  const int G = gridDim.x;
  int buf = 0;
  int eA, eB, hasB;
  pair_elems(idx, eA, eB, hasB);
  {  // prologue: stage the first pair
    EntryOffsets<P, NT> oa, ob;
    oa.load(a.offsets, eA);
    ob.load(a.offsets, eB);
    oa.store(sO[0][0]);
    ob.store(sO[0][1]);
    gather_lane_async<P, NT>(oa, p.dq, sN, 0);
    gather_lane_async<P, NT>(ob, p.dq, sN, 1);
    if (threadIdx.x == 0) {
      stage_qdata(eA, eB);
      warm_jd(eA, eB);
    }
    cp_async_commit();
  }
  unsigned phase = 0;
  int nA = -1, nB = -1, nhasB = 0;
  if (idx + G < npairs) pair_elems(idx + G, nA, nB, nhasB);
  EntryOffsets<P, NT> nxa, nxb;
  if (nA >= 0) {
    nxa.load(a.offsets, nA);
    nxb.load(a.offsets, nB);
  }
  for (; idx < npairs; idx += G) {
    const int cA = eA, cB = eB, chasB = hasB;
    cp_async_wait_group<0>();  // the pair's node values have landed
    if (threadIdx.x == 0 && !mbar_wait_bounded(mbar, phase)) {
      s_bail = 1;
      atomicOr(a.status, 1);
    }
    __syncthreads();
    if (s_bail) break;
    phase ^= 1;
    if (nA >= 0 && threadIdx.x == 0) warm_jd(nA, nB);
    pass_x_staged<P, Q, 5, NT, f2>(a.basis, sN, s1);
    __syncthreads();
    if (nA >= 0) {
      gather_lane_async<P, NT>(nxa, p.dq, sN, 0);
      gather_lane_async<P, NT>(nxb, p.dq, sN, 1);
      cp_async_commit();
      nxa.store(sO[buf ^ 1][0]);
      nxb.store(sO[buf ^ 1][1]);
    }
    forward_yz<P, Q, 5, NT, f2, true>(a.basis, s1, s2, sU, sG, sFib);
    const int q = threadIdx.x;
    if (q < Q3) {
      f2 dq[5], gref[3][5], wdetJ, X[3][3], v[5], gv[3][5], jd[15];
#pragma unroll
      for (int c = 0; c < 5; c++) {
        dq[c] = sU[c * Q3 + q];
#pragma unroll
        for (int d = 0; d < 3; d++) gref[d][c] = sG[(d * 5 + c) * Q3 + q];
      }
      const float *jA = p.jac_data + (int64_t)cA * njd * Q3 + q, *jB = p.jac_data + (int64_t)cB * njd * Q3 + q;
#pragma unroll
      for (int c = 0; c < 14; c++) jd[c] = f2(__ldg(jA + c * Q3), __ldg(jB + c * Q3));
      jd[14] = njd > 14 ? f2(__ldg(jA + 14 * Q3), __ldg(jB + 14 * Q3)) : f2(0.0);
      const double *qA = sQD + q, *qB = sQD + 10 * Q3 + q;
      wdetJ = f2(float(qA[0]), float(qB[0]));
#pragma unroll
      for (int k = 0; k < 9; k++) X[k / 3][k % 3] = f2(float(qA[(1 + k) * Q3]), float(qB[(1 + k) * Q3]));
      ijacobian_point_stream<f2, SV>(a.pc, jd, dq, gref, wdetJ, X, v, gv);
#pragma unroll
      for (int c = 0; c < 5; c++) {
        sU[c * Q3 + q] = v[c];
#pragma unroll
        for (int d = 0; d < 3; d++) sG[(d * 5 + c) * Q3 + q] = gv[d][c];
      }
    }
    __syncthreads();
    if (nA >= 0) {
      if (threadIdx.x == 0) {
        fence_proxy_async_smem();
        stage_qdata(nA, nB);
      }
      cp_async_commit();
    }
    transpose_passes<P, Q, NT, f2, true>(a.basis, sU, sG, sW1, s2, s1, sG, s2, sFib);
    {  // scatter: each lane to its own element's nodes, by reductions (scatter_add)
      const int32_t *oA = sO[buf][0], *oB = sO[buf][1];
      for (int t = threadIdx.x; t < 5 * P3; t += NT) {
        const f2 r = s2[t];
        atomicAdd(p.v + oA[t], r.x());
        if (chasB) atomicAdd(p.v + oB[t], r.y());
      }
    }  // no barrier: the next iteration's top barrier orders the scatter before any shared-memory write
    buf ^= 1;
    eA = nA;
    eB = nB;
    hasB = nhasB;
    if (idx + 2 * G < npairs) {
      pair_elems(idx + 2 * G, nA, nB, nhasB);
      nxa.load(a.offsets, nA);
      nxb.load(a.offsets, nB);
    } else {
      nA = nB = -1;
      nhasB = 0;
    }
  }
  cp_async_wait_all();
  if (s_bail && threadIdx.x == 0) mbar_wait_bounded(mbar, phase);
}

// ---------------------------------------------------------------------------------------------------------------------
// Diagonal of the IJacobian operator (libCEED CeedOperatorLinearAssembleDiagonal semantics): at every quadrature point
// linearise the point-wise Jacobian for each component c with unit inputs in the four eval modes (interp, grad x/y/z),
// keep the 4x4 block A_c[m][n] = d out(m,c) / d in(n,c), and contract sum_q phi_m(q,p) A_c[m][n](q) phi_n(q,p) by sum
// factorisation with products of 1D basis rows.  The 16 (m,n) pairs share 10 distinct product triples (combinations).
//
// The point blocks come from the explicit linearisation of the point function (diag_point_blocks: per component one
// value tangent and three physical-gradient tangents with their unit inputs folded in, the reference-direction blocks
// assembled as X R X^T), so a point costs about four Jacobian evaluations, not twenty.  The per-point Jacobian data and
// qdata are read once per element.  The 50 combination arrays [5][10][Q^3] are contracted in three batched passes whose
// partial sums are grouped by the basis factors still to apply: after the x pass the ten combinations of a component
// collapse into six (y, z) groups, after the y pass into three z groups.

template <typename T>
struct DiagArgs {
  const T *jac_data;
  T *diag;
  T G1[kMaxP * kMaxP];        // reference 1D gradient [Q][P]
  T W[3][kMaxP * kMaxP];      // squared basis rows [Q][P]: B*B, B*G, G*G
};

// combination order: II, IGx, IGy, IGz, GxGx, GyGy, GzGz, GxGy, GxGz, GyGz.  The six x-pass groups by their (y, z)
// factors, each member given as (combination, x factor): (0,0): II/BB, IGx/BG, GxGx/GG; (1,0): IGy/BB, GxGy/BG;
// (0,1): IGz/BB, GxGz/BG; (2,0): GyGy/BB; (0,2): GzGz/BB; (1,1): GyGz/BB.  The three y-pass groups by their z factor,
// members (x group, y factor): z=0: (0,0)/BB, (1,0)/BG, (2,0)/GG; z=1: (0,1)/BB, (1,1)/BG; z=2: (0,2)/BB.
__host__ __device__ constexpr int diag_xgroup_size(int g) { return g == 0 ? 3 : (g < 3 ? 2 : 1); }
__host__ __device__ constexpr int diag_xmember(int g, int i) {
  return g == 0 ? (i == 0 ? 0 : (i == 1 ? 1 : 4)) : g == 1 ? (i == 0 ? 2 : 7) : g == 2 ? (i == 0 ? 3 : 8) : g == 3 ? 5 : (g == 4 ? 6 : 9);
}
__host__ __device__ constexpr int diag_xfactor(int g, int i) { return g < 3 ? i : 0; }
__host__ __device__ constexpr int diag_ygroup_size(int h) { return 3 - h; }
__host__ __device__ constexpr int diag_ymember(int h, int i) { return h == 0 ? (i == 0 ? 0 : (i == 1 ? 1 : 3)) : h == 1 ? (i == 0 ? 2 : 5) : 4; }
__host__ __device__ constexpr int diag_yfactor(int h, int i) { return i; }

template <int P, int Q>
struct DiagPlan {
  // FP64 at Q = 5: 74 KB, three CTAs per SM
  static constexpr int P2 = P * P, P3 = P2 * P, Q2 = Q * Q, Q3 = Q2 * Q, PX = P;  // PX: pa stride of the x-pass output
  static constexpr int nA = 50 * Q3;                                               // [5][10][Q3]; after the y pass: T2 [5][3][Q][P][P]
  static constexpr int nT1 = 5 * 6 * Q2 * PX;                                      // [5][6][Q][Q][PX]
  static constexpr int nT2 = 5 * 3 * Q * P2;
  static_assert(nT2 <= nA, "the y-pass output fits in the combination arrays");
  template <typename T>
  static constexpr size_t t1_bytes() { return (sizeof(T) * nT1 + 15) & ~(size_t)15; }
  template <typename T>
  static constexpr size_t bytes() { return ((sizeof(T) * nA + 15) & ~(size_t)15) + t1_bytes<T>(); }
};

// resident CTAs per SM: three at Q <= 5; at Q = 6 two for FP32 (65 KB of shared memory, 146 registers, no spills: 1.03 ->
// 0.74 ms per 32^3 apply at P = 5) and one for FP64 (130 KB)
template <int P, int Q, typename T, int SV = HB_STATEVAR_CONSERVATIVE>
__global__ void __launch_bounds__(nthreads_for<T>(Q), (Q <= 5 ? 3 : (sizeof(T) == 4 && Q == 6 ? 2 : 1))) k_diagonal(const ElemArgs<T> a, const DiagArgs<T> p) {
  constexpr int NT = nthreads_for<T>(Q);
  using L = DiagPlan<P, Q>;
  constexpr int P2 = L::P2, P3 = L::P3, Q2 = L::Q2, Q3 = L::Q3, PX = L::PX;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *sA = reinterpret_cast<T *>(smem_raw);                                        // [5][10][Q3]
  unsigned char *t1_raw = smem_raw + ((sizeof(T) * L::nA + 15) & ~(size_t)15);
  T *sT1 = reinterpret_cast<T *>(t1_raw);                                         // [5][6][Q2][PX]
  T *sT2 = sA;                                                                    // [5][3][Q][P][P]
  const int njd = a.num_jd;
  // The point data (qdata and Jacobian data) are read at the point from global memory (coalesced: thread q reads entry q
  // of each [Q3] row), warmed in L2 one element ahead.  Staging them by cp.async into the x-pass region after the y pass
  // measured slower (7.42 against 7.08 ms FP64, 3.00 against 2.81 ms FP32 per 64^3 apply at P = 4, Q = 5).
  auto warm = [&](int e) {
    prefetch_l2_bulk(p.jac_data + (int64_t)e * njd * Q3, sizeof(T) * njd * Q3);
    prefetch_l2_bulk(a.qdata + (int64_t)e * 10 * Q3, sizeof(double) * 10 * Q3);
  };
  if (blockIdx.x < a.n_elems && threadIdx.x == 0) warm(a.elems[blockIdx.x]);
  for (int idx = blockIdx.x; idx < a.n_elems; idx += gridDim.x) {
    const int e = a.elems[idx];
    const int en = idx + (int)gridDim.x < a.n_elems ? a.elems[idx + gridDim.x] : -1;
    if (threadIdx.x == 0 && en >= 0) warm(en);
    __syncthreads();  // the previous element's z pass has read sT2 (= sA) before the point phase writes sA
    const int q = threadIdx.x;
    if (q < Q3) {
      T jd[15], wdetJ, X[3][3];
      const T *gJD = p.jac_data + (int64_t)e * njd * Q3 + q;
      const double *gQD = a.qdata + (int64_t)e * 10 * Q3 + q;
#pragma unroll
      for (int k = 0; k < 14; k++) jd[k] = gJD[k * Q3];
      jd[14] = njd > 14 ? gJD[14 * Q3] : T(0);
      wdetJ = T(gQD[0]);
#pragma unroll
      for (int k = 0; k < 9; k++) X[k / 3][k % 3] = T(gQD[(1 + k) * Q3]);
      T *sAq = sA + q;
      diag_point_blocks<SV>(a.pc, jd, wdetJ, X, [&](int c, int m, T v) { sAq[(c * 10 + m) * Q3] = v; });
    }
    __syncthreads();
    // x pass, one (component, k j) fibre per work item and x group: T1[c][g][kj][pa] = sum_members sum_i W(i,pa) A[c][m][kj][i]
#pragma unroll
    for (int g = 0; g < 6; g++) {
      for (int t = threadIdx.x; t < 5 * Q2; t += NT) {
        const int c = t / Q2, kj = t % Q2;
        T acc[P];
#pragma unroll
        for (int pa = 0; pa < P; pa++) acc[pa] = 0;
#pragma unroll
        for (int mi = 0; mi < diag_xgroup_size(g); mi++) {
          const T *src = sA + (c * 10 + diag_xmember(g, mi)) * Q3 + kj * Q;
          T in[Q];
#pragma unroll
          for (int i = 0; i < Q; i++) in[i] = src[i];
#pragma unroll
          for (int pa = 0; pa < P; pa++)
#pragma unroll
            for (int i = 0; i < Q; i++) acc[pa] += p.W[diag_xfactor(g, mi)][i * P + pa] * in[i];
        }
        T *dst = sT1 + ((c * 6 + g) * Q2 + kj) * PX;
#pragma unroll
        for (int pa = 0; pa < P; pa++) dst[pa] = acc[pa];
      }
    }
    __syncthreads();
    // y pass, one (component, k, pa) fibre per work item and y group: T2[c][h][k][pb][pa]
#pragma unroll
    for (int h = 0; h < 3; h++) {
      for (int t = threadIdx.x; t < 5 * Q * P; t += NT) {
        const int c = t / (Q * P), k = (t / P) % Q, pa = t % P;
        T acc[P];
#pragma unroll
        for (int pb = 0; pb < P; pb++) acc[pb] = 0;
#pragma unroll
        for (int mi = 0; mi < diag_ygroup_size(h); mi++) {
          const T *src = sT1 + ((c * 6 + diag_ymember(h, mi)) * Q2 + k * Q) * PX + pa;
          T in[Q];
#pragma unroll
          for (int j = 0; j < Q; j++) in[j] = src[j * PX];
#pragma unroll
          for (int pb = 0; pb < P; pb++)
#pragma unroll
            for (int j = 0; j < Q; j++) acc[pb] += p.W[diag_yfactor(h, mi)][j * P + pb] * in[j];
        }
        T *dst = sT2 + ((c * 3 + h) * Q + k) * P2 + pa;
#pragma unroll
        for (int pb = 0; pb < P; pb++) dst[pb * P] = acc[pb];
      }
    }
    __syncthreads();
    // z pass over the three z groups, then the scatter: elements of one colour share no node, so each entry receives one
    // addition per launch; a reduction without return (red.global.add) leaves no thread waiting for the old value
    const int32_t *off = a.offsets + (int64_t)e * P3;
    for (int t = threadIdx.x; t < 5 * P2; t += NT) {
      const int c = t / P2, pab = t % P2;
      T acc[P];
#pragma unroll
      for (int pc = 0; pc < P; pc++) acc[pc] = 0;
#pragma unroll
      for (int h = 0; h < 3; h++) {
        T in[Q];
#pragma unroll
        for (int k = 0; k < Q; k++) in[k] = sT2[((c * 3 + h) * Q + k) * P2 + pab];
#pragma unroll
        for (int pc = 0; pc < P; pc++)
#pragma unroll
          for (int k = 0; k < Q; k++) acc[pc] += p.W[h][k * P + pc] * in[k];
      }
#pragma unroll
      for (int pc = 0; pc < P; pc++) atomicAdd(p.diag + __ldg(off + pc * P2 + pab) + c, acc[pc]);
    }
  }
}

// ---------------------------------------------------------------------------------------------------------------------
// Point-block diagonal of the IJacobian operator with batched contractions.
//
// The element matrix restricted to a node p and components (i out, j in) is
//   sum_q sum_{a,b} phi_a(p,q) A_q[(a,i),(b,j)] phi_b(p,q),   a, b in {value, d/dX0, d/dX1, d/dX2}
// with A_q the linearised point function (20 x 20, the columns taken by forward products with unit inputs).  phi_a phi_b is
// symmetric in (a,b), so the ten combinations {a,b} carry A[(a,i),(b,j)] + A[(b,i),(a,j)] (one term when a = b), and each is
// a tensor product of per-direction squared-basis rows (B B, B G or G G).  A round covers one input component j and NI
// output components: the point phase accumulates the NI x 10 combination arrays in shared memory, one thread per point,
// then three batched passes contract them all, and the last pass sums the ten combinations before the coloured scatter.
// This is libCEED's point-block semantics (CeedOperatorLinearAssemblePointBlockDiagonal: a 5 x 5 block
// [component out][component in] per node, what MatCEED hands PCVPBJACOBI, src/mat-ceed.c:76-153).  Like k_diagonal the
// cost is the 20 forward products per point; the batched contraction keeps the 25 blocks at about 2.5x the diagonal.
__host__ __device__ constexpr int blockdiag_ni(int P, int Q, int elem_bytes) {
  // the largest output-component group whose combination arrays [NI*10][Q^3] and first-pass buffer [NI*10][Q^2 P] fit
  return (50 * (Q * Q * Q + Q * Q * P) * elem_bytes <= 200 * 1024)   ? 5
         : (30 * (Q * Q * Q + Q * Q * P) * elem_bytes <= 200 * 1024) ? 3
         : (20 * (Q * Q * Q + Q * Q * P) * elem_bytes <= 200 * 1024) ? 2
                                                                     : 1;
}
template <int P, int Q, typename T>
constexpr size_t blockdiag_smem() {
  return sizeof(T) * (size_t)blockdiag_ni(P, Q, sizeof(T)) * 10 * (Q * Q * Q + Q * Q * P);
}

__device__ __forceinline__ int combo_sel(int m, int d) {
  // derivatives in direction d of combination m (order: II, IGx, IGy, IGz, GxGx, GyGy, GzGz, GxGy, GxGz, GyGz)
  if (d == 0) return (m == 1 || m == 7 || m == 8) ? 1 : (m == 4 ? 2 : 0);
  if (d == 1) return (m == 2 || m == 7 || m == 9) ? 1 : (m == 5 ? 2 : 0);
  return (m == 3 || m == 8 || m == 9) ? 1 : (m == 6 ? 2 : 0);
}
__host__ __device__ constexpr int combo_of(int a, int b) {
  // unordered pair {a, b} of {value, Gx, Gy, Gz} -> combination index
  return a > b ? combo_of(b, a)
               : (a == b ? (a == 0 ? 0 : 3 + a) : (a == 0 ? b : (a == 1 ? (b == 2 ? 7 : 8) : 9)));
}

template <int P, int Q, typename T, int SV = HB_STATEVAR_CONSERVATIVE>
__global__ void __launch_bounds__(nthreads_for<T>(Q), 1) k_blockdiag(const ElemArgs<T> a, const DiagArgs<T> p) {
  constexpr int NT = nthreads_for<T>(Q);
  constexpr int P2 = P * P, P3 = P2 * P, Q2 = Q * Q, Q3 = Q2 * Q, Q2P = Q2 * P, QP2 = Q * P2;
  constexpr int NI = blockdiag_ni(P, Q, sizeof(T)), NA = NI * 10, NG = (5 + NI - 1) / NI;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *sA = reinterpret_cast<T *>(smem_raw);  // [NA][Q3]; after the second pass [NA][Q][P][P]
  T *sY = sA + NA * Q3;                     // [NA][Q][Q][P]
  __shared__ T sW[3][kMaxP * kMaxP];        // B*B, B*G, G*G  [Q][P]
  for (int t = threadIdx.x; t < Q * P; t += NT) {
    T b = 0, g = 0;
#pragma unroll
    for (int i = 0; i < Q * P; i++)
      if (i == t) {
        b = a.basis.B[i];
        g = p.G1[i];
      }
    sW[0][t] = b * b;
    sW[1][t] = b * g;
    sW[2][t] = g * g;
  }
  __syncthreads();
  constexpr int kRounds = 5 * NG;
  for (int idx = blockIdx.x; idx < a.n_elems; idx += gridDim.x) {
    const int e = a.elems[idx];
    const int32_t *off = a.offsets + (int64_t)e * P3;
    for (int r = 0; r < kRounds; r++) {
      const int j_in = r / NG, i0 = (r % NG) * NI;  // input component j_in, output components [i0, i0 + NI)
      const int q = threadIdx.x;
      if (q < Q3) {
        T jd[15], wdetJ, X[3][3];
        const T *jdp = p.jac_data + (int64_t)e * a.num_jd * Q3 + q;
#pragma unroll
        for (int k = 0; k < 14; k++) jd[k] = jdp[k * Q3];
        jd[14] = a.num_jd > 14 ? jdp[14 * Q3] : T(0);
        load_qdata(a.qdata + (int64_t)e * 10 * Q3, Q3, q, wdetJ, X);
        for (int t = 0; t < NA; t++) sA[t * Q3 + q] = 0;
        {
          const int jj = j_in;
#pragma unroll
          for (int n = 0; n < 4; n++) {
            T dq[5] = {0, 0, 0, 0, 0}, gref[3][5] = {{0, 0, 0, 0, 0}, {0, 0, 0, 0, 0}, {0, 0, 0, 0, 0}}, v[5], gv[3][5];
#pragma unroll
            for (int k = 0; k < 5; k++) {
              if (n == 0 && k == jj) dq[k] = 1;
#pragma unroll
              for (int d = 0; d < 3; d++)
                if (n == d + 1 && k == jj) gref[d][k] = 1;
            }
            ijacobian_point_stream<T, SV>(a.pc, jd, dq, gref, wdetJ, X, v, gv);
#pragma unroll
            for (int k = 0; k < 5; k++) {
              if (k < i0 || k >= i0 + NI) continue;
              T *row = sA + (k - i0) * 10 * Q3 + q;
              // A[(mo, k), (n, jj)] for mo = value, Gx, Gy, Gz
              row[combo_of(0, n) * Q3] += v[k];
              row[combo_of(1, n) * Q3] += gv[0][k];
              row[combo_of(2, n) * Q3] += gv[1][k];
              row[combo_of(3, n) * Q3] += gv[2][k];
            }
          }
        }
      }
      __syncthreads();
      for (int f = threadIdx.x; f < NA * Q2P; f += NT) {  // x: [a][k][j][pa]
        const int t = f / Q2P, rem = f % Q2P, pa = rem % P, kj = rem / P;
        const T *W = sW[combo_sel(t % 10, 0)];
        T acc = 0;
#pragma unroll
        for (int i = 0; i < Q; i++) acc += W[i * P + pa] * sA[t * Q3 + kj * Q + i];
        sY[f] = acc;
      }
      __syncthreads();
      for (int f = threadIdx.x; f < NA * QP2; f += NT) {  // y: [a][k][pb][pa]
        const int t = f / QP2, rem = f % QP2, pa = rem % P, pb = (rem / P) % P, k = rem / P2;
        const T *W = sW[combo_sel(t % 10, 1)];
        T acc = 0;
#pragma unroll
        for (int j = 0; j < Q; j++) acc += W[j * P + pb] * sY[t * Q2P + (k * Q + j) * P + pa];
        sA[f] = acc;
      }
      __syncthreads();
      for (int f = threadIdx.x; f < NI * P3; f += NT) {  // z, summed over the ten combinations, and the scatter
        const int il = f / P3, pp = f % P3, pab = pp % P2, pc_ = pp / P2;
        const int i = i0 + il;
        if (i >= 5) continue;
        T acc = 0;
#pragma unroll
        for (int m = 0; m < 10; m++) {
          const T *W = sW[combo_sel(m, 2)];
#pragma unroll
          for (int k = 0; k < Q; k++) acc += W[k * P + pc_] * sA[(il * 10 + m) * QP2 + k * P2 + pab];
        }
        p.diag[(int64_t)__ldg(off + pp) * 5 + i * 5 + j_in] += acc;
      }
      __syncthreads();
    }
  }
}

// ---------------------------------------------------------------------------------------------------------------------
// Geometric factors (qfunctions/setupgeo.h:42-56, utils.h:201-216): trilinear coordinates -> w detJ, dX/dx.

__global__ void k_setup_qdata(int num_elem, int Q, const double *__restrict__ x_elem, QRef qref, QRef qw, double *__restrict__ qdata) {
  const int Q3 = Q * Q * Q;
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (int64_t)num_elem * Q3) return;
  const int64_t e = gid / Q3;
  const int q = (int)(gid % Q3);
  const int ii[3] = {q % Q, (q / Q) % Q, q / (Q * Q)};
  const double *xe = x_elem + e * 24;
  double J[3][3];  // J[c][d] = dx_c / dX_d
  for (int c = 0; c < 3; c++)
    for (int d = 0; d < 3; d++) {
      double s = 0;
      for (int v = 0; v < 8; v++) {
        double w = 1;
        for (int dd = 0; dd < 3; dd++) {
          const int bit = (v >> dd) & 1;
          const double xi = qref.x[ii[dd]];
          w *= (dd == d) ? (bit ? 0.5 : -0.5) : (bit ? 0.5 * (1 + xi) : 0.5 * (1 - xi));
        }
        s += w * xe[c * 8 + v];
      }
      J[c][d] = s;
    }
  double A[3][3];
  A[0][0] = J[1][1] * J[2][2] - J[1][2] * J[2][1];
  A[0][1] = J[0][2] * J[2][1] - J[0][1] * J[2][2];
  A[0][2] = J[0][1] * J[1][2] - J[0][2] * J[1][1];
  A[1][0] = J[1][2] * J[2][0] - J[1][0] * J[2][2];
  A[1][1] = J[0][0] * J[2][2] - J[0][2] * J[2][0];
  A[1][2] = J[0][2] * J[1][0] - J[0][0] * J[1][2];
  A[2][0] = J[1][0] * J[2][1] - J[1][1] * J[2][0];
  A[2][1] = J[0][1] * J[2][0] - J[0][0] * J[2][1];
  A[2][2] = J[0][0] * J[1][1] - J[0][1] * J[1][0];
  const double det = J[0][0] * A[0][0] + J[1][0] * A[0][1] + J[2][0] * A[0][2];
  const double inv = 1 / det;
  double *qd = qdata + e * 10 * Q3 + q;
  qd[0] = qw.x[ii[0]] * qw.x[ii[1]] * qw.x[ii[2]] * det;
  for (int k = 0; k < 9; k++) qd[(1 + k) * Q3] = A[k / 3][k % 3] * inv;
}

// ---------------------------------------------------------------------------------------------------------------------
// host side

template <typename T>
static PhysConst<T> make_phys(const HbNewtonianContext &c) {
  PhysConst<T> p;
  p.mu = T(c.gas.mu);
  p.lambda = T(c.gas.lambda);
  p.k = T(c.gas.k);
  p.cv = T(c.gas.cv);
  p.inv_cv = T(1.0 / c.gas.cv);
  p.gm1 = T(c.gas.cp / c.gas.cv - 1);
  p.Rgas = T(c.gas.cp - c.gas.cv);
  for (int i = 0; i < 3; i++) p.g[i] = T(c.g[i]);
  p.shift = T(c.ijacobian_time_shift);
  p.Ctau_C = T(c.tau_coeffs.Ctau_C);
  p.Ctau_M = T(c.tau_coeffs.Ctau_M);
  p.Ctau_E = T(c.tau_coeffs.Ctau_E);
  p.Ctau_v = T(c.tau_coeffs.Ctau_v);
  p.dts = T(c.tau_coeffs.Ctau_t / c.dt);
  p.stab = (int)c.stabilization;
  p.idl_enable = c.idl_enable ? 1 : 0;
  p.idl_amplitude = T(c.idl_amplitude);
  p.idl_start = T(c.idl_start);
  p.idl_length = T(c.idl_length);
  p.idl_pressure = T(c.idl_pressure);
  return p;
}

template <typename T>
static void fill_basis(const HbElemOp *op, Basis1D<T> &b) {
  memset(&b, 0, sizeof b);
  for (int i = 0; i < op->Q * op->P; i++) b.B[i] = T(op->interp1d[i]);
  for (int i = 0; i < op->Q * op->Q; i++) b.D[i] = T(op->colo_grad1d[i]);
}

template <typename T>
static ElemArgs<T> make_args(const HbElemOp *op, const HbNewtonianContext &ctx, const double *qdata, int color) {
  ElemArgs<T> a;
  a.offsets = op->d_offsets;
  a.elems = op->d_color_elem + op->h_color_ptr[color];
  a.n_elems = op->h_color_ptr[color + 1] - op->h_color_ptr[color];
  fill_basis<T>(op, a.basis);
  a.pc = make_phys<T>(ctx);
  a.qdata = qdata;
  a.x_elem = op->d_x_elem;
  a.num_jd = ctx.idl_enable ? 15 : 14;
  a.status = op->d_status;
  return a;
}

template <typename K>
static int grid_for(const HbElemOp *op, int n_elems, K kernel, int nthreads, size_t smem) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, nthreads, smem) != cudaSuccess || per_sm < 1) per_sm = 1;
  const int g = op->num_sms * per_sm;
  return n_elems < g ? n_elems : g;
}

template <typename T>
static size_t smem_bytes(int P, int Q) {
  const int P3 = P * P * P, Q3 = Q * Q * Q;
  return sizeof(T) * (size_t)(10 * P3 + 10 * P * P * Q + 10 * P * Q * Q + 10 * Q3 + 15 * Q3);
}

template <int P, int Q, int SGS = 0, int SV = HB_STATEVAR_CONSERVATIVE>
static int launch_ifunction_v(const HbElemOp *op, const HbNewtonianContext &ctx, const HbIFunctionIO *io, cudaStream_t s,
                              const SgsArg<SGS> &sg = SgsArg<SGS>{}) {
  using L = Plan<P, Q, 2, double, false, false>;
  const size_t sm = L::bytes;
  cudaFuncSetAttribute(k_ifunction<P, Q, SGS, SV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  IfunctionPtrs p;
  p.q = io->q;
  p.q_dot = io->q_dot;
  p.jac_data = io->jac_data;
  p.jac_f32 = io->jac_data_f32;
  p.v = io->v;
  for (int i = 0; i < kMaxP; i++) p.qref.x[i] = i < Q ? op->qref1d[i] : 0;
  for (int c = 0; c < op->num_colors; c++) {
    ElemArgs<double> a = make_args<double>(op, ctx, io->qdata, c);
    if (a.n_elems == 0) continue;
    k_ifunction<P, Q, SGS, SV><<<grid_for(op, a.n_elems, k_ifunction<P, Q, SGS, SV>, nthreads_for<double>(Q), sm), nthreads_for<double>(Q), sm, s>>>(a, p, sg);
  }
  return cudaGetLastError() == cudaSuccess ? HB_SUCCESS : HB_ERROR_CUDA;
}
template <int P, int Q, int SV = HB_STATEVAR_CONSERVATIVE>
static int launch_ifunction(const HbElemOp *op, const HbNewtonianContext &ctx, const HbIFunctionIO *io, cudaStream_t s) {
  return launch_ifunction_v<P, Q, 0, SV>(op, ctx, io, s);
}

template <int P, int Q, typename T, bool ST, int SV = HB_STATEVAR_CONSERVATIVE>
static int launch_ijacobian_v(const HbElemOp *op, const HbNewtonianContext &ctx, const double *qdata, const T *jd, const T *dq, T *v,
                              cudaStream_t s) {
  using L = Plan<P, Q, 1, T, true, ST>;
  const size_t sm = L::bytes;
  cudaFuncSetAttribute(k_ijacobian<P, Q, T, ST, SV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  IjacobianPtrs<T> p;
  p.dq = dq;
  p.jac_data = jd;
  p.v = v;
  const int njd = ctx.idl_enable ? 15 : 14;
  p.qdata_tma = ((uintptr_t)qdata % 16) == 0;
  p.jd_tma = ((uintptr_t)jd % 16) == 0 && (sizeof(T) * njd * L::Q3) % 16 == 0;
  for (int c = 0; c < op->num_colors; c++) {
    ElemArgs<T> a = make_args<T>(op, ctx, qdata, c);
    if (a.n_elems == 0) continue;
    k_ijacobian<P, Q, T, ST, SV><<<grid_for(op, a.n_elems, k_ijacobian<P, Q, T, ST, SV>, nthreads_for<T>(Q), sm), nthreads_for<T>(Q), sm, s>>>(a, p);
  }
  return cudaGetLastError() == cudaSuccess ? HB_SUCCESS : HB_ERROR_CUDA;
}

template <int P, int Q, typename T, int SV = HB_STATEVAR_CONSERVATIVE>
static int launch_ijacobian(const HbElemOp *op, const HbNewtonianContext &ctx, const double *qdata, const T *jd, const T *dq, T *v,
                            cudaStream_t s) {
  return launch_ijacobian_v<P, Q, T, true, SV>(op, ctx, qdata, jd, dq, v, s);
}

// The paired FP32 Jacobian (two elements of a colour per CTA pass, packed FP32): needs qdata 16-byte aligned (TMA).
template <int P, int Q, int SV = HB_STATEVAR_CONSERVATIVE>
static int launch_ijacobian_pair(const HbElemOp *op, const HbNewtonianContext &ctx, const double *qdata, const float *jd, const float *dq, float *v,
                                 cudaStream_t s) {
  using L = Plan<P, Q, 1, f2, false, false>;
  const size_t sm = L::qd_offset_bytes + 2 * sizeof(double) * 10 * L::Q3 + 16;
  if (cudaFuncSetAttribute(k_ijacobian_pair<P, Q, SV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess) return HB_ERROR_CUDA;
  IjacobianPairPtrs p;
  p.dq = dq;
  p.jac_data = jd;
  p.v = v;
  for (int c = 0; c < op->num_colors; c++) {
    ElemArgs<f2> a = make_args<f2>(op, ctx, qdata, c);
    if (a.n_elems == 0) continue;
    const int npairs = (a.n_elems + 1) / 2;
    k_ijacobian_pair<P, Q, SV><<<grid_for(op, npairs, k_ijacobian_pair<P, Q, SV>, nthreads_for<float>(Q), sm), nthreads_for<float>(Q), sm, s>>>(a, p);
  }
  return cudaGetLastError() == cudaSuccess ? HB_SUCCESS : HB_ERROR_CUDA;
}

template <int P, int Q, int SV>
static int pair_case(const HbElemOp *op, const HbNewtonianContext &ctx, const double *qdata, const float *jd, const float *dq, float *v, cudaStream_t s) {
  if constexpr (Q <= 5) return launch_ijacobian_pair<P, Q, SV>(op, ctx, qdata, jd, dq, v, s);
  return launch_ijacobian<P, Q, float, SV>(op, ctx, qdata, jd, dq, v, s);
}

template <int P, int Q, typename T, int SV = HB_STATEVAR_CONSERVATIVE>
static int launch_diagonal(const HbElemOp *op, const HbNewtonianContext &ctx, const double *qdata, const T *jd, T *diag, cudaStream_t s) {
  const size_t sm = DiagPlan<P, Q>::template bytes<T>();
  cudaFuncSetAttribute(k_diagonal<P, Q, T, SV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  DiagArgs<T> p;
  memset(&p, 0, sizeof p);
  p.jac_data = jd;
  p.diag = diag;
  for (int i = 0; i < Q * P; i++) {
    const double b = op->interp1d[i], g = op->grad1d[i];
    p.G1[i] = T(g);
    p.W[0][i] = T(b * b);
    p.W[1][i] = T(b * g);
    p.W[2][i] = T(g * g);
  }
  for (int c = 0; c < op->num_colors; c++) {
    ElemArgs<T> a = make_args<T>(op, ctx, qdata, c);
    if (a.n_elems == 0) continue;
    k_diagonal<P, Q, T, SV><<<grid_for(op, a.n_elems, k_diagonal<P, Q, T, SV>, nthreads_for<T>(Q), sm), nthreads_for<T>(Q), sm, s>>>(a, p);
  }
  return cudaGetLastError() == cudaSuccess ? HB_SUCCESS : HB_ERROR_CUDA;
}

// ---------------------------------------------------------------------------------------------------------------------
// Mass operator of the explicit path (Mass_N with N = 5, qfunctions/mass.h:19-26, on the state restriction and basis:
// src/setuplibceed.c:15-53): v += B^T (wdetJ .* (B u)) per component, and its diagonal sum_q B_p(q)^2 wdetJ_q.
// Memory-bound (the state read once, the output read-modify-written once, one of the ten qdata components read), so
// one CTA per element of a colour: node-interleaved gather staged in shared memory, then the three 1D contractions per
// direction for all five components at once, qdata read as one contiguous Q^3 block.
constexpr int kMassThreads = 256;

template <int P, int Q>
__device__ __forceinline__ void mass_basis_to_smem(const Basis1D<double> &bas, double *sB, bool squared) {
  for (int t = threadIdx.x; t < Q * P; t += kMassThreads) {
    double b = 0;
#pragma unroll
    for (int i = 0; i < Q * P; i++)  // compile-time indices: the parameter array stays in the constant bank
      if (i == t) b = bas.B[i];
    sB[t] = squared ? b * b : b;
  }
}

template <int P, int Q>
__global__ void __launch_bounds__(kMassThreads) k_mass(const ElemArgs<double> a, const double *__restrict__ u, double *__restrict__ v) {
  constexpr int NT = kMassThreads, P2 = P * P, P3 = P2 * P, Q2 = Q * Q, Q3 = Q2 * Q, P2Q = P2 * Q, PQ2 = P * Q2;
  __shared__ double sB[Q * P];
  __shared__ double sX[5 * Q3], sY[5 * Q3];  // ping-pong; Q >= P so Q^3 bounds every intermediate
  mass_basis_to_smem<P, Q>(a.basis, sB, false);
  for (int idx = blockIdx.x; idx < a.n_elems; idx += gridDim.x) {
    const int e = a.elems[idx];
    const int32_t *off = a.offsets + (int64_t)e * P3;
    for (int i = threadIdx.x; i < 5 * P3; i += NT) sX[(i % 5) * P3 + i / 5] = u[off[i / 5] + i % 5];
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
    const double *wq = a.qdata + (int64_t)e * 10 * Q3;  // component 0: w detJ
    for (int f = threadIdx.x; f < 5 * Q3; f += NT) {  // z, times w detJ: [c][qk][qj][qi]
      const int qji = f % Q2, qk = (f / Q2) % Q, c = f / Q3;
      double s = 0;
#pragma unroll
      for (int k = 0; k < P; k++) s += sB[qk * P + k] * sX[c * PQ2 + k * Q2 + qji];
      sY[f] = s * __ldg(wq + qk * Q2 + qji);
    }
    __syncthreads();
    for (int f = threadIdx.x; f < 5 * PQ2; f += NT) {  // z^T: [c][pc][qj][qi]
      const int qji = f % Q2, pc = (f / Q2) % P, c = f / PQ2;
      double s = 0;
#pragma unroll
      for (int k = 0; k < Q; k++) s += sB[k * P + pc] * sY[c * Q3 + k * Q2 + qji];
      sX[f] = s;
    }
    __syncthreads();
    for (int f = threadIdx.x; f < 5 * P2Q; f += NT) {  // y^T: [c][pc][pb][qi]
      const int qi = f % Q, pb = (f / Q) % P, pc = (f / (Q * P)) % P, c = f / P2Q;
      double s = 0;
#pragma unroll
      for (int j = 0; j < Q; j++) s += sB[j * P + pb] * sX[c * PQ2 + (pc * Q + j) * Q + qi];
      sY[f] = s;
    }
    __syncthreads();
    for (int f = threadIdx.x; f < 5 * P3; f += NT) {  // x^T and the scatter, components fastest (node-interleaved)
      const int c = f % 5, p = f / 5, pa = p % P, pcb = p / P;
      double s = 0;
#pragma unroll
      for (int i = 0; i < Q; i++) s += sB[i * P + pa] * sY[c * P2Q + pcb * Q + i];
      v[off[p] + c] += s;
    }
    // the next gather writes sX, last read before the barrier above; the x^T pass reads sY, next written after a barrier
  }
}

template <int P, int Q>
__global__ void __launch_bounds__(kMassThreads) k_mass_diag(const ElemArgs<double> a, double *__restrict__ diag, int block) {
  constexpr int NT = kMassThreads, P2 = P * P, P3 = P2 * P, Q2 = Q * Q, Q3 = Q2 * Q;
  __shared__ double sW[Q * P];  // B^2
  __shared__ double sX[Q3], sY[Q3];
  mass_basis_to_smem<P, Q>(a.basis, sW, true);
  for (int idx = blockIdx.x; idx < a.n_elems; idx += gridDim.x) {
    const int e = a.elems[idx];
    const double *wq = a.qdata + (int64_t)e * 10 * Q3;
    for (int q = threadIdx.x; q < Q3; q += NT) sX[q] = __ldg(wq + q);
    __syncthreads();
    for (int f = threadIdx.x; f < P * Q2; f += NT) {  // [pc][qj][qi]
      const int qji = f % Q2, pc = f / Q2;
      double s = 0;
#pragma unroll
      for (int k = 0; k < Q; k++) s += sW[k * P + pc] * sX[k * Q2 + qji];
      sY[f] = s;
    }
    __syncthreads();
    for (int f = threadIdx.x; f < P2 * Q; f += NT) {  // [pc][pb][qi]
      const int qi = f % Q, pb = (f / Q) % P, pc = f / (Q * P);
      double s = 0;
#pragma unroll
      for (int j = 0; j < Q; j++) s += sW[j * P + pb] * sY[(pc * Q + j) * Q + qi];
      sX[f] = s;
    }
    __syncthreads();
    for (int f = threadIdx.x; f < 5 * P3; f += NT) {
      const int c = f % 5, p = f / 5, pa = p % P, pcb = p / P;
      double s = 0;
#pragma unroll
      for (int i = 0; i < Q; i++) s += sW[i * P + pa] * sX[pcb * Q + i];
      const int64_t o = a.offsets[(int64_t)e * P3 + p];
      diag[block ? o * 5 + c * 6 : o + c] += s;  // block: entry (c, c) of the node's 5 x 5 block
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------------------------------------------------
// SUPG-stabilized mass of the explicit path (MassFunction_Newtonian, qfunctions/newtonian.h:44-86; HONEE builds it instead of
// Mass_5 when stab = supg and the run is explicit, problems/newtonian.c:212-265, 795): for a rate u at the state q,
//   v = wdetJ u,  grad v = wdetJ dXdx stab(u),  stab = dF(StateFromY_fwd(tau . u)) with tau = Tau_diagPrim(q).
// One CTA per element of a colour: both fields gathered and interpolated, the point function, then the value and the three
// gradient transposes grouped by their remaining factors (z: {B v + G gv_z, B gv_y, B gv_x}; y: {B, G, B}; x: {B, B, G}).
template <typename T>
__device__ __forceinline__ void mass_stab_point(const PhysConst<T> &c, const T q[5], const T u[5], T wdetJ, const T X[3][3], T v[5], T gv[3][5]) {
  St<T> s;
  T inv_rho, etot, eint;
  state_from_u(c, q, s, inv_rho, etot, eint);
#pragma unroll
  for (int i = 0; i < 5; i++) v[i] = wdetJ * u[i];
  St<T> gs[3];
  memset(gs, 0, sizeof gs);
  const T body[5] = {0, 0, 0, 0, 0};
  T tau[3], stab[5][3];
  tau_diag(c, s, X, tau);
  stabilization(c, s, eint, tau, gs, u, body, stab);
#pragma unroll
  for (int k = 0; k < 3; k++)
#pragma unroll
    for (int j = 0; j < 5; j++) gv[k][j] = wdetJ * (stab[j][0] * X[k][0] + stab[j][1] * X[k][1] + stab[j][2] * X[k][2]);
}

template <int P, int Q>
struct MassStabPlan {
  static constexpr int P2 = P * P, P3 = P2 * P, Q2 = Q * Q, Q3 = Q2 * Q, P2Q = P2 * Q, PQ2 = P * Q2;
  static constexpr int oN = 0, oA = oN + 5 * P3, oB = oA + 5 * P2Q, oU = oB + 5 * PQ2, oQ = oU + 5 * Q3, oG = oQ + 5 * Q3, oZ = oG + 15 * Q3,
                       oY = oZ + 15 * PQ2, total = oY + 10 * P2Q;
  static constexpr size_t bytes = sizeof(double) * (size_t)total;
};

// interpolate the 5-component field gathered in sN [5][P3] to sOut [5][Q3] (x, y, z passes through sA, sB)
template <int P, int Q>
__device__ __forceinline__ void interp5(const double *sB1, const double *sN, double *sA, double *sBt, double *sOut) {
  using L = MassStabPlan<P, Q>;
  for (int f = threadIdx.x; f < 5 * L::P2Q; f += kMassThreads) {
    const int qi = f % Q, pcb = (f / Q) % L::P2, c = f / L::P2Q;
    double acc = 0;
#pragma unroll
    for (int i = 0; i < P; i++) acc += sB1[qi * P + i] * sN[c * L::P3 + pcb * P + i];
    sA[f] = acc;
  }
  __syncthreads();
  for (int f = threadIdx.x; f < 5 * L::PQ2; f += kMassThreads) {
    const int qi = f % Q, qj = (f / Q) % Q, pc = (f / L::Q2) % P, c = f / L::PQ2;
    double acc = 0;
#pragma unroll
    for (int j = 0; j < P; j++) acc += sB1[qj * P + j] * sA[c * L::P2Q + (pc * P + j) * Q + qi];
    sBt[f] = acc;
  }
  __syncthreads();
  for (int f = threadIdx.x; f < 5 * L::Q3; f += kMassThreads) {
    const int qji = f % L::Q2, qk = (f / L::Q2) % Q, c = f / L::Q3;
    double acc = 0;
#pragma unroll
    for (int k = 0; k < P; k++) acc += sB1[qk * P + k] * sBt[c * L::PQ2 + k * L::Q2 + qji];
    sOut[f] = acc;
  }
}

struct Grad1D {
  double G[kMaxP * kMaxP];  // reference 1D gradient [Q][P]
};

template <int P, int Q>
__global__ void __launch_bounds__(kMassThreads) k_mass_stab(const ElemArgs<double> a, const Grad1D bg, const double *__restrict__ qs,
                                                            const double *__restrict__ u, double *__restrict__ v) {
  using L = MassStabPlan<P, Q>;
  constexpr int P3 = L::P3, Q2 = L::Q2, Q3 = L::Q3, P2Q = L::P2Q, PQ2 = L::PQ2, NT = kMassThreads;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *sm = reinterpret_cast<double *>(smem_raw);
  double *sN = sm + L::oN, *sA = sm + L::oA, *sBt = sm + L::oB, *sU = sm + L::oU, *sQ = sm + L::oQ, *sG = sm + L::oG, *sZ = sm + L::oZ,
         *sY = sm + L::oY;
  __shared__ double sB1[Q * P], sG1[Q * P];
  for (int t = threadIdx.x; t < Q * P; t += NT) {
    double b = 0, g = 0;
#pragma unroll
    for (int i = 0; i < Q * P; i++)  // compile-time indices: the parameter arrays stay in the constant bank
      if (i == t) {
        b = a.basis.B[i];
        g = bg.G[i];
      }
    sB1[t] = b;
    sG1[t] = g;
  }
  __syncthreads();
  for (int idx = blockIdx.x; idx < a.n_elems; idx += gridDim.x) {
    const int e = a.elems[idx];
    const int32_t *off = a.offsets + (int64_t)e * P3;
    // rate and state at the quadrature points
    for (int i = threadIdx.x; i < 5 * P3; i += NT) sN[(i % 5) * P3 + i / 5] = u[off[i / 5] + i % 5];
    __syncthreads();
    interp5<P, Q>(sB1, sN, sA, sBt, sU);
    __syncthreads();
    for (int i = threadIdx.x; i < 5 * P3; i += NT) sN[(i % 5) * P3 + i / 5] = qs[off[i / 5] + i % 5];
    __syncthreads();
    interp5<P, Q>(sB1, sN, sA, sBt, sQ);
    __syncthreads();
    const double *qd = a.qdata + (int64_t)e * 10 * Q3;
    for (int q = threadIdx.x; q < Q3; q += NT) {
      double wdetJ, X[3][3], qv[5], uv[5], vv[5], gv[3][5];
      load_qdata(qd, Q3, q, wdetJ, X);
#pragma unroll
      for (int c = 0; c < 5; c++) {
        qv[c] = sQ[c * Q3 + q];
        uv[c] = sU[c * Q3 + q];
      }
      mass_stab_point<double>(a.pc, qv, uv, wdetJ, X, vv, gv);
#pragma unroll
      for (int c = 0; c < 5; c++) {
        sU[c * Q3 + q] = vv[c];
#pragma unroll
        for (int d = 0; d < 3; d++) sG[(d * 5 + c) * Q3 + q] = gv[d][c];
      }
    }
    __syncthreads();
    // z: three arrays [g][c][pc][qj][qi]: g0 = B v + G gv_z, g1 = B gv_y, g2 = B gv_x
    for (int f = threadIdx.x; f < 15 * PQ2; f += NT) {
      const int qji = f % Q2, pc = (f / Q2) % P, c = (f / PQ2) % 5, g = f / (5 * PQ2);
      double acc = 0;
#pragma unroll
      for (int k = 0; k < Q; k++) {
        const int qq = k * Q2 + qji;
        if (g == 0) acc += sB1[k * P + pc] * sU[c * Q3 + qq] + sG1[k * P + pc] * sG[(10 + c) * Q3 + qq];
        else acc += sB1[k * P + pc] * sG[((g == 1 ? 5 : 0) + c) * Q3 + qq];
      }
      sZ[f] = acc;
    }
    __syncthreads();
    // y: two arrays [h][c][pc][pb][qi]: h0 = B g0 + G g1 (x factor B), h1 = B g2 (x factor G)
    for (int f = threadIdx.x; f < 10 * P2Q; f += NT) {
      const int qi = f % Q, pb = (f / Q) % P, pc = (f / (Q * P)) % P, c = (f / P2Q) % 5, h = f / (5 * P2Q);
      double acc = 0;
#pragma unroll
      for (int j = 0; j < Q; j++) {
        const int zz = c * PQ2 + (pc * Q + j) * Q + qi;
        if (h == 0) acc += sB1[j * P + pb] * sZ[zz] + sG1[j * P + pb] * sZ[5 * PQ2 + zz];
        else acc += sB1[j * P + pb] * sZ[10 * PQ2 + zz];
      }
      sY[f] = acc;
    }
    __syncthreads();
    for (int f = threadIdx.x; f < 5 * P3; f += NT) {  // x and the scatter, components fastest
      const int c = f % 5, p = f / 5, pa = p % P, pcb = p / P;
      double acc = 0;
#pragma unroll
      for (int i = 0; i < Q; i++) acc += sB1[i * P + pa] * sY[c * P2Q + pcb * Q + i] + sG1[i * P + pa] * sY[5 * P2Q + c * P2Q + pcb * Q + i];
      v[off[p] + c] += acc;
    }
    __syncthreads();
  }
}

// Diagonal of the stabilized mass at the state q: for node p and component c, sum over points of phi_p^2 wdetJ plus
// sum_k phi_p dphi_p/dX_k wdetJ (dXdx stab_c)_k, stab_c the stabilization row c for the unit rate e_c.  Twenty combination
// arrays per element (5 components x {value, X0, X1, X2}) contracted together in three passes.
template <int P, int Q>
struct MassStabDiagPlan {
  static constexpr int P2 = P * P, P3 = P2 * P, Q2 = Q * Q, Q3 = Q2 * Q, P2Q = P2 * Q, PQ2 = P * Q2;
  static constexpr int oN = 0, oTa = oN + 5 * P3, oTb = oTa + 5 * P2Q, oQ = oTb + 5 * PQ2, oA = oQ + 5 * Q3, oY = oA + 20 * Q3,
                       total = oY + 20 * Q2 * P;
  static constexpr size_t bytes = sizeof(double) * (size_t)total;
};

template <int P, int Q>
__global__ void __launch_bounds__(kMassThreads) k_mass_stab_diag(const ElemArgs<double> a, const Grad1D bg, const double *__restrict__ qs,
                                                                 double *__restrict__ diag) {
  using L = MassStabDiagPlan<P, Q>;
  constexpr int P2 = L::P2, P3 = L::P3, Q2 = L::Q2, Q3 = L::Q3, QP2 = Q * L::P2, NT = kMassThreads;  // QP2: [Q][P][P] after the y pass
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *sm = reinterpret_cast<double *>(smem_raw);
  double *sN = sm + L::oN, *sTa = sm + L::oTa, *sTb = sm + L::oTb, *sQ = sm + L::oQ, *sA = sm + L::oA, *sY = sm + L::oY;
  __shared__ double sB1[Q * P], sW[3][Q * P];
  for (int t = threadIdx.x; t < Q * P; t += NT) {
    double b = 0, g = 0;
#pragma unroll
    for (int i = 0; i < Q * P; i++)
      if (i == t) {
        b = a.basis.B[i];
        g = bg.G[i];
      }
    sB1[t] = b;
    sW[0][t] = b * b;
    sW[1][t] = b * g;
    sW[2][t] = g * g;
  }
  __syncthreads();
  for (int idx = blockIdx.x; idx < a.n_elems; idx += gridDim.x) {
    const int e = a.elems[idx];
    const int32_t *off = a.offsets + (int64_t)e * P3;
    for (int i = threadIdx.x; i < 5 * P3; i += NT) sN[(i % 5) * P3 + i / 5] = qs[off[i / 5] + i % 5];
    __syncthreads();
    interp5<P, Q>(sB1, sN, sTa, sTb, sQ);
    __syncthreads();
    const double *qd = a.qdata + (int64_t)e * 10 * Q3;
    for (int q = threadIdx.x; q < Q3; q += NT) {
      double wdetJ, X[3][3], qv[5];
      load_qdata(qd, Q3, q, wdetJ, X);
#pragma unroll
      for (int c = 0; c < 5; c++) qv[c] = sQ[c * Q3 + q];
#pragma unroll
      for (int c = 0; c < 5; c++) {
        double uv[5] = {0, 0, 0, 0, 0}, vv[5], gv[3][5];
        uv[c] = 1.0;
        mass_stab_point<double>(a.pc, qv, uv, wdetJ, X, vv, gv);
        sA[(c * 4 + 0) * Q3 + q] = vv[c];
#pragma unroll
        for (int k = 0; k < 3; k++) sA[(c * 4 + 1 + k) * Q3 + q] = gv[k][c];
      }
    }
    __syncthreads();
    for (int f = threadIdx.x; f < 20 * Q2 * P; f += NT) {  // x: [t][k][j][pa]
      const int t = f / (Q2 * P), rem = f % (Q2 * P), pa = rem % P, kj = rem / P;
      const double *W = sW[combo_sel(t % 4, 0)];
      double acc = 0;
#pragma unroll
      for (int i = 0; i < Q; i++) acc += W[i * P + pa] * sA[t * Q3 + kj * Q + i];
      sY[f] = acc;
    }
    __syncthreads();
    for (int f = threadIdx.x; f < 20 * QP2; f += NT) {  // y: [t][k][pb][pa]
      const int t = f / QP2, rem = f % QP2, pa = rem % P, pb = (rem / P) % P, k = rem / P2;
      const double *W = sW[combo_sel(t % 4, 1)];
      double acc = 0;
#pragma unroll
      for (int j = 0; j < Q; j++) acc += W[j * P + pb] * sY[t * Q2 * P + (k * Q + j) * P + pa];
      sA[f] = acc;
    }
    __syncthreads();
    for (int f = threadIdx.x; f < 5 * P3; f += NT) {  // z, summed over the four combinations, and the scatter
      const int c = f % 5, pp = f / 5, pab = pp % P2, pc_ = pp / P2;
      double acc = 0;
#pragma unroll
      for (int m = 0; m < 4; m++) {
        const double *W = sW[combo_sel(m, 2)];
#pragma unroll
        for (int k = 0; k < Q; k++) acc += W[k * P + pc_] * sA[(c * 4 + m) * QP2 + k * P2 + pab];
      }
      diag[off[pp] + c] += acc;
    }
    __syncthreads();
  }
}

template <int P, int Q>
static int launch_mass_stab(const HbElemOp *op, const HbNewtonianContext &ctx, const double *qdata, const double *qs, const double *u, double *v,
                            bool diagonal, cudaStream_t s) {
  Grad1D bg;
  memset(&bg, 0, sizeof bg);
  for (int i = 0; i < Q * P; i++) bg.G[i] = op->grad1d[i];
  const size_t sm = diagonal ? MassStabDiagPlan<P, Q>::bytes : MassStabPlan<P, Q>::bytes;
  if (diagonal) {
    if (cudaFuncSetAttribute(k_mass_stab_diag<P, Q>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess) return HB_ERROR_CUDA;
  } else {
    if (cudaFuncSetAttribute(k_mass_stab<P, Q>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess) return HB_ERROR_CUDA;
  }
  for (int c = 0; c < op->num_colors; c++) {
    ElemArgs<double> a = make_args<double>(op, ctx, qdata, c);
    if (a.n_elems == 0) continue;
    if (diagonal)
      k_mass_stab_diag<P, Q><<<grid_for(op, a.n_elems, k_mass_stab_diag<P, Q>, kMassThreads, sm), kMassThreads, sm, s>>>(a, bg, qs, v);
    else
      k_mass_stab<P, Q><<<grid_for(op, a.n_elems, k_mass_stab<P, Q>, kMassThreads, sm), kMassThreads, sm, s>>>(a, bg, qs, u, v);
  }
  return cudaGetLastError() == cudaSuccess ? HB_SUCCESS : HB_ERROR_CUDA;
}

template <int P, int Q>
static int launch_mass(const HbElemOp *op, const double *qdata, const double *u, double *v, bool diagonal, cudaStream_t s, int block = 0) {
  for (int c = 0; c < op->num_colors; c++) {
    ElemArgs<double> a;
    memset(&a, 0, sizeof a);
    a.offsets = op->d_offsets;
    a.elems = op->d_color_elem + op->h_color_ptr[c];
    a.n_elems = op->h_color_ptr[c + 1] - op->h_color_ptr[c];
    fill_basis<double>(op, a.basis);
    a.qdata = qdata;
    a.status = op->d_status;
    if (a.n_elems == 0) continue;
    if (diagonal)
      k_mass_diag<P, Q><<<grid_for(op, a.n_elems, k_mass_diag<P, Q>, kMassThreads, 0), kMassThreads, 0, s>>>(a, v, block);
    else
      k_mass<P, Q><<<grid_for(op, a.n_elems, k_mass<P, Q>, kMassThreads, 0), kMassThreads, 0, s>>>(a, u, v);
  }
  return cudaGetLastError() == cudaSuccess ? HB_SUCCESS : HB_ERROR_CUDA;
}

template <int P, int Q, typename T, int SV = HB_STATEVAR_CONSERVATIVE>
static int launch_blockdiag(const HbElemOp *op, const HbNewtonianContext &ctx, const double *qdata, const T *jd, T *out, cudaStream_t s) {
  const size_t sm = blockdiag_smem<P, Q, T>();
  if (cudaFuncSetAttribute(k_blockdiag<P, Q, T, SV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess) return HB_ERROR_CUDA;
  DiagArgs<T> p;
  p.jac_data = jd;
  p.diag = out;
  memset(p.G1, 0, sizeof p.G1);
  for (int i = 0; i < Q * P; i++) p.G1[i] = T(op->grad1d[i]);
  for (int c = 0; c < op->num_colors; c++) {
    ElemArgs<T> a = make_args<T>(op, ctx, qdata, c);
    if (a.n_elems == 0) continue;
    k_blockdiag<P, Q, T, SV><<<grid_for(op, a.n_elems, k_blockdiag<P, Q, T, SV>, nthreads_for<T>(Q), sm), nthreads_for<T>(Q), sm, s>>>(a, p);
  }
  return cudaGetLastError() == cudaSuccess ? HB_SUCCESS : HB_ERROR_CUDA;
}

// (P, Q) pairs compiled: polynomial degree 1..5 with q_extra 0 or 1 (Q = P or P + 1), and q_extra 2 for degrees 1 and 2
// (the channel example's q_extra 2); the benchmark configurations use (3,3), (4,5) and (5,6).
// The compiled (P, Q) lists.  A build with -DHB_BASES_P4Q5_ONLY compiles the degree-3 basis with q_extra 1 alone (every
// kernel, conservative variables only): a quick build for kernel work, not a product configuration.
#ifdef HB_BASES_P4Q5_ONLY
#define HB_PQ_LIST(X) X(4, 5)
#define HB_SGS_PQ_LIST(X)
#define HB_SV_PQ_LIST(X)
#endif
#ifndef HB_PQ_LIST
#define HB_PQ_LIST(X) X(2, 2) X(2, 3) X(2, 4) X(3, 3) X(3, 4) X(3, 5) X(4, 4) X(4, 5) X(5, 5) X(5, 6) X(6, 6) X(6, 7)
#endif
// bases the residual with the fused SGS closure is built for (the coarse LES runs at degree 2 and 3)
#ifndef HB_SGS_PQ_LIST
#define HB_SGS_PQ_LIST(X) X(3, 3) X(3, 4) X(4, 5)
#endif
// bases compiled for the primitive and entropy state variables (degree 1-3 with q_extra 0-2 as HONEE's examples use them)
#ifndef HB_SV_PQ_LIST
#define HB_SV_PQ_LIST(X) X(2, 2) X(2, 3) X(2, 4) X(3, 3) X(3, 4) X(3, 5) X(4, 4) X(4, 5)
#endif

}  // namespace hb

using namespace hb;

static int check_op(const HbElemOp *op) {
  if (!op || op->P < 2 || op->P > kMaxP || op->Q < op->P || op->Q > kMaxP) return HB_ERROR_UNSUPPORTED;
  return HB_SUCCESS;
}

// (P, Q) dispatch for one state variable: every compiled pair for conservative variables, HB_SV_PQ_LIST for the others
template <int SV>
static int ifunction_pq(const HbElemOp *op, const HbNewtonianContext &ctx, const HbIFunctionIO *io, cudaStream_t s) {
#define HB_CASE(PP, QQ) \
  if (op->P == PP && op->Q == QQ) return launch_ifunction<PP, QQ, SV>(op, ctx, io, s);
  if constexpr (SV == HB_STATEVAR_CONSERVATIVE) {
    HB_PQ_LIST(HB_CASE)
  } else {
    HB_SV_PQ_LIST(HB_CASE)
  }
#undef HB_CASE
  return HB_ERROR_UNSUPPORTED;
}

extern "C" int hb_ifunction_apply(const HbElemOp *op, const void *ctx184, const HbIFunctionIO *io, void *stream) {
  int err = check_op(op);
  if (err) return err;
  HbNewtonianContext ctx;
  memcpy(&ctx, ctx184, sizeof ctx);
  if (ctx.divFdiff_method != HB_DIV_DIFF_FLUX_PROJ_NONE) return HB_ERROR_UNSUPPORTED;
  if (ctx.idl_enable && !op->d_x_elem) return HB_ERROR_INVALID;
  if (ctx.state_var != HB_STATEVAR_CONSERVATIVE && ctx.state_var != HB_STATEVAR_PRIMITIVE && ctx.state_var != HB_STATEVAR_ENTROPY)
    return HB_ERROR_UNSUPPORTED;
  cudaStream_t s = (cudaStream_t)stream;
  if (!io->add && cudaMemsetAsync(io->v, 0, sizeof(double) * op->l_size, s) != cudaSuccess) return HB_ERROR_CUDA;
  if (ctx.state_var == HB_STATEVAR_PRIMITIVE) return ifunction_pq<HB_STATEVAR_PRIMITIVE>(op, ctx, io, s);
  if (ctx.state_var == HB_STATEVAR_ENTROPY) return ifunction_pq<HB_STATEVAR_ENTROPY>(op, ctx, io, s);
  return ifunction_pq<HB_STATEVAR_CONSERVATIVE>(op, ctx, io, s);
}

template <int SGS>
static int fill_sgs(const HbMlpDesc *d, const float *w, SgsArg<SGS> &sg) {
  const int np = hb_mlp_num_params(d);
  if (np != (int)(sizeof sg.w / sizeof sg.w[0])) return HB_ERROR_INVALID;
  memcpy(sg.w, w, sizeof sg.w);
  sg.alpha = d->leaky_alpha;
  memcpy(sg.b, d->out_bounds, sizeof sg.b);
  sg.clamp = d->clamp_outputs;
  sg.no_backscatter = d->no_backscatter;
  return HB_SUCCESS;
}

template <int SGS, int SV>
static int ifunction_sgs_pq(const HbElemOp *op, const HbNewtonianContext &ctx, const HbIFunctionIO *io, const SgsArg<SGS> &sg, cudaStream_t s) {
#define HB_CASE(PP, QQ) \
  if (op->P == PP && op->Q == QQ) return launch_ifunction_v<PP, QQ, SGS, SV>(op, ctx, io, s, sg);
  HB_SGS_PQ_LIST(HB_CASE)
#undef HB_CASE
  return HB_ERROR_UNSUPPORTED;
}
template <int SGS>
static int ifunction_sgs_sv(const HbElemOp *op, const HbNewtonianContext &ctx, const HbIFunctionIO *io, const SgsArg<SGS> &sg, cudaStream_t s) {
  if (ctx.state_var == HB_STATEVAR_PRIMITIVE) return ifunction_sgs_pq<SGS, HB_STATEVAR_PRIMITIVE>(op, ctx, io, sg, s);
  if (ctx.state_var == HB_STATEVAR_ENTROPY) return ifunction_sgs_pq<SGS, HB_STATEVAR_ENTROPY>(op, ctx, io, sg, s);
  return ifunction_sgs_pq<SGS, HB_STATEVAR_CONSERVATIVE>(op, ctx, io, sg, s);
}

extern "C" int hb_ifunction_apply_sgs(const HbElemOp *op, const void *ctx184, const HbIFunctionIO *io, const HbMlpDesc *d, const float *h_weights,
                                      void *stream) {
  int err = check_op(op);
  if (err) return err;
  if (!d || !h_weights || d->hidden1 != 20 || (d->hidden2 != 0 && d->hidden2 != 20)) return HB_ERROR_INVALID;
  HbNewtonianContext ctx;
  memcpy(&ctx, ctx184, sizeof ctx);
  if (ctx.divFdiff_method != HB_DIV_DIFF_FLUX_PROJ_NONE) return HB_ERROR_UNSUPPORTED;
  if (ctx.state_var != HB_STATEVAR_CONSERVATIVE && ctx.state_var != HB_STATEVAR_PRIMITIVE && ctx.state_var != HB_STATEVAR_ENTROPY)
    return HB_ERROR_UNSUPPORTED;
  if (ctx.idl_enable && !op->d_x_elem) return HB_ERROR_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  if (!io->add && cudaMemsetAsync(io->v, 0, sizeof(double) * op->l_size, s) != cudaSuccess) return HB_ERROR_CUDA;
  if (d->hidden2 == 20) {
    SgsArg<2> sg;
    if ((err = fill_sgs<2>(d, h_weights, sg))) return err;
    return ifunction_sgs_sv<2>(op, ctx, io, sg, s);
  }
  SgsArg<1> sg;
  if ((err = fill_sgs<1>(d, h_weights, sg))) return err;
  return ifunction_sgs_sv<1>(op, ctx, io, sg, s);
}

template <typename T, int SV>
static int ijacobian_pq(const HbElemOp *op, const HbNewtonianContext &ctx, const double *qdata, const T *jd, const T *dq, T *v, cudaStream_t s) {
  if constexpr (sizeof(T) == 4 && SV == HB_STATEVAR_CONSERVATIVE) {  // FP32: element pairs in packed FP32 where the basis allows
    if (((uintptr_t)qdata % 16) == 0 && op->Q <= 5) {  // three CTAs per SM; at Q = 6 the pair kernel would run one
#define HB_CASE(PP, QQ) \
  if (op->P == PP && op->Q == QQ) return pair_case<PP, QQ, SV>(op, ctx, qdata, (const float *)jd, (const float *)dq, (float *)v, s);
      HB_PQ_LIST(HB_CASE)
#undef HB_CASE
    }
  }
#define HB_CASE(PP, QQ) \
  if (op->P == PP && op->Q == QQ) return launch_ijacobian<PP, QQ, T, SV>(op, ctx, qdata, jd, dq, v, s);
  if constexpr (SV == HB_STATEVAR_CONSERVATIVE) {
    HB_PQ_LIST(HB_CASE)
  } else {
    HB_SV_PQ_LIST(HB_CASE)
  }
#undef HB_CASE
  return HB_ERROR_UNSUPPORTED;
}

extern "C" int hb_ijacobian_apply_f64(const HbElemOp *op, const void *ctx184, const double *qdata, const double *jac_data, const double *dq,
                                      double *v, int add, void *stream) {
  int err = check_op(op);
  if (err) return err;
  HbNewtonianContext ctx;
  memcpy(&ctx, ctx184, sizeof ctx);
  if (ctx.state_var != HB_STATEVAR_CONSERVATIVE && ctx.state_var != HB_STATEVAR_PRIMITIVE && ctx.state_var != HB_STATEVAR_ENTROPY)
    return HB_ERROR_UNSUPPORTED;
  cudaStream_t s = (cudaStream_t)stream;
  if (!add && cudaMemsetAsync(v, 0, sizeof(double) * op->l_size, s) != cudaSuccess) return HB_ERROR_CUDA;
  if (ctx.state_var == HB_STATEVAR_PRIMITIVE) return ijacobian_pq<double, HB_STATEVAR_PRIMITIVE>(op, ctx, qdata, jac_data, dq, v, s);
  if (ctx.state_var == HB_STATEVAR_ENTROPY) return ijacobian_pq<double, HB_STATEVAR_ENTROPY>(op, ctx, qdata, jac_data, dq, v, s);
  return ijacobian_pq<double, HB_STATEVAR_CONSERVATIVE>(op, ctx, qdata, jac_data, dq, v, s);
}

extern "C" int hb_ijacobian_apply_f32(const HbElemOp *op, const void *ctx184, const double *qdata, const float *jac_data, const float *dq,
                                      float *v, int add, void *stream) {
  int err = check_op(op);
  if (err) return err;
  HbNewtonianContext ctx;
  memcpy(&ctx, ctx184, sizeof ctx);
  if (ctx.state_var != HB_STATEVAR_CONSERVATIVE && ctx.state_var != HB_STATEVAR_PRIMITIVE && ctx.state_var != HB_STATEVAR_ENTROPY)
    return HB_ERROR_UNSUPPORTED;
  cudaStream_t s = (cudaStream_t)stream;
  if (!add && cudaMemsetAsync(v, 0, sizeof(float) * op->l_size, s) != cudaSuccess) return HB_ERROR_CUDA;
  if (ctx.state_var == HB_STATEVAR_PRIMITIVE) return ijacobian_pq<float, HB_STATEVAR_PRIMITIVE>(op, ctx, qdata, jac_data, dq, v, s);
  if (ctx.state_var == HB_STATEVAR_ENTROPY) return ijacobian_pq<float, HB_STATEVAR_ENTROPY>(op, ctx, qdata, jac_data, dq, v, s);
  return ijacobian_pq<float, HB_STATEVAR_CONSERVATIVE>(op, ctx, qdata, jac_data, dq, v, s);
}

template <typename T, int SV>
static int diagonal_pq(const HbElemOp *op, const HbNewtonianContext &ctx, const double *qdata, const T *jd, T *diag, cudaStream_t s) {
#define HB_CASE(PP, QQ) \
  if (op->P == PP && op->Q == QQ) return launch_diagonal<PP, QQ, T, SV>(op, ctx, qdata, jd, diag, s);
  if constexpr (SV == HB_STATEVAR_CONSERVATIVE) {
    HB_PQ_LIST(HB_CASE)
  } else {
    HB_SV_PQ_LIST(HB_CASE)
  }
#undef HB_CASE
  return HB_ERROR_UNSUPPORTED;
}

extern "C" int hb_diagonal_assemble_f64(const HbElemOp *op, const void *ctx184, const double *qdata, const double *jac_data, double *diag, int add,
                                        void *stream) {
  int err = check_op(op);
  if (err) return err;
  HbNewtonianContext ctx;
  memcpy(&ctx, ctx184, sizeof ctx);
  if (ctx.state_var != HB_STATEVAR_CONSERVATIVE && ctx.state_var != HB_STATEVAR_PRIMITIVE && ctx.state_var != HB_STATEVAR_ENTROPY)
    return HB_ERROR_UNSUPPORTED;
  cudaStream_t s = (cudaStream_t)stream;
  if (!add && cudaMemsetAsync(diag, 0, sizeof(double) * op->l_size, s) != cudaSuccess) return HB_ERROR_CUDA;
  if (ctx.state_var == HB_STATEVAR_PRIMITIVE) return diagonal_pq<double, HB_STATEVAR_PRIMITIVE>(op, ctx, qdata, jac_data, diag, s);
  if (ctx.state_var == HB_STATEVAR_ENTROPY) return diagonal_pq<double, HB_STATEVAR_ENTROPY>(op, ctx, qdata, jac_data, diag, s);
  return diagonal_pq<double, HB_STATEVAR_CONSERVATIVE>(op, ctx, qdata, jac_data, diag, s);
}

extern "C" int hb_diagonal_assemble_f32(const HbElemOp *op, const void *ctx184, const double *qdata, const float *jac_data, float *diag, int add,
                                        void *stream) {
  int err = check_op(op);
  if (err) return err;
  HbNewtonianContext ctx;
  memcpy(&ctx, ctx184, sizeof ctx);
  if (ctx.state_var != HB_STATEVAR_CONSERVATIVE && ctx.state_var != HB_STATEVAR_PRIMITIVE && ctx.state_var != HB_STATEVAR_ENTROPY)
    return HB_ERROR_UNSUPPORTED;
  cudaStream_t s = (cudaStream_t)stream;
  if (!add && cudaMemsetAsync(diag, 0, sizeof(float) * op->l_size, s) != cudaSuccess) return HB_ERROR_CUDA;
  if (ctx.state_var == HB_STATEVAR_PRIMITIVE) return diagonal_pq<float, HB_STATEVAR_PRIMITIVE>(op, ctx, qdata, jac_data, diag, s);
  if (ctx.state_var == HB_STATEVAR_ENTROPY) return diagonal_pq<float, HB_STATEVAR_ENTROPY>(op, ctx, qdata, jac_data, diag, s);
  return diagonal_pq<float, HB_STATEVAR_CONSERVATIVE>(op, ctx, qdata, jac_data, diag, s);
}

extern "C" int hb_setup_qdata(int num_elem, int Q, const double *qref1d, const double *qweight1d, const double *x_elem, double *qdata, void *stream) {
  if (Q < 1 || Q > kMaxP || num_elem <= 0) return HB_ERROR_INVALID;
  QRef r, w;
  for (int i = 0; i < kMaxP; i++) {
    r.x[i] = i < Q ? qref1d[i] : 0;
    w.x[i] = i < Q ? qweight1d[i] : 0;
  }
  const int64_t n = (int64_t)num_elem * Q * Q * Q;
  const int bs = 256;
  k_setup_qdata<<<(unsigned)((n + bs - 1) / bs), bs, 0, (cudaStream_t)stream>>>(num_elem, Q, x_elem, r, w, qdata);
  return cudaGetLastError() == cudaSuccess ? HB_SUCCESS : HB_ERROR_CUDA;
}

#ifdef HB_PHASE_TIMING
extern "C" HB_EXPORT int hb_debug_phase_cycles(unsigned long long *out, int reset) {
  if (cudaDeviceSynchronize() != cudaSuccess) return HB_ERROR_CUDA;
  if (cudaMemcpyFromSymbol(out, hb_phase_cycles, sizeof(unsigned long long) * 16) != cudaSuccess) return HB_ERROR_CUDA;
  if (reset) {
    unsigned long long z[16] = {0};
    cudaMemcpyToSymbol(hb_phase_cycles, z, sizeof z);
  }
  return HB_SUCCESS;
}
#endif

extern "C" int hb_mass_apply(const HbElemOp *op, const double *qdata, const double *u, double *v, int add, void *stream) {
  int err = check_op(op);
  if (err) return err;
  if (!qdata || !u || !v) return HB_ERROR_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  if (!add && cudaMemsetAsync(v, 0, sizeof(double) * op->l_size, s) != cudaSuccess) return HB_ERROR_CUDA;
#define HB_CASE(PP, QQ) \
  if (op->P == PP && op->Q == QQ) return launch_mass<PP, QQ>(op, qdata, u, v, false, s);
  HB_PQ_LIST(HB_CASE)
#undef HB_CASE
  return HB_ERROR_UNSUPPORTED;
}

extern "C" int hb_mass_diagonal(const HbElemOp *op, const double *qdata, double *diag, int add, void *stream) {
  int err = check_op(op);
  if (err) return err;
  if (!qdata || !diag) return HB_ERROR_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  if (!add && cudaMemsetAsync(diag, 0, sizeof(double) * op->l_size, s) != cudaSuccess) return HB_ERROR_CUDA;
#define HB_CASE(PP, QQ) \
  if (op->P == PP && op->Q == QQ) return launch_mass<PP, QQ>(op, qdata, NULL, diag, true, s);
  HB_PQ_LIST(HB_CASE)
#undef HB_CASE
  return HB_ERROR_UNSUPPORTED;
}

// Point-block diagonal of the IJacobian operator: out[(node * 5 + i) * 5 + j] (+)= d v_(node,i) / d dq_(node,j), i.e. one
// row-major 5 x 5 block per node of the node-interleaved L-vector (out holds l_size * 5 values).
template <typename T, int SV>
static int pbdiag_pq(const HbElemOp *op, const HbNewtonianContext &ctx, const double *qdata, const T *jd, T *out, cudaStream_t s) {
#define HB_CASE(PP, QQ) \
  if (op->P == PP && op->Q == QQ) return launch_blockdiag<PP, QQ, T, SV>(op, ctx, qdata, jd, out, s);
  if constexpr (SV == HB_STATEVAR_CONSERVATIVE) {
    HB_PQ_LIST(HB_CASE)
  } else {
    HB_SV_PQ_LIST(HB_CASE)
  }
#undef HB_CASE
  return HB_ERROR_UNSUPPORTED;
}

template <typename T>
static int pbdiag_dispatch(const HbElemOp *op, const void *ctx184, const double *qdata, const T *jac_data, T *out, int add, void *stream) {
  int err = check_op(op);
  if (err) return err;
  if (!ctx184 || !qdata || !jac_data || !out) return HB_ERROR_INVALID;
  HbNewtonianContext ctx;
  memcpy(&ctx, ctx184, sizeof ctx);
  if (ctx.state_var != HB_STATEVAR_CONSERVATIVE && ctx.state_var != HB_STATEVAR_PRIMITIVE && ctx.state_var != HB_STATEVAR_ENTROPY)
    return HB_ERROR_UNSUPPORTED;
  cudaStream_t s = (cudaStream_t)stream;
  if (!add && cudaMemsetAsync(out, 0, sizeof(T) * (size_t)op->l_size * 5, s) != cudaSuccess) return HB_ERROR_CUDA;
  if (ctx.state_var == HB_STATEVAR_PRIMITIVE) return pbdiag_pq<T, HB_STATEVAR_PRIMITIVE>(op, ctx, qdata, jac_data, out, s);
  if (ctx.state_var == HB_STATEVAR_ENTROPY) return pbdiag_pq<T, HB_STATEVAR_ENTROPY>(op, ctx, qdata, jac_data, out, s);
  return pbdiag_pq<T, HB_STATEVAR_CONSERVATIVE>(op, ctx, qdata, jac_data, out, s);
}

extern "C" int hb_point_block_diagonal_f64(const HbElemOp *op, const void *ctx184, const double *qdata, const double *jac_data, double *out, int add,
                                           void *stream) {
  return pbdiag_dispatch<double>(op, ctx184, qdata, jac_data, out, add, stream);
}
extern "C" int hb_point_block_diagonal_f32(const HbElemOp *op, const void *ctx184, const double *qdata, const float *jac_data, float *out, int add,
                                           void *stream) {
  return pbdiag_dispatch<float>(op, ctx184, qdata, jac_data, out, add, stream);
}

// the mass operator's point blocks: its diagonal on the diagonal of each node's 5 x 5 block (the components decouple)
extern "C" int hb_mass_point_block_diagonal(const HbElemOp *op, const double *qdata, double *out, int add, void *stream) {
  int err = check_op(op);
  if (err) return err;
  if (!qdata || !out) return HB_ERROR_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  if (!add && cudaMemsetAsync(out, 0, sizeof(double) * op->l_size * 5, s) != cudaSuccess) return HB_ERROR_CUDA;
#define HB_CASE(PP, QQ) \
  if (op->P == PP && op->Q == QQ) return launch_mass<PP, QQ>(op, qdata, NULL, out, true, s, 1);
  HB_PQ_LIST(HB_CASE)
#undef HB_CASE
  return HB_ERROR_UNSUPPORTED;
}

// SUPG-stabilized mass (MassFunction_Newtonian) at the state qs: v (+)= M_stab(qs) u, and its diagonal
template <bool DIAG>
static int mass_stab_dispatch(const HbElemOp *op, const void *ctx184, const double *qdata, const double *qs, const double *u, double *v, int add,
                              void *stream) {
  int err = check_op(op);
  if (err) return err;
  if (!ctx184 || !qdata || !qs || (!DIAG && !u) || !v) return HB_ERROR_INVALID;
  HbNewtonianContext ctx;
  memcpy(&ctx, ctx184, sizeof ctx);
  if (ctx.state_var != HB_STATEVAR_CONSERVATIVE) return HB_ERROR_UNSUPPORTED;
  cudaStream_t s = (cudaStream_t)stream;
  if (!add && cudaMemsetAsync(v, 0, sizeof(double) * op->l_size, s) != cudaSuccess) return HB_ERROR_CUDA;
#define HB_CASE(PP, QQ) \
  if (op->P == PP && op->Q == QQ) return launch_mass_stab<PP, QQ>(op, ctx, qdata, qs, u, v, DIAG, s);
  HB_PQ_LIST(HB_CASE)
#undef HB_CASE
  return HB_ERROR_UNSUPPORTED;
}

extern "C" int hb_mass_stab_apply(const HbElemOp *op, const void *ctx184, const double *qdata, const double *q_state, const double *u, double *v,
                                  int add, void *stream) {
  return mass_stab_dispatch<false>(op, ctx184, qdata, q_state, u, v, add, stream);
}
extern "C" int hb_mass_stab_diagonal(const HbElemOp *op, const void *ctx184, const double *qdata, const double *q_state, double *diag, int add,
                                     void *stream) {
  return mass_stab_dispatch<true>(op, ctx184, qdata, q_state, NULL, diag, add, stream);
}
