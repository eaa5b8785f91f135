/* honee_oracle.h -- CPU oracle for the HONEE Newtonian operator (TEST INFRASTRUCTURE ONLY).
 *
 * This is the checker, not the product: only tests/, the smoke check of __graft_entry__.py and the cpu_baseline /
 * reference legs of bench.py load it.  The product library (honee-4aiad_b200/) never links or calls it.
 *
 * It restates, in plain C99, (1) the point-wise QFunction arithmetic of the reference (qfunctions/newtonian*.h,
 * stabilization.h, setupgeo.h, utils.h, monitor_totalkineticenergy.h, taylorgreen.h) and (2) the libCEED operator
 * semantics HONEE relies on (element restriction, tensor-product H1 basis, operator apply, diagonal assembly), which
 * live in the un-vendored third-party libCEED (pinned by the reference's goldens as libCEED 0.12.0,
 * v0.12.0-1263-ge205ca3fa, tests/output/taylorgreen_totalke.csv:3-4).  Each function cites the reference lines it
 * follows.  The restatement is pinned against the reference's own QFunctions compiled unchanged into oracle/_ref
 * (oracle/Makefile) and against the reference's known-answer tests (problems/newtonian.c:947-987 state round trips,
 * tests/output/taylorgreen_totalke.csv step-0 kinetic energy).
 */
#ifndef HONEE_ORACLE_H
#define HONEE_ORACLE_H

#include <stdint.h>

#include "honee_b200_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* libCEED QFunction calling convention: in[i]/out[i] are component-major arrays [num_comp][Q]
 * (gradients [dim][num_comp][Q]). */
typedef int (*OracleQF)(void *ctx, int Q, const double *const *in, double *const *out);

/* ---- point-wise state algebra (qfunctions/newtonian_state.h) ---- */
typedef struct {
  double U[5]; /* density, momentum[3], total energy */
  double Y[5]; /* pressure, velocity[3], temperature */
} OracleState;

OracleState oracle_state_from_q(const HbGasProperties *gas, const double q[5], int state_var);
OracleState oracle_state_from_q_fwd(const HbGasProperties *gas, const OracleState *s, const double dq[5], int state_var);
void        oracle_state_to_q(const HbGasProperties *gas, const OracleState *s, double q[5], int state_var);
void        oracle_state_to_q_fwd(const HbGasProperties *gas, const OracleState *s, const OracleState *ds, double dq[5], int state_var);

/* ---- QFunctions (libCEED batch interface) ---- */
int oracle_qf_ifunction_conserv(void *ctx, int Q, const double *const *in, double *const *out);
int oracle_qf_ifunction_prim(void *ctx, int Q, const double *const *in, double *const *out);
int oracle_qf_ifunction_entropy(void *ctx, int Q, const double *const *in, double *const *out);
int oracle_qf_ijacobian_conserv(void *ctx, int Q, const double *const *in, double *const *out);
int oracle_qf_ijacobian_prim(void *ctx, int Q, const double *const *in, double *const *out);
int oracle_qf_ijacobian_entropy(void *ctx, int Q, const double *const *in, double *const *out);
int oracle_qf_setup(void *ctx, int Q, const double *const *in, double *const *out);
int oracle_qf_monitor_ke_conserv(void *ctx, int Q, const double *const *in, double *const *out);
int oracle_qf_ics_taylorgreen(void *ctx, int Q, const double *const *in, double *const *out);

/* ---- 1D tabulation (PETSc Lagrange on Gauss-Lobatto nodes, Gauss-Legendre quadrature; src/dm-utils.c:594-735) ---- */
void oracle_gauss_legendre(int Q, double *x, double *w);
void oracle_gauss_lobatto(int P, double *x);
void oracle_lagrange_tabulate(int P, const double *nodes, int Q, const double *pts, double *interp, double *grad);

/* ---- structured hex box (stand-in for DMPlex box meshes) ----
 * Elements are numbered lexicographically (x fastest); nodes of the order-(P-1) mesh likewise.  L-vectors are
 * node-interleaved [node][ncomp] (src/setupdm.c:51), offsets are int32 node*ncomp with comp_stride 1
 * (src/dm-utils.c:83-137).  Periodic directions identify the last node plane with the first. */
int64_t oracle_box_num_nodes(const int n[3], int P, const int periodic[3]);
void    oracle_box_offsets(const int n[3], int P, const int periodic[3], int ncomp, int32_t *offsets);
/* Element-local vertex coordinates x_elem [elem][3][8] (E-vector of the P=2 coordinate field, vertex a+2(b+2c))
 * of the tensor mesh whose vertex planes are xs[0..n0], ys[0..n1], zs[0..n2]. */
void oracle_box_elem_coords(const int n[3], const double *xs, const double *ys, const double *zs, double *x_elem);

/* ---- libCEED operator semantics ----
 * A "volume operator" is one interior QFunction over all elements with
 *   active input  : restriction (offsets, ncomp=5, comp_stride 1) + H1 tensor basis (P, Q), eval modes listed in
 *                   in_modes (bit 1 = INTERP, bit 2 = GRAD) -- the QFunction's first inputs
 *   passive inputs: per-element strided arrays [elem][comp][Q^3] (qdata, jac_data) or an E-vector interpolated field
 *   active output : INTERP + GRAD summed back through the transpose basis and restriction.
 * Strided layout follows libCEED's CEED_STRIDES_BACKEND for /cpu/self ([elem][comp][qpt]). */
typedef struct {
  int            num_elem, P, Q;
  const int32_t *offsets;                /* [num_elem][P^3] */
  const double  *interp1d, *grad1d;      /* [Q][P] row major */
  const double  *qweight1d;              /* [Q] */
  int            num_threads;            /* OpenMP threads, <=0: runtime default */
  const int32_t *color_ptr, *color_elem; /* optional element colouring (CSR): used for race-free threading */
  int            num_colors;
} OracleMesh;

/* IFunction: v = F(q, q_dot) and jac_data (optional, [elem][num_jd][Q^3]); x_e is [elem][3][Q^3] coordinates at
 * quadrature points (only read when the context enables the IDL); v is overwritten. */
int oracle_apply_ifunction(const OracleMesh *m, OracleQF qf, void *ctx, const double *q, const double *q_dot, const double *qdata,
                           const double *x_q, double *jac_data, int num_jd, double *v, int64_t l_size);
/* IJacobian action: v = J dq using stored jac_data (read-only); v is overwritten. */
int oracle_apply_ijacobian(const OracleMesh *m, OracleQF qf, void *ctx, const double *dq, const double *qdata, const double *jac_data,
                           int num_jd, double *v, int64_t l_size);
/* Point-wise diagonal of the IJacobian operator (CeedOperatorLinearAssembleDiagonal semantics): linearise the
 * QFunction at each quadrature point with unit inputs, then contract with the squared basis rows. diag overwritten. */
int oracle_assemble_diagonal(const OracleMesh *m, OracleQF qf, void *ctx, const double *qdata, const double *jac_data, int num_jd,
                             double *diag, int64_t l_size);
/* Explicit path.  RHSFunction_Newtonian (qfunctions/newtonian.h:133-202) applied as an operator: inputs q (INTERP),
 * Grad_q (GRAD), qdata, x; outputs v (INTERP) and Grad_v (GRAD) (src/setuplibceed.c:179-205).  v is overwritten. */
int oracle_apply_rhs(const OracleMesh *m, OracleQF qf, void *ctx, const double *q, const double *qdata, const double *x_q, double *v,
                     int64_t l_size);
/* The restatement of RHSFunction_Newtonian: the IFunction integrand at q_dot = 0 with the sign reversed (same in/out
 * layout as the reference QFunction). */
int oracle_qf_rhs_conserv(void *ctx, int Q, const double *const *in, double *const *out);
/* Mass operator (Mass_N, N = 5, qfunctions/mass.h:19-26; src/setuplibceed.c:15-53): v = M u through the QFunction qf
 * (in: u [5][Q], qdata [10][Q]; out: v [5][Q]) -- oracle_qf_mass or the reference's Mass_5.  v is overwritten. */
int oracle_apply_mass(const OracleMesh *m, OracleQF qf, const double *u, const double *qdata, double *v, int64_t l_size);
int oracle_qf_mass(void *ctx, int Q, const double *const *in, double *const *out);
/* The SUPG-stabilized mass operator (MassFunction_Newtonian: in q_dot [5][Q], q [5][Q], qdata [10][Q]; out v [5][Q],
 * Grad_v [3][5][Q]), applied to q_dot at the state q.  v is overwritten. */
int oracle_apply_mass_stab(const OracleMesh *m, OracleQF qf, void *ctx, const double *q_dot, const double *q, const double *qdata, double *v,
                           int64_t l_size);
int oracle_qf_mass_stab_conserv(void *ctx, int Q, const double *const *in, double *const *out);
int oracle_assemble_mass_stab_diagonal(const OracleMesh *m, OracleQF qf, void *ctx, const double *q, const double *qdata, double *diag,
                                       int64_t l_size);

/* Point-block diagonal of the IJacobian operator (CeedOperatorLinearAssemblePointBlockDiagonal semantics): a row-major
 * 5 x 5 block per node, out[(node * 5 + i) * 5 + j] (5 * l_size values), overwritten. */
int oracle_assemble_point_block(const OracleMesh *m, OracleQF qf, void *ctx, const double *qdata, const double *jac_data, int num_jd, double *out,
                                int64_t l_size);

/* Geometric factors: qdata [elem][10][Q^3] from vertex coordinates x_elem [elem][3][8] (P=2 linear coordinate basis
 * with the same Gauss rule; src/qdata.c:133-190, qfunctions/setupgeo.h:42-56). */
int oracle_setup_qdata(int num_elem, int Q, const double *x_elem, double *qdata);
/* Coordinates at quadrature points [elem][3][Q^3] from x_elem (interpolation with the linear coordinate basis). */
int oracle_coords_at_qpts(int num_elem, int Q, const double *x_elem, double *x_q);
/* Total kinetic energy monitor sums (5 values, not yet divided by the volume; src/monitor_totalkineticenergy.c:134-163). */
int oracle_monitor_ke(const OracleMesh *m, void *ctx, const double *q, const double *qdata, double sums[5]);

/* Element gather/scatter (libCEED restriction NOTRANSPOSE/TRANSPOSE) for tests of the restriction maps. */
void oracle_restrict(int num_elem, int elem_size, int ncomp, int comp_stride, const int32_t *offsets, const double *l, double *e);
void oracle_restrict_t(int num_elem, int elem_size, int ncomp, int comp_stride, const int32_t *offsets, const double *e, double *l);

#ifdef __cplusplus
}
#endif
#endif
