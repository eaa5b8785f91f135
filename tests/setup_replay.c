/* setup_replay.c -- HONEE's set-up and first applies, call for call, against the libCEED API of libceed_b200.so.
 *
 * Test driver compiled by tests/test_gpu_setup_replay.py into a small shared library (gcc, include/ceed/ceed.h, linked
 * against libceed_b200.so).  replay() makes the calls navierstokes makes, in its order, with the structured box mesh
 * standing in for DMPlex (restriction offsets and coordinates come from the test):
 *   SetupLibceed (src/setuplibceed.c:97-340): solution basis and restriction, jac_data, q / q_dot / g vectors, the
 *     coordinate field, QDataGet (src/qdata.c:133-190, the Setup QFunction), the initial-condition operator on the
 *     projection basis (CeedBasisCreateProjection, :143-175), the IFunction and IJacobian volume operators (:209-269)
 *     and their composites (:295-306), the context labels (:318-326)
 *   ICs_FixMultiplicity (src/misc.c:16-45): op_ics applied to the coordinates, the multiplicity of the solution
 *     restriction (CeedElemRestrictionGetMultiplicity), the state divided by it
 *   IFunction_NS (src/setupts.c:78-125): labels "solution time" and "timestep size" set, the composite applied
 *   FormIJacobian_NS / MatMult_Ceed / MatGetDiagonal_Ceed (src/setupts.c:131-157, src/mat-ceed.c:1603-1700): shift label,
 *     the IJacobian composite applied and its diagonal assembled
 *   SetupMontiorTotalKineticEnergy / TSMonitor_TotalKineticEnergy (src/monitor_totalkineticenergy.c:49-163) and the CFL
 *     monitor (src/monitor_cfl.c:49-167): the monitor operators on the collocated strided restrictions, summed / min-maxed
 * Every call goes through PetscCallCeed-style error checking: the first failure returns with the stored message. */
#include <ceed.h>
#include <stddef.h>
#include <stdio.h>
#include <string.h>

typedef struct {
  const char   *resource;
  int           num_elem, P, Q;
  long long     l_size;
  const int    *offsets; /* [E][P^3] node * 5 */
  const double *x_coord; /* element-local coordinates [E][8][3] */
  const void   *newt_ctx; /* 184 bytes */
  const char   *ic_name;  /* e.g. "taylorgreen.h:ICsTaylorGreen" */
  const void   *ic_ctx;
  size_t        ic_ctx_size;
  const double *q_dot, *dq;
  double        time, dt, shift;
  int           state_var; /* of the Newtonian context: selects the *_Conserv / *_Prim / *_Entropy QFunctions */
} ReplayIn;

typedef struct {
  double *q0, *mult, *v, *jv, *diag; /* l_size each */
  double  ke[5], cfl[2];
  char    msg[512];
} ReplayOut;

#define CKR(x)                                                            \
  do {                                                                    \
    int ierr_ = (x);                                                      \
    if (ierr_) {                                                          \
      const char *m_ = "";                                                \
      CeedGetErrorMessage(ceed, &m_);                                     \
      snprintf(out->msg, sizeof out->msg, "%s -> %d: %s", #x, ierr_, m_); \
      return ierr_;                                                       \
    }                                                                     \
  } while (0)

static int read_host(Ceed ceed, CeedVector v, double *dst, long long n, ReplayOut *out) {
  const CeedScalar *a;
  CKR(CeedVectorGetArrayRead(v, CEED_MEM_HOST, &a));
  memcpy(dst, a, sizeof(double) * (size_t)n);
  CKR(CeedVectorRestoreArrayRead(v, &a));
  return 0;
}

int replay(const ReplayIn *in, ReplayOut *out) {
  Ceed ceed = NULL;
  out->msg[0] = 0;
  if (CeedInit(in->resource, &ceed)) {
    const char *m = "";
    CeedGetErrorMessage(NULL, &m);
    snprintf(out->msg, sizeof out->msg, "CeedInit: %s", m);
    return 1;
  }
  CKR(CeedSetErrorHandler(ceed, CeedErrorStore));
  const int   E = in->num_elem, P = in->P, Q = in->Q, P3 = P * P * P, Q3 = Q * Q * Q, njd = 14;
  const char *sv = in->state_var == 1 ? "Prim" : (in->state_var == 2 ? "Entropy" : "Conserv");
  char        name[128];

  /* -- bases and restrictions (src/setuplibceed.c:113-135; DMPlexCeedBasisCreate / DMPlexCeedElemRestrictionCreate) */
  CeedBasis           basis_q, basis_x, basis_xc;
  CeedElemRestriction elem_restr_q, elem_restr_x, elem_restr_qd, elem_restr_jd_i;
  CeedVector          q_ceed, q_dot_ceed, g_ceed, jac_data, x_coord, q_data;
  CKR(CeedBasisCreateTensorH1Lagrange(ceed, 3, 5, P, Q, CEED_GAUSS, &basis_q));
  CKR(CeedElemRestrictionCreate(ceed, E, P3, 5, 1, in->l_size, CEED_MEM_HOST, CEED_COPY_VALUES, in->offsets, &elem_restr_q));
  CKR(CeedElemRestrictionCreateStrided(ceed, E, Q3, njd, (CeedSize)E * Q3 * njd, CEED_STRIDES_BACKEND, &elem_restr_jd_i));
  CKR(CeedElemRestrictionCreateVector(elem_restr_jd_i, &jac_data, NULL));
  CKR(CeedElemRestrictionCreateVector(elem_restr_q, &q_ceed, NULL));
  CKR(CeedElemRestrictionCreateVector(elem_restr_q, &q_dot_ceed, NULL));
  CKR(CeedElemRestrictionCreateVector(elem_restr_q, &g_ceed, NULL));
  {  /* DMPlexCeedCoordinateCreateField: trilinear coordinate field */
    CeedInt off_x[8 * 4096];
    if (E > 4096) {
      snprintf(out->msg, sizeof out->msg, "replay handles at most 4096 elements");
      return 1;
    }
    for (int t = 0; t < E * 8; t++) off_x[t] = 3 * t;
    CKR(CeedElemRestrictionCreate(ceed, E, 8, 3, 1, (CeedSize)E * 24, CEED_MEM_HOST, CEED_COPY_VALUES, off_x, &elem_restr_x));
  }
  CKR(CeedBasisCreateTensorH1Lagrange(ceed, 3, 3, 2, Q, CEED_GAUSS, &basis_x));
  CKR(CeedVectorCreate(ceed, (CeedSize)E * 24, &x_coord));
  CKR(CeedVectorSetArray(x_coord, CEED_MEM_HOST, CEED_COPY_VALUES, (CeedScalar *)in->x_coord));

  /* -- QDataGet (src/qdata.c:153-178) */
  {
    CeedQFunction qf_setup;
    CeedOperator  op_setup;
    CKR(CeedQFunctionCreateInterior(ceed, 1, NULL, "setupgeo.h:Setup", &qf_setup));
    CKR(CeedQFunctionSetUserFlopsEstimate(qf_setup, 0));
    CKR(CeedQFunctionAddInput(qf_setup, "dx", 9, CEED_EVAL_GRAD));
    CKR(CeedQFunctionAddInput(qf_setup, "weight", 1, CEED_EVAL_WEIGHT));
    CKR(CeedQFunctionAddOutput(qf_setup, "surface qdata", 10, CEED_EVAL_NONE));
    CKR(CeedElemRestrictionCreateStrided(ceed, E, Q3, 10, (CeedSize)E * Q3 * 10, CEED_STRIDES_BACKEND, &elem_restr_qd));
    CKR(CeedElemRestrictionCreateVector(elem_restr_qd, &q_data, NULL));
    CKR(CeedOperatorCreate(ceed, qf_setup, NULL, NULL, &op_setup));
    CKR(CeedOperatorSetField(op_setup, "dx", elem_restr_x, basis_x, CEED_VECTOR_ACTIVE));
    CKR(CeedOperatorSetField(op_setup, "weight", CEED_ELEMRESTRICTION_NONE, basis_x, CEED_VECTOR_NONE));
    CKR(CeedOperatorSetField(op_setup, "surface qdata", elem_restr_qd, CEED_BASIS_NONE, CEED_VECTOR_ACTIVE));
    CKR(CeedOperatorApply(op_setup, x_coord, q_data, CEED_REQUEST_IMMEDIATE));
    CKR(CeedOperatorDestroy(&op_setup));
    CKR(CeedQFunctionDestroy(&qf_setup));
  }

  /* -- contexts (problems/newtonian.c:744-753) */
  CeedQFunctionContext newt_qfctx, ics_qfctx;
  CKR(CeedQFunctionContextCreate(ceed, &newt_qfctx));
  CKR(CeedQFunctionContextSetData(newt_qfctx, CEED_MEM_HOST, CEED_COPY_VALUES, 184, (void *)in->newt_ctx));
  CKR(CeedQFunctionContextRegisterDouble(newt_qfctx, "timestep size", 168, 1, "Size of timestep, delta t"));
  CKR(CeedQFunctionContextRegisterDouble(newt_qfctx, "ijacobian time shift", 72, 1, "Shift for mass matrix in IJacobian"));
  CKR(CeedQFunctionContextRegisterDouble(newt_qfctx, "solution time", 64, 1, "Current solution time"));
  CKR(CeedQFunctionContextCreate(ceed, &ics_qfctx));
  CKR(CeedQFunctionContextSetData(ics_qfctx, CEED_MEM_HOST, CEED_COPY_VALUES, in->ic_ctx_size, (void *)in->ic_ctx));

  /* -- initial conditions (src/setuplibceed.c:143-175) */
  CeedOperator          op_ics;
  CeedContextFieldLabel ics_time_label;
  {
    CeedQFunction qf_ics;
    CKR(CeedBasisCreateProjection(basis_x, basis_q, &basis_xc));
    CKR(CeedQFunctionCreateInterior(ceed, 1, NULL, in->ic_name, &qf_ics));
    CKR(CeedQFunctionSetContext(qf_ics, ics_qfctx));
    CKR(CeedQFunctionSetUserFlopsEstimate(qf_ics, 0));
    CKR(CeedQFunctionAddInput(qf_ics, "x", 3, CEED_EVAL_INTERP));
    CKR(CeedQFunctionAddInput(qf_ics, "dx", 9, CEED_EVAL_GRAD));
    CKR(CeedQFunctionAddOutput(qf_ics, "q0", 5, CEED_EVAL_NONE));
    CKR(CeedOperatorCreate(ceed, qf_ics, NULL, NULL, &op_ics));
    CKR(CeedOperatorSetField(op_ics, "x", elem_restr_x, basis_xc, CEED_VECTOR_ACTIVE));
    CKR(CeedOperatorSetField(op_ics, "dx", elem_restr_x, basis_xc, CEED_VECTOR_ACTIVE));
    CKR(CeedOperatorSetField(op_ics, "q0", elem_restr_q, CEED_BASIS_NONE, CEED_VECTOR_ACTIVE));
    CKR(CeedOperatorGetContextFieldLabel(op_ics, "evaluation time", &ics_time_label));
    CKR(CeedBasisDestroy(&basis_xc));
    CKR(CeedQFunctionDestroy(&qf_ics));
  }

  /* -- IFunction and IJacobian volume operators and composites (src/setuplibceed.c:209-306) */
  CeedOperator op_ifunction, op_ijacobian, op_ifunction_vol, op_ijacobian_vol;
  {
    CeedQFunction qf_ifunction_vol, qf_ijacobian_vol;
    snprintf(name, sizeof name, "newtonian.h:IFunction_Newtonian_%s", sv);
    CKR(CeedQFunctionCreateInterior(ceed, 1, NULL, name, &qf_ifunction_vol));
    CKR(CeedQFunctionSetContext(qf_ifunction_vol, newt_qfctx));
    CKR(CeedQFunctionSetUserFlopsEstimate(qf_ifunction_vol, 0));
    CKR(CeedQFunctionAddInput(qf_ifunction_vol, "q", 5, CEED_EVAL_INTERP));
    CKR(CeedQFunctionAddInput(qf_ifunction_vol, "Grad_q", 15, CEED_EVAL_GRAD));
    CKR(CeedQFunctionAddInput(qf_ifunction_vol, "q dot", 5, CEED_EVAL_INTERP));
    CKR(CeedQFunctionAddInput(qf_ifunction_vol, "qdata", 10, CEED_EVAL_NONE));
    CKR(CeedQFunctionAddInput(qf_ifunction_vol, "x", 3, CEED_EVAL_INTERP));
    CKR(CeedQFunctionAddOutput(qf_ifunction_vol, "v", 5, CEED_EVAL_INTERP));
    CKR(CeedQFunctionAddOutput(qf_ifunction_vol, "Grad_v", 15, CEED_EVAL_GRAD));
    CKR(CeedQFunctionAddOutput(qf_ifunction_vol, "jac_data", njd, CEED_EVAL_NONE));
    CKR(CeedOperatorCreate(ceed, qf_ifunction_vol, NULL, NULL, &op_ifunction_vol));
    CKR(CeedOperatorSetName(op_ifunction_vol, "IFunction Domain Operator"));
    CKR(CeedOperatorSetField(op_ifunction_vol, "q", elem_restr_q, basis_q, CEED_VECTOR_ACTIVE));
    CKR(CeedOperatorSetField(op_ifunction_vol, "Grad_q", elem_restr_q, basis_q, CEED_VECTOR_ACTIVE));
    CKR(CeedOperatorSetField(op_ifunction_vol, "q dot", elem_restr_q, basis_q, q_dot_ceed));
    CKR(CeedOperatorSetField(op_ifunction_vol, "qdata", elem_restr_qd, CEED_BASIS_NONE, q_data));
    CKR(CeedOperatorSetField(op_ifunction_vol, "x", elem_restr_x, basis_x, x_coord));
    CKR(CeedOperatorSetField(op_ifunction_vol, "v", elem_restr_q, basis_q, CEED_VECTOR_ACTIVE));
    CKR(CeedOperatorSetField(op_ifunction_vol, "Grad_v", elem_restr_q, basis_q, CEED_VECTOR_ACTIVE));
    CKR(CeedOperatorSetField(op_ifunction_vol, "jac_data", elem_restr_jd_i, CEED_BASIS_NONE, jac_data));
    CKR(CeedQFunctionDestroy(&qf_ifunction_vol));

    snprintf(name, sizeof name, "newtonian.h:IJacobian_Newtonian_%s", sv);
    CKR(CeedQFunctionCreateInterior(ceed, 1, NULL, name, &qf_ijacobian_vol));
    CKR(CeedQFunctionSetContext(qf_ijacobian_vol, newt_qfctx));
    CKR(CeedQFunctionSetUserFlopsEstimate(qf_ijacobian_vol, 0));
    CKR(CeedQFunctionAddInput(qf_ijacobian_vol, "dq", 5, CEED_EVAL_INTERP));
    CKR(CeedQFunctionAddInput(qf_ijacobian_vol, "Grad_dq", 15, CEED_EVAL_GRAD));
    CKR(CeedQFunctionAddInput(qf_ijacobian_vol, "qdata", 10, CEED_EVAL_NONE));
    CKR(CeedQFunctionAddInput(qf_ijacobian_vol, "jac_data", njd, CEED_EVAL_NONE));
    CKR(CeedQFunctionAddOutput(qf_ijacobian_vol, "v", 5, CEED_EVAL_INTERP));
    CKR(CeedQFunctionAddOutput(qf_ijacobian_vol, "Grad_v", 15, CEED_EVAL_GRAD));
    CKR(CeedOperatorCreate(ceed, qf_ijacobian_vol, NULL, NULL, &op_ijacobian_vol));
    CKR(CeedOperatorSetName(op_ijacobian_vol, "IJacobian Domain Operator"));
    CKR(CeedOperatorSetField(op_ijacobian_vol, "dq", elem_restr_q, basis_q, CEED_VECTOR_ACTIVE));
    CKR(CeedOperatorSetField(op_ijacobian_vol, "Grad_dq", elem_restr_q, basis_q, CEED_VECTOR_ACTIVE));
    CKR(CeedOperatorSetField(op_ijacobian_vol, "qdata", elem_restr_qd, CEED_BASIS_NONE, q_data));
    CKR(CeedOperatorSetField(op_ijacobian_vol, "jac_data", elem_restr_jd_i, CEED_BASIS_NONE, jac_data));
    CKR(CeedOperatorSetField(op_ijacobian_vol, "v", elem_restr_q, basis_q, CEED_VECTOR_ACTIVE));
    CKR(CeedOperatorSetField(op_ijacobian_vol, "Grad_v", elem_restr_q, basis_q, CEED_VECTOR_ACTIVE));
    CKR(CeedQFunctionDestroy(&qf_ijacobian_vol));

    CKR(CeedOperatorCreateComposite(ceed, &op_ifunction));
    CKR(CeedOperatorCompositeAddSub(op_ifunction, op_ifunction_vol));
    CKR(CeedOperatorCreateComposite(ceed, &op_ijacobian));
    CKR(CeedOperatorCompositeAddSub(op_ijacobian, op_ijacobian_vol));
  }
  CeedContextFieldLabel solution_time_label, timestep_size_label, ijacobian_time_shift_label;
  CKR(CeedOperatorGetContextFieldLabel(op_ifunction, "solution time", &solution_time_label));
  CKR(CeedOperatorGetContextFieldLabel(op_ifunction, "timestep size", &timestep_size_label));
  CKR(CeedOperatorGetContextFieldLabel(op_ijacobian, "ijacobian time shift", &ijacobian_time_shift_label));

  /* -- ICs_FixMultiplicity (src/misc.c:16-45) */
  {
    double     t = in->time;
    CeedVector mult_vec;
    if (ics_time_label) CKR(CeedOperatorSetContextDouble(op_ics, ics_time_label, &t));
    CKR(CeedOperatorApply(op_ics, x_coord, q_ceed, CEED_REQUEST_IMMEDIATE));
    CKR(CeedElemRestrictionCreateVector(elem_restr_q, &mult_vec, NULL));
    CKR(CeedElemRestrictionGetMultiplicity(elem_restr_q, mult_vec));
    if (read_host(ceed, q_ceed, out->q0, in->l_size, out)) return 1;
    if (read_host(ceed, mult_vec, out->mult, in->l_size, out)) return 1;
    for (long long i = 0; i < in->l_size; i++) out->q0[i] /= out->mult[i];
    CKR(CeedVectorSetArray(q_ceed, CEED_MEM_HOST, CEED_COPY_VALUES, out->q0));
    CKR(CeedVectorDestroy(&mult_vec));
  }

  /* -- IFunction_NS (src/setupts.c:78-125) */
  {
    double t = in->time, dt = in->dt;
    CKR(CeedOperatorSetContextDouble(op_ifunction, solution_time_label, &t));
    CKR(CeedOperatorSetContextDouble(op_ifunction, timestep_size_label, &dt));
    CKR(CeedVectorSetArray(q_dot_ceed, CEED_MEM_HOST, CEED_COPY_VALUES, (CeedScalar *)in->q_dot));
    CKR(CeedOperatorApply(op_ifunction, q_ceed, g_ceed, CEED_REQUEST_IMMEDIATE));
    if (read_host(ceed, g_ceed, out->v, in->l_size, out)) return 1;
  }
  /* -- FormIJacobian_NS, MatMult_Ceed and MatGetDiagonal_Ceed (src/setupts.c:131-157, src/mat-ceed.c:1603-1700) */
  {
    double     shift = in->shift;
    CeedVector x_loc, y_loc, diag;
    CKR(CeedOperatorSetContextDouble(op_ijacobian, ijacobian_time_shift_label, &shift));
    CKR(CeedElemRestrictionCreateVector(elem_restr_q, &x_loc, NULL));
    CKR(CeedElemRestrictionCreateVector(elem_restr_q, &y_loc, NULL));
    CKR(CeedElemRestrictionCreateVector(elem_restr_q, &diag, NULL));
    CKR(CeedVectorSetArray(x_loc, CEED_MEM_HOST, CEED_COPY_VALUES, (CeedScalar *)in->dq));
    CKR(CeedOperatorApply(op_ijacobian, x_loc, y_loc, CEED_REQUEST_IMMEDIATE));
    CKR(CeedVectorSetValue(diag, 0.0));
    CKR(CeedOperatorLinearAssembleDiagonal(op_ijacobian, diag, CEED_REQUEST_IMMEDIATE));
    if (read_host(ceed, y_loc, out->jv, in->l_size, out) || read_host(ceed, diag, out->diag, in->l_size, out)) return 1;
    CKR(CeedVectorDestroy(&x_loc));
    CKR(CeedVectorDestroy(&y_loc));
    CKR(CeedVectorDestroy(&diag));
  }

  /* -- monitors (src/monitor_totalkineticenergy.c:80-163, src/monitor_cfl.c:90-164), volume operator's context */
  for (int m = 0; m < 2; m++) {
    const int            ke = m == 0, ncomp = ke ? 5 : 1;
    const CeedInt        strides[3] = {ncomp, 1, Q3 * ncomp};
    CeedElemRestriction  elem_restr_mon;
    CeedQFunction        qf_monitor;
    CeedOperator         op_monitor, *sub_ops;
    CeedQFunctionContext ctx_vol = NULL;
    CeedVector           values;
    CKR(CeedOperatorCompositeGetSubList(op_ifunction, &sub_ops));
    CKR(CeedOperatorGetContext(sub_ops[0], &ctx_vol));
    CKR(CeedElemRestrictionCreateStrided(ceed, E, Q3, ncomp, (CeedSize)ncomp * E * Q3, strides, &elem_restr_mon));
    snprintf(name, sizeof name, ke ? "monitor_totalkineticenergy.h:MonitorTotalKineticEnergy_%s" : "monitor_cfl.h:MonitorCFL_3D_%s", sv);
    CKR(CeedQFunctionCreateInterior(ceed, 1, NULL, name, &qf_monitor));
    CKR(CeedQFunctionSetContext(qf_monitor, ctx_vol));
    CKR(CeedQFunctionAddInput(qf_monitor, "q", 5, CEED_EVAL_INTERP));
    if (ke) CKR(CeedQFunctionAddInput(qf_monitor, "Grad_q", 15, CEED_EVAL_GRAD));
    CKR(CeedQFunctionAddInput(qf_monitor, "q_data", 10, CEED_EVAL_NONE));
    CKR(CeedQFunctionAddOutput(qf_monitor, "v", ncomp, CEED_EVAL_NONE));
    CKR(CeedOperatorCreate(ceed, qf_monitor, NULL, NULL, &op_monitor));
    CKR(CeedOperatorSetField(op_monitor, "q", elem_restr_q, basis_q, CEED_VECTOR_ACTIVE));
    if (ke) CKR(CeedOperatorSetField(op_monitor, "Grad_q", elem_restr_q, basis_q, CEED_VECTOR_ACTIVE));
    CKR(CeedOperatorSetField(op_monitor, "q_data", elem_restr_qd, CEED_BASIS_NONE, q_data));
    CKR(CeedOperatorSetField(op_monitor, "v", elem_restr_mon, CEED_BASIS_NONE, CEED_VECTOR_ACTIVE));
    CKR(CeedElemRestrictionCreateVector(elem_restr_mon, &values, NULL));
    CKR(CeedOperatorApply(op_monitor, q_ceed, values, CEED_REQUEST_IMMEDIATE));
    const CeedScalar *a;
    CKR(CeedVectorGetArrayRead(values, CEED_MEM_HOST, &a));
    if (ke) { /* VecStrideSum per component */
      for (int c = 0; c < 5; c++) out->ke[c] = 0;
      for (long long i = 0; i < (long long)E * Q3; i++)
        for (int c = 0; c < 5; c++) out->ke[c] += a[i * 5 + c];
    } else { /* VecMin / VecMax, times dt */
      double mn = a[0], mx = a[0];
      for (long long i = 1; i < (long long)E * Q3; i++) {
        mn = a[i] < mn ? a[i] : mn;
        mx = a[i] > mx ? a[i] : mx;
      }
      out->cfl[0] = mn * in->dt;
      out->cfl[1] = mx * in->dt;
    }
    CKR(CeedVectorRestoreArrayRead(values, &a));
    CKR(CeedVectorDestroy(&values));
    CKR(CeedOperatorDestroy(&op_monitor));
    CKR(CeedQFunctionDestroy(&qf_monitor));
    CKR(CeedQFunctionContextDestroy(&ctx_vol));
    CKR(CeedElemRestrictionDestroy(&elem_restr_mon));
  }

  CKR(CeedOperatorDestroy(&op_ics));
  CKR(CeedOperatorDestroy(&op_ifunction_vol));
  CKR(CeedOperatorDestroy(&op_ijacobian_vol));
  CKR(CeedOperatorDestroy(&op_ifunction));
  CKR(CeedOperatorDestroy(&op_ijacobian));
  CKR(CeedQFunctionContextDestroy(&newt_qfctx));
  CKR(CeedQFunctionContextDestroy(&ics_qfctx));
  CKR(CeedVectorDestroy(&q_ceed));
  CKR(CeedVectorDestroy(&q_dot_ceed));
  CKR(CeedVectorDestroy(&g_ceed));
  CKR(CeedVectorDestroy(&jac_data));
  CKR(CeedVectorDestroy(&x_coord));
  CKR(CeedVectorDestroy(&q_data));
  CKR(CeedElemRestrictionDestroy(&elem_restr_q));
  CKR(CeedElemRestrictionDestroy(&elem_restr_x));
  CKR(CeedElemRestrictionDestroy(&elem_restr_qd));
  CKR(CeedElemRestrictionDestroy(&elem_restr_jd_i));
  CKR(CeedBasisDestroy(&basis_q));
  CKR(CeedBasisDestroy(&basis_x));
  return CeedDestroy(&ceed);
}
