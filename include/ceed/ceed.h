/* ceed/ceed.h -- the libCEED C API subset HONEE calls, served by the B200 backend (libceed_b200.so).
 *
 * This is the drop-in boundary: HONEE's `navierstokes` is compiled against libCEED's <ceed.h> and selects a backend
 * with `-ceed <resource>` (src/cloptions.c:101, examples/navierstokes.c:64).  Linking it against libceed_b200.so with
 * this header gives it the resources "/gpu/b200" (FP64 everywhere) and "/gpu/b200/mixed" (FP64 residual, FP32
 * Jacobian action and diagonal); "/gpu/cuda", "/gpu/cuda/shared", "/gpu/cuda/gen" are accepted as aliases of
 * "/gpu/b200".  Types, enum values and signatures follow libCEED (third-party, un-vendored; the reference's goldens pin
 * libCEED 0.12.0 v0.12.0-1263-ge205ca3fa, tests/output/taylorgreen_totalke.csv:3-4) so that the caller compiles
 * unchanged.  Every group cites the HONEE call sites it serves (grep counts in parentheses are from src/, problems/,
 * examples/, include/).
 *
 * Scope: the operators of the Newtonian hot path -- QFunctions named (by their `*_loc` source string)
 * "Setup", "IFunction_Newtonian_Conserv", "IJacobian_Newtonian_Conserv" -- run as fused sm_100a kernels.  Any other
 * QFunction is refused with CEED_ERROR_UNSUPPORTED when its operator is applied: there is no CPU fallback.
 */
#ifndef CEED_B200_CEED_H
#define CEED_B200_CEED_H

#include <stdarg.h>
#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CEED_EXTERN extern __attribute__((visibility("default")))
#define CEED_VERSION_MAJOR 0
#define CEED_VERSION_MINOR 12
#define CEED_VERSION_PATCH 0
#define CEED_VERSION_RELEASE false
#define CEED_VERSION_GE(major, minor, patch) \
  (!CEED_VERSION_RELEASE ||                  \
   (CEED_VERSION_MAJOR > major ||            \
    (CEED_VERSION_MAJOR == major && (CEED_VERSION_MINOR > minor || (CEED_VERSION_MINOR == minor && CEED_VERSION_PATCH >= patch)))))

#include "ceed/types.h"

typedef struct Ceed_private                 *Ceed;
typedef struct CeedRequest_private          *CeedRequest;
typedef struct CeedVector_private           *CeedVector;
typedef struct CeedElemRestriction_private  *CeedElemRestriction;
typedef struct CeedBasis_private            *CeedBasis;
typedef struct CeedQFunctionField_private   *CeedQFunctionField;
typedef struct CeedQFunction_private        *CeedQFunction;
typedef struct CeedOperatorField_private    *CeedOperatorField;
typedef struct CeedQFunctionContext_private *CeedQFunctionContext;
typedef struct CeedContextFieldLabel_private *CeedContextFieldLabel;
typedef struct CeedOperator_private         *CeedOperator;
typedef struct CeedObject_private           *CeedObject; /* every object starts with its Ceed, so any handle casts to this */
typedef struct CeedOperatorAssemblyData_private *CeedOperatorAssemblyData;

typedef int (*CeedQFunctionUser)(void *ctx, const CeedInt Q, const CeedScalar *const *in, CeedScalar *const *out);
typedef int (*CeedQFunctionContextDataDestroyUser)(void *data);
typedef int (*CeedErrorHandler)(Ceed, const char *, int, const char *, int, const char *, va_list *);

typedef enum { CEED_CONTEXT_FIELD_DOUBLE = 1, CEED_CONTEXT_FIELD_INT32 = 2, CEED_CONTEXT_FIELD_BOOL = 3 } CeedContextFieldType;

CEED_EXTERN CeedRequest *const        CEED_REQUEST_IMMEDIATE;
CEED_EXTERN CeedRequest *const        CEED_REQUEST_ORDERED;
CEED_EXTERN const CeedInt             CEED_STRIDES_BACKEND[3];
CEED_EXTERN const CeedVector          CEED_VECTOR_ACTIVE;
CEED_EXTERN const CeedVector          CEED_VECTOR_NONE;
CEED_EXTERN const CeedBasis           CEED_BASIS_NONE;
CEED_EXTERN const CeedElemRestriction CEED_ELEMRESTRICTION_NONE;
CEED_EXTERN const CeedQFunction       CEED_QFUNCTION_NONE;

/* ---- Ceed (examples/navierstokes.c:64-112, src/cloptions.c:101,169-172, include/petsc-ceed.h:25-36) ---- */
CEED_EXTERN int CeedInit(const char *resource, Ceed *ceed);
CEED_EXTERN int CeedDestroy(Ceed *ceed);
CEED_EXTERN int CeedReferenceCopy(Ceed ceed, Ceed *ceed_copy);
CEED_EXTERN int CeedGetResource(Ceed ceed, const char **resource);
CEED_EXTERN int CeedGetPreferredMemType(Ceed ceed, CeedMemType *type);
CEED_EXTERN int CeedIsDeterministic(Ceed ceed, bool *is_deterministic);
CEED_EXTERN int CeedSetStream(Ceed ceed, void *handle);
CEED_EXTERN int CeedGetVersion(int *major, int *minor, int *patch, bool *release);
CEED_EXTERN int CeedSetErrorHandler(Ceed ceed, CeedErrorHandler handler);
CEED_EXTERN int CeedGetErrorMessage(Ceed ceed, const char **err_msg);
CEED_EXTERN int CeedResetErrorMessage(Ceed ceed, const char **err_msg);
CEED_EXTERN int CeedErrorReturn(Ceed ceed, const char *filename, int line_no, const char *func, int ecode, const char *format, va_list *args);
CEED_EXTERN int CeedErrorStore(Ceed ceed, const char *filename, int line_no, const char *func, int ecode, const char *format, va_list *args);
CEED_EXTERN int CeedErrorAbort(Ceed ceed, const char *filename, int line_no, const char *func, int ecode, const char *format, va_list *args);
CEED_EXTERN int CeedErrorExit(Ceed ceed, const char *filename, int line_no, const char *func, int ecode, const char *format, va_list *args);
CEED_EXTERN int CeedGetGitVersion(const char **git_version);
CEED_EXTERN int CeedErrorImpl(Ceed ceed, const char *filename, int line_no, const char *func, int ecode, const char *format, ...);
#define CeedError(ceed, ecode, ...) (CeedErrorImpl((ceed), __FILE__, __LINE__, __func__, (ecode), __VA_ARGS__) ?: (ecode))
CEED_EXTERN Ceed CeedObjectReturnCeed(CeedObject obj);

/* ---- CeedVector (include/petsc-ceed-utils.h:127-219 zero-copy wrapping, src/qdata.c:42-45, src/mat-ceed.c) ---- */
CEED_EXTERN int CeedVectorCreate(Ceed ceed, CeedSize len, CeedVector *vec);
CEED_EXTERN int CeedVectorReferenceCopy(CeedVector vec, CeedVector *vec_copy);
CEED_EXTERN int CeedVectorSetArray(CeedVector vec, CeedMemType mem_type, CeedCopyMode copy_mode, CeedScalar *array);
CEED_EXTERN int CeedVectorSetValue(CeedVector vec, CeedScalar value);
CEED_EXTERN int CeedVectorSyncArray(CeedVector vec, CeedMemType mem_type);
CEED_EXTERN int CeedVectorTakeArray(CeedVector vec, CeedMemType mem_type, CeedScalar **array);
CEED_EXTERN int CeedVectorGetArray(CeedVector vec, CeedMemType mem_type, CeedScalar **array);
CEED_EXTERN int CeedVectorGetArrayRead(CeedVector vec, CeedMemType mem_type, const CeedScalar **array);
CEED_EXTERN int CeedVectorGetArrayWrite(CeedVector vec, CeedMemType mem_type, CeedScalar **array);
CEED_EXTERN int CeedVectorRestoreArray(CeedVector vec, CeedScalar **array);
CEED_EXTERN int CeedVectorRestoreArrayRead(CeedVector vec, const CeedScalar **array);
CEED_EXTERN int CeedVectorGetLength(CeedVector vec, CeedSize *length);
CEED_EXTERN int CeedVectorNorm(CeedVector vec, CeedNormType type, CeedScalar *norm);
CEED_EXTERN int CeedVectorCopy(CeedVector vec, CeedVector vec_copy);
CEED_EXTERN int CeedVectorScale(CeedVector x, CeedScalar alpha);
CEED_EXTERN int CeedVectorAXPY(CeedVector y, CeedScalar alpha, CeedVector x);
CEED_EXTERN int CeedVectorAXPBY(CeedVector y, CeedScalar alpha, CeedScalar beta, CeedVector x);
CEED_EXTERN int CeedVectorPointwiseMult(CeedVector w, CeedVector x, CeedVector y);
CEED_EXTERN int CeedVectorReciprocal(CeedVector vec);
CEED_EXTERN int CeedVectorGetCeed(CeedVector vec, Ceed *ceed);
CEED_EXTERN Ceed CeedVectorReturnCeed(CeedVector vec);
CEED_EXTERN int CeedVectorDestroy(CeedVector *vec);

/* ---- CeedElemRestriction (src/dm-utils.c:83-137, :235, src/setuplibceed.c:121-129) ---- */
CEED_EXTERN int CeedElemRestrictionCreate(Ceed ceed, CeedInt num_elem, CeedInt elem_size, CeedInt num_comp, CeedInt comp_stride, CeedSize l_size,
                                          CeedMemType mem_type, CeedCopyMode copy_mode, const CeedInt *offsets, CeedElemRestriction *rstr);
CEED_EXTERN int CeedElemRestrictionCreateStrided(Ceed ceed, CeedInt num_elem, CeedInt elem_size, CeedInt num_comp, CeedSize l_size,
                                                 const CeedInt strides[3], CeedElemRestriction *rstr);
CEED_EXTERN int CeedElemRestrictionReferenceCopy(CeedElemRestriction rstr, CeedElemRestriction *rstr_copy);
CEED_EXTERN int CeedElemRestrictionCreateVector(CeedElemRestriction rstr, CeedVector *l_vec, CeedVector *e_vec);
CEED_EXTERN int CeedElemRestrictionApply(CeedElemRestriction rstr, CeedTransposeMode t_mode, CeedVector u, CeedVector ru, CeedRequest *request);
CEED_EXTERN int CeedElemRestrictionGetNumElements(CeedElemRestriction rstr, CeedInt *num_elem);
CEED_EXTERN int CeedElemRestrictionGetElementSize(CeedElemRestriction rstr, CeedInt *elem_size);
CEED_EXTERN int CeedElemRestrictionGetLVectorSize(CeedElemRestriction rstr, CeedSize *l_size);
CEED_EXTERN int CeedElemRestrictionGetEVectorSize(CeedElemRestriction rstr, CeedSize *e_size);
CEED_EXTERN int CeedElemRestrictionGetNumComponents(CeedElemRestriction rstr, CeedInt *num_comp);
CEED_EXTERN int CeedElemRestrictionGetCompStride(CeedElemRestriction rstr, CeedInt *comp_stride);
CEED_EXTERN int CeedElemRestrictionGetMultiplicity(CeedElemRestriction rstr, CeedVector mult);
CEED_EXTERN int CeedElemRestrictionGetCeed(CeedElemRestriction rstr, Ceed *ceed);
CEED_EXTERN Ceed CeedElemRestrictionReturnCeed(CeedElemRestriction rstr);
CEED_EXTERN int CeedElemRestrictionDestroy(CeedElemRestriction *rstr);

/* ---- CeedBasis (src/dm-utils.c:766-879) ---- */
CEED_EXTERN int CeedBasisCreateTensorH1(Ceed ceed, CeedInt dim, CeedInt num_comp, CeedInt P_1d, CeedInt Q_1d, const CeedScalar *interp_1d,
                                        const CeedScalar *grad_1d, const CeedScalar *q_ref_1d, const CeedScalar *q_weight_1d, CeedBasis *basis);
CEED_EXTERN int CeedBasisCreateTensorH1Lagrange(Ceed ceed, CeedInt dim, CeedInt num_comp, CeedInt P, CeedInt Q, CeedQuadMode quad_mode,
                                                CeedBasis *basis);
CEED_EXTERN int CeedBasisCreateH1(Ceed ceed, CeedElemTopology topo, CeedInt num_comp, CeedInt num_nodes, CeedInt nqpts, const CeedScalar *interp,
                                  const CeedScalar *grad, const CeedScalar *q_ref, const CeedScalar *q_weights, CeedBasis *basis);
CEED_EXTERN int CeedBasisCreateProjection(CeedBasis basis_from, CeedBasis basis_to, CeedBasis *basis_project);
CEED_EXTERN int CeedBasisReferenceCopy(CeedBasis basis, CeedBasis *basis_copy);
CEED_EXTERN int CeedBasisApply(CeedBasis basis, CeedInt num_elem, CeedTransposeMode t_mode, CeedEvalMode eval_mode, CeedVector u, CeedVector v);
CEED_EXTERN int CeedBasisGetDimension(CeedBasis basis, CeedInt *dim);
CEED_EXTERN int CeedBasisGetNumComponents(CeedBasis basis, CeedInt *num_comp);
CEED_EXTERN int CeedBasisGetNumNodes(CeedBasis basis, CeedInt *P);
CEED_EXTERN int CeedBasisGetNumNodes1D(CeedBasis basis, CeedInt *P_1d);
CEED_EXTERN int CeedBasisGetNumQuadraturePoints(CeedBasis basis, CeedInt *Q);
CEED_EXTERN int CeedBasisGetNumQuadraturePoints1D(CeedBasis basis, CeedInt *Q_1d);
CEED_EXTERN Ceed CeedBasisReturnCeed(CeedBasis basis);
CEED_EXTERN int CeedBasisDestroy(CeedBasis *basis);
CEED_EXTERN int CeedLobattoQuadrature(CeedInt Q, CeedScalar *q_ref_1d, CeedScalar *q_weight_1d);
CEED_EXTERN int CeedGaussQuadrature(CeedInt Q, CeedScalar *q_ref_1d, CeedScalar *q_weight_1d);

/* ---- CeedQFunctionContext (problems/newtonian.c:744-753, src/setupts.c:91-93,141, src/mat-ceed.c:889-906) ---- */
CEED_EXTERN int CeedQFunctionContextCreate(Ceed ceed, CeedQFunctionContext *ctx);
CEED_EXTERN int CeedQFunctionContextReferenceCopy(CeedQFunctionContext ctx, CeedQFunctionContext *ctx_copy);
CEED_EXTERN int CeedQFunctionContextSetData(CeedQFunctionContext ctx, CeedMemType mem_type, CeedCopyMode copy_mode, size_t size, void *data);
CEED_EXTERN int CeedQFunctionContextGetData(CeedQFunctionContext ctx, CeedMemType mem_type, void *data);
CEED_EXTERN int CeedQFunctionContextGetDataRead(CeedQFunctionContext ctx, CeedMemType mem_type, void *data);
CEED_EXTERN int CeedQFunctionContextRestoreData(CeedQFunctionContext ctx, void *data);
CEED_EXTERN int CeedQFunctionContextRestoreDataRead(CeedQFunctionContext ctx, void *data);
CEED_EXTERN int CeedQFunctionContextSetDataDestroy(CeedQFunctionContext ctx, CeedMemType f_mem_type, CeedQFunctionContextDataDestroyUser f);
CEED_EXTERN int CeedQFunctionContextRegisterDouble(CeedQFunctionContext ctx, const char *field_name, size_t field_offset, size_t num_values,
                                                   const char *field_description);
CEED_EXTERN int CeedQFunctionContextGetContextSize(CeedQFunctionContext ctx, size_t *ctx_size);
CEED_EXTERN int CeedQFunctionContextReference(CeedQFunctionContext ctx);
CEED_EXTERN int CeedQFunctionContextDestroy(CeedQFunctionContext *ctx);

/* ---- CeedQFunction (src/setuplibceed.c:209-266, src/qdata.c:153-170) ---- */
CEED_EXTERN int CeedQFunctionCreateInterior(Ceed ceed, CeedInt vec_length, CeedQFunctionUser f, const char *source, CeedQFunction *qf);
CEED_EXTERN int CeedQFunctionReferenceCopy(CeedQFunction qf, CeedQFunction *qf_copy);
CEED_EXTERN int CeedQFunctionAddInput(CeedQFunction qf, const char *field_name, CeedInt size, CeedEvalMode eval_mode);
CEED_EXTERN int CeedQFunctionAddOutput(CeedQFunction qf, const char *field_name, CeedInt size, CeedEvalMode eval_mode);
CEED_EXTERN int CeedQFunctionSetContext(CeedQFunction qf, CeedQFunctionContext ctx);
CEED_EXTERN int CeedQFunctionGetContext(CeedQFunction qf, CeedQFunctionContext *ctx);
CEED_EXTERN int CeedQFunctionSetUserFlopsEstimate(CeedQFunction qf, CeedSize flops);
CEED_EXTERN int CeedQFunctionGetKernelName(CeedQFunction qf, const char **kernel_name);
CEED_EXTERN int CeedQFunctionCreateIdentity(Ceed ceed, CeedInt size, CeedEvalMode in_mode, CeedEvalMode out_mode, CeedQFunction *qf);
CEED_EXTERN int CeedQFunctionDestroy(CeedQFunction *qf);

/* ---- CeedOperator (src/setuplibceed.c:209-318, src/setupts.c:109, src/mat-ceed.c:1603-1700, src/petsc_ops.c:232-234) ---- */
CEED_EXTERN int CeedOperatorCreate(Ceed ceed, CeedQFunction qf, CeedQFunction dqf, CeedQFunction dqfT, CeedOperator *op);
CEED_EXTERN int CeedOperatorCreateComposite(Ceed ceed, CeedOperator *op);
CEED_EXTERN int CeedCompositeOperatorCreate(Ceed ceed, CeedOperator *op);
CEED_EXTERN int CeedOperatorReferenceCopy(CeedOperator op, CeedOperator *op_copy);
CEED_EXTERN int CeedOperatorSetField(CeedOperator op, const char *field_name, CeedElemRestriction rstr, CeedBasis basis, CeedVector vec);
CEED_EXTERN int CeedOperatorCompositeAddSub(CeedOperator composite_op, CeedOperator sub_op);
CEED_EXTERN int CeedCompositeOperatorAddSub(CeedOperator composite_op, CeedOperator sub_op);
CEED_EXTERN int CeedOperatorCompositeGetNumSub(CeedOperator op, CeedInt *num_suboperators);
CEED_EXTERN int CeedOperatorCompositeGetSubList(CeedOperator op, CeedOperator **sub_operators);
CEED_EXTERN int CeedOperatorSetName(CeedOperator op, const char *name);
CEED_EXTERN int CeedOperatorCheckReady(CeedOperator op);
CEED_EXTERN int CeedOperatorGetActiveVectorLengths(CeedOperator op, CeedSize *input_size, CeedSize *output_size);
CEED_EXTERN int CeedOperatorGetContextFieldLabel(CeedOperator op, const char *field_name, CeedContextFieldLabel *field_label);
CEED_EXTERN int CeedOperatorSetContextDouble(CeedOperator op, CeedContextFieldLabel field_label, double *values);
CEED_EXTERN int CeedOperatorGetContextDoubleRead(CeedOperator op, CeedContextFieldLabel field_label, size_t *num_values, const double **values);
CEED_EXTERN int CeedOperatorRestoreContextDoubleRead(CeedOperator op, CeedContextFieldLabel field_label, const double **values);
CEED_EXTERN int CeedOperatorApply(CeedOperator op, CeedVector in, CeedVector out, CeedRequest *request);
CEED_EXTERN int CeedOperatorApplyAdd(CeedOperator op, CeedVector in, CeedVector out, CeedRequest *request);
CEED_EXTERN int CeedOperatorLinearAssembleDiagonal(CeedOperator op, CeedVector assembled, CeedRequest *request);
CEED_EXTERN int CeedOperatorLinearAssembleAddDiagonal(CeedOperator op, CeedVector assembled, CeedRequest *request);
CEED_EXTERN int CeedOperatorGetFlopsEstimate(CeedOperator op, CeedSize *flops);
CEED_EXTERN int CeedOperatorGetCeed(CeedOperator op, Ceed *ceed);
CEED_EXTERN Ceed CeedOperatorReturnCeed(CeedOperator op);
CEED_EXTERN int CeedOperatorIsComposite(CeedOperator op, bool *is_composite);
CEED_EXTERN int CeedOperatorGetContext(CeedOperator op, CeedQFunctionContext *ctx);
CEED_EXTERN int CeedOperatorGetFieldByName(CeedOperator op, const char *field_name, CeedOperatorField *op_field);
CEED_EXTERN int CeedOperatorFieldGetElemRestriction(CeedOperatorField op_field, CeedElemRestriction *rstr);
CEED_EXTERN int CeedOperatorFieldGetVector(CeedOperatorField op_field, CeedVector *vec);
CEED_EXTERN int CeedOperatorFieldGetData(CeedOperatorField op_field, const char **field_name, CeedElemRestriction *rstr, CeedBasis *basis,
                                         CeedVector *vec);
CEED_EXTERN int CeedOperatorView(CeedOperator op, FILE *stream);
CEED_EXTERN int CeedOperatorViewTerse(CeedOperator op, FILE *stream);
CEED_EXTERN int CeedOperatorSetNumViewTabs(CeedOperator op, CeedInt num_tabs);
CEED_EXTERN int CeedOperatorGetNumViewTabs(CeedOperator op, CeedInt *num_tabs);
CEED_EXTERN int CeedOperatorSetQFunctionAssemblyDataUpdateNeeded(CeedOperator op, bool needs_data_update);
/* Full (COO) assembly and point-block diagonals are not provided on /gpu/b200 (assembled matrices are not matrix-free; the
 * point-block Jacobi preconditioner is listed as next): these return CEED_ERROR_UNSUPPORTED. */
CEED_EXTERN int CeedOperatorLinearAssembleSymbolic(CeedOperator op, CeedSize *num_entries, CeedInt **rows, CeedInt **cols);
CEED_EXTERN int CeedOperatorLinearAssemble(CeedOperator op, CeedVector values);
CEED_EXTERN int CeedOperatorLinearAssembleGetNumEntries(CeedOperator op, CeedSize *num_entries);
CEED_EXTERN int CeedOperatorLinearAssemblePointBlockDiagonal(CeedOperator op, CeedVector assembled, CeedRequest *request);
CEED_EXTERN int CeedOperatorLinearAssembleAddPointBlockDiagonal(CeedOperator op, CeedVector assembled, CeedRequest *request);
CEED_EXTERN int CeedOperatorLinearAssemblePointBlockDiagonalSymbolic(CeedOperator op, CeedSize *num_entries, CeedInt **rows, CeedInt **cols);
CEED_EXTERN int CeedOperatorGetOperatorAssemblyData(CeedOperator op, CeedOperatorAssemblyData *data);
CEED_EXTERN int CeedOperatorAssemblyDataGetBases(CeedOperatorAssemblyData data, CeedInt *num_active_bases_in, CeedBasis **active_bases_in,
                                                 const CeedScalar ***assembled_bases_in, CeedInt *num_active_bases_out,
                                                 CeedBasis **active_bases_out, const CeedScalar ***assembled_bases_out);
CEED_EXTERN int CeedOperatorDestroy(CeedOperator *op);

#ifdef __cplusplus
}
#endif
#endif
