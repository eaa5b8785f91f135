/* ceed_b200.c -- libCEED-compatible host layer of the B200 backend (declared in include/ceed/ceed.h).
 *
 * HONEE builds its operators through the libCEED C API (src/setuplibceed.c:97-340, src/qdata.c:133-190) and applies
 * them through CeedOperatorApply / CeedOperatorApplyAdd / CeedOperatorLinearAssembleDiagonal (src/setupts.c:109,
 * src/mat-ceed.c:1603-1700).  This file implements that object model (Ceed, CeedVector, CeedElemRestriction, CeedBasis,
 * CeedQFunctionContext, CeedQFunction, CeedOperator, composite operators, context field labels, error handling) and,
 * when an operator is first applied, recognises the HONEE QFunction by the kernel name in its source string
 * ("newtonian.h:IFunction_Newtonian_Conserv" -> "IFunction_Newtonian_Conserv") and binds it to a fused sm_100a kernel
 * (include/honee_b200.h).  An operator whose QFunction has no fused kernel fails with CEED_ERROR_UNSUPPORTED; the user
 * function pointer is never called, so nothing runs on the CPU.
 *
 * Memory follows libCEED's CUDA backends: a CeedVector mirrors host and device arrays with validity flags, wraps
 * caller arrays zero-copy with CEED_USE_POINTER (include/petsc-ceed-utils.h:127-191), and copies lazily on access.
 * All device work is stream-ordered on the Ceed's stream (the legacy default stream unless CeedSetStream is called);
 * host reads synchronise it.
 */
#include <cuda_runtime.h>
#include <math.h>
#include <stdarg.h>
#include <stdbool.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ceed/ceed.h"
#include "hb_internal.h"
#include "honee_b200.h"

#define MAX_FIELDS 16
#define MAX_SUBS 16
#define MAX_LABELS 16
#define NAME_LEN 128

/* ------------------------------------------------------------------------------------------------------------------ */
/* object layouts                                                                                                     */

struct Ceed_private {
  int              ref;
  char             resource[256];
  int              mixed;  /* 1: FP32 Jacobian action and diagonal */
  cudaStream_t     stream;
  CeedErrorHandler handler;
  char             err_msg[2048];
  double          *d_scratch; /* 1024 doubles for reductions */
  HbElemOp        *ops[64];   /* element operators whose kernel status words are checked at host synchronisation */
  int              nops;
  /* host <-> device copies of host-backed vectors run on their own streams, ordered against the compute stream by
   * events, so an input copy overlaps the kernels before it and an output read-back the kernels after its producer */
  cudaStream_t     s_h2d, s_d2h;
  cudaEvent_t      ev_tmp;
  int              copy_streams;
  int             *h_status; /* pinned: the status words read back beside an output read-back on s_d2h */
};

struct CeedVector_private {
  Ceed     ceed;
  int      ref;
  CeedSize length;
  double  *h, *d;
  int      h_own, d_own, h_valid, d_valid;
  float   *d_f32;      /* FP32 shadow (mixed-precision jac_data) */
  int      f32_valid;  /* shadow holds the current values */
  int      f64_stale;  /* FP64 copies are out of date: rebuild from the shadow on access */
  cudaEvent_t ev_h2d;  /* end of the last host-to-device copy (on the Ceed's copy stream) */
  cudaEvent_t ev_use;  /* recorded on the compute stream after the last operator that used the device array */
  int      events, h2d_pending, use_known; /* use_known: ev_use covers every use of d handed out so far */
};

struct CeedElemRestriction_private {
  Ceed     ceed;
  int      ref;
  CeedInt  num_elem, elem_size, num_comp, comp_stride;
  CeedSize l_size;
  int      strided;
  CeedInt  strides[3];
  int32_t *h_off, *d_off, *d_strides;
  int64_t *d_tptr, *d_teidx; /* transpose CSR, built on first transpose apply */
};

struct CeedBasis_private {
  Ceed    ceed;
  int     ref;
  int     dim, num_comp, P1d, Q1d, tensor;
  double  interp1d[HB_MAX_P * HB_MAX_P], grad1d[HB_MAX_P * HB_MAX_P], qref1d[HB_MAX_P], qweight1d[HB_MAX_P];
  double *d_B, *d_G, *d_w;
};

typedef struct {
  char   name[NAME_LEN];
  size_t offset, num_values;
  int    type;
} CtxLabel;

struct CeedQFunctionContext_private {
  Ceed                                ceed;
  int                                 ref;
  size_t                              size;
  void                               *data;
  int                                 own;
  CeedQFunctionContextDataDestroyUser destroy;
  int                                 nlabels;
  CtxLabel                            labels[MAX_LABELS];
};

typedef struct {
  char         name[NAME_LEN];
  CeedInt      size;
  CeedEvalMode emode;
} QFField;

struct CeedQFunction_private {
  Ceed                 ceed;
  int                  ref;
  CeedInt              vlength;
  CeedQFunctionUser    f;
  char                 source[512], kernel[NAME_LEN];
  int                  nin, nout;
  QFField              in[MAX_FIELDS], out[MAX_FIELDS];
  CeedQFunctionContext ctx;
  CeedSize             user_flops;
};

typedef struct {
  CeedElemRestriction r;
  CeedBasis           b;
  CeedVector          v;
  int                 set;
} OpField;

enum {
  PLAN_NONE = 0,
  PLAN_SETUP,
  PLAN_IFUNCTION,
  PLAN_IJACOBIAN,
  PLAN_SETUP_SUR,
  PLAN_FREESTREAM,
  PLAN_FREESTREAM_JAC,
  PLAN_RHS,
  PLAN_MASS,
  PLAN_MASS_STAB,
  PLAN_ICS,     /* initial condition at the solution nodes (src/setuplibceed.c:143-175) */
  PLAN_MON_KE,  /* MonitorTotalKineticEnergy_* per-point integrands (src/monitor_totalkineticenergy.c:80-103) */
  PLAN_MON_CFL, /* MonitorCFL_3D_* per-point CFL numbers (src/monitor_cfl.c:60-110) */
  PLAN_MASS_N,  /* Mass_N on N != 5 node-interleaved fields (src/honee-mass.c:20-60) */
  PLAN_VELGRAD, /* VelocityGradientProjectionRHS_* (src/velocity_gradient_projection.c:61-103) */
  PLAN_ANISO,   /* AnisotropyTensorProjection (src/grid_anisotropy_tensor.c:49-69) */
  PLAN_INV_MULT,/* InverseMultiplicity (src/inverse_multiplicity.c:63-73) */
  PLAN_SGS_NODAL, /* ComputeSgsDDNodal_* (problems/sgs_dd_model.c:149-185) */
  PLAN_SGS_IF   /* IFunction_NodalSgs_* (problems/sgs_dd_model.c:533-550) */
};

struct CeedOperator_private {
  Ceed          ceed;
  int           ref;
  int           composite;
  char          name[NAME_LEN];
  CeedQFunction qf;
  OpField       in[MAX_FIELDS], out[MAX_FIELDS];
  int           nsub;
  CeedOperator  subs[MAX_SUBS];
  /* backend plan */
  int       plan;
  HbElemOp *eop;
  int       idl_coords_set;
  float    *d_tmp_in32, *d_tmp_out32; /* mixed-precision staging of L-vectors */
  double   *d_tmp_e;                  /* coordinate E-vector for the Setup operator */
  HbFaceOp *fop;                      /* boundary-face sub-operators */
  double   *d_zero, *d_tmp_rhs;       /* explicit right-hand side: zero rate and the residual it is negated from */
  float    *d_tmp_pb32;               /* mixed-precision point blocks before they are widened into the FP64 output */
  int       flux_type;                /* 0 HLL, 1 HLLC */
  double   *d_tmp_e2;                 /* output E-vector of the initial-condition and monitor operators */
  int       ic_kind, ic_state_var;    /* initial-condition QFunction (HB_IC_*) and the state variable it writes */
  int       nc, state_var;            /* fields of a Mass_N operator; state variable of the nodal SGS operators */
  double   *d_node_w;                 /* per-node weight of the nodal SGS closure (transposed inverse multiplicity) */
};

struct CeedContextFieldLabel_private {
  int    n;
  struct {
    CeedQFunctionContext ctx;
    size_t               offset, num_values;
  } ent[MAX_SUBS];
  char name[NAME_LEN];
};

struct CeedRequest_private {
  int unused;
};

/* sentinels */
static struct CeedVector_private          vec_active_obj, vec_none_obj;
static struct CeedBasis_private           basis_none_obj;
static struct CeedElemRestriction_private rstr_none_obj;
static struct CeedQFunction_private       qf_none_obj;
static CeedRequest                        req_immediate_obj, req_ordered_obj;
CeedRequest *const                        CEED_REQUEST_IMMEDIATE    = &req_immediate_obj;
CeedRequest *const                        CEED_REQUEST_ORDERED      = &req_ordered_obj;
const CeedInt                             CEED_STRIDES_BACKEND[3]   = {0, 0, 0};
const CeedVector                          CEED_VECTOR_ACTIVE        = &vec_active_obj;
const CeedVector                          CEED_VECTOR_NONE          = &vec_none_obj;
const CeedBasis                           CEED_BASIS_NONE           = &basis_none_obj;
const CeedElemRestriction                 CEED_ELEMRESTRICTION_NONE = &rstr_none_obj;
const CeedQFunction                       CEED_QFUNCTION_NONE       = &qf_none_obj;

/* ------------------------------------------------------------------------------------------------------------------ */
/* errors                                                                                                             */

/* CeedErrorImpl: route an error through the Ceed's handler (CeedErrorStore by default, as HONEE installs it,
 * examples/navierstokes.c:66); the CeedError macro of the public header calls this. */
int CeedErrorImpl(Ceed ceed, const char *file, int line, const char *func, int ecode, const char *fmt, ...) {
  va_list args;
  va_start(args, fmt);
  int r = ecode;
  if (ceed && ceed->handler) r = ceed->handler(ceed, file, line, func, ecode, fmt, &args);
  else r = CeedErrorStore(ceed, file, line, func, ecode, fmt, &args);
  va_end(args);
  return r;
}
#define CK(call)            \
  do {                      \
    int ierr_ = (call);     \
    if (ierr_) return ierr_; \
  } while (0)
#define CUDA_CK(ceed, call)                                                                                          \
  do {                                                                                                               \
    cudaError_t cerr_ = (call);                                                                                      \
    if (cerr_ != cudaSuccess) return CeedError((ceed), CEED_ERROR_BACKEND, "CUDA error %s in %s", cudaGetErrorString(cerr_), #call); \
  } while (0)
#define HB_CK(ceed, call)                                                                             \
  do {                                                                                                \
    int herr_ = (call);                                                                               \
    if (herr_) return CeedError((ceed), herr_ == HB_ERROR_UNSUPPORTED ? CEED_ERROR_UNSUPPORTED : CEED_ERROR_BACKEND, \
                                "backend call %s failed with status %d", #call, herr_);              \
  } while (0)

static char fallback_msg[2048];

int CeedErrorStore(Ceed ceed, const char *filename, int line_no, const char *func, int ecode, const char *format, va_list *args) {
  char *buf = ceed ? ceed->err_msg : fallback_msg;
  int   n   = snprintf(buf, 2048, "%s:%d in %s(): ", filename, line_no, func);
  if (n < 0 || n >= 2048) n = 0;
  vsnprintf(buf + n, (size_t)(2048 - n), format, *args);
  return ecode;
}
int CeedErrorReturn(Ceed ceed, const char *filename, int line_no, const char *func, int ecode, const char *format, va_list *args) {
  return CeedErrorStore(ceed, filename, line_no, func, ecode, format, args);
}
int CeedErrorAbort(Ceed ceed, const char *filename, int line_no, const char *func, int ecode, const char *format, va_list *args) {
  CeedErrorStore(ceed, filename, line_no, func, ecode, format, args);
  fprintf(stderr, "%s\n", ceed ? ceed->err_msg : fallback_msg);
  abort();
  return ecode;
}
int CeedErrorExit(Ceed ceed, const char *filename, int line_no, const char *func, int ecode, const char *format, va_list *args) {
  CeedErrorStore(ceed, filename, line_no, func, ecode, format, args);
  fprintf(stderr, "%s\n", ceed ? ceed->err_msg : fallback_msg);
  exit(ecode);
  return ecode;
}
int CeedSetErrorHandler(Ceed ceed, CeedErrorHandler handler) {
  ceed->handler = handler;
  return CEED_ERROR_SUCCESS;
}
int CeedGetErrorMessage(Ceed ceed, const char **err_msg) {
  *err_msg = ceed ? ceed->err_msg : fallback_msg;
  return CEED_ERROR_SUCCESS;
}
int CeedResetErrorMessage(Ceed ceed, const char **err_msg) {
  if (ceed) ceed->err_msg[0] = 0;
  if (err_msg) *err_msg = ceed ? ceed->err_msg : fallback_msg;
  return CEED_ERROR_SUCCESS;
}

/* ------------------------------------------------------------------------------------------------------------------ */
/* Ceed                                                                                                               */

int CeedInit(const char *resource, Ceed *ceed) {
  *ceed = NULL;
  if (!resource) return CEED_ERROR_MAJOR;
  int mixed = 0;
  if (!strcmp(resource, "/gpu/b200") || !strcmp(resource, "/gpu/cuda") || !strcmp(resource, "/gpu/cuda/shared") ||
      !strcmp(resource, "/gpu/cuda/gen") || !strcmp(resource, "/gpu/cuda/ref") || !strcmp(resource, "/gpu/b200/fp64"))
    mixed = 0;
  else if (!strcmp(resource, "/gpu/b200/mixed")) mixed = 1;
  else {
    snprintf(fallback_msg, sizeof fallback_msg, "CeedInit: resource '%s' is not provided by the B200 backend (use /gpu/b200 or /gpu/b200/mixed)",
             resource);
    return CEED_ERROR_UNSUPPORTED;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
    snprintf(fallback_msg, sizeof fallback_msg, "CeedInit: resource '%s' needs a CUDA device and none is visible", resource);
    return CEED_ERROR_BACKEND;
  }
  Ceed c = (Ceed)calloc(1, sizeof(*c));
  c->ref   = 1;
  c->mixed = mixed;
  snprintf(c->resource, sizeof c->resource, "%s", resource);
  c->stream  = NULL;
  c->handler = CeedErrorStore;
  if (cudaMalloc((void **)&c->d_scratch, 1024 * sizeof(double)) != cudaSuccess) {
    free(c);
    return CEED_ERROR_BACKEND;
  }
  *ceed = c;
  return CEED_ERROR_SUCCESS;
}

int CeedReferenceCopy(Ceed ceed, Ceed *ceed_copy) {
  ceed->ref++;
  CK(CeedDestroy(ceed_copy));
  *ceed_copy = ceed;
  return CEED_ERROR_SUCCESS;
}

int CeedDestroy(Ceed *ceed) {
  if (!*ceed) return CEED_ERROR_SUCCESS;
  if (--(*ceed)->ref > 0) {
    *ceed = NULL;
    return CEED_ERROR_SUCCESS;
  }
  cudaFree((*ceed)->d_scratch);
  if ((*ceed)->copy_streams) {
    cudaStreamDestroy((*ceed)->s_h2d);
    cudaStreamDestroy((*ceed)->s_d2h);
    cudaEventDestroy((*ceed)->ev_tmp);
  }
  if ((*ceed)->h_status) cudaFreeHost((*ceed)->h_status);
  free(*ceed);
  *ceed = NULL;
  return CEED_ERROR_SUCCESS;
}

int CeedGetResource(Ceed ceed, const char **resource) {
  *resource = ceed->resource;
  return CEED_ERROR_SUCCESS;
}
int CeedGetPreferredMemType(Ceed ceed, CeedMemType *type) {
  (void)ceed;
  *type = CEED_MEM_DEVICE;
  return CEED_ERROR_SUCCESS;
}
int CeedIsDeterministic(Ceed ceed, bool *is_deterministic) {
  (void)ceed;
  *is_deterministic = true; /* coloured scatters: one addition per output entry and launch, colours in stream order */
  return CEED_ERROR_SUCCESS;
}
int CeedSetStream(Ceed ceed, void *handle) {
  ceed->stream = (cudaStream_t)handle;
  return CEED_ERROR_SUCCESS;
}
int CeedGetVersion(int *major, int *minor, int *patch, bool *release) {
  if (major) *major = CEED_VERSION_MAJOR;
  if (minor) *minor = CEED_VERSION_MINOR;
  if (patch) *patch = CEED_VERSION_PATCH;
  if (release) *release = CEED_VERSION_RELEASE;
  return CEED_ERROR_SUCCESS;
}

/* ------------------------------------------------------------------------------------------------------------------ */
/* CeedVector                                                                                                         */

int CeedVectorCreate(Ceed ceed, CeedSize len, CeedVector *vec) {
  if (len < 0) return CeedError(ceed, CEED_ERROR_DIMENSION, "negative vector length");
  CeedVector v = (CeedVector)calloc(1, sizeof(*v));
  v->ceed      = ceed;
  ceed->ref++;
  v->ref    = 1;
  v->length = len;
  *vec      = v;
  return CEED_ERROR_SUCCESS;
}

int CeedVectorReferenceCopy(CeedVector vec, CeedVector *vec_copy) {
  vec->ref++;
  CK(CeedVectorDestroy(vec_copy));
  *vec_copy = vec;
  return CEED_ERROR_SUCCESS;
}

static int vec_alloc_host(CeedVector v) {
  if (!v->h) {
    v->h     = (double *)malloc(sizeof(double) * (size_t)(v->length ? v->length : 1));
    v->h_own = 1;
    if (!v->h) return CeedError(v->ceed, CEED_ERROR_MAJOR, "host allocation of %td doubles failed", v->length);
  }
  return CEED_ERROR_SUCCESS;
}
static int vec_alloc_dev(CeedVector v) {
  if (!v->d) {
    CUDA_CK(v->ceed, cudaMalloc((void **)&v->d, sizeof(double) * (size_t)(v->length ? v->length : 1)));
    v->d_own = 1;
  }
  return CEED_ERROR_SUCCESS;
}
/* bring the FP64 device copy up to date from the FP32 shadow */
static int vec_unstale(CeedVector v) {
  if (!v->f64_stale) return CEED_ERROR_SUCCESS;
  CK(vec_alloc_dev(v));
  HB_CK(v->ceed, hb_vec_f32_to_f64(v->d_f32, v->d, v->length, 0, v->ceed->stream));
  v->use_known = 0; /* d written on the compute stream after the last operator's ev_use */
  v->f64_stale = 0;
  v->d_valid   = 1;
  v->h_valid   = 0;
  return CEED_ERROR_SUCCESS;
}
static int ceed_copy_streams(Ceed c) {
  if (c->copy_streams) return CEED_ERROR_SUCCESS;
  if (!c->h_status) CUDA_CK(c, cudaMallocHost((void **)&c->h_status, sizeof(int) * 64));
  CUDA_CK(c, cudaStreamCreateWithFlags(&c->s_h2d, cudaStreamNonBlocking));
  CUDA_CK(c, cudaStreamCreateWithFlags(&c->s_d2h, cudaStreamNonBlocking));
  CUDA_CK(c, cudaEventCreateWithFlags(&c->ev_tmp, cudaEventDisableTiming));
  c->copy_streams = 1;
  return CEED_ERROR_SUCCESS;
}
static int vec_events(CeedVector v) {
  if (v->events) return CEED_ERROR_SUCCESS;
  CUDA_CK(v->ceed, cudaEventCreateWithFlags(&v->ev_h2d, cudaEventDisableTiming));
  CUDA_CK(v->ceed, cudaEventCreateWithFlags(&v->ev_use, cudaEventDisableTiming));
  v->events = 1;
  return CEED_ERROR_SUCCESS;
}
/* A host array handed over with CEED_USE_POINTER is read by an asynchronous copy: wait for it before the host array is
 * given back, replaced, overwritten or freed. */
static int vec_wait_h2d(CeedVector v) {
  if (v->h2d_pending) {
    CUDA_CK(v->ceed, cudaEventSynchronize(v->ev_h2d));
    v->h2d_pending = 0;
  }
  return CEED_ERROR_SUCCESS;
}
/* Host -> device on the copy stream, after every earlier use of the device array on the compute stream (ev_use when an
 * operator recorded it, else everything enqueued so far); later compute work waits for the copy. */
static int vec_sync_dev(CeedVector v) {
  CK(vec_unstale(v));
  CK(vec_alloc_dev(v));
  if (!v->d_valid) {
    if (!v->h_valid) return CeedError(v->ceed, CEED_ERROR_INCOMPLETE, "vector has no valid data");
    Ceed c = v->ceed;
    CK(ceed_copy_streams(c));
    CK(vec_events(v));
    CK(vec_wait_h2d(v));
    if (v->use_known) CUDA_CK(c, cudaStreamWaitEvent(c->s_h2d, v->ev_use, 0));
    else {
      CUDA_CK(c, cudaEventRecord(c->ev_tmp, c->stream));
      CUDA_CK(c, cudaStreamWaitEvent(c->s_h2d, c->ev_tmp, 0));
    }
    CUDA_CK(c, cudaMemcpyAsync(v->d, v->h, sizeof(double) * (size_t)v->length, cudaMemcpyHostToDevice, c->s_h2d));
    CUDA_CK(c, cudaEventRecord(v->ev_h2d, c->s_h2d));
    CUDA_CK(c, cudaStreamWaitEvent(c->stream, v->ev_h2d, 0));
    v->h2d_pending = 1;
    v->d_valid     = 1;
  }
  return CEED_ERROR_SUCCESS;
}
static int ceed_status_error(Ceed ceed, int i, int st) {
  cudaMemset(ceed->ops[i]->d_status, 0, sizeof(int));
  return CeedError(ceed, CEED_ERROR_BACKEND, "a fused kernel abandoned a bounded wait (status %d); its output is incomplete", st);
}
/* Kernels never trap: a bounded wait that gives up sets a status word.  Surface it at the next host synchronisation. */
static int ceed_check_status(Ceed ceed) {
  for (int i = 0; i < ceed->nops; i++) {
    int st = 0;
    if (cudaMemcpy(&st, ceed->ops[i]->d_status, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
      return CeedError(ceed, CEED_ERROR_BACKEND, "could not read the kernel status word");
    if (st) return ceed_status_error(ceed, i, st);
  }
  return CEED_ERROR_SUCCESS;
}
/* The same check beside a read-back on the copy stream s_d2h, after the producer's ev_use: the words are read in that
 * stream's order, so the check covers the producer and does not wait for kernels enqueued after it (a blocking
 * cudaMemcpy would, on the legacy default stream, and so serialise a pipelined host loop).  A word that a later kernel
 * is still writing reads as 0 or as its error; the error is then reported here or at a later synchronisation. */
static int ceed_check_status_d2h(Ceed ceed) {
  const int n = ceed->nops;
  for (int i = 0; i < n; i++)
    CUDA_CK(ceed, cudaMemcpyAsync(ceed->h_status + i, ceed->ops[i]->d_status, sizeof(int), cudaMemcpyDeviceToHost, ceed->s_d2h));
  CUDA_CK(ceed, cudaStreamSynchronize(ceed->s_d2h));
  for (int i = 0; i < n; i++)
    if (ceed->h_status[i]) return ceed_status_error(ceed, i, ceed->h_status[i]);
  return CEED_ERROR_SUCCESS;
}
static void ceed_register_op(Ceed ceed, HbElemOp *op) {
  if (ceed->nops < 64) ceed->ops[ceed->nops++] = op;
}
static void ceed_unregister_op(Ceed ceed, HbElemOp *op) {
  for (int i = 0; i < ceed->nops; i++)
    if (ceed->ops[i] == op) {
      ceed->ops[i] = ceed->ops[--ceed->nops];
      return;
    }
}

/* Device -> host.  When the last operator that touched the vector recorded ev_use, the read-back waits only for that
 * operator (on the copy stream), so it overlaps kernels enqueued after it; otherwise it follows the compute stream. */
static int vec_sync_host(CeedVector v) {
  CK(vec_unstale(v));
  CK(vec_alloc_host(v));
  CK(vec_wait_h2d(v));
  if (!v->h_valid) {
    if (!v->d_valid) return CeedError(v->ceed, CEED_ERROR_INCOMPLETE, "vector has no valid data");
    Ceed c = v->ceed;
    if (v->use_known) {
      CK(ceed_copy_streams(c));
      CUDA_CK(c, cudaStreamWaitEvent(c->s_d2h, v->ev_use, 0));
      CUDA_CK(c, cudaMemcpyAsync(v->h, v->d, sizeof(double) * (size_t)v->length, cudaMemcpyDeviceToHost, c->s_d2h));
      v->h_valid = 1;
      CK(ceed_check_status_d2h(c));
    } else {
      CUDA_CK(c, cudaMemcpyAsync(v->h, v->d, sizeof(double) * (size_t)v->length, cudaMemcpyDeviceToHost, c->stream));
      CUDA_CK(c, cudaStreamSynchronize(c->stream));
      v->h_valid = 1;
      CK(ceed_check_status(v->ceed));
    }
  }
  return CEED_ERROR_SUCCESS;
}
/* device array for a kernel that reads the vector */
static int vec_dev_read(CeedVector v, const double **d) {
  CK(vec_sync_dev(v));
  v->use_known = 0; /* a new use of d: ev_use no longer covers it */
  *d = v->d;
  return CEED_ERROR_SUCCESS;
}
/* device array for a kernel that writes (write_only: contents may be discarded) */
static int vec_dev_write(CeedVector v, double **d, int write_only) {
  v->use_known = 0;
  if (write_only) {
    v->f64_stale = 0;
    CK(vec_alloc_dev(v));
  } else CK(vec_sync_dev(v));
  v->d_valid   = 1;
  v->h_valid   = 0;
  v->f32_valid = 0;
  *d           = v->d;
  return CEED_ERROR_SUCCESS;
}

/* Any call that hands the device array out (GetArray*, TakeArray) or replaces or writes it outside an operator (SetArray
 * on the device, including a device-to-device copy on the compute stream) clears use_known: ev_use then no longer covers
 * every use of d, so the next copy between host and device follows the whole compute stream instead of the last
 * operator's event.  SetArray on the host leaves d untouched, so ev_use still covers it: the upload of the new host array
 * waits only for the last operator that used the vector, and overlaps the kernels enqueued after that one. */
int CeedVectorSetArray(CeedVector v, CeedMemType mem_type, CeedCopyMode copy_mode, CeedScalar *array) {
  CK(vec_wait_h2d(v));
  v->f64_stale = 0;
  v->f32_valid = 0;
  if (mem_type == CEED_MEM_HOST) {
    if (copy_mode == CEED_COPY_VALUES) {
      CK(vec_alloc_host(v));
      if (array) memcpy(v->h, array, sizeof(double) * (size_t)v->length);
    } else {
      if (v->h_own) free(v->h);
      v->h     = array;
      v->h_own = copy_mode == CEED_OWN_POINTER;
    }
    v->h_valid = array != NULL;
    v->d_valid = 0;
  } else {
    v->use_known = 0;
    if (copy_mode == CEED_COPY_VALUES) {
      CK(vec_alloc_dev(v));
      if (array) CUDA_CK(v->ceed, cudaMemcpyAsync(v->d, array, sizeof(double) * (size_t)v->length, cudaMemcpyDeviceToDevice, v->ceed->stream));
    } else {
      if (v->d_own) cudaFree(v->d);
      v->d     = array;
      v->d_own = copy_mode == CEED_OWN_POINTER;
    }
    v->d_valid = array != NULL;
    v->h_valid = 0;
  }
  return CEED_ERROR_SUCCESS;
}

int CeedVectorSetValue(CeedVector v, CeedScalar value) {
  double *d;
  CK(vec_dev_write(v, &d, 1));
  HB_CK(v->ceed, hb_vec_set_f64(d, v->length, value, v->ceed->stream));
  return CEED_ERROR_SUCCESS;
}

int CeedVectorSyncArray(CeedVector v, CeedMemType mem_type) { return mem_type == CEED_MEM_HOST ? vec_sync_host(v) : vec_sync_dev(v); }

int CeedVectorTakeArray(CeedVector v, CeedMemType mem_type, CeedScalar **array) {
  CK(vec_wait_h2d(v));
  v->use_known = 0;
  if (mem_type == CEED_MEM_HOST) {
    if (v->h && !v->h_valid && (v->d_valid || v->f64_stale)) CK(vec_sync_host(v));
    *array     = v->h;
    v->h       = NULL;
    v->h_own   = 0;
    v->h_valid = 0;
  } else {
    if (v->d && !v->d_valid && (v->h_valid || v->f64_stale)) CK(vec_sync_dev(v));
    *array     = v->d;
    v->d       = NULL;
    v->d_own   = 0;
    v->d_valid = 0;
  }
  return CEED_ERROR_SUCCESS;
}

int CeedVectorGetArrayRead(CeedVector v, CeedMemType mem_type, const CeedScalar **array) {
  if (mem_type == CEED_MEM_HOST) {
    CK(vec_sync_host(v));
    *array = v->h;
  } else {
    CK(vec_sync_dev(v));
    v->use_known = 0;
    *array = v->d;
  }
  return CEED_ERROR_SUCCESS;
}

int CeedVectorGetArray(CeedVector v, CeedMemType mem_type, CeedScalar **array) {
  CK(vec_wait_h2d(v));
  if (mem_type == CEED_MEM_HOST) {
    CK(vec_sync_host(v));
    v->d_valid = 0;
    *array     = v->h;
  } else {
    CK(vec_sync_dev(v));
    v->use_known = 0;
    v->h_valid   = 0;
    *array       = v->d;
  }
  v->f32_valid = 0;
  return CEED_ERROR_SUCCESS;
}

int CeedVectorGetArrayWrite(CeedVector v, CeedMemType mem_type, CeedScalar **array) {
  CK(vec_wait_h2d(v));
  v->f64_stale = 0;
  v->f32_valid = 0;
  if (mem_type == CEED_MEM_HOST) {
    CK(vec_alloc_host(v));
    v->h_valid = 1;
    v->d_valid = 0;
    *array     = v->h;
  } else {
    CK(vec_alloc_dev(v));
    v->use_known = 0;
    v->d_valid   = 1;
    v->h_valid   = 0;
    *array       = v->d;
  }
  return CEED_ERROR_SUCCESS;
}

int CeedVectorRestoreArray(CeedVector v, CeedScalar **array) {
  (void)v;
  *array = NULL;
  return CEED_ERROR_SUCCESS;
}
int CeedVectorRestoreArrayRead(CeedVector v, const CeedScalar **array) {
  (void)v;
  *array = NULL;
  return CEED_ERROR_SUCCESS;
}
int CeedVectorGetLength(CeedVector v, CeedSize *length) {
  *length = v->length;
  return CEED_ERROR_SUCCESS;
}

int CeedVectorNorm(CeedVector v, CeedNormType type, CeedScalar *norm) {
  const double *d;
  CK(vec_dev_read(v, &d));
  double r  = 0;
  int    tp = type == CEED_NORM_1 ? 0 : (type == CEED_NORM_2 ? 1 : 2);
  HB_CK(v->ceed, hb_vec_reduce_f64(d, NULL, v->length, tp, v->ceed->d_scratch, &r, v->ceed->stream));
  CK(ceed_check_status(v->ceed));
  *norm = type == CEED_NORM_2 ? sqrt(r) : r;
  return CEED_ERROR_SUCCESS;
}

int CeedVectorCopy(CeedVector vec, CeedVector vec_copy) {
  if (vec->length != vec_copy->length) return CeedError(vec->ceed, CEED_ERROR_INCOMPATIBLE, "vector lengths differ");
  const double *s;
  double       *d;
  CK(vec_dev_read(vec, &s));
  CK(vec_dev_write(vec_copy, &d, 1));
  CUDA_CK(vec->ceed, cudaMemcpyAsync(d, s, sizeof(double) * (size_t)vec->length, cudaMemcpyDeviceToDevice, vec->ceed->stream));
  return CEED_ERROR_SUCCESS;
}
int CeedVectorScale(CeedVector x, CeedScalar alpha) {
  double *d;
  CK(vec_dev_write(x, &d, 0));
  HB_CK(x->ceed, hb_vec_scale_f64(d, x->length, alpha, x->ceed->stream));
  return CEED_ERROR_SUCCESS;
}
int CeedVectorAXPY(CeedVector y, CeedScalar alpha, CeedVector x) {
  if (x->length != y->length) return CeedError(y->ceed, CEED_ERROR_INCOMPATIBLE, "vector lengths differ");
  const double *xd;
  double       *yd;
  CK(vec_dev_read(x, &xd));
  CK(vec_dev_write(y, &yd, 0));
  HB_CK(y->ceed, hb_vec_axpy_f64(yd, alpha, xd, y->length, y->ceed->stream));
  return CEED_ERROR_SUCCESS;
}
int CeedVectorAXPBY(CeedVector y, CeedScalar alpha, CeedScalar beta, CeedVector x) {
  if (x->length != y->length) return CeedError(y->ceed, CEED_ERROR_INCOMPATIBLE, "vector lengths differ");
  const double *xd;
  double       *yd;
  CK(vec_dev_read(x, &xd));
  CK(vec_dev_write(y, &yd, 0));
  HB_CK(y->ceed, hb_vec_axpby_f64(yd, alpha, beta, xd, y->length, y->ceed->stream));
  return CEED_ERROR_SUCCESS;
}
int CeedVectorPointwiseMult(CeedVector w, CeedVector x, CeedVector y) {
  if (x->length != w->length || y->length != w->length) return CeedError(w->ceed, CEED_ERROR_INCOMPATIBLE, "vector lengths differ");
  const double *xd, *yd;
  double       *wd;
  CK(vec_dev_read(x, &xd));
  CK(vec_dev_read(y, &yd));
  CK(vec_dev_write(w, &wd, w != x && w != y));
  HB_CK(w->ceed, hb_vec_pointwise_mult_f64(wd, xd, yd, w->length, w->ceed->stream));
  return CEED_ERROR_SUCCESS;
}
int CeedVectorReciprocal(CeedVector v) {
  double *d;
  CK(vec_dev_write(v, &d, 0));
  HB_CK(v->ceed, hb_vec_reciprocal_f64(d, v->length, v->ceed->stream));
  return CEED_ERROR_SUCCESS;
}

int CeedVectorDestroy(CeedVector *vec) {
  CeedVector v = *vec;
  if (!v || v == CEED_VECTOR_ACTIVE || v == CEED_VECTOR_NONE) {
    *vec = NULL;
    return CEED_ERROR_SUCCESS;
  }
  if (--v->ref > 0) {
    *vec = NULL;
    return CEED_ERROR_SUCCESS;
  }
  vec_wait_h2d(v);
  if (v->h_own) free(v->h);
  if (v->d_own) cudaFree(v->d);
  if (v->d_f32) cudaFree(v->d_f32);
  if (v->events) {
    cudaEventDestroy(v->ev_h2d);
    cudaEventDestroy(v->ev_use);
  }
  Ceed ceed = v->ceed;
  free(v);
  *vec = NULL;
  return CeedDestroy(&ceed);
}

/* ------------------------------------------------------------------------------------------------------------------ */
/* CeedElemRestriction                                                                                                */

int CeedElemRestrictionCreate(Ceed ceed, CeedInt num_elem, CeedInt elem_size, CeedInt num_comp, CeedInt comp_stride, CeedSize l_size,
                              CeedMemType mem_type, CeedCopyMode copy_mode, const CeedInt *offsets, CeedElemRestriction *rstr) {
  (void)copy_mode;
  if (num_elem < 0 || elem_size < 1 || num_comp < 1) return CeedError(ceed, CEED_ERROR_DIMENSION, "invalid restriction dimensions");
  const size_t n = (size_t)num_elem * elem_size;
  int32_t     *h = (int32_t *)malloc(sizeof(int32_t) * (n ? n : 1));
  if (mem_type == CEED_MEM_HOST) memcpy(h, offsets, sizeof(int32_t) * n);
  else CUDA_CK(ceed, cudaMemcpy(h, offsets, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
  /* host-side bounds validation: every entry offset + c*comp_stride must lie in [0, l_size) */
  const int64_t span = (int64_t)(num_comp - 1) * comp_stride;
  for (size_t i = 0; i < n; i++)
    if (h[i] < 0 || (int64_t)h[i] + span >= l_size) {
      const int32_t bad = h[i];
      free(h);
      return CeedError(ceed, CEED_ERROR_DIMENSION, "restriction offset %d at entry %zu outside the L-vector of size %td", bad, i, l_size);
    }
  CeedElemRestriction r = (CeedElemRestriction)calloc(1, sizeof(*r));
  r->ceed               = ceed;
  ceed->ref++;
  r->ref         = 1;
  r->num_elem    = num_elem;
  r->elem_size   = elem_size;
  r->num_comp    = num_comp;
  r->comp_stride = comp_stride;
  r->l_size      = l_size;
  r->h_off       = h;
  *rstr          = r;
  return CEED_ERROR_SUCCESS;
}

int CeedElemRestrictionCreateStrided(Ceed ceed, CeedInt num_elem, CeedInt elem_size, CeedInt num_comp, CeedSize l_size, const CeedInt strides[3],
                                     CeedElemRestriction *rstr) {
  CeedElemRestriction r = (CeedElemRestriction)calloc(1, sizeof(*r));
  r->ceed               = ceed;
  ceed->ref++;
  r->ref       = 1;
  r->num_elem  = num_elem;
  r->elem_size = elem_size;
  r->num_comp  = num_comp;
  r->l_size    = l_size;
  r->strided   = 1;
  if (strides == CEED_STRIDES_BACKEND) {
    /* backend layout [elem][comp][node]: the layout the fused kernels read qdata and write jac_data in */
    r->strides[0] = 1;
    r->strides[1] = elem_size;
    r->strides[2] = elem_size * num_comp;
  } else {
    memcpy(r->strides, strides, sizeof(r->strides));
    if (strides[0] < 0 || strides[1] < 0 || strides[2] < 0) {
      CeedElemRestrictionDestroy(&r);
      return CeedError(ceed, CEED_ERROR_DIMENSION, "negative restriction strides are not supported");
    }
  }
  const int64_t last = (int64_t)(elem_size - 1) * r->strides[0] + (int64_t)(num_comp - 1) * r->strides[1] + (int64_t)(num_elem - 1) * r->strides[2];
  if (num_elem > 0 && (last >= l_size || last < 0)) {
    CeedElemRestrictionDestroy(&r);
    return CeedError(ceed, CEED_ERROR_DIMENSION, "strided restriction exceeds the L-vector size %td", l_size);
  }
  *rstr = r;
  return CEED_ERROR_SUCCESS;
}

int CeedElemRestrictionReferenceCopy(CeedElemRestriction rstr, CeedElemRestriction *rstr_copy) {
  rstr->ref++;
  CK(CeedElemRestrictionDestroy(rstr_copy));
  *rstr_copy = rstr;
  return CEED_ERROR_SUCCESS;
}

int CeedElemRestrictionCreateVector(CeedElemRestriction r, CeedVector *l_vec, CeedVector *e_vec) {
  if (l_vec) CK(CeedVectorCreate(r->ceed, r->l_size, l_vec));
  if (e_vec) CK(CeedVectorCreate(r->ceed, (CeedSize)r->num_elem * r->elem_size * r->num_comp, e_vec));
  return CEED_ERROR_SUCCESS;
}

static int rstr_upload(CeedElemRestriction r) {
  if (r->strided) {
    if (!r->d_strides) {
      CUDA_CK(r->ceed, cudaMalloc((void **)&r->d_strides, sizeof(int32_t) * 3));
      CUDA_CK(r->ceed, cudaMemcpy(r->d_strides, r->strides, sizeof(int32_t) * 3, cudaMemcpyHostToDevice));
    }
  } else if (!r->d_off) {
    const size_t n = (size_t)r->num_elem * r->elem_size;
    CUDA_CK(r->ceed, cudaMalloc((void **)&r->d_off, sizeof(int32_t) * (n ? n : 1)));
    CUDA_CK(r->ceed, cudaMemcpy(r->d_off, r->h_off, sizeof(int32_t) * n, cudaMemcpyHostToDevice));
  }
  return CEED_ERROR_SUCCESS;
}

/* transpose map: for each L entry, the E entries that map to it, in increasing E order (a serial scatter's order) */
static int rstr_build_transpose(CeedElemRestriction r) {
  if (r->d_tptr) return CEED_ERROR_SUCCESS;
  const int64_t ne = (int64_t)r->num_elem * r->elem_size * r->num_comp;
  int64_t      *ptr = (int64_t *)calloc((size_t)r->l_size + 1, sizeof(int64_t));
  int64_t      *idx = (int64_t *)malloc(sizeof(int64_t) * (size_t)(ne ? ne : 1));
  for (int64_t t = 0; t < ne; t++) {
    const int64_t p = t % r->elem_size, rr = t / r->elem_size, c = rr % r->num_comp, el = rr / r->num_comp;
    ptr[r->h_off[el * r->elem_size + p] + c * r->comp_stride + 1]++;
  }
  for (int64_t i = 0; i < r->l_size; i++) ptr[i + 1] += ptr[i];
  int64_t *fill = (int64_t *)malloc(sizeof(int64_t) * (size_t)(r->l_size ? r->l_size : 1));
  memcpy(fill, ptr, sizeof(int64_t) * (size_t)r->l_size);
  /* E entries visited element by element, node by node: within one L entry this is increasing element order */
  for (int64_t el = 0; el < r->num_elem; el++)
    for (int64_t p = 0; p < r->elem_size; p++)
      for (int64_t c = 0; c < r->num_comp; c++) {
        const int64_t li = r->h_off[el * r->elem_size + p] + c * r->comp_stride;
        idx[fill[li]++]  = (el * r->num_comp + c) * r->elem_size + p;
      }
  free(fill);
  int err = 0;
  if (cudaMalloc((void **)&r->d_tptr, sizeof(int64_t) * ((size_t)r->l_size + 1)) != cudaSuccess ||
      cudaMalloc((void **)&r->d_teidx, sizeof(int64_t) * (size_t)(ne ? ne : 1)) != cudaSuccess ||
      cudaMemcpy(r->d_tptr, ptr, sizeof(int64_t) * ((size_t)r->l_size + 1), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(r->d_teidx, idx, sizeof(int64_t) * (size_t)ne, cudaMemcpyHostToDevice) != cudaSuccess)
    err = 1;
  free(ptr);
  free(idx);
  if (err) return CeedError(r->ceed, CEED_ERROR_BACKEND, "could not upload the transpose restriction map");
  return CEED_ERROR_SUCCESS;
}

int CeedElemRestrictionApply(CeedElemRestriction r, CeedTransposeMode t_mode, CeedVector u, CeedVector ru, CeedRequest *request) {
  (void)request;
  const CeedSize e_size = (CeedSize)r->num_elem * r->elem_size * r->num_comp;
  const CeedSize in_len = t_mode == CEED_NOTRANSPOSE ? r->l_size : e_size, out_len = t_mode == CEED_NOTRANSPOSE ? e_size : r->l_size;
  if (u->length < in_len || ru->length < out_len)
    return CeedError(r->ceed, CEED_ERROR_DIMENSION, "restriction apply vectors too short (need %td in, %td out)", in_len, out_len);
  CK(rstr_upload(r));
  const double *in;
  double       *out;
  CK(vec_dev_read(u, &in));
  if (t_mode == CEED_NOTRANSPOSE) {
    CK(vec_dev_write(ru, &out, 1));
    HB_CK(r->ceed, hb_restrict_apply(r->num_elem, r->elem_size, r->num_comp, r->comp_stride, r->strided ? NULL : r->d_off,
                                     r->strided ? r->d_strides : NULL, in, out, r->ceed->stream));
  } else {
    /* libCEED semantics: the transpose adds into ru */
    CK(vec_dev_write(ru, &out, 0));
    if (r->strided) HB_CK(r->ceed, hb_restrict_apply_t_strided(r->num_elem, r->elem_size, r->num_comp, r->d_strides, in, out, r->ceed->stream));
    else {
      CK(rstr_build_transpose(r));
      HB_CK(r->ceed, hb_restrict_apply_t_csr(r->l_size, r->d_tptr, r->d_teidx, in, out, r->ceed->stream));
    }
  }
  return CEED_ERROR_SUCCESS;
}

int CeedElemRestrictionGetNumElements(CeedElemRestriction r, CeedInt *num_elem) {
  *num_elem = r->num_elem;
  return CEED_ERROR_SUCCESS;
}
int CeedElemRestrictionGetElementSize(CeedElemRestriction r, CeedInt *elem_size) {
  *elem_size = r->elem_size;
  return CEED_ERROR_SUCCESS;
}
int CeedElemRestrictionGetLVectorSize(CeedElemRestriction r, CeedSize *l_size) {
  *l_size = r->l_size;
  return CEED_ERROR_SUCCESS;
}
int CeedElemRestrictionGetEVectorSize(CeedElemRestriction r, CeedSize *e_size) {
  *e_size = (CeedSize)r->num_elem * r->elem_size * r->num_comp;
  return CEED_ERROR_SUCCESS;
}
int CeedElemRestrictionGetNumComponents(CeedElemRestriction r, CeedInt *num_comp) {
  *num_comp = r->num_comp;
  return CEED_ERROR_SUCCESS;
}
int CeedElemRestrictionGetCompStride(CeedElemRestriction r, CeedInt *comp_stride) {
  *comp_stride = r->comp_stride;
  return CEED_ERROR_SUCCESS;
}
int CeedElemRestrictionGetMultiplicity(CeedElemRestriction r, CeedVector mult) {
  CeedVector e;
  CK(CeedVectorCreate(r->ceed, (CeedSize)r->num_elem * r->elem_size * r->num_comp, &e));
  CK(CeedVectorSetValue(e, 1.0));
  CK(CeedVectorSetValue(mult, 0.0));
  CK(CeedElemRestrictionApply(r, CEED_TRANSPOSE, e, mult, CEED_REQUEST_IMMEDIATE));
  return CeedVectorDestroy(&e);
}

int CeedElemRestrictionDestroy(CeedElemRestriction *rstr) {
  CeedElemRestriction r = *rstr;
  if (!r || r == CEED_ELEMRESTRICTION_NONE) {
    *rstr = NULL;
    return CEED_ERROR_SUCCESS;
  }
  if (--r->ref > 0) {
    *rstr = NULL;
    return CEED_ERROR_SUCCESS;
  }
  free(r->h_off);
  cudaFree(r->d_off);
  cudaFree(r->d_strides);
  cudaFree(r->d_tptr);
  cudaFree(r->d_teidx);
  Ceed ceed = r->ceed;
  free(r);
  *rstr = NULL;
  return CeedDestroy(&ceed);
}

/* ------------------------------------------------------------------------------------------------------------------ */
/* CeedBasis                                                                                                          */

int CeedBasisCreateTensorH1(Ceed ceed, CeedInt dim, CeedInt num_comp, CeedInt P_1d, CeedInt Q_1d, const CeedScalar *interp_1d, const CeedScalar *grad_1d,
                            const CeedScalar *q_ref_1d, const CeedScalar *q_weight_1d, CeedBasis *basis) {
  if (dim < 1 || dim > 3 || P_1d < 1 || Q_1d < 1) return CeedError(ceed, CEED_ERROR_DIMENSION, "invalid tensor basis dimensions");
  if (P_1d > HB_MAX_P || Q_1d > HB_MAX_P)
    return CeedError(ceed, CEED_ERROR_UNSUPPORTED, "tensor bases with more than %d nodes or points per direction are not supported", HB_MAX_P);
  CeedBasis b = (CeedBasis)calloc(1, sizeof(*b));
  b->ceed     = ceed;
  ceed->ref++;
  b->ref      = 1;
  b->dim      = dim;
  b->num_comp = num_comp;
  b->P1d      = P_1d;
  b->Q1d      = Q_1d;
  b->tensor   = 1;
  memcpy(b->interp1d, interp_1d, sizeof(double) * P_1d * Q_1d);
  memcpy(b->grad1d, grad_1d, sizeof(double) * P_1d * Q_1d);
  if (q_ref_1d) memcpy(b->qref1d, q_ref_1d, sizeof(double) * Q_1d);
  if (q_weight_1d) memcpy(b->qweight1d, q_weight_1d, sizeof(double) * Q_1d);
  *basis = b;
  return CEED_ERROR_SUCCESS;
}

static void legendre(int n, double x, double *p, double *dp) {
  double p0 = 1, p1 = x;
  if (n == 0) {
    *p  = 1;
    *dp = 0;
    return;
  }
  for (int k = 2; k <= n; k++) {
    const double p2 = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k;
    p0              = p1;
    p1              = p2;
  }
  *p  = p1;
  *dp = n * (x * p1 - p0) / (x * x - 1);
}

int CeedGaussQuadrature(CeedInt Q, CeedScalar *x, CeedScalar *w) {
  for (int i = 0; i < Q; i++) {
    double z = -cos(M_PI * (i + 0.75) / (Q + 0.5)), p, dp;
    for (int it = 0; it < 100; it++) {
      legendre(Q, z, &p, &dp);
      const double dz = p / dp;
      z -= dz;
      if (fabs(dz) < 1e-16) break;
    }
    legendre(Q, z, &p, &dp);
    x[i] = z;
    if (w) w[i] = 2 / ((1 - z * z) * dp * dp);
  }
  return CEED_ERROR_SUCCESS;
}

int CeedLobattoQuadrature(CeedInt P, CeedScalar *x, CeedScalar *w) {
  const int N = P - 1;
  x[0]        = -1;
  x[N]        = 1;
  for (int i = 1; i < N; i++) {
    double z = -cos(M_PI * i / N);
    for (int it = 0; it < 100; it++) {
      double p, dp;
      legendre(N, z, &p, &dp);
      const double ddp = (2 * z * dp - N * (N + 1) * p) / (1 - z * z), dz = dp / ddp;
      z -= dz;
      if (fabs(dz) < 1e-16) break;
    }
    x[i] = z;
  }
  if (w)
    for (int i = 0; i <= N; i++) {
      double p, dp;
      legendre(N, x[i], &p, &dp);
      w[i] = 2.0 / (N * (N + 1) * p * p);
    }
  return CEED_ERROR_SUCCESS;
}

int CeedBasisCreateTensorH1Lagrange(Ceed ceed, CeedInt dim, CeedInt num_comp, CeedInt P, CeedInt Q, CeedQuadMode quad_mode, CeedBasis *basis) {
  if (P > HB_MAX_P || Q > HB_MAX_P || P < 2) return CeedError(ceed, CEED_ERROR_UNSUPPORTED, "unsupported Lagrange basis size");
  double nodes[HB_MAX_P], qx[HB_MAX_P], qw[HB_MAX_P], B[HB_MAX_P * HB_MAX_P], G[HB_MAX_P * HB_MAX_P];
  CeedLobattoQuadrature(P, nodes, NULL);
  if (quad_mode == CEED_GAUSS) CeedGaussQuadrature(Q, qx, qw);
  else CeedLobattoQuadrature(Q, qx, qw);
  for (int q = 0; q < Q; q++)
    for (int j = 0; j < P; j++) {
      double l = 1, dl = 0;
      for (int m = 0; m < P; m++) {
        if (m == j) continue;
        const double f = (qx[q] - nodes[m]) / (nodes[j] - nodes[m]);
        dl             = dl * f + l / (nodes[j] - nodes[m]);
        l *= f;
      }
      B[q * P + j] = l;
      G[q * P + j] = dl;
    }
  return CeedBasisCreateTensorH1(ceed, dim, num_comp, P, Q, B, G, qx, qw, basis);
}

int CeedBasisCreateH1(Ceed ceed, CeedElemTopology topo, CeedInt num_comp, CeedInt num_nodes, CeedInt nqpts, const CeedScalar *interp,
                      const CeedScalar *grad, const CeedScalar *q_ref, const CeedScalar *q_weights, CeedBasis *basis) {
  (void)topo, (void)num_comp, (void)num_nodes, (void)nqpts, (void)interp, (void)grad, (void)q_ref, (void)q_weights, (void)basis;
  return CeedError(ceed, CEED_ERROR_UNSUPPORTED, "non-tensor H1 bases are outside the B200 backend's hex-element scope");
}
/* libCEED's CeedBasisCreateProjection, which SetupLibceed calls for its initial-condition operator
 * (src/setuplibceed.c:150): a basis from the nodes of basis_from to the nodes of basis_to with interp = B_to^+ B_from
 * and grad = B_to^+ G_from, B_to^+ the least-squares pseudo-inverse over the quadrature both bases share, so a field
 * given at basis_from's nodes is evaluated (value and reference gradient) at basis_to's nodes.  Tensor bases take the
 * 1D rule per direction; the new basis has P = P_from, Q = P_to and no quadrature weights.  The pseudo-inverse comes
 * from the normal equations solved by Cholesky in long double (B_to has full column rank for Q >= P_to); when the
 * from-space lies in the to-space (a trilinear coordinate field projected onto a higher-degree solution basis) the
 * result is the from-basis evaluated at the to-nodes, to rounding. */
int CeedBasisCreateProjection(CeedBasis basis_from, CeedBasis basis_to, CeedBasis *basis_project) {
  Ceed ceed = basis_from->ceed;
  if (!basis_from->tensor || !basis_to->tensor || basis_from->dim != basis_to->dim)
    return CeedError(ceed, CEED_ERROR_UNSUPPORTED, "projection bases need two tensor H1 bases of the same dimension");
  if (basis_from->Q1d != basis_to->Q1d) return CeedError(ceed, CEED_ERROR_DIMENSION, "bases for a projection must share their quadrature points");
  const int Q = basis_to->Q1d, Pt = basis_to->P1d, Pf = basis_from->P1d;
  if (Pt > Q) return CeedError(ceed, CEED_ERROR_DIMENSION, "projection needs at least as many quadrature points as target nodes");
  long double M[HB_MAX_P][HB_MAX_P], L[HB_MAX_P][HB_MAX_P];
  for (int a = 0; a < Pt; a++)
    for (int b = 0; b < Pt; b++) {
      long double s = 0;
      for (int q = 0; q < Q; q++) s += (long double)basis_to->interp1d[q * Pt + a] * basis_to->interp1d[q * Pt + b];
      M[a][b] = s;
    }
  for (int a = 0; a < Pt; a++)
    for (int b = 0; b <= a; b++) {
      long double s = M[a][b];
      for (int k = 0; k < b; k++) s -= L[a][k] * L[b][k];
      if (a == b) {
        if (s <= 0) return CeedError(ceed, CEED_ERROR_DIMENSION, "target basis is rank deficient on the shared quadrature");
        L[a][a] = sqrtl(s);
      } else L[a][b] = s / L[b][b];
    }
  double interp[HB_MAX_P * HB_MAX_P], grad[HB_MAX_P * HB_MAX_P], zeros[HB_MAX_P] = {0};
  for (int m = 0; m < 2; m++) {
    const double *src = m ? basis_from->grad1d : basis_from->interp1d;
    double       *dst = m ? grad : interp;
    for (int j = 0; j < Pf; j++) {
      long double y[HB_MAX_P], x[HB_MAX_P];
      for (int a = 0; a < Pt; a++) {  /* rhs = B_to^T src[:, j], then forward and back substitution */
        long double r = 0;
        for (int q = 0; q < Q; q++) r += (long double)basis_to->interp1d[q * Pt + a] * src[q * Pf + j];
        for (int k = 0; k < a; k++) r -= L[a][k] * y[k];
        y[a] = r / L[a][a];
      }
      for (int a = Pt - 1; a >= 0; a--) {
        long double r = y[a];
        for (int k = a + 1; k < Pt; k++) r -= L[k][a] * x[k];
        x[a] = r / L[a][a];
      }
      for (int a = 0; a < Pt; a++) dst[a * Pf + j] = (double)x[a];
    }
  }
  return CeedBasisCreateTensorH1(ceed, basis_from->dim, basis_from->num_comp, Pf, Pt, interp, grad, zeros, zeros, basis_project);
}

int CeedBasisReferenceCopy(CeedBasis basis, CeedBasis *basis_copy) {
  basis->ref++;
  CK(CeedBasisDestroy(basis_copy));
  *basis_copy = basis;
  return CEED_ERROR_SUCCESS;
}

static int basis_upload(CeedBasis b) {
  if (b->d_B) return CEED_ERROR_SUCCESS;
  const size_t n = sizeof(double) * b->P1d * b->Q1d;
  CUDA_CK(b->ceed, cudaMalloc((void **)&b->d_B, n));
  CUDA_CK(b->ceed, cudaMalloc((void **)&b->d_G, n));
  CUDA_CK(b->ceed, cudaMalloc((void **)&b->d_w, sizeof(double) * b->Q1d));
  CUDA_CK(b->ceed, cudaMemcpy(b->d_B, b->interp1d, n, cudaMemcpyHostToDevice));
  CUDA_CK(b->ceed, cudaMemcpy(b->d_G, b->grad1d, n, cudaMemcpyHostToDevice));
  CUDA_CK(b->ceed, cudaMemcpy(b->d_w, b->qweight1d, sizeof(double) * b->Q1d, cudaMemcpyHostToDevice));
  return CEED_ERROR_SUCCESS;
}

/* Layouts: nodal input/output [elem][comp][P^dim]; quadrature values [elem][comp][Q^dim], gradients
 * [elem][dim][comp][Q^dim], weights [elem][Q^dim]. */
int CeedBasisApply(CeedBasis b, CeedInt num_elem, CeedTransposeMode t_mode, CeedEvalMode eval_mode, CeedVector u, CeedVector v) {
  if (eval_mode != CEED_EVAL_INTERP && eval_mode != CEED_EVAL_GRAD && eval_mode != CEED_EVAL_WEIGHT)
    return CeedError(b->ceed, CEED_ERROR_UNSUPPORTED, "eval mode %d not supported", eval_mode);
  CK(basis_upload(b));
  CeedSize Pn = 1, Qn = 1;
  for (int d = 0; d < b->dim; d++) Pn *= b->P1d, Qn *= b->Q1d;
  const CeedSize nq = (CeedSize)num_elem * b->num_comp * (eval_mode == CEED_EVAL_GRAD ? b->dim : 1) * Qn, np = (CeedSize)num_elem * b->num_comp * Pn;
  const CeedSize need_in = eval_mode == CEED_EVAL_WEIGHT ? 0 : (t_mode == CEED_TRANSPOSE ? nq : np);
  const CeedSize need_out = eval_mode == CEED_EVAL_WEIGHT ? (CeedSize)num_elem * Qn : (t_mode == CEED_TRANSPOSE ? np : nq);
  if ((need_in && (!u || u == CEED_VECTOR_NONE || u->length < need_in)) || v->length < need_out)
    return CeedError(b->ceed, CEED_ERROR_DIMENSION, "basis apply vectors too short (need %td in, %td out)", need_in, need_out);
  const double *in = NULL;
  double       *out;
  if (eval_mode != CEED_EVAL_WEIGHT) CK(vec_dev_read(u, &in));
  CK(vec_dev_write(v, &out, 1));
  HB_CK(b->ceed, hb_basis_apply_generic(num_elem, b->num_comp, b->dim, b->P1d, b->Q1d, t_mode == CEED_TRANSPOSE, eval_mode, b->d_B, b->d_G, b->d_w,
                                        in, out, b->ceed->stream));
  return CEED_ERROR_SUCCESS;
}

int CeedBasisGetDimension(CeedBasis b, CeedInt *dim) {
  *dim = b->dim;
  return CEED_ERROR_SUCCESS;
}
int CeedBasisGetNumComponents(CeedBasis b, CeedInt *num_comp) {
  *num_comp = b->num_comp;
  return CEED_ERROR_SUCCESS;
}
int CeedBasisGetNumNodes(CeedBasis b, CeedInt *P) {
  int n = 1;
  for (int d = 0; d < b->dim; d++) n *= b->P1d;
  *P = n;
  return CEED_ERROR_SUCCESS;
}
int CeedBasisGetNumNodes1D(CeedBasis b, CeedInt *P_1d) {
  *P_1d = b->P1d;
  return CEED_ERROR_SUCCESS;
}
int CeedBasisGetNumQuadraturePoints(CeedBasis b, CeedInt *Q) {
  int n = 1;
  for (int d = 0; d < b->dim; d++) n *= b->Q1d;
  *Q = n;
  return CEED_ERROR_SUCCESS;
}
int CeedBasisGetNumQuadraturePoints1D(CeedBasis b, CeedInt *Q_1d) {
  *Q_1d = b->Q1d;
  return CEED_ERROR_SUCCESS;
}

int CeedBasisDestroy(CeedBasis *basis) {
  CeedBasis b = *basis;
  if (!b || b == CEED_BASIS_NONE) {
    *basis = NULL;
    return CEED_ERROR_SUCCESS;
  }
  if (--b->ref > 0) {
    *basis = NULL;
    return CEED_ERROR_SUCCESS;
  }
  cudaFree(b->d_B);
  cudaFree(b->d_G);
  cudaFree(b->d_w);
  Ceed ceed = b->ceed;
  free(b);
  *basis = NULL;
  return CeedDestroy(&ceed);
}

/* ------------------------------------------------------------------------------------------------------------------ */
/* CeedQFunctionContext                                                                                               */

int CeedQFunctionContextCreate(Ceed ceed, CeedQFunctionContext *ctx) {
  CeedQFunctionContext c = (CeedQFunctionContext)calloc(1, sizeof(*c));
  c->ceed                = ceed;
  ceed->ref++;
  c->ref = 1;
  *ctx   = c;
  return CEED_ERROR_SUCCESS;
}
int CeedQFunctionContextReferenceCopy(CeedQFunctionContext ctx, CeedQFunctionContext *ctx_copy) {
  ctx->ref++;
  CK(CeedQFunctionContextDestroy(ctx_copy));
  *ctx_copy = ctx;
  return CEED_ERROR_SUCCESS;
}
int CeedQFunctionContextSetData(CeedQFunctionContext ctx, CeedMemType mem_type, CeedCopyMode copy_mode, size_t size, void *data) {
  if (mem_type != CEED_MEM_HOST) return CeedError(ctx->ceed, CEED_ERROR_UNSUPPORTED, "contexts are read from host memory at apply time");
  if (ctx->own) free(ctx->data);
  if (copy_mode == CEED_COPY_VALUES) {
    ctx->data = malloc(size);
    memcpy(ctx->data, data, size);
    ctx->own = 1;
  } else {
    ctx->data = data;
    ctx->own  = copy_mode == CEED_OWN_POINTER;
  }
  ctx->size = size;
  return CEED_ERROR_SUCCESS;
}
int CeedQFunctionContextGetData(CeedQFunctionContext ctx, CeedMemType mem_type, void *data) {
  if (mem_type != CEED_MEM_HOST) return CeedError(ctx->ceed, CEED_ERROR_UNSUPPORTED, "context data lives in host memory");
  *(void **)data = ctx->data;
  return CEED_ERROR_SUCCESS;
}
int CeedQFunctionContextGetDataRead(CeedQFunctionContext ctx, CeedMemType mem_type, void *data) { return CeedQFunctionContextGetData(ctx, mem_type, data); }
int CeedQFunctionContextRestoreData(CeedQFunctionContext ctx, void *data) {
  (void)ctx;
  *(void **)data = NULL;
  return CEED_ERROR_SUCCESS;
}
int CeedQFunctionContextRestoreDataRead(CeedQFunctionContext ctx, void *data) { return CeedQFunctionContextRestoreData(ctx, data); }
int CeedQFunctionContextSetDataDestroy(CeedQFunctionContext ctx, CeedMemType f_mem_type, CeedQFunctionContextDataDestroyUser f) {
  (void)f_mem_type;
  ctx->destroy = f;
  return CEED_ERROR_SUCCESS;
}
int CeedQFunctionContextRegisterDouble(CeedQFunctionContext ctx, const char *field_name, size_t field_offset, size_t num_values,
                                       const char *field_description) {
  (void)field_description;
  for (int i = 0; i < ctx->nlabels; i++)
    if (!strcmp(ctx->labels[i].name, field_name)) return CeedError(ctx->ceed, CEED_ERROR_MINOR, "context field '%s' already registered", field_name);
  if (ctx->nlabels >= MAX_LABELS) return CeedError(ctx->ceed, CEED_ERROR_UNSUPPORTED, "too many context fields");
  if (ctx->size && field_offset + num_values * sizeof(double) > ctx->size)
    return CeedError(ctx->ceed, CEED_ERROR_DIMENSION, "context field '%s' exceeds the context size", field_name);
  CtxLabel *l = &ctx->labels[ctx->nlabels++];
  snprintf(l->name, sizeof l->name, "%s", field_name);
  l->offset     = field_offset;
  l->num_values = num_values;
  l->type       = CEED_CONTEXT_FIELD_DOUBLE;
  return CEED_ERROR_SUCCESS;
}
int CeedQFunctionContextGetContextSize(CeedQFunctionContext ctx, size_t *ctx_size) {
  *ctx_size = ctx->size;
  return CEED_ERROR_SUCCESS;
}
int CeedQFunctionContextReference(CeedQFunctionContext ctx) {
  ctx->ref++;
  return CEED_ERROR_SUCCESS;
}
int CeedQFunctionContextDestroy(CeedQFunctionContext *ctx) {
  CeedQFunctionContext c = *ctx;
  if (!c) return CEED_ERROR_SUCCESS;
  if (--c->ref > 0) {
    *ctx = NULL;
    return CEED_ERROR_SUCCESS;
  }
  if (c->destroy) c->destroy(c->data);
  else if (c->own) free(c->data);
  Ceed ceed = c->ceed;
  free(c);
  *ctx = NULL;
  return CeedDestroy(&ceed);
}

/* ------------------------------------------------------------------------------------------------------------------ */
/* CeedQFunction                                                                                                      */

int CeedQFunctionCreateInterior(Ceed ceed, CeedInt vec_length, CeedQFunctionUser f, const char *source, CeedQFunction *qf) {
  if (!source) return CeedError(ceed, CEED_ERROR_INCOMPLETE, "QFunction source location is required");
  CeedQFunction q = (CeedQFunction)calloc(1, sizeof(*q));
  q->ceed         = ceed;
  ceed->ref++;
  q->ref     = 1;
  q->vlength = vec_length;
  q->f       = f;
  snprintf(q->source, sizeof q->source, "%s", source);
  const char *colon = strrchr(source, ':');
  snprintf(q->kernel, sizeof q->kernel, "%s", colon ? colon + 1 : source);
  *qf = q;
  return CEED_ERROR_SUCCESS;
}
int CeedQFunctionReferenceCopy(CeedQFunction qf, CeedQFunction *qf_copy) {
  qf->ref++;
  CK(CeedQFunctionDestroy(qf_copy));
  *qf_copy = qf;
  return CEED_ERROR_SUCCESS;
}
static int qf_add(CeedQFunction qf, QFField *arr, int *n, const char *name, CeedInt size, CeedEvalMode emode) {
  if (*n >= MAX_FIELDS) return CeedError(qf->ceed, CEED_ERROR_UNSUPPORTED, "too many QFunction fields");
  QFField *f = &arr[(*n)++];
  snprintf(f->name, sizeof f->name, "%s", name);
  f->size  = size;
  f->emode = emode;
  return CEED_ERROR_SUCCESS;
}
int CeedQFunctionAddInput(CeedQFunction qf, const char *field_name, CeedInt size, CeedEvalMode eval_mode) {
  return qf_add(qf, qf->in, &qf->nin, field_name, size, eval_mode);
}
int CeedQFunctionAddOutput(CeedQFunction qf, const char *field_name, CeedInt size, CeedEvalMode eval_mode) {
  return qf_add(qf, qf->out, &qf->nout, field_name, size, eval_mode);
}
int CeedQFunctionSetContext(CeedQFunction qf, CeedQFunctionContext ctx) {
  if (ctx) ctx->ref++;
  CK(CeedQFunctionContextDestroy(&qf->ctx));
  qf->ctx = ctx;
  return CEED_ERROR_SUCCESS;
}
int CeedQFunctionGetContext(CeedQFunction qf, CeedQFunctionContext *ctx) {
  *ctx = qf->ctx;
  return CEED_ERROR_SUCCESS;
}
int CeedQFunctionSetUserFlopsEstimate(CeedQFunction qf, CeedSize flops) {
  qf->user_flops = flops;
  return CEED_ERROR_SUCCESS;
}
int CeedQFunctionGetKernelName(CeedQFunction qf, const char **kernel_name) {
  *kernel_name = qf->kernel;
  return CEED_ERROR_SUCCESS;
}
int CeedQFunctionDestroy(CeedQFunction *qf) {
  CeedQFunction q = *qf;
  if (!q || q == CEED_QFUNCTION_NONE) {
    *qf = NULL;
    return CEED_ERROR_SUCCESS;
  }
  if (--q->ref > 0) {
    *qf = NULL;
    return CEED_ERROR_SUCCESS;
  }
  CeedQFunctionContextDestroy(&q->ctx);
  Ceed ceed = q->ceed;
  free(q);
  *qf = NULL;
  return CeedDestroy(&ceed);
}

/* ------------------------------------------------------------------------------------------------------------------ */
/* CeedOperator: object model                                                                                         */

int CeedOperatorCreate(Ceed ceed, CeedQFunction qf, CeedQFunction dqf, CeedQFunction dqfT, CeedOperator *op) {
  (void)dqf, (void)dqfT;
  if (!qf || qf == CEED_QFUNCTION_NONE) return CeedError(ceed, CEED_ERROR_INCOMPLETE, "operator needs a QFunction");
  CeedOperator o = (CeedOperator)calloc(1, sizeof(*o));
  o->ceed        = ceed;
  ceed->ref++;
  o->ref = 1;
  qf->ref++;
  o->qf = qf;
  *op   = o;
  return CEED_ERROR_SUCCESS;
}
int CeedOperatorCreateComposite(Ceed ceed, CeedOperator *op) {
  CeedOperator o = (CeedOperator)calloc(1, sizeof(*o));
  o->ceed        = ceed;
  ceed->ref++;
  o->ref       = 1;
  o->composite = 1;
  *op          = o;
  return CEED_ERROR_SUCCESS;
}
int CeedCompositeOperatorCreate(Ceed ceed, CeedOperator *op) { return CeedOperatorCreateComposite(ceed, op); }
int CeedOperatorReferenceCopy(CeedOperator op, CeedOperator *op_copy) {
  op->ref++;
  CK(CeedOperatorDestroy(op_copy));
  *op_copy = op;
  return CEED_ERROR_SUCCESS;
}

int CeedOperatorSetField(CeedOperator op, const char *field_name, CeedElemRestriction rstr, CeedBasis basis, CeedVector vec) {
  if (op->composite) return CeedError(op->ceed, CEED_ERROR_INCOMPATIBLE, "cannot set a field on a composite operator");
  OpField *f = NULL;
  for (int i = 0; i < op->qf->nin && !f; i++)
    if (!strcmp(op->qf->in[i].name, field_name)) f = &op->in[i];
  for (int i = 0; i < op->qf->nout && !f; i++)
    if (!strcmp(op->qf->out[i].name, field_name)) f = &op->out[i];
  if (!f) return CeedError(op->ceed, CEED_ERROR_INCOMPLETE, "QFunction has no field named '%s'", field_name);
  if (rstr && rstr != CEED_ELEMRESTRICTION_NONE) rstr->ref++;
  if (basis && basis != CEED_BASIS_NONE) basis->ref++;
  if (vec && vec != CEED_VECTOR_ACTIVE && vec != CEED_VECTOR_NONE) vec->ref++;
  if (f->set) {
    CeedElemRestrictionDestroy(&f->r);
    CeedBasisDestroy(&f->b);
    CeedVectorDestroy(&f->v);
  }
  f->r   = rstr;
  f->b   = basis;
  f->v   = vec;
  f->set = 1;
  /* re-plan on next apply, with kernels built from the new fields */
  op->plan = PLAN_NONE;
  if (op->eop) {
    ceed_unregister_op(op->ceed, op->eop);
    hb_elemop_destroy(op->eop);
    op->eop            = NULL;
    op->idl_coords_set = 0;
  }
  hb_faceop_destroy(op->fop);
  op->fop = NULL;
  /* work buffers sized by the old fields */
  cudaFree(op->d_zero);
  cudaFree(op->d_tmp_rhs);
  cudaFree(op->d_tmp_in32);
  cudaFree(op->d_tmp_out32);
  cudaFree(op->d_tmp_e);
  cudaFree(op->d_tmp_pb32);
  cudaFree(op->d_tmp_e2);
  cudaFree(op->d_node_w);
  op->d_node_w = NULL;
  op->d_tmp_pb32 = NULL;
  op->d_zero = op->d_tmp_rhs = op->d_tmp_e = op->d_tmp_e2 = NULL;
  op->d_tmp_in32 = op->d_tmp_out32 = NULL;
  return CEED_ERROR_SUCCESS;
}

int CeedOperatorCompositeAddSub(CeedOperator composite_op, CeedOperator sub_op) {
  if (!composite_op->composite) return CeedError(composite_op->ceed, CEED_ERROR_MINOR, "not a composite operator");
  if (composite_op->nsub >= MAX_SUBS) return CeedError(composite_op->ceed, CEED_ERROR_UNSUPPORTED, "too many sub-operators");
  sub_op->ref++;
  composite_op->subs[composite_op->nsub++] = sub_op;
  return CEED_ERROR_SUCCESS;
}
int CeedCompositeOperatorAddSub(CeedOperator composite_op, CeedOperator sub_op) { return CeedOperatorCompositeAddSub(composite_op, sub_op); }
int CeedOperatorCompositeGetNumSub(CeedOperator op, CeedInt *num_suboperators) {
  *num_suboperators = op->nsub;
  return CEED_ERROR_SUCCESS;
}
int CeedOperatorCompositeGetSubList(CeedOperator op, CeedOperator **sub_operators) {
  *sub_operators = op->subs;
  return CEED_ERROR_SUCCESS;
}
int CeedOperatorSetName(CeedOperator op, const char *name) {
  snprintf(op->name, sizeof op->name, "%s", name);
  return CEED_ERROR_SUCCESS;
}

static int op_check_fields(CeedOperator op) {
  for (int i = 0; i < op->qf->nin; i++)
    if (!op->in[i].set) return CeedError(op->ceed, CEED_ERROR_INCOMPLETE, "operator field '%s' not set", op->qf->in[i].name);
  for (int i = 0; i < op->qf->nout; i++)
    if (!op->out[i].set) return CeedError(op->ceed, CEED_ERROR_INCOMPLETE, "operator field '%s' not set", op->qf->out[i].name);
  return CEED_ERROR_SUCCESS;
}
int CeedOperatorCheckReady(CeedOperator op) {
  if (op->composite) {
    for (int i = 0; i < op->nsub; i++) CK(CeedOperatorCheckReady(op->subs[i]));
    return CEED_ERROR_SUCCESS;
  }
  return op_check_fields(op);
}

static CeedElemRestriction op_active_rstr(CeedOperator op, int output) {
  const int n = output ? op->qf->nout : op->qf->nin;
  for (int i = 0; i < n; i++) {
    OpField *f = output ? &op->out[i] : &op->in[i];
    if (f->set && f->v == CEED_VECTOR_ACTIVE) return f->r;
  }
  return NULL;
}
int CeedOperatorGetActiveVectorLengths(CeedOperator op, CeedSize *input_size, CeedSize *output_size) {
  CeedOperator o = op->composite ? (op->nsub ? op->subs[0] : NULL) : op;
  if (!o) return CeedError(op->ceed, CEED_ERROR_INCOMPLETE, "empty composite operator");
  CeedElemRestriction ri = op_active_rstr(o, 0), ro = op_active_rstr(o, 1);
  if (input_size) *input_size = ri ? ri->l_size : -1;
  if (output_size) *output_size = ro ? ro->l_size : -1;
  return CEED_ERROR_SUCCESS;
}

/* context labels: every QFunction context of op (or of its sub-operators) that registered field_name */
static void label_collect(CeedOperator op, const char *name, CeedContextFieldLabel lab) {
  if (op->composite) {
    for (int i = 0; i < op->nsub; i++) label_collect(op->subs[i], name, lab);
    return;
  }
  CeedQFunctionContext ctx = op->qf->ctx;
  if (!ctx) return;
  for (int k = 0; k < lab->n; k++)
    if (lab->ent[k].ctx == ctx) return;
  for (int i = 0; i < ctx->nlabels; i++)
    if (!strcmp(ctx->labels[i].name, name) && lab->n < MAX_SUBS) {
      lab->ent[lab->n].ctx        = ctx;
      lab->ent[lab->n].offset     = ctx->labels[i].offset;
      lab->ent[lab->n].num_values = ctx->labels[i].num_values;
      lab->n++;
    }
}

/* labels are owned by a small global pool so callers never free them (libCEED ties them to the operator) */
#define LABEL_POOL 256
static struct CeedContextFieldLabel_private label_pool[LABEL_POOL];
static int                                  label_pool_n;

int CeedOperatorGetContextFieldLabel(CeedOperator op, const char *field_name, CeedContextFieldLabel *field_label) {
  struct CeedContextFieldLabel_private tmp;
  memset(&tmp, 0, sizeof tmp);
  label_collect(op, field_name, &tmp);
  if (!tmp.n) {
    *field_label = NULL;
    return CEED_ERROR_SUCCESS;
  }
  snprintf(tmp.name, sizeof tmp.name, "%s", field_name);
  for (int i = 0; i < label_pool_n; i++)
    if (!memcmp(&label_pool[i], &tmp, sizeof tmp)) {
      *field_label = &label_pool[i];
      return CEED_ERROR_SUCCESS;
    }
  if (label_pool_n >= LABEL_POOL) return CeedError(op->ceed, CEED_ERROR_UNSUPPORTED, "too many context labels");
  label_pool[label_pool_n] = tmp;
  *field_label             = &label_pool[label_pool_n++];
  return CEED_ERROR_SUCCESS;
}

int CeedOperatorSetContextDouble(CeedOperator op, CeedContextFieldLabel lab, double *values) {
  if (!lab) return CeedError(op->ceed, CEED_ERROR_UNSUPPORTED, "invalid context field label");
  for (int k = 0; k < lab->n; k++) {
    CeedQFunctionContext ctx = lab->ent[k].ctx;
    memcpy((char *)ctx->data + lab->ent[k].offset, values, sizeof(double) * lab->ent[k].num_values);
  }
  return CEED_ERROR_SUCCESS;
}
int CeedOperatorGetContextDoubleRead(CeedOperator op, CeedContextFieldLabel lab, size_t *num_values, const double **values) {
  if (!lab || !lab->n) return CeedError(op->ceed, CEED_ERROR_UNSUPPORTED, "invalid context field label");
  *num_values = lab->ent[0].num_values;
  *values     = (const double *)((const char *)lab->ent[0].ctx->data + lab->ent[0].offset);
  return CEED_ERROR_SUCCESS;
}
int CeedOperatorRestoreContextDoubleRead(CeedOperator op, CeedContextFieldLabel lab, const double **values) {
  (void)op, (void)lab;
  *values = NULL;
  return CEED_ERROR_SUCCESS;
}

/* ------------------------------------------------------------------------------------------------------------------ */
/* CeedOperator: backend plans                                                                                        */

static int is_tensor3(CeedBasis b, int ncomp) { return b && b != CEED_BASIS_NONE && b->tensor && b->dim == 3 && b->num_comp == ncomp; }
static int is_tensor2(CeedBasis b, int ncomp) { return b && b != CEED_BASIS_NONE && b->tensor && b->dim == 2 && b->num_comp == ncomp; }

static int plan_fail(CeedOperator op, const char *why) {
  return CeedError(op->ceed, CEED_ERROR_UNSUPPORTED, "operator '%s' (QFunction %s) has no B200 kernel: %s", op->name, op->qf->kernel, why);
}

/* element-level restriction + basis pair of the Newtonian state fields */
static int plan_elemop(CeedOperator op, CeedElemRestriction r, CeedBasis b) {
  if (!r || r == CEED_ELEMRESTRICTION_NONE || r->strided) return plan_fail(op, "state field needs an offset restriction");
  if (r->num_comp != 5 || r->comp_stride != 1) return plan_fail(op, "state restriction must be 5 node-interleaved components (comp_stride 1)");
  if (!is_tensor3(b, 5)) return plan_fail(op, "state basis must be a 3D tensor H1 basis with 5 components");
  if (r->elem_size != b->P1d * b->P1d * b->P1d) return plan_fail(op, "restriction element size does not match the basis");
  if (!op->eop) {
    HB_CK(op->ceed, hb_elemop_create(r->num_elem, b->P1d, b->Q1d, r->h_off, r->l_size, b->interp1d, b->grad1d, b->qref1d, b->qweight1d, &op->eop));
    ceed_register_op(op->ceed, op->eop);
  }
  return CEED_ERROR_SUCCESS;
}

static int check_qdata_rstr(CeedOperator op, CeedElemRestriction r, int ncomp, int Q3, const char *what) {
  if (!r || r == CEED_ELEMRESTRICTION_NONE || !r->strided || r->num_comp != ncomp || r->elem_size != Q3)
    return CeedError(op->ceed, CEED_ERROR_UNSUPPORTED, "%s must use a strided restriction with %d components at %d points", what, ncomp, Q3);
  if (r->strides[0] != 1 || r->strides[1] != Q3 || r->strides[2] != Q3 * ncomp)
    return CeedError(op->ceed, CEED_ERROR_UNSUPPORTED, "%s must use the backend [elem][comp][point] layout (CEED_STRIDES_BACKEND)", what);
  return CEED_ERROR_SUCCESS;
}

/* every vector a planned operator touches must be at least as long as its restriction says (device safety) */
static int need_len(CeedOperator op, CeedVector v, CeedSize n, const char *what) {
  if (!v || v == CEED_VECTOR_ACTIVE || v == CEED_VECTOR_NONE || v->length < n)
    return CeedError(op->ceed, CEED_ERROR_DIMENSION, "operator '%s': %s vector missing or shorter than %td", op->name, what, n);
  return CEED_ERROR_SUCCESS;
}

/* gather the coordinate field of an input (restriction with 3 comps, basis of P nodes per direction, elem_size nodes
 * per element) into an E-vector [E][3][elem_size] */
static int gather_coords_n(CeedOperator op, OpField *fx, CeedVector xvec, int P, int elem_size, double **d_xe) {
  CeedElemRestriction r = fx->r;
  if (!r || r == CEED_ELEMRESTRICTION_NONE || r->num_comp != 3 || r->elem_size != elem_size || !fx->b || fx->b == CEED_BASIS_NONE ||
      fx->b->P1d != P)
    return CeedError(op->ceed, CEED_ERROR_UNSUPPORTED, "coordinate field must be a 3-component field with %d nodes per direction", P);
  CK(need_len(op, xvec, r->l_size, "coordinate"));
  CK(rstr_upload(r));
  const size_t nb = sizeof(double) * 3 * elem_size * (size_t)r->num_elem;
  if (!*d_xe) CUDA_CK(op->ceed, cudaMalloc((void **)d_xe, nb));
  const double *x;
  CK(vec_dev_read(xvec, &x));
  HB_CK(op->ceed, hb_restrict_apply(r->num_elem, elem_size, 3, r->comp_stride, r->strided ? NULL : r->d_off, r->strided ? r->d_strides : NULL, x,
                                    *d_xe, op->ceed->stream));
  return CEED_ERROR_SUCCESS;
}

/* the trilinear (P=2) volume coordinate field: E-vector [E][3][8] */
static int gather_coords(CeedOperator op, OpField *fx, CeedVector xvec, double **d_xe) { return gather_coords_n(op, fx, xvec, 2, 8, d_xe); }

/* The free-stream boundary sub-operators HONEE adds to its composites (HoneeBCCreateIFunctionQF / HoneeBCCreateIJacobianQF
 * and HoneeBCAddIFunctionOp / HoneeBCAddIJacobianOp, src/boundary_condition.c:276-470; QFunctions of
 * qfunctions/bc_freestream.h:54-138).  Inputs "q"/"dq" (INTERP), "Grad_q"/"Grad_dq" (GRAD, unused by the flux),
 * "surface qdata" (NONE, 10), "x" (INTERP, unused); IFunction outputs "v" (INTERP) and, for implicit runs, "surface
 * jacobian data" (NONE, 5); the IJacobian reads that data as its fifth input.  Returns the flux type through the name. */
/* "Freestream[_Jacobian]_{Conserv,Prim,Entropy}_{HLL,HLLC}" (qfunctions/bc_freestream.h:54-76, 116-138) */
static int freestream_kernel(const char *k, int *jacobian, int *flux_type, int *state_var) {
  static const char *sv_names[3] = {"Conserv", "Prim", "Entropy"};
  for (int jac = 0; jac < 2; jac++)
    for (int sv = 0; sv < 3; sv++)
      for (int flux = 0; flux < 2; flux++) {
        char name[64];
        snprintf(name, sizeof name, "Freestream_%s%s_%s", jac ? "Jacobian_" : "", sv_names[sv], flux ? "HLLC" : "HLL");
        if (!strcmp(k, name)) {
          *jacobian  = jac;
          *flux_type = flux;
          *state_var = sv;
          return 1;
        }
      }
  return 0;
}

static int plan_freestream(CeedOperator op, int jacobian, int flux_type, int state_var) {
  CeedQFunction qf = op->qf;
  const int     nin = jacobian ? 5 : 4, nout = jacobian ? 1 : (qf->nout == 2 ? 2 : 1);
  if (qf->nin != nin || qf->nout != nout || qf->in[0].emode != CEED_EVAL_INTERP || qf->in[0].size != 5 || qf->in[1].emode != CEED_EVAL_GRAD ||
      qf->in[2].emode != CEED_EVAL_NONE || qf->in[2].size != 10 || qf->in[3].emode != CEED_EVAL_INTERP || qf->out[0].emode != CEED_EVAL_INTERP ||
      qf->out[0].size != 5 || (jacobian && (qf->in[4].emode != CEED_EVAL_NONE || qf->in[4].size != 5)) ||
      (nout == 2 && (qf->out[1].emode != CEED_EVAL_NONE || qf->out[1].size != 5)))
    return plan_fail(op, "unexpected free-stream field layout (src/boundary_condition.c:276-364)");
  if (op->in[0].v != CEED_VECTOR_ACTIVE || op->in[1].v != CEED_VECTOR_ACTIVE || op->out[0].v != CEED_VECTOR_ACTIVE)
    return plan_fail(op, "the state and test fields must be active");
  CeedElemRestriction r = op->in[0].r;
  CeedBasis           b = op->in[0].b;
  if (op->in[1].r != r || op->out[0].r != r || op->in[1].b != b || op->out[0].b != b) return plan_fail(op, "state fields must share one face restriction and basis");
  if (!r || r == CEED_ELEMRESTRICTION_NONE || r->strided || r->num_comp != 5 || r->comp_stride != 1)
    return plan_fail(op, "face restriction must be 5 node-interleaved components (comp_stride 1) with offsets");
  if (!is_tensor2(b, 5) || r->elem_size != b->P1d * b->P1d) return plan_fail(op, "face basis must be a 2D tensor H1 basis with 5 components");
  if (!qf->ctx || qf->ctx->size != sizeof(HbFreestreamContext)) return plan_fail(op, "context must be the 264-byte FreestreamContext_");
  if (((const HbFreestreamContext *)qf->ctx->data)->newt.state_var != state_var)
    return plan_fail(op, "the free-stream context's state_var differs from the QFunction's");
  const int Q2 = b->Q1d * b->Q1d;
  CK(check_qdata_rstr(op, op->in[2].r, 10, Q2, "surface qdata"));
  if (jacobian) CK(check_qdata_rstr(op, op->in[4].r, 5, Q2, "surface jacobian data"));
  if (nout == 2) CK(check_qdata_rstr(op, op->out[1].r, 5, Q2, "surface jacobian data"));
  if (!op->fop) {
    int rc = hb_faceop_create(r->num_elem, b->P1d, b->Q1d, r->h_off, r->l_size, b->interp1d, b->grad1d, b->qweight1d, &op->fop);
    if (rc) return CeedError(op->ceed, CEED_ERROR_BACKEND, "face operator creation failed (%d): offsets outside the L-vector or sizes too large", rc);
  }
  op->flux_type = flux_type;
  op->plan      = jacobian ? PLAN_FREESTREAM_JAC : PLAN_FREESTREAM;
  return CEED_ERROR_SUCCESS;
}


/* Initial-condition operator: the coordinates' restriction (3 components, trilinear) with the projection basis onto the
 * solution nodes, the IC QFunction's context, and the output through the solution's node restriction. */
static int plan_ics(CeedOperator op, int kind, int sv) {
  CeedQFunction qf = op->qf;
  if (qf->nin > 2) return plan_fail(op, "initial conditions from the wall distance (ics_use_wall_distance) are not supported");
  if (qf->nin != 2 || qf->nout != 1 || qf->in[0].emode != CEED_EVAL_INTERP || qf->in[0].size != 3 || qf->in[1].emode != CEED_EVAL_GRAD ||
      qf->out[0].emode != CEED_EVAL_NONE || qf->out[0].size != 5)
    return plan_fail(op, "unexpected initial-condition field layout (src/setuplibceed.c:153-166)");
  if (op->in[0].v != CEED_VECTOR_ACTIVE || op->out[0].v != CEED_VECTOR_ACTIVE) return plan_fail(op, "the coordinates and q0 must be active");
  CeedBasis bx = op->in[0].b;
  if (!is_tensor3(bx, 3) || bx->P1d != 2 || op->in[1].b != bx || op->in[1].r != op->in[0].r)
    return plan_fail(op, "x and dx must share the trilinear coordinate restriction and its projection basis");
  CeedElemRestriction rq = op->out[0].r;
  if (!rq || rq == CEED_ELEMRESTRICTION_NONE || rq->strided || rq->num_comp != 5 || rq->elem_size != bx->Q1d * bx->Q1d * bx->Q1d ||
      rq->num_elem != op->in[0].r->num_elem)
    return plan_fail(op, "q0 must use a 5-component node restriction with one entry per projected node");
  static const size_t sizes[4] = {sizeof(HbSetupContext), sizeof(HbTaylorGreenContext), sizeof(HbChannelContext), sizeof(HbGaussianWaveContext)};
  if (!qf->ctx || qf->ctx->size != sizes[kind]) return plan_fail(op, "the initial-condition context has an unexpected size");
  if (kind == HB_IC_TAYLOR_GREEN) sv = ((const HbTaylorGreenContext *)qf->ctx->data)->newt_ctx.state_var;
  if (kind == HB_IC_CHANNEL) sv = ((const HbChannelContext *)qf->ctx->data)->newt_ctx.state_var;
  op->ic_kind      = kind;
  op->ic_state_var = sv;
  op->plan         = PLAN_ICS;
  return CEED_ERROR_SUCCESS;
}

/* Monitor operators: the state (INTERP, and GRAD for the kinetic energy) and qdata -> per-point values through a strided
 * collocated restriction (CreateElemRestrColloc_CompMajor, src/monitor_totalkineticenergy.c:35-47). */
static int plan_monitor(CeedOperator op, int ke, int sv) {
  CeedQFunction qf = op->qf;
  const int     nin = ke ? 3 : 2, ncomp = ke ? 5 : 1;
  if (qf->nin != nin || qf->nout != 1 || qf->in[0].emode != CEED_EVAL_INTERP || qf->in[0].size != 5 ||
      (ke && qf->in[1].emode != CEED_EVAL_GRAD) || qf->in[nin - 1].emode != CEED_EVAL_NONE || qf->in[nin - 1].size != 10 ||
      qf->out[0].emode != CEED_EVAL_NONE || qf->out[0].size != ncomp)
    return plan_fail(op, ke ? "unexpected kinetic-energy monitor field layout (src/monitor_totalkineticenergy.c:96-105)"
                            : "unexpected CFL monitor field layout (src/monitor_cfl.c:100-107)");
  if (op->in[0].v != CEED_VECTOR_ACTIVE || op->out[0].v != CEED_VECTOR_ACTIVE || (ke && op->in[1].v != CEED_VECTOR_ACTIVE))
    return plan_fail(op, "the state and the monitor values must be active");
  if (ke && (op->in[1].r != op->in[0].r || op->in[1].b != op->in[0].b)) return plan_fail(op, "q and Grad_q must share restriction and basis");
  if (!qf->ctx || qf->ctx->size != sizeof(HbNewtonianContext)) return plan_fail(op, "context must be the 184-byte NewtonianIdealGasContext_");
  if (((const HbNewtonianContext *)qf->ctx->data)->state_var != sv) return plan_fail(op, "the context's state_var differs from the QFunction's");
  CK(plan_elemop(op, op->in[0].r, op->in[0].b));
  const int           Q3 = op->eop->Q * op->eop->Q * op->eop->Q;
  CeedElemRestriction ro = op->out[0].r;
  CK(check_qdata_rstr(op, op->in[nin - 1].r, 10, Q3, "qdata"));
  if (!ro || ro == CEED_ELEMRESTRICTION_NONE || !ro->strided || ro->num_comp != ncomp || ro->elem_size != Q3 || ro->num_elem != op->eop->num_elem)
    return plan_fail(op, "monitor values must use a strided restriction with one entry per quadrature point and component");
  op->plan = ke ? PLAN_MON_KE : PLAN_MON_CFL;
  return CEED_ERROR_SUCCESS;
}

/* ---- nodal data-driven SGS pipeline (problems/sgs_dd_model.c:98-200, 508-560, 645-737) ----------------------------------
 * Every field of these operators lives on one node set: the state (5 fields), the velocity gradient (9), the anisotropy
 * tensor (7) and the SGS stress (6) each come from a clone of the solution DM (DMSetupByOrder_FEM with the solution's
 * degree, src/velocity_gradient_projection.c:12-36, src/grid_anisotropy_tensor.c:23-45, problems/sgs_dd_model.c:75-96), so
 * their restrictions number the nodes alike and differ only in the fields per node.  The plans check exactly that. */

/* a node restriction of nc node-interleaved fields: offsets node * nc (comp_stride 1) */
static int node_rstr(CeedElemRestriction r, int nc) {
  return r && r != CEED_ELEMRESTRICTION_NONE && !r->strided && r->num_comp == nc && r->comp_stride == 1 && r->l_size % nc == 0;
}

/* 1 when restrictions a (na fields) and b (nb fields) put every element node on the same node */
static int same_nodes(CeedElemRestriction a, int na, CeedElemRestriction b, int nb) {
  if (a->num_elem != b->num_elem || a->elem_size != b->elem_size || a->l_size / na != b->l_size / nb) return 0;
  const int64_t n = (int64_t)a->num_elem * a->elem_size;
  for (int64_t i = 0; i < n; i++)
    if (a->h_off[i] % na || b->h_off[i] % nb || a->h_off[i] / na != b->h_off[i] / nb) return 0;
  return 1;
}

/* the element operator of an nc-field node restriction and its basis: offsets rewritten as node * 5 */
static int plan_elemop_nc(CeedOperator op, CeedElemRestriction r, CeedBasis b, int nc, const char *what) {
  if (nc == 5) {
    if (!is_tensor3(b, 5)) return plan_fail(op, "state basis must be a 3D tensor H1 basis with 5 components");
    return plan_elemop(op, r, b);
  }
  char why[160];
  snprintf(why, sizeof why, "%s needs a %d-component node restriction (comp_stride 1) and a 3D tensor basis with %d components", what, nc, nc);
  if (!node_rstr(r, nc) || !is_tensor3(b, nc) || r->elem_size != b->P1d * b->P1d * b->P1d) return plan_fail(op, why);
  if (op->eop) return CEED_ERROR_SUCCESS;
  const int64_t n   = (int64_t)r->num_elem * r->elem_size;
  int32_t      *off = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n ? n : 1));
  if (!off) return CeedError(op->ceed, CEED_ERROR_BACKEND, "out of host memory");
  for (int64_t i = 0; i < n; i++) {
    if (r->h_off[i] % nc) {
      free(off);
      return plan_fail(op, why);
    }
    off[i] = (r->h_off[i] / nc) * 5;
  }
  const int rc = hb_elemop_create(r->num_elem, b->P1d, b->Q1d, off, (r->l_size / nc) * 5, b->interp1d, b->grad1d, b->qref1d, b->qweight1d, &op->eop);
  free(off);
  HB_CK(op->ceed, rc);
  ceed_register_op(op->ceed, op->eop);
  return CEED_ERROR_SUCCESS;
}

/* "Mass_<N>" (src/honee-mass.c:20-60): u (INTERP, N) and qdata (NONE) -> v (INTERP, N) */
static int plan_mass_n(CeedOperator op, int nc) {
  CeedQFunction qf = op->qf;
  if (qf->nin != 2 || qf->nout != 1 || qf->in[0].emode != CEED_EVAL_INTERP || qf->in[0].size != nc || qf->in[1].emode != CEED_EVAL_NONE ||
      qf->in[1].size != 10 || qf->out[0].emode != CEED_EVAL_INTERP || qf->out[0].size != nc)
    return plan_fail(op, "unexpected Mass_N field layout (src/honee-mass.c:58-60)");
  if (op->in[0].v != CEED_VECTOR_ACTIVE || op->out[0].v != CEED_VECTOR_ACTIVE) return plan_fail(op, "u and v must be active");
  if (op->in[0].r != op->out[0].r || op->in[0].b != op->out[0].b) return plan_fail(op, "u and v must share restriction and basis");
  CK(plan_elemop_nc(op, op->in[0].r, op->in[0].b, nc, "the mass operator"));
  CK(check_qdata_rstr(op, op->in[1].r, 10, op->eop->Q * op->eop->Q * op->eop->Q, "qdata"));
  op->nc   = nc;
  op->plan = PLAN_MASS_N;
  return CEED_ERROR_SUCCESS;
}

/* "VelocityGradientProjectionRHS_*": q (INTERP), Grad_q (GRAD), qdata (NONE), x (INTERP, unused by the point function)
 * -> velocity gradient (INTERP, 9) */
static int plan_velgrad(CeedOperator op, int sv) {
  CeedQFunction qf = op->qf;
  if (qf->nin != 4 || qf->nout != 1 || qf->in[0].emode != CEED_EVAL_INTERP || qf->in[0].size != 5 || qf->in[1].emode != CEED_EVAL_GRAD ||
      qf->in[2].emode != CEED_EVAL_NONE || qf->in[2].size != 10 || qf->in[3].emode != CEED_EVAL_INTERP || qf->out[0].emode != CEED_EVAL_INTERP ||
      qf->out[0].size != 9)
    return plan_fail(op, "unexpected velocity-gradient projection field layout (src/velocity_gradient_projection.c:86-97)");
  if (op->in[0].v != CEED_VECTOR_ACTIVE || op->in[1].v != CEED_VECTOR_ACTIVE || op->out[0].v != CEED_VECTOR_ACTIVE)
    return plan_fail(op, "q, Grad_q and the velocity gradient must be active");
  if (op->in[1].r != op->in[0].r || op->in[1].b != op->in[0].b) return plan_fail(op, "q and Grad_q must share restriction and basis");
  if (!qf->ctx || qf->ctx->size != sizeof(HbNewtonianContext)) return plan_fail(op, "context must be the 184-byte NewtonianIdealGasContext_");
  CK(plan_elemop(op, op->in[0].r, op->in[0].b));
  CeedElemRestriction ro = op->out[0].r;
  CeedBasis           bo = op->out[0].b;
  if (!node_rstr(ro, 9) || !is_tensor3(bo, 9) || bo->P1d != op->eop->P || bo->Q1d != op->eop->Q || !same_nodes(op->in[0].r, 5, ro, 9))
    return plan_fail(op, "the velocity gradient must use the solution's nodes with 9 fields and the solution's basis");
  CK(check_qdata_rstr(op, op->in[2].r, 10, op->eop->Q * op->eop->Q * op->eop->Q, "qdata"));
  op->state_var = sv;
  op->plan      = PLAN_VELGRAD;
  return CEED_ERROR_SUCCESS;
}

/* "AnisotropyTensorProjection": qdata (NONE) -> v (INTERP, 7) */
static int plan_aniso(CeedOperator op) {
  CeedQFunction qf = op->qf;
  if (qf->nin != 1 || qf->nout != 1 || qf->in[0].emode != CEED_EVAL_NONE || qf->in[0].size != 10 || qf->out[0].emode != CEED_EVAL_INTERP ||
      qf->out[0].size != 7)
    return plan_fail(op, "unexpected anisotropy-tensor projection field layout (src/grid_anisotropy_tensor.c:56-62)");
  if (op->out[0].v != CEED_VECTOR_ACTIVE) return plan_fail(op, "the projected tensor must be active");
  CK(plan_elemop_nc(op, op->out[0].r, op->out[0].b, 7, "the anisotropy tensor"));
  CK(check_qdata_rstr(op, op->in[0].r, 10, op->eop->Q * op->eop->Q * op->eop->Q, "qdata"));
  op->plan = PLAN_ANISO;
  return CEED_ERROR_SUCCESS;
}

/* "InverseMultiplicity": multiplicity (NONE, any fields, node restriction) -> inverse multiplicity (NONE, 1, strided) */
static int plan_inv_mult(CeedOperator op) {
  CeedQFunction qf = op->qf;
  if (qf->nin != 1 || qf->nout != 1 || qf->in[0].emode != CEED_EVAL_NONE || qf->out[0].emode != CEED_EVAL_NONE || qf->out[0].size != 1)
    return plan_fail(op, "unexpected inverse-multiplicity field layout (src/inverse_multiplicity.c:63-71)");
  if (op->in[0].v != CEED_VECTOR_ACTIVE || op->out[0].v != CEED_VECTOR_ACTIVE) return plan_fail(op, "multiplicity and its inverse must be active");
  CeedElemRestriction ri = op->in[0].r, ro = op->out[0].r;
  if (!ri || ri == CEED_ELEMRESTRICTION_NONE || ri->strided || ri->num_comp != qf->in[0].size)
    return plan_fail(op, "the multiplicity must come through a node restriction");
  CK(check_qdata_rstr(op, ro, 1, ri->elem_size, "the inverse multiplicity"));
  if (ro->num_elem != ri->num_elem) return plan_fail(op, "both restrictions must cover the same elements");
  op->plan = PLAN_INV_MULT;
  return CEED_ERROR_SUCCESS;
}

/* "ComputeSgsDDNodal_*": q (NONE, 5), x (INTERP, unused), gradient velocity (NONE, 9), anisotropy tensor (NONE, 7),
 * inverse multiplicity (NONE, 1, strided) -> km_sgs (NONE, 6); context SgsDDContext_ */
static int plan_sgs_nodal(CeedOperator op, int sv) {
  CeedQFunction qf = op->qf;
  static const int sizes[5] = {5, 3, 9, 7, 1};
  int              ok       = qf->nin == 5 && qf->nout == 1 && qf->out[0].emode == CEED_EVAL_NONE && qf->out[0].size == 6;
  for (int i = 0; ok && i < 5; i++) ok = qf->in[i].size == sizes[i] && qf->in[i].emode == (i == 1 ? CEED_EVAL_INTERP : CEED_EVAL_NONE);
  if (!ok) return plan_fail(op, "unexpected nodal SGS field layout (problems/sgs_dd_model.c:168-173)");
  if (op->in[2].v != CEED_VECTOR_ACTIVE || op->out[0].v != CEED_VECTOR_ACTIVE) return plan_fail(op, "the velocity gradient and km_sgs must be active");
  for (int i = 0; i < 5; i++)
    if (i != 2 && (!op->in[i].v || op->in[i].v == CEED_VECTOR_ACTIVE || op->in[i].v == CEED_VECTOR_NONE))
      return plan_fail(op, "q, x, the anisotropy tensor and the inverse multiplicity must be passive vectors");
  if (!qf->ctx || qf->ctx->size < sizeof(HbSgsDDContext)) return plan_fail(op, "context must be an SgsDDContext_ with its network data");
  const HbSgsDDContext *c = (const HbSgsDDContext *)qf->ctx->data;
  if (c->num_inputs != 6 || c->num_outputs != 6 || c->num_neurons != 20)
    return plan_fail(op, "the fused nodal closure is built for the 6-20-6 network of SgsDDSetup (problems/sgs_dd_model.c:665-671)");
  if (c->newt_ctx.state_var != sv) return plan_fail(op, "the context's state_var differs from the QFunction's");
  CeedElemRestriction rs = op->out[0].r;
  if (!node_rstr(rs, 6)) return plan_fail(op, "km_sgs must use a 6-field node restriction");
  if (!node_rstr(op->in[0].r, 5) || !same_nodes(rs, 6, op->in[0].r, 5) || !node_rstr(op->in[2].r, 9) || !same_nodes(rs, 6, op->in[2].r, 9) ||
      !node_rstr(op->in[3].r, 7) || !same_nodes(rs, 6, op->in[3].r, 7))
    return plan_fail(op, "q, the velocity gradient, the anisotropy tensor and km_sgs must number the nodes alike");
  CK(check_qdata_rstr(op, op->in[4].r, 1, rs->elem_size, "the inverse multiplicity"));
  CeedBasis bx = op->in[1].b;
  if (!is_tensor3(bx, 3) || bx->Q1d * bx->Q1d * bx->Q1d != rs->elem_size) return plan_fail(op, "x must be projected onto the solution nodes");
  /* the node weights are summed per element colour: an element operator on the stress nodes (its basis is not used) */
  if (!op->eop) {
    const int P = (int)(cbrt((double)rs->elem_size) + 0.5);
    if (P * P * P != rs->elem_size) return plan_fail(op, "km_sgs elements must be tensor-product node sets");
    double        I[HB_MAX_P * HB_MAX_P] = {0}, w[HB_MAX_P] = {0};
    const int64_t n                      = (int64_t)rs->num_elem * rs->elem_size;
    int32_t      *off                    = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n ? n : 1));
    if (!off) return CeedError(op->ceed, CEED_ERROR_BACKEND, "out of host memory");
    for (int64_t i = 0; i < n; i++) off[i] = (rs->h_off[i] / 6) * 5;
    for (int i = 0; i < P; i++) I[i * P + i] = 1;
    const int rc = hb_elemop_create(rs->num_elem, P, P, off, (rs->l_size / 6) * 5, I, I, NULL, w, &op->eop);
    free(off);
    HB_CK(op->ceed, rc);
    ceed_register_op(op->ceed, op->eop);
  }
  op->state_var = sv;
  op->plan      = PLAN_SGS_NODAL;
  return CEED_ERROR_SUCCESS;
}

/* "IFunction_NodalSgs_*": q (INTERP, 5), qdata (NONE), km_sgs (INTERP, 6) -> Grad_v (GRAD) */
static int plan_sgs_if(CeedOperator op, int sv) {
  CeedQFunction qf = op->qf;
  if (qf->nin != 3 || qf->nout != 1 || qf->in[0].emode != CEED_EVAL_INTERP || qf->in[0].size != 5 || qf->in[1].emode != CEED_EVAL_NONE ||
      qf->in[1].size != 10 || qf->in[2].emode != CEED_EVAL_INTERP || qf->in[2].size != 6 || qf->out[0].emode != CEED_EVAL_GRAD || qf->out[0].size != 15)
    return plan_fail(op, "unexpected nodal SGS residual field layout (problems/sgs_dd_model.c:533-545)");
  if (op->in[0].v != CEED_VECTOR_ACTIVE || op->out[0].v != CEED_VECTOR_ACTIVE) return plan_fail(op, "q and Grad_v must be active");
  if (!op->in[2].v || op->in[2].v == CEED_VECTOR_ACTIVE || op->in[2].v == CEED_VECTOR_NONE) return plan_fail(op, "km_sgs must be a passive vector");
  if (op->out[0].r != op->in[0].r || op->out[0].b != op->in[0].b) return plan_fail(op, "q and Grad_v must share restriction and basis");
  if (!qf->ctx || qf->ctx->size != sizeof(HbNewtonianContext)) return plan_fail(op, "context must be the 184-byte NewtonianIdealGasContext_");
  if (((const HbNewtonianContext *)qf->ctx->data)->state_var != sv) return plan_fail(op, "the context's state_var differs from the QFunction's");
  CK(plan_elemop(op, op->in[0].r, op->in[0].b));
  CeedElemRestriction rk = op->in[2].r;
  CeedBasis           bk = op->in[2].b;
  if (!node_rstr(rk, 6) || !is_tensor3(bk, 6) || bk->P1d != op->eop->P || bk->Q1d != op->eop->Q || !same_nodes(op->in[0].r, 5, rk, 6))
    return plan_fail(op, "km_sgs must use the solution's nodes with 6 fields and the solution's basis");
  CK(check_qdata_rstr(op, op->in[1].r, 10, op->eop->Q * op->eop->Q * op->eop->Q, "qdata"));
  op->state_var = sv;
  op->plan      = PLAN_SGS_IF;
  return CEED_ERROR_SUCCESS;
}

/* The state variable a Newtonian QFunction name selects (newtonian.h:259-269, 313-323): "<prefix>Conserv" 0, "<prefix>Prim" 1,
 * "<prefix>Entropy" 2, anything else -1. */
static int newtonian_state_var(const char *k, const char *prefix) {
  const size_t n = strlen(prefix);
  if (strncmp(k, prefix, n)) return -1;
  if (!strcmp(k + n, "Conserv")) return HB_STATEVAR_CONSERVATIVE;
  if (!strcmp(k + n, "Prim")) return HB_STATEVAR_PRIMITIVE;
  if (!strcmp(k + n, "Entropy")) return HB_STATEVAR_ENTROPY;
  return -1;
}

static int op_plan(CeedOperator op) {
  if (op->plan != PLAN_NONE) return CEED_ERROR_SUCCESS;
  CK(op_check_fields(op));
  CeedQFunction qf = op->qf;
  const char   *k  = qf->kernel;
  if (!strcmp(k, "Setup")) {
    /* inputs: "dx" (GRAD of coordinates), "weight" (WEIGHT); output: qdata (NONE, strided) */
    if (qf->nin != 2 || qf->nout != 1 || qf->in[0].emode != CEED_EVAL_GRAD || qf->in[1].emode != CEED_EVAL_WEIGHT ||
        qf->out[0].emode != CEED_EVAL_NONE || qf->out[0].size != 10)
      return plan_fail(op, "unexpected Setup field layout");
    if (op->in[0].v != CEED_VECTOR_ACTIVE) return plan_fail(op, "Setup expects the coordinates as the active input");
    CeedBasis bx = op->in[0].b;
    if (!is_tensor3(bx, 3) || bx->P1d != 2) return plan_fail(op, "Setup needs a trilinear coordinate basis");
    CK(check_qdata_rstr(op, op->out[0].r, 10, bx->Q1d * bx->Q1d * bx->Q1d, "qdata"));
    op->plan = PLAN_SETUP;
    return CEED_ERROR_SUCCESS;
  }
  const int sv_if = newtonian_state_var(k, "IFunction_Newtonian_"), sv_ij = newtonian_state_var(k, "IJacobian_Newtonian_");
  if (sv_if >= 0) {
    if (qf->nin < 5 || qf->nout != 3 || qf->in[0].emode != CEED_EVAL_INTERP || qf->in[1].emode != CEED_EVAL_GRAD ||
        qf->in[2].emode != CEED_EVAL_INTERP || qf->in[3].emode != CEED_EVAL_NONE || qf->out[0].emode != CEED_EVAL_INTERP ||
        qf->out[1].emode != CEED_EVAL_GRAD || qf->out[2].emode != CEED_EVAL_NONE)
      return plan_fail(op, "unexpected IFunction field layout (src/setuplibceed.c:216-230)");
    if (qf->nin > 5) return plan_fail(op, "projected divergence of the diffusive flux is not supported");
    if (op->in[0].v != CEED_VECTOR_ACTIVE || op->in[1].v != CEED_VECTOR_ACTIVE || op->out[0].v != CEED_VECTOR_ACTIVE ||
        op->out[1].v != CEED_VECTOR_ACTIVE)
      return plan_fail(op, "q/Grad_q and v/Grad_v must be active");
    if (op->in[0].r != op->in[1].r || op->in[0].r != op->in[2].r || op->in[0].r != op->out[0].r || op->in[0].r != op->out[1].r)
      return plan_fail(op, "state fields must share one restriction");
    if (op->in[0].b != op->in[1].b || op->in[0].b != op->in[2].b || op->in[0].b != op->out[0].b || op->in[0].b != op->out[1].b)
      return plan_fail(op, "state fields must share one basis");
    if (!qf->ctx || qf->ctx->size != sizeof(HbNewtonianContext)) return plan_fail(op, "context must be the 184-byte NewtonianIdealGasContext_");
    if (((const HbNewtonianContext *)qf->ctx->data)->state_var != sv_if) return plan_fail(op, "the context's state_var differs from the QFunction's");
    CK(plan_elemop(op, op->in[0].r, op->in[0].b));
    const int Q3 = op->eop->Q * op->eop->Q * op->eop->Q;
    CK(check_qdata_rstr(op, op->in[3].r, 10, Q3, "qdata"));
    const int njd = qf->out[2].size;
    if (njd != 14 && njd != 15) return plan_fail(op, "jac_data must have 14 or 15 components");
    CK(check_qdata_rstr(op, op->out[2].r, njd, Q3, "jac_data"));
    op->plan = PLAN_IFUNCTION;
    return CEED_ERROR_SUCCESS;
  }
  if (sv_ij >= 0) {
    if (qf->nin != 4 || qf->nout != 2 || qf->in[0].emode != CEED_EVAL_INTERP || qf->in[1].emode != CEED_EVAL_GRAD ||
        qf->in[2].emode != CEED_EVAL_NONE || qf->in[3].emode != CEED_EVAL_NONE || qf->out[0].emode != CEED_EVAL_INTERP ||
        qf->out[1].emode != CEED_EVAL_GRAD)
      return plan_fail(op, "unexpected IJacobian field layout (src/setuplibceed.c:252-266)");
    if (op->in[0].v != CEED_VECTOR_ACTIVE || op->in[1].v != CEED_VECTOR_ACTIVE || op->out[0].v != CEED_VECTOR_ACTIVE ||
        op->out[1].v != CEED_VECTOR_ACTIVE)
      return plan_fail(op, "dq/Grad_dq and v/Grad_v must be active");
    if (op->in[0].r != op->in[1].r || op->in[0].r != op->out[0].r || op->in[0].r != op->out[1].r) return plan_fail(op, "shared restriction expected");
    if (op->in[0].b != op->in[1].b || op->in[0].b != op->out[0].b || op->in[0].b != op->out[1].b) return plan_fail(op, "shared basis expected");
    if (!qf->ctx || qf->ctx->size != sizeof(HbNewtonianContext)) return plan_fail(op, "context must be the 184-byte NewtonianIdealGasContext_");
    if (((const HbNewtonianContext *)qf->ctx->data)->state_var != sv_ij) return plan_fail(op, "the context's state_var differs from the QFunction's");
    CK(plan_elemop(op, op->in[0].r, op->in[0].b));
    const int Q3 = op->eop->Q * op->eop->Q * op->eop->Q;
    CK(check_qdata_rstr(op, op->in[2].r, 10, Q3, "qdata"));
    const int njd = qf->in[3].size;
    if (njd != 14 && njd != 15) return plan_fail(op, "jac_data must have 14 or 15 components");
    CK(check_qdata_rstr(op, op->in[3].r, njd, Q3, "jac_data"));
    op->plan = PLAN_IJACOBIAN;
    return CEED_ERROR_SUCCESS;
  }
  if (!strcmp(k, "RHSFunction_Newtonian")) {
    /* explicit right-hand side (src/setuplibceed.c:179-205): q (INTERP), Grad_q (GRAD), qdata (NONE, 10), x (INTERP) ->
     * v (INTERP), Grad_v (GRAD) */
    if (qf->nin != 4 || qf->nout != 2 || qf->in[0].emode != CEED_EVAL_INTERP || qf->in[1].emode != CEED_EVAL_GRAD ||
        qf->in[2].emode != CEED_EVAL_NONE || qf->in[3].emode != CEED_EVAL_INTERP || qf->out[0].emode != CEED_EVAL_INTERP ||
        qf->out[1].emode != CEED_EVAL_GRAD)
      return plan_fail(op, qf->nin > 4 ? "projected divergence of the diffusive flux is not supported"
                                       : "unexpected RHSFunction field layout (src/setuplibceed.c:185-192)");
    if (op->in[0].v != CEED_VECTOR_ACTIVE || op->in[1].v != CEED_VECTOR_ACTIVE || op->out[0].v != CEED_VECTOR_ACTIVE ||
        op->out[1].v != CEED_VECTOR_ACTIVE)
      return plan_fail(op, "q/Grad_q and v/Grad_v must be active");
    if (op->in[0].r != op->in[1].r || op->in[0].r != op->out[0].r || op->in[0].r != op->out[1].r) return plan_fail(op, "shared restriction expected");
    if (op->in[0].b != op->in[1].b || op->in[0].b != op->out[0].b || op->in[0].b != op->out[1].b) return plan_fail(op, "shared basis expected");
    if (!qf->ctx || qf->ctx->size != sizeof(HbNewtonianContext)) return plan_fail(op, "context must be the 184-byte NewtonianIdealGasContext_");
    CK(plan_elemop(op, op->in[0].r, op->in[0].b));
    CK(check_qdata_rstr(op, op->in[2].r, 10, op->eop->Q * op->eop->Q * op->eop->Q, "qdata"));
    op->plan = PLAN_RHS;
    return CEED_ERROR_SUCCESS;
  }
  if (!strcmp(k, "Mass_5")) {
    /* HoneeMassQFunctionCreate (src/honee-mass.c:20-60) on the state fields: u (INTERP), qdata (NONE) -> v (INTERP) */
    if (qf->nin != 2 || qf->nout != 1 || qf->in[0].emode != CEED_EVAL_INTERP || qf->in[0].size != 5 || qf->in[1].emode != CEED_EVAL_NONE ||
        qf->out[0].emode != CEED_EVAL_INTERP || qf->out[0].size != 5)
      return plan_fail(op, "unexpected Mass_5 field layout (src/setuplibceed.c:40-45)");
    if (op->in[0].v != CEED_VECTOR_ACTIVE || op->out[0].v != CEED_VECTOR_ACTIVE) return plan_fail(op, "u and v must be active");
    if (op->in[0].r != op->out[0].r || op->in[0].b != op->out[0].b) return plan_fail(op, "u and v must share restriction and basis");
    CK(plan_elemop(op, op->in[0].r, op->in[0].b));
    CK(check_qdata_rstr(op, op->in[1].r, qf->in[1].size, op->eop->Q * op->eop->Q * op->eop->Q, "qdata"));
    if (qf->in[1].size != 10) return plan_fail(op, "mass qdata must be the 10-component volume qdata");
    op->plan = PLAN_MASS;
    return CEED_ERROR_SUCCESS;
  }
  if (!strcmp(k, "MassFunction_Newtonian_Conserv")) {
    /* CreateKSPMassOperator_NewtonianStabilized (problems/newtonian.c:212-265): q_dot (active, INTERP), q (passive, INTERP),
     * qdata (NONE) -> v (INTERP), Grad_v (GRAD) */
    if (qf->nin != 3 || qf->nout != 2 || qf->in[0].emode != CEED_EVAL_INTERP || qf->in[1].emode != CEED_EVAL_INTERP ||
        qf->in[2].emode != CEED_EVAL_NONE || qf->in[2].size != 10 || qf->out[0].emode != CEED_EVAL_INTERP || qf->out[1].emode != CEED_EVAL_GRAD)
      return plan_fail(op, "unexpected stabilized-mass field layout (problems/newtonian.c:244-256)");
    if (op->in[0].v != CEED_VECTOR_ACTIVE || op->out[0].v != CEED_VECTOR_ACTIVE || op->out[1].v != CEED_VECTOR_ACTIVE)
      return plan_fail(op, "q_dot, v and Grad_v must be active");
    if (!op->in[1].v || op->in[1].v == CEED_VECTOR_ACTIVE || op->in[1].v == CEED_VECTOR_NONE) return plan_fail(op, "the state q must be a passive vector");
    if (op->in[0].r != op->in[1].r || op->in[0].r != op->out[0].r || op->in[0].r != op->out[1].r) return plan_fail(op, "shared restriction expected");
    if (op->in[0].b != op->in[1].b || op->in[0].b != op->out[0].b || op->in[0].b != op->out[1].b) return plan_fail(op, "shared basis expected");
    if (!qf->ctx || qf->ctx->size != sizeof(HbNewtonianContext)) return plan_fail(op, "context must be the 184-byte NewtonianIdealGasContext_");
    CK(plan_elemop(op, op->in[0].r, op->in[0].b));
    CK(check_qdata_rstr(op, op->in[2].r, 10, op->eop->Q * op->eop->Q * op->eop->Q, "qdata"));
    op->plan = PLAN_MASS_STAB;
    return CEED_ERROR_SUCCESS;
  }
  if (!strcmp(k, "SetupBoundary")) {
    /* inputs "dx" (GRAD of the face coordinates), "weight" (WEIGHT); output "surface qdata" (NONE, 10, strided) --
     * QDataBoundaryGet, src/qdata.c:228-261 */
    if (qf->nin != 2 || qf->nout != 1 || qf->in[0].emode != CEED_EVAL_GRAD || qf->in[1].emode != CEED_EVAL_WEIGHT ||
        qf->out[0].emode != CEED_EVAL_NONE || qf->out[0].size != 10)
      return plan_fail(op, "unexpected SetupBoundary field layout (src/qdata.c:251-255)");
    if (op->in[0].v != CEED_VECTOR_ACTIVE) return plan_fail(op, "SetupBoundary expects the face coordinates as the active input");
    CeedBasis bx = op->in[0].b;
    if (!is_tensor2(bx, 3)) return plan_fail(op, "SetupBoundary needs a 2D tensor coordinate basis with 3 components");
    CK(check_qdata_rstr(op, op->out[0].r, 10, bx->Q1d * bx->Q1d, "surface qdata"));
    op->plan = PLAN_SETUP_SUR;
    return CEED_ERROR_SUCCESS;
  }
  {  /* initial conditions (src/setuplibceed.c:143-175): "x" (INTERP) and "dx" (GRAD) of the coordinates through the
      * projection basis onto the solution nodes -> "q0" (NONE) through the state restriction */
    int kind = -1, sv = -1;
    if ((sv = newtonian_state_var(k, "ICsNewtonianIG_")) >= 0) kind = HB_IC_NEWTONIAN;
    else if ((sv = newtonian_state_var(k, "IC_GaussianWave_")) >= 0) kind = HB_IC_GAUSSIAN_WAVE;
    else if (!strcmp(k, "ICsTaylorGreen")) kind = HB_IC_TAYLOR_GREEN;
    else if (!strcmp(k, "ICsChannel")) kind = HB_IC_CHANNEL;
    if (kind >= 0) return plan_ics(op, kind, sv);
  }
  {
    int nc = 0, used = 0;
    if (sscanf(k, "Mass_%d%n", &nc, &used) == 1 && k[used] == 0 && nc != 5 && nc >= 1 && nc <= 64) return plan_mass_n(op, nc);
  }
  {
    int sv;
    if ((sv = newtonian_state_var(k, "VelocityGradientProjectionRHS_")) >= 0) return plan_velgrad(op, sv);
    if ((sv = newtonian_state_var(k, "ComputeSgsDDNodal_")) >= 0) return plan_sgs_nodal(op, sv);
    if ((sv = newtonian_state_var(k, "IFunction_NodalSgs_")) >= 0) return plan_sgs_if(op, sv);
    if (!strcmp(k, "AnisotropyTensorProjection")) return plan_aniso(op);
    if (!strcmp(k, "InverseMultiplicity")) return plan_inv_mult(op);
  }
  const int sv_ke = newtonian_state_var(k, "MonitorTotalKineticEnergy_"), sv_cfl = newtonian_state_var(k, "MonitorCFL_3D_");
  if (sv_ke >= 0 || sv_cfl >= 0) return plan_monitor(op, sv_ke >= 0, sv_ke >= 0 ? sv_ke : sv_cfl);
  int jacobian, flux_type, fs_sv;
  if (freestream_kernel(k, &jacobian, &flux_type, &fs_sv)) return plan_freestream(op, jacobian, flux_type, fs_sv);
  return plan_fail(op, "no fused kernel for this QFunction (no CPU fallback on /gpu/b200)");
}

static int vec_f32_shadow(CeedVector v) {
  if (!v->d_f32) CUDA_CK(v->ceed, cudaMalloc((void **)&v->d_f32, sizeof(float) * (size_t)(v->length ? v->length : 1)));
  return CEED_ERROR_SUCCESS;
}

/* apply one non-composite operator, adding into out (out already holds what should be kept) */
/* An operator over zero elements (a partition that owns none, libCEED's CeedElemRestrictionCreate with num_elem 0)
 * contributes nothing: its apply, diagonal and point-block diagonal add zero, and no plan (no kernel) is built. */
static int op_empty(CeedOperator op) {
  if (op->composite) return 0;
  for (int i = 0; i < MAX_FIELDS; i++) {
    const CeedElemRestriction r = op->in[i].r;
    if (r && r != CEED_ELEMRESTRICTION_NONE) return r->num_elem == 0;
  }
  return 0;
}

static int op_apply_add_single(CeedOperator op, CeedVector in, CeedVector out) {
  if (op_empty(op)) return CEED_ERROR_SUCCESS;
  CK(op_plan(op));
  Ceed         ceed = op->ceed;
  cudaStream_t s    = ceed->stream;
  switch (op->plan) {
    case PLAN_SETUP: {
      CeedBasis bx = op->in[0].b;
      CK(need_len(op, in, op->in[0].r->l_size, "coordinate"));
      CK(need_len(op, out, op->out[0].r->l_size, "qdata"));
      CK(gather_coords(op, &op->in[0], in, &op->d_tmp_e));
      double *qd;
      CK(vec_dev_write(out, &qd, 1));
      /* Setup writes (not adds) qdata: libCEED's strided output of an EVAL_NONE field is overwritten per element */
      HB_CK(ceed, hb_setup_qdata(op->in[0].r->num_elem, bx->Q1d, bx->qref1d, bx->qweight1d, op->d_tmp_e, qd, s));
      return CEED_ERROR_SUCCESS;
    }
    case PLAN_SETUP_SUR: {
      CeedBasis bx = op->in[0].b;
      CK(need_len(op, out, op->out[0].r->l_size, "surface qdata"));
      CK(gather_coords_n(op, &op->in[0], in, bx->P1d, bx->P1d * bx->P1d, &op->d_tmp_e));
      double *qd;
      CK(vec_dev_write(out, &qd, 1));
      HB_CK(ceed, hb_face_setup_qdata_nodes(op->in[0].r->num_elem, bx->P1d, bx->Q1d, bx->interp1d, bx->grad1d, bx->qweight1d, op->d_tmp_e, qd, s));
      return CEED_ERROR_SUCCESS;
    }
    case PLAN_FREESTREAM: {
      /* FP64 in both precisions: the boundary is O(E^(2/3)) of the work; in the mixed run its jac data stays FP64 */
      const int64_t n = op->fop->l_size;
      CK(need_len(op, in, n, "input"));
      CK(need_len(op, out, n, "output"));
      CK(need_len(op, op->in[2].v, op->in[2].r->l_size, "surface qdata"));
      const double *q, *qd;
      double       *jd = NULL, *v;
      CK(vec_dev_read(in, &q));
      CK(vec_dev_read(op->in[2].v, &qd));
      if (op->qf->nout == 2) {
        CK(need_len(op, op->out[1].v, op->out[1].r->l_size, "surface jacobian data"));
        CK(vec_dev_write(op->out[1].v, &jd, 1));
      }
      CK(vec_dev_write(out, &v, 0));
      if (((const HbFreestreamContext *)op->qf->ctx->data)->newt.is_implicit) {
        HB_CK(ceed, hb_freestream_apply(op->fop, op->qf->ctx->data, op->flux_type, qd, q, jd, v, s));
      } else {
        /* explicit (RHS) form: the QFunction returns -wdetJb F (bc_freestream.h:45-48) */
        if (!op->d_tmp_rhs) CUDA_CK(ceed, cudaMalloc((void **)&op->d_tmp_rhs, sizeof(double) * (size_t)n));
        CUDA_CK(ceed, cudaMemsetAsync(op->d_tmp_rhs, 0, sizeof(double) * (size_t)n, s));
        HB_CK(ceed, hb_freestream_apply(op->fop, op->qf->ctx->data, op->flux_type, qd, q, NULL, op->d_tmp_rhs, s));
        HB_CK(ceed, hb_vec_axpy_f64(v, -1.0, op->d_tmp_rhs, n, s));
      }
      return CEED_ERROR_SUCCESS;
    }
    case PLAN_FREESTREAM_JAC: {
      const int64_t n = op->fop->l_size;
      CK(need_len(op, in, n, "input"));
      CK(need_len(op, out, n, "output"));
      CK(need_len(op, op->in[2].v, op->in[2].r->l_size, "surface qdata"));
      CK(need_len(op, op->in[4].v, op->in[4].r->l_size, "surface jacobian data"));
      const double *dq, *qd, *jd;
      double       *v;
      CK(vec_dev_read(in, &dq));
      CK(vec_dev_read(op->in[2].v, &qd));
      CK(vec_dev_read(op->in[4].v, &jd));
      CK(vec_dev_write(out, &v, 0));
      HB_CK(ceed, hb_freestream_jacobian_apply(op->fop, op->qf->ctx->data, op->flux_type, qd, jd, dq, v, s));
      return CEED_ERROR_SUCCESS;
    }
    case PLAN_RHS: {
      /* RHS(q) = -F(q, q_dot = 0): the IFunction kernel at zero rate, negated into the output */
      const HbNewtonianContext *ctx = (const HbNewtonianContext *)op->qf->ctx->data;
      const int64_t             n   = op->eop->l_size;
      CK(need_len(op, in, n, "input"));
      CK(need_len(op, out, n, "output"));
      CK(need_len(op, op->in[2].v, op->in[2].r->l_size, "qdata"));
      if (ctx->idl_enable && !op->idl_coords_set) {
        CeedVector xv = op->in[3].v;
        if (!xv || xv == CEED_VECTOR_ACTIVE || xv == CEED_VECTOR_NONE) return plan_fail(op, "IDL needs the coordinate field 'x'");
        CK(gather_coords(op, &op->in[3], xv, &op->eop->d_x_elem));
        op->idl_coords_set = 1;
      }
      if (!op->d_zero) {
        CUDA_CK(ceed, cudaMalloc((void **)&op->d_zero, sizeof(double) * (size_t)n));
        CUDA_CK(ceed, cudaMalloc((void **)&op->d_tmp_rhs, sizeof(double) * (size_t)n));
        CUDA_CK(ceed, cudaMemsetAsync(op->d_zero, 0, sizeof(double) * (size_t)n, s));
      }
      HbIFunctionIO io;
      memset(&io, 0, sizeof io);
      CK(vec_dev_read(in, &io.q));
      CK(vec_dev_read(op->in[2].v, &io.qdata));
      io.q_dot = op->d_zero;
      io.v     = op->d_tmp_rhs;
      io.add   = 0;
      HB_CK(ceed, hb_ifunction_apply(op->eop, ctx, &io, s));
      double *v;
      CK(vec_dev_write(out, &v, 0));
      HB_CK(ceed, hb_vec_axpy_f64(v, -1.0, op->d_tmp_rhs, n, s));
      return CEED_ERROR_SUCCESS;
    }
    case PLAN_MASS_STAB: {
      const int64_t n = op->eop->l_size;
      CK(need_len(op, in, n, "input"));
      CK(need_len(op, out, n, "output"));
      CK(need_len(op, op->in[1].v, n, "state"));
      CK(need_len(op, op->in[2].v, op->in[2].r->l_size, "qdata"));
      const double *u, *qs, *qd;
      double       *v;
      CK(vec_dev_read(in, &u));
      CK(vec_dev_read(op->in[1].v, &qs));
      CK(vec_dev_read(op->in[2].v, &qd));
      CK(vec_dev_write(out, &v, 0));
      HB_CK(ceed, hb_mass_stab_apply(op->eop, op->qf->ctx->data, qd, qs, u, v, 1, s));
      return CEED_ERROR_SUCCESS;
    }
    case PLAN_ICS: {
      CeedBasis           bx = op->in[0].b;
      CeedElemRestriction rq = op->out[0].r;
      CK(need_len(op, out, rq->l_size, "initial state"));
      CK(gather_coords(op, &op->in[0], in, &op->d_tmp_e));
      const size_t ne = (size_t)rq->num_elem * 5 * rq->elem_size;
      if (!op->d_tmp_e2) CUDA_CK(ceed, cudaMalloc((void **)&op->d_tmp_e2, sizeof(double) * (ne ? ne : 1)));
      HB_CK(ceed, hb_ics_apply(op->ic_kind, op->ic_state_var, op->qf->ctx->data, op->qf->ctx->size, rq->num_elem, bx->Q1d, bx->interp1d, op->d_tmp_e,
                               op->d_tmp_e2, s));
      CK(rstr_upload(rq));
      CK(rstr_build_transpose(rq));
      double *v;
      CK(vec_dev_write(out, &v, 0));
      HB_CK(ceed, hb_restrict_apply_t_csr(rq->l_size, rq->d_tptr, rq->d_teidx, op->d_tmp_e2, v, s));
      return CEED_ERROR_SUCCESS;
    }
    case PLAN_MON_KE:
    case PLAN_MON_CFL: {
      const int           ke = op->plan == PLAN_MON_KE, iq = ke ? 2 : 1;
      CeedElemRestriction ro = op->out[0].r;
      CK(need_len(op, in, op->eop->l_size, "state"));
      CK(need_len(op, out, ro->l_size, "monitor values"));
      CK(need_len(op, op->in[iq].v, op->in[iq].r->l_size, "qdata"));
      const size_t ne = (size_t)ro->num_elem * ro->num_comp * ro->elem_size;
      if (!op->d_tmp_e2) CUDA_CK(ceed, cudaMalloc((void **)&op->d_tmp_e2, sizeof(double) * (ne ? ne : 1)));
      const double *q, *qd;
      CK(vec_dev_read(in, &q));
      CK(vec_dev_read(op->in[iq].v, &qd));
      if (ke) HB_CK(ceed, hb_monitor_ke_points(op->eop, op->qf->ctx->data, q, qd, op->d_tmp_e2, s));
      else HB_CK(ceed, hb_monitor_cfl_points(op->eop, op->qf->ctx->data, q, qd, op->d_tmp_e2, s));
      CK(rstr_upload(ro));
      double *v;
      CK(vec_dev_write(out, &v, 0));
      HB_CK(ceed, hb_restrict_apply_t_strided(ro->num_elem, ro->elem_size, ro->num_comp, ro->d_strides, op->d_tmp_e2, v, s));
      return CEED_ERROR_SUCCESS;
    }
    case PLAN_MASS_N: {
      const int64_t n = op->in[0].r->l_size;
      CK(need_len(op, in, n, "input"));
      CK(need_len(op, out, n, "output"));
      CK(need_len(op, op->in[1].v, op->in[1].r->l_size, "qdata"));
      const double *u, *qd;
      double       *v;
      CK(vec_dev_read(in, &u));
      CK(vec_dev_read(op->in[1].v, &qd));
      CK(vec_dev_write(out, &v, 0));
      HB_CK(ceed, hb_mass_n_apply(op->eop, op->nc, qd, u, v, s));
      return CEED_ERROR_SUCCESS;
    }
    case PLAN_VELGRAD: {
      CK(need_len(op, in, op->eop->l_size, "state"));
      CK(need_len(op, out, op->out[0].r->l_size, "velocity gradient"));
      CK(need_len(op, op->in[2].v, op->in[2].r->l_size, "qdata"));
      const double *q, *qd;
      double       *v;
      CK(vec_dev_read(in, &q));
      CK(vec_dev_read(op->in[2].v, &qd));
      CK(vec_dev_write(out, &v, 0));
      HB_CK(ceed, hb_velocity_gradient_rhs(op->eop, op->qf->ctx->data, op->state_var, qd, q, v, s));
      return CEED_ERROR_SUCCESS;
    }
    case PLAN_ANISO: {
      CK(need_len(op, out, op->out[0].r->l_size, "anisotropy tensor"));
      CK(need_len(op, op->in[0].v, op->in[0].r->l_size, "qdata"));
      const double *qd;
      double       *v;
      CK(vec_dev_read(op->in[0].v, &qd));
      CK(vec_dev_write(out, &v, 0));
      HB_CK(ceed, hb_anisotropy_rhs(op->eop, qd, v, s));
      return CEED_ERROR_SUCCESS;
    }
    case PLAN_INV_MULT: {
      CeedElemRestriction ri = op->in[0].r, ro = op->out[0].r;
      CK(need_len(op, in, ri->l_size, "multiplicity"));
      CK(need_len(op, out, ro->l_size, "inverse multiplicity"));
      CK(rstr_upload(ri));
      CK(rstr_upload(ro));
      const size_t ne = (size_t)ro->num_elem * ro->elem_size;
      if (!op->d_tmp_e2) CUDA_CK(ceed, cudaMalloc((void **)&op->d_tmp_e2, sizeof(double) * (ne ? ne : 1)));
      const double *m;
      double       *v;
      CK(vec_dev_read(in, &m));
      CUDA_CK(ceed, cudaMemsetAsync(op->d_tmp_e2, 0, sizeof(double) * ne, s));
      HB_CK(ceed, hb_inverse_multiplicity((int64_t)ne, ri->d_off, m, op->d_tmp_e2, s));
      CK(vec_dev_write(out, &v, 0));
      HB_CK(ceed, hb_restrict_apply_t_strided(ro->num_elem, ro->elem_size, 1, ro->d_strides, op->d_tmp_e2, v, s));
      return CEED_ERROR_SUCCESS;
    }
    case PLAN_SGS_NODAL: {
      CeedElemRestriction rs = op->out[0].r;
      const int64_t       nodes = rs->l_size / 6;
      CK(need_len(op, in, op->in[2].r->l_size, "velocity gradient"));
      CK(need_len(op, out, rs->l_size, "km_sgs"));
      CK(need_len(op, op->in[0].v, op->in[0].r->l_size, "q"));
      CK(need_len(op, op->in[3].v, op->in[3].r->l_size, "anisotropy tensor"));
      CK(need_len(op, op->in[4].v, op->in[4].r->l_size, "inverse multiplicity"));
      if (!op->d_node_w) CUDA_CK(ceed, cudaMalloc((void **)&op->d_node_w, sizeof(double) * (size_t)(nodes ? nodes : 1)));
      const double *q, *G, *A, *im;
      double       *v;
      CK(vec_dev_read(op->in[0].v, &q));
      CK(vec_dev_read(in, &G));
      CK(vec_dev_read(op->in[3].v, &A));
      CK(vec_dev_read(op->in[4].v, &im));
      /* the inverse multiplicity arrives in the backend E-vector order [elem][node] (strided, one field) */
      CUDA_CK(ceed, cudaMemsetAsync(op->d_node_w, 0, sizeof(double) * (size_t)nodes, s));
      HB_CK(ceed, hb_node_weight_sum(op->eop, im, op->d_node_w, s));
      CK(vec_dev_write(out, &v, 0));
      HB_CK(ceed, hb_sgs_nodal_closure(nodes, op->qf->ctx->data, op->qf->ctx->size, op->state_var, q, G, A, op->d_node_w, v, s));
      return CEED_ERROR_SUCCESS;
    }
    case PLAN_SGS_IF: {
      CK(need_len(op, in, op->eop->l_size, "state"));
      CK(need_len(op, out, op->eop->l_size, "residual"));
      CK(need_len(op, op->in[1].v, op->in[1].r->l_size, "qdata"));
      CK(need_len(op, op->in[2].v, op->in[2].r->l_size, "km_sgs"));
      const double *q, *qd, *km;
      double       *v;
      CK(vec_dev_read(in, &q));
      CK(vec_dev_read(op->in[1].v, &qd));
      CK(vec_dev_read(op->in[2].v, &km));
      CK(vec_dev_write(out, &v, 0));
      HB_CK(ceed, hb_sgs_nodal_ifunction(op->eop, op->qf->ctx->data, op->state_var, qd, q, km, v, s));
      return CEED_ERROR_SUCCESS;
    }
    case PLAN_MASS: {
      const int64_t n = op->eop->l_size;
      CK(need_len(op, in, n, "input"));
      CK(need_len(op, out, n, "output"));
      CK(need_len(op, op->in[1].v, op->in[1].r->l_size, "qdata"));
      const double *u, *qd;
      double       *v;
      CK(vec_dev_read(in, &u));
      CK(vec_dev_read(op->in[1].v, &qd));
      CK(vec_dev_write(out, &v, 0));
      HB_CK(ceed, hb_mass_apply(op->eop, qd, u, v, 1, s));
      return CEED_ERROR_SUCCESS;
    }
    case PLAN_IFUNCTION: {
      const HbNewtonianContext *ctx = (const HbNewtonianContext *)op->qf->ctx->data;
      if ((ctx->idl_enable ? 15 : 14) != op->qf->out[2].size)
        return plan_fail(op, "jac_data must have 15 components with the IDL enabled and 14 without (problems/newtonian.c:756-757)");
      CK(need_len(op, in, op->eop->l_size, "input"));
      CK(need_len(op, out, op->eop->l_size, "output"));
      CK(need_len(op, op->in[2].v, op->eop->l_size, "q dot"));
      CK(need_len(op, op->in[3].v, op->in[3].r->l_size, "qdata"));
      CK(need_len(op, op->out[2].v, op->out[2].r->l_size, "jac_data"));
      if (ctx->idl_enable && !op->idl_coords_set) {
        CeedVector xv = op->in[4].v;
        if (!xv || xv == CEED_VECTOR_ACTIVE || xv == CEED_VECTOR_NONE) return plan_fail(op, "IDL needs the coordinate field 'x'");
        CK(gather_coords(op, &op->in[4], xv, &op->eop->d_x_elem));
        op->idl_coords_set = 1;
      }
      HbIFunctionIO io;
      memset(&io, 0, sizeof io);
      CK(vec_dev_read(in, &io.q));
      CK(vec_dev_read(op->in[2].v, &io.q_dot));
      CK(vec_dev_read(op->in[3].v, &io.qdata));
      CeedVector jd = op->out[2].v;
      if (ceed->mixed) {
        CK(vec_f32_shadow(jd));
        io.jac_data_f32 = jd->d_f32;
        jd->f32_valid   = 1;
        jd->f64_stale   = 1;
        jd->h_valid = jd->d_valid = 0;
      } else {
        double *jdd;
        CK(vec_dev_write(jd, &jdd, 1));
        io.jac_data = jdd;
      }
      double *v;
      CK(vec_dev_write(out, &v, 0));
      io.v   = v;
      io.add = 1;
      HB_CK(ceed, hb_ifunction_apply(op->eop, ctx, &io, s));
      return CEED_ERROR_SUCCESS;
    }
    case PLAN_IJACOBIAN: {
      const HbNewtonianContext *ctx = (const HbNewtonianContext *)op->qf->ctx->data;
      if ((ctx->idl_enable ? 15 : 14) != op->qf->in[3].size)
        return plan_fail(op, "jac_data must have 15 components with the IDL enabled and 14 without (problems/newtonian.c:756-757)");
      CK(need_len(op, in, op->eop->l_size, "input"));
      CK(need_len(op, out, op->eop->l_size, "output"));
      CK(need_len(op, op->in[2].v, op->in[2].r->l_size, "qdata"));
      CK(need_len(op, op->in[3].v, op->in[3].r->l_size, "jac_data"));
      const double             *qd;
      CK(vec_dev_read(op->in[2].v, &qd));
      CeedVector jd = op->in[3].v;
      if (ceed->mixed) {
        if (!jd->f32_valid) {
          const double *j64;
          CK(vec_dev_read(jd, &j64));
          CK(vec_f32_shadow(jd));
          HB_CK(ceed, hb_vec_f64_to_f32(j64, jd->d_f32, jd->length, 0, s));
          jd->f32_valid = 1;
        }
        const int64_t n = op->eop->l_size;
        if (!op->d_tmp_in32) {
          CUDA_CK(ceed, cudaMalloc((void **)&op->d_tmp_in32, sizeof(float) * (size_t)n));
          CUDA_CK(ceed, cudaMalloc((void **)&op->d_tmp_out32, sizeof(float) * (size_t)n));
        }
        const double *x;
        double       *y;
        CK(vec_dev_read(in, &x));
        CK(vec_dev_write(out, &y, 0));
        HB_CK(ceed, hb_vec_f64_to_f32(x, op->d_tmp_in32, n, 0, s));
        HB_CK(ceed, hb_ijacobian_apply_f32(op->eop, ctx, qd, jd->d_f32, op->d_tmp_in32, op->d_tmp_out32, 0, s));
        HB_CK(ceed, hb_vec_f32_to_f64(op->d_tmp_out32, y, n, 1, s));
      } else {
        const double *j64, *x;
        double       *y;
        CK(vec_dev_read(jd, &j64));
        CK(vec_dev_read(in, &x));
        CK(vec_dev_write(out, &y, 0));
        HB_CK(ceed, hb_ijacobian_apply_f64(op->eop, ctx, qd, j64, x, y, 1, s));
      }
      return CEED_ERROR_SUCCESS;
    }
  }
  return plan_fail(op, "unplanned operator");
}

static int op_apply_add(CeedOperator op, CeedVector in, CeedVector out) {
  if (op->composite) {
    for (int i = 0; i < op->nsub; i++) CK(op_apply_add_single(op->subs[i], in, out));
    return CEED_ERROR_SUCCESS;
  }
  return op_apply_add_single(op, in, out);
}

/* After an operator's kernels are enqueued, record on the compute stream that every vector it touched has been used up
 * to here: later copies into or out of those vectors wait for this point only, not for work enqueued after it. */
static int vec_mark_used(CeedVector v) {
  if (!v || v == CEED_VECTOR_ACTIVE || v == CEED_VECTOR_NONE || !v->d) return CEED_ERROR_SUCCESS;
  CK(vec_events(v));
  CUDA_CK(v->ceed, cudaEventRecord(v->ev_use, v->ceed->stream));
  v->use_known = 1;
  return CEED_ERROR_SUCCESS;
}
static int op_mark_used(CeedOperator op) {
  for (int i = 0; i < MAX_FIELDS; i++) {
    CK(vec_mark_used(op->in[i].v));
    CK(vec_mark_used(op->out[i].v));
  }
  for (int i = 0; i < op->nsub; i++) CK(op_mark_used(op->subs[i]));
  return CEED_ERROR_SUCCESS;
}
static int op_apply_marked(CeedOperator op, CeedVector in, CeedVector out) {
  CK(op_apply_add(op, in, out));
  CK(op_mark_used(op));
  CK(vec_mark_used(in));
  return vec_mark_used(out);
}

int CeedOperatorApply(CeedOperator op, CeedVector in, CeedVector out, CeedRequest *request) {
  (void)request;
  if (out && out != CEED_VECTOR_NONE) {
    /* Setup overwrites; everything else accumulates after zeroing */
    int only_setup = !op->composite && !op_empty(op) && (op_plan(op) == 0) && (op->plan == PLAN_SETUP || op->plan == PLAN_SETUP_SUR);
    if (!only_setup) CK(CeedVectorSetValue(out, 0.0));
  }
  return op_apply_marked(op, in, out);
}

int CeedOperatorApplyAdd(CeedOperator op, CeedVector in, CeedVector out, CeedRequest *request) {
  (void)request;
  return op_apply_marked(op, in, out);
}

static int op_diag_add_single(CeedOperator op, CeedVector assembled) {
  if (op_empty(op)) return CEED_ERROR_SUCCESS;
  CK(op_plan(op));
  if (op->plan == PLAN_FREESTREAM_JAC) {
    CK(need_len(op, assembled, op->fop->l_size, "diagonal"));
    CK(need_len(op, op->in[2].v, op->in[2].r->l_size, "surface qdata"));
    CK(need_len(op, op->in[4].v, op->in[4].r->l_size, "surface jacobian data"));
    const double *qd, *jd;
    double       *y;
    CK(vec_dev_read(op->in[2].v, &qd));
    CK(vec_dev_read(op->in[4].v, &jd));
    CK(vec_dev_write(assembled, &y, 0));
    HB_CK(op->ceed, hb_freestream_diagonal(op->fop, op->qf->ctx->data, op->flux_type, qd, jd, y, op->ceed->stream));
    return CEED_ERROR_SUCCESS;
  }
  if (op->plan == PLAN_MASS_STAB) {
    CK(need_len(op, assembled, op->eop->l_size, "diagonal"));
    CK(need_len(op, op->in[1].v, op->eop->l_size, "state"));
    CK(need_len(op, op->in[2].v, op->in[2].r->l_size, "qdata"));
    const double *qs, *qd;
    double       *y;
    CK(vec_dev_read(op->in[1].v, &qs));
    CK(vec_dev_read(op->in[2].v, &qd));
    CK(vec_dev_write(assembled, &y, 0));
    HB_CK(op->ceed, hb_mass_stab_diagonal(op->eop, op->qf->ctx->data, qd, qs, y, 1, op->ceed->stream));
    return CEED_ERROR_SUCCESS;
  }
  if (op->plan == PLAN_MASS_N) {
    CK(need_len(op, assembled, op->in[0].r->l_size, "diagonal"));
    CK(need_len(op, op->in[1].v, op->in[1].r->l_size, "qdata"));
    const double *qd;
    double       *y;
    CK(vec_dev_read(op->in[1].v, &qd));
    CK(vec_dev_write(assembled, &y, 0));
    HB_CK(op->ceed, hb_mass_n_diagonal(op->eop, op->nc, qd, y, op->ceed->stream));
    return CEED_ERROR_SUCCESS;
  }
  if (op->plan == PLAN_MASS) {
    CK(need_len(op, assembled, op->eop->l_size, "diagonal"));
    CK(need_len(op, op->in[1].v, op->in[1].r->l_size, "qdata"));
    const double *qd;
    double       *y;
    CK(vec_dev_read(op->in[1].v, &qd));
    CK(vec_dev_write(assembled, &y, 0));
    HB_CK(op->ceed, hb_mass_diagonal(op->eop, qd, y, 1, op->ceed->stream));
    return CEED_ERROR_SUCCESS;
  }
  if (op->plan != PLAN_IJACOBIAN)
    return plan_fail(op, "diagonal assembly is provided for the IJacobian operators (volume and free-stream faces) and the mass operator");
  CK(need_len(op, assembled, op->eop->l_size, "diagonal"));
  CK(need_len(op, op->in[2].v, op->in[2].r->l_size, "qdata"));
  CK(need_len(op, op->in[3].v, op->in[3].r->l_size, "jac_data"));
  if ((((const HbNewtonianContext *)op->qf->ctx->data)->idl_enable ? 15 : 14) != op->qf->in[3].size)
    return plan_fail(op, "jac_data component count does not match the IDL setting");
  Ceed                      ceed = op->ceed;
  cudaStream_t              s    = ceed->stream;
  const HbNewtonianContext *ctx  = (const HbNewtonianContext *)op->qf->ctx->data;
  const double             *qd;
  CK(vec_dev_read(op->in[2].v, &qd));
  CeedVector jd = op->in[3].v;
  double    *y;
  if (ceed->mixed) {
    if (!jd->f32_valid) {
      const double *j64;
      CK(vec_dev_read(jd, &j64));
      CK(vec_f32_shadow(jd));
      HB_CK(ceed, hb_vec_f64_to_f32(j64, jd->d_f32, jd->length, 0, s));
      jd->f32_valid = 1;
    }
    const int64_t n = op->eop->l_size;
    if (!op->d_tmp_out32) {
      CUDA_CK(ceed, cudaMalloc((void **)&op->d_tmp_in32, sizeof(float) * (size_t)n));
      CUDA_CK(ceed, cudaMalloc((void **)&op->d_tmp_out32, sizeof(float) * (size_t)n));
    }
    CK(vec_dev_write(assembled, &y, 0));
    HB_CK(ceed, hb_diagonal_assemble_f32(op->eop, ctx, qd, jd->d_f32, op->d_tmp_out32, 0, s));
    HB_CK(ceed, hb_vec_f32_to_f64(op->d_tmp_out32, y, n, 1, s));
  } else {
    const double *j64;
    CK(vec_dev_read(jd, &j64));
    CK(vec_dev_write(assembled, &y, 0));
    HB_CK(ceed, hb_diagonal_assemble_f64(op->eop, ctx, qd, j64, y, 1, s));
  }
  return CEED_ERROR_SUCCESS;
}

int CeedOperatorLinearAssembleAddDiagonal(CeedOperator op, CeedVector assembled, CeedRequest *request) {
  (void)request;
  if (op->composite) {
    for (int i = 0; i < op->nsub; i++) CK(op_diag_add_single(op->subs[i], assembled));
    return CEED_ERROR_SUCCESS;
  }
  return op_diag_add_single(op, assembled);
}

int CeedOperatorLinearAssembleDiagonal(CeedOperator op, CeedVector assembled, CeedRequest *request) {
  CK(CeedVectorSetValue(assembled, 0.0));
  return CeedOperatorLinearAssembleAddDiagonal(op, assembled, request);
}

/* Flop estimate: sum-factorised basis (interp + collocated gradient and their transposes) plus the point-wise counts
 * of the fused kernels (measured with the oracle's counting build: about 700 flops per IFunction point and 520 per
 * IJacobian point at conservative variables with SUPG). */
int CeedOperatorGetFlopsEstimate(CeedOperator op, CeedSize *flops) {
  *flops = 0;
  if (op->composite) {
    for (int i = 0; i < op->nsub; i++) {
      CeedSize f;
      CK(CeedOperatorGetFlopsEstimate(op->subs[i], &f));
      *flops += f;
    }
    return CEED_ERROR_SUCCESS;
  }
  CK(op_plan(op));
  if (!op->eop) return CEED_ERROR_SUCCESS;
  const CeedSize P = op->eop->P, Q = op->eop->Q, E = op->eop->num_elem, Q3 = Q * Q * Q;
  const CeedSize interp = 2 * (Q * P * P * P + Q * Q * P * P + Q * Q * Q * P), deriv = 2 * 3 * Q3 * Q;
  if (op->plan == PLAN_IFUNCTION || op->plan == PLAN_RHS) *flops = E * (5 * (2 * (interp + deriv)) + 5 * interp + 700 * Q3);
  else if (op->plan == PLAN_MASS) *flops = E * (5 * 2 * interp + 5 * Q3);
  else if (op->plan == PLAN_IJACOBIAN) *flops = E * (5 * (2 * (interp + deriv)) + 520 * Q3);
  else if (op->plan == PLAN_MASS_N) *flops = E * (op->nc * (2 * interp + Q3));
  else if (op->plan == PLAN_VELGRAD) *flops = E * (5 * (interp + deriv) + 9 * interp + 150 * Q3);
  else if (op->plan == PLAN_ANISO) *flops = E * (7 * interp + 400 * Q3);
  else if (op->plan == PLAN_SGS_IF) *flops = E * (11 * interp + 5 * (interp + deriv) + 90 * Q3);
  else if (op->plan == PLAN_SGS_NODAL) *flops = (op->out[0].r->l_size / 6) * 1500;
  return CEED_ERROR_SUCCESS;
}

int CeedOperatorDestroy(CeedOperator *op) {
  CeedOperator o = *op;
  if (!o) return CEED_ERROR_SUCCESS;
  if (--o->ref > 0) {
    *op = NULL;
    return CEED_ERROR_SUCCESS;
  }
  if (o->composite) {
    for (int i = 0; i < o->nsub; i++) CeedOperatorDestroy(&o->subs[i]);
  } else {
    for (int i = 0; i < o->qf->nin; i++)
      if (o->in[i].set) {
        CeedElemRestrictionDestroy(&o->in[i].r);
        CeedBasisDestroy(&o->in[i].b);
        CeedVectorDestroy(&o->in[i].v);
      }
    for (int i = 0; i < o->qf->nout; i++)
      if (o->out[i].set) {
        CeedElemRestrictionDestroy(&o->out[i].r);
        CeedBasisDestroy(&o->out[i].b);
        CeedVectorDestroy(&o->out[i].v);
      }
    CeedQFunctionDestroy(&o->qf);
  }
  if (o->eop) ceed_unregister_op(o->ceed, o->eop);
  hb_elemop_destroy(o->eop);
  hb_faceop_destroy(o->fop);
  cudaFree(o->d_zero);
  cudaFree(o->d_tmp_rhs);
  cudaFree(o->d_tmp_pb32);
  cudaFree(o->d_tmp_in32);
  cudaFree(o->d_tmp_out32);
  cudaFree(o->d_tmp_e);
  cudaFree(o->d_tmp_e2);
  Ceed ceed = o->ceed;
  free(o);
  *op = NULL;
  return CeedDestroy(&ceed);
}

/* ------------------------------------------------------------------------------------------------------------------ */
/* Accessors, views and the assembly entry points HONEE links against (src/mat-ceed.c, src/misc.c, src/petsc_ops.c)      */

int CeedGetGitVersion(const char **git_version) {
  *git_version = "honee-b200";
  return CEED_ERROR_SUCCESS;
}
Ceed CeedObjectReturnCeed(CeedObject obj) { return obj ? *(Ceed *)obj : NULL; }
int  CeedVectorGetCeed(CeedVector vec, Ceed *ceed) {
  *ceed = NULL;
  return CeedReferenceCopy(vec->ceed, ceed);
}
Ceed CeedVectorReturnCeed(CeedVector vec) { return vec->ceed; }
int  CeedElemRestrictionGetCeed(CeedElemRestriction rstr, Ceed *ceed) {
  *ceed = NULL;
  return CeedReferenceCopy(rstr->ceed, ceed);
}
Ceed CeedElemRestrictionReturnCeed(CeedElemRestriction rstr) { return rstr->ceed; }
Ceed CeedBasisReturnCeed(CeedBasis basis) { return basis->ceed; }
int  CeedOperatorGetCeed(CeedOperator op, Ceed *ceed) {
  *ceed = NULL;
  return CeedReferenceCopy(op->ceed, ceed);
}
Ceed CeedOperatorReturnCeed(CeedOperator op) { return op->ceed; }
int  CeedOperatorIsComposite(CeedOperator op, bool *is_composite) {
  *is_composite = op->composite != 0;
  return CEED_ERROR_SUCCESS;
}
int CeedOperatorGetContext(CeedOperator op, CeedQFunctionContext *ctx) {
  *ctx = NULL;
  if (op->composite) return CeedError(op->ceed, CEED_ERROR_INCOMPATIBLE, "composite operators have no single context");
  if (op->qf->ctx) return CeedQFunctionContextReferenceCopy(op->qf->ctx, ctx);
  return CEED_ERROR_SUCCESS;
}

int CeedQFunctionCreateIdentity(Ceed ceed, CeedInt size, CeedEvalMode in_mode, CeedEvalMode out_mode, CeedQFunction *qf) {
  CK(CeedQFunctionCreateInterior(ceed, 1, NULL, "Identity", qf));
  CK(CeedQFunctionAddInput(*qf, "input", size, in_mode));
  return CeedQFunctionAddOutput(*qf, "output", size, out_mode);
}

/* Operator fields are addressed through a handle encoding (operator, field index); the layout is private to this file. */
struct CeedOperatorField_private {
  CeedOperator op;
  int          out, index;
};
#define FIELD_POOL 1024
static struct CeedOperatorField_private field_pool[FIELD_POOL];
static int                              field_pool_n;

int CeedOperatorGetFieldByName(CeedOperator op, const char *field_name, CeedOperatorField *op_field) {
  *op_field = NULL;
  if (op->composite) return CeedError(op->ceed, CEED_ERROR_INCOMPATIBLE, "composite operators have no fields");
  for (int o = 0; o < 2; o++) {
    const int n = o ? op->qf->nout : op->qf->nin;
    for (int i = 0; i < n; i++) {
      const char *nm = o ? op->qf->out[i].name : op->qf->in[i].name;
      if (strcmp(nm, field_name)) continue;
      for (int k = 0; k < field_pool_n; k++)
        if (field_pool[k].op == op && field_pool[k].out == o && field_pool[k].index == i) {
          *op_field = &field_pool[k];
          return CEED_ERROR_SUCCESS;
        }
      if (field_pool_n >= FIELD_POOL) return CeedError(op->ceed, CEED_ERROR_UNSUPPORTED, "too many operator field handles");
      field_pool[field_pool_n] = (struct CeedOperatorField_private){op, o, i};
      *op_field                = &field_pool[field_pool_n++];
      return CEED_ERROR_SUCCESS;
    }
  }
  return CeedError(op->ceed, CEED_ERROR_INCOMPLETE, "operator has no field named '%s'", field_name);
}
static OpField *field_of(CeedOperatorField f) { return f->out ? &f->op->out[f->index] : &f->op->in[f->index]; }
int CeedOperatorFieldGetElemRestriction(CeedOperatorField op_field, CeedElemRestriction *rstr) {
  *rstr = field_of(op_field)->r;
  return CEED_ERROR_SUCCESS;
}
int CeedOperatorFieldGetVector(CeedOperatorField op_field, CeedVector *vec) {
  *vec = field_of(op_field)->v;
  return CEED_ERROR_SUCCESS;
}
int CeedOperatorFieldGetData(CeedOperatorField op_field, const char **field_name, CeedElemRestriction *rstr, CeedBasis *basis, CeedVector *vec) {
  OpField *f = field_of(op_field);
  if (field_name) *field_name = op_field->out ? op_field->op->qf->out[op_field->index].name : op_field->op->qf->in[op_field->index].name;
  if (rstr) *rstr = f->r;
  if (basis) *basis = f->b;
  if (vec) *vec = f->v;
  return CEED_ERROR_SUCCESS;
}

static int view_tabs_default;
int CeedOperatorSetNumViewTabs(CeedOperator op, CeedInt num_tabs) {
  (void)op;
  view_tabs_default = num_tabs;
  return CEED_ERROR_SUCCESS;
}
int CeedOperatorGetNumViewTabs(CeedOperator op, CeedInt *num_tabs) {
  (void)op;
  *num_tabs = view_tabs_default;
  return CEED_ERROR_SUCCESS;
}
static void op_view(CeedOperator op, FILE *stream, int terse, int depth) {
  const int tabs = view_tabs_default + depth;
  for (int t = 0; t < tabs; t++) fputs("  ", stream);
  if (op->composite) {
    fprintf(stream, "Composite CeedOperator '%s' (%d sub-operators) on %s\n", op->name, op->nsub, op->ceed->resource);
    for (int i = 0; i < op->nsub; i++) op_view(op->subs[i], stream, terse, depth + 1);
    return;
  }
  fprintf(stream, "CeedOperator '%s': QFunction %s, %d inputs, %d outputs, backend plan %s\n", op->name, op->qf->kernel, op->qf->nin,
          op->qf->nout,
          op->plan == PLAN_IFUNCTION   ? "fused IFunction"
          : op->plan == PLAN_IJACOBIAN ? "fused IJacobian"
          : op->plan == PLAN_SETUP     ? "qdata setup"
          : op->plan == PLAN_SETUP_SUR ? "surface qdata setup"
          : op->plan == PLAN_FREESTREAM ? "free-stream faces"
          : op->plan == PLAN_FREESTREAM_JAC ? "free-stream faces Jacobian"
          : op->plan == PLAN_RHS       ? "explicit right-hand side"
          : op->plan == PLAN_MASS      ? "mass"
          : op->plan == PLAN_MASS_STAB ? "stabilized mass"
          : op->plan == PLAN_MASS_N    ? "mass (N fields)"
          : op->plan == PLAN_VELGRAD   ? "velocity-gradient projection right-hand side"
          : op->plan == PLAN_ANISO     ? "anisotropy-tensor projection right-hand side"
          : op->plan == PLAN_INV_MULT  ? "inverse multiplicity"
          : op->plan == PLAN_SGS_NODAL ? "nodal data-driven SGS closure"
          : op->plan == PLAN_SGS_IF    ? "nodal SGS residual"
                                       : "not planned");
  if (terse) return;
  for (int o = 0; o < 2; o++)
    for (int i = 0; i < (o ? op->qf->nout : op->qf->nin); i++) {
      const QFField *qf = o ? &op->qf->out[i] : &op->qf->in[i];
      for (int t = 0; t < tabs + 1; t++) fputs("  ", stream);
      fprintf(stream, "%s field '%s': size %d, eval mode %d\n", o ? "output" : "input", qf->name, qf->size, qf->emode);
    }
}
int CeedOperatorView(CeedOperator op, FILE *stream) {
  op_view(op, stream, 0, 0);
  return CEED_ERROR_SUCCESS;
}
int CeedOperatorViewTerse(CeedOperator op, FILE *stream) {
  op_view(op, stream, 1, 0);
  return CEED_ERROR_SUCCESS;
}
int CeedOperatorSetQFunctionAssemblyDataUpdateNeeded(CeedOperator op, bool needs_data_update) {
  (void)op, (void)needs_data_update; /* the diagonal is linearised on the fly from the stored Jacobian data */
  return CEED_ERROR_SUCCESS;
}

#define ASSEMBLY_UNSUPPORTED(op) \
  CeedError((op)->ceed, CEED_ERROR_UNSUPPORTED, "assembled (COO) and point-block operators are not provided by /gpu/b200 (matrix-free only)")
int CeedOperatorLinearAssembleSymbolic(CeedOperator op, CeedSize *num_entries, CeedInt **rows, CeedInt **cols) {
  (void)num_entries, (void)rows, (void)cols;
  return ASSEMBLY_UNSUPPORTED(op);
}
int CeedOperatorLinearAssemble(CeedOperator op, CeedVector values) {
  (void)values;
  return ASSEMBLY_UNSUPPORTED(op);
}
int CeedOperatorLinearAssembleGetNumEntries(CeedOperator op, CeedSize *num_entries) {
  (void)num_entries;
  return ASSEMBLY_UNSUPPORTED(op);
}
/* Point-block diagonal (MatCEED's COO assembly for PCVPBJACOBI, src/mat-ceed.c:76-153): per node of the active
 * node-interleaved L-vector a row-major 5 x 5 block [component out][component in]; values[(node * 5 + i) * 5 + j].  The
 * symbolic call returns the matching COO rows/cols (malloc'd; the caller frees them with free(), as HONEE's
 * IntArrayCeedToPetsc does). */
static int pb_rstr(CeedOperator op, CeedElemRestriction *r) {
  CeedOperator o = op;
  while (o->composite) {
    if (o->nsub < 1) return CeedError(op->ceed, CEED_ERROR_INCOMPLETE, "composite operator '%s' has no sub-operators", op->name);
    o = o->subs[0];
  }
  *r = op_active_rstr(o, 0);
  if (!*r || (*r)->num_comp != 5 || (*r)->comp_stride != 1 || (*r)->strided)
    return CeedError(op->ceed, CEED_ERROR_UNSUPPORTED, "point blocks need the 5-component node-interleaved active restriction");
  return CEED_ERROR_SUCCESS;
}

static int op_pbdiag_add_single(CeedOperator op, CeedVector assembled) {
  if (op_empty(op)) return CEED_ERROR_SUCCESS;
  CK(op_plan(op));
  Ceed         ceed = op->ceed;
  cudaStream_t s    = ceed->stream;
  double      *y;
  switch (op->plan) {
    case PLAN_FREESTREAM_JAC: {
      CK(need_len(op, assembled, 5 * op->fop->l_size, "point-block"));
      CK(need_len(op, op->in[2].v, op->in[2].r->l_size, "surface qdata"));
      CK(need_len(op, op->in[4].v, op->in[4].r->l_size, "surface jacobian data"));
      const double *qd, *jd;
      CK(vec_dev_read(op->in[2].v, &qd));
      CK(vec_dev_read(op->in[4].v, &jd));
      CK(vec_dev_write(assembled, &y, 0));
      HB_CK(ceed, hb_freestream_point_block_diagonal(op->fop, op->qf->ctx->data, op->flux_type, qd, jd, y, s));
      return CEED_ERROR_SUCCESS;
    }
    case PLAN_MASS: {
      CK(need_len(op, assembled, 5 * op->eop->l_size, "point-block"));
      CK(need_len(op, op->in[1].v, op->in[1].r->l_size, "qdata"));
      const double *qd;
      CK(vec_dev_read(op->in[1].v, &qd));
      CK(vec_dev_write(assembled, &y, 0));
      HB_CK(ceed, hb_mass_point_block_diagonal(op->eop, qd, y, 1, s));
      return CEED_ERROR_SUCCESS;
    }
    case PLAN_IJACOBIAN: break;
    default: return plan_fail(op, "point-block assembly is provided for the IJacobian operators (volume and free-stream faces) and the mass operator");
  }
  const HbNewtonianContext *ctx = (const HbNewtonianContext *)op->qf->ctx->data;
  if ((ctx->idl_enable ? 15 : 14) != op->qf->in[3].size) return plan_fail(op, "jac_data component count does not match the IDL setting");
  const int64_t n = op->eop->l_size;
  CK(need_len(op, assembled, 5 * n, "point-block"));
  CK(need_len(op, op->in[2].v, op->in[2].r->l_size, "qdata"));
  CK(need_len(op, op->in[3].v, op->in[3].r->l_size, "jac_data"));
  const double *qd;
  CK(vec_dev_read(op->in[2].v, &qd));
  CeedVector jd = op->in[3].v;
  if (ceed->mixed) {
    if (!jd->f32_valid) {
      const double *j64;
      CK(vec_dev_read(jd, &j64));
      CK(vec_f32_shadow(jd));
      HB_CK(ceed, hb_vec_f64_to_f32(j64, jd->d_f32, jd->length, 0, s));
      jd->f32_valid = 1;
    }
    if (!op->d_tmp_pb32) CUDA_CK(ceed, cudaMalloc((void **)&op->d_tmp_pb32, sizeof(float) * 5 * (size_t)n));
    CK(vec_dev_write(assembled, &y, 0));
    HB_CK(ceed, hb_point_block_diagonal_f32(op->eop, ctx, qd, jd->d_f32, op->d_tmp_pb32, 0, s));
    HB_CK(ceed, hb_vec_f32_to_f64(op->d_tmp_pb32, y, 5 * n, 1, s));
  } else {
    const double *j64;
    CK(vec_dev_read(jd, &j64));
    CK(vec_dev_write(assembled, &y, 0));
    HB_CK(ceed, hb_point_block_diagonal_f64(op->eop, ctx, qd, j64, y, 1, s));
  }
  return CEED_ERROR_SUCCESS;
}

int CeedOperatorLinearAssembleAddPointBlockDiagonal(CeedOperator op, CeedVector assembled, CeedRequest *request) {
  (void)request;
  if (op->composite) {
    for (int i = 0; i < op->nsub; i++) CK(op_pbdiag_add_single(op->subs[i], assembled));
    return CEED_ERROR_SUCCESS;
  }
  return op_pbdiag_add_single(op, assembled);
}

int CeedOperatorLinearAssemblePointBlockDiagonal(CeedOperator op, CeedVector assembled, CeedRequest *request) {
  CK(CeedVectorSetValue(assembled, 0.0));
  return CeedOperatorLinearAssembleAddPointBlockDiagonal(op, assembled, request);
}

int CeedOperatorLinearAssemblePointBlockDiagonalSymbolic(CeedOperator op, CeedSize *num_entries, CeedInt **rows, CeedInt **cols) {
  CeedElemRestriction r;
  CK(pb_rstr(op, &r));
  const CeedSize nodes = r->l_size / 5, ne = nodes * 25;
  CeedInt *ro = (CeedInt *)malloc(sizeof(CeedInt) * (size_t)ne), *co = (CeedInt *)malloc(sizeof(CeedInt) * (size_t)ne);
  if (!ro || !co) {
    free(ro);
    free(co);
    return CeedError(op->ceed, CEED_ERROR_MAJOR, "out of host memory for %td point-block entries", ne);
  }
  for (CeedSize k = 0; k < ne; k++) {
    const CeedSize node = k / 25;
    ro[k] = (CeedInt)(node * 5 + (k / 5) % 5);
    co[k] = (CeedInt)(node * 5 + k % 5);
  }
  *num_entries = ne;
  *rows        = ro;
  *cols        = co;
  return CEED_ERROR_SUCCESS;
}
int CeedOperatorGetOperatorAssemblyData(CeedOperator op, CeedOperatorAssemblyData *data) {
  (void)data;
  return ASSEMBLY_UNSUPPORTED(op);
}
int CeedOperatorAssemblyDataGetBases(CeedOperatorAssemblyData data, CeedInt *num_active_bases_in, CeedBasis **active_bases_in,
                                     const CeedScalar ***assembled_bases_in, CeedInt *num_active_bases_out, CeedBasis **active_bases_out,
                                     const CeedScalar ***assembled_bases_out) {
  (void)data, (void)num_active_bases_in, (void)active_bases_in, (void)assembled_bases_in, (void)num_active_bases_out, (void)active_bases_out,
      (void)assembled_bases_out;
  snprintf(fallback_msg, sizeof fallback_msg, "operator assembly data is not provided by /gpu/b200");
  return CEED_ERROR_UNSUPPORTED;
}
