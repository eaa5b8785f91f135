/* ceed/types.h -- scalar types, enums and QFunction macros of the libCEED API (B200 backend).
 *
 * HONEE QFunction headers (the qfunctions directory) include <ceed/types.h>; so does include/ceed/ceed.h.  Names and values follow
 * libCEED so those sources compile unchanged: CEED_QFUNCTION(name) declares the user function and the `name_loc` source
 * string ("file:name") that HONEE passes to CeedQFunctionCreateInterior (problems/newtonian.c:773-787) and that the
 * backend uses to bind the fused kernel. */
#ifndef CEED_B200_TYPES_H
#define CEED_B200_TYPES_H

#ifndef CEED_RUNNING_JIT_PASS
#include <float.h>
#include <math.h>
#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>
#endif

typedef int32_t   CeedInt;
typedef int8_t    CeedInt8;
typedef ptrdiff_t CeedSize;
typedef double    CeedScalar;
#define CEED_SCALAR_TYPE CEED_SCALAR_FP64
#define CEED_EPSILON 0x1p-52

typedef enum {
  CEED_ERROR_SUCCESS      = 0,
  CEED_ERROR_MINOR        = 1,
  CEED_ERROR_DIMENSION    = 2,
  CEED_ERROR_INCOMPLETE   = 3,
  CEED_ERROR_INCOMPATIBLE = 4,
  CEED_ERROR_ACCESS       = 5,
  CEED_ERROR_MAJOR        = -1,
  CEED_ERROR_BACKEND      = -2,
  CEED_ERROR_UNSUPPORTED  = -3,
} CeedErrorType;

typedef enum { CEED_MEM_HOST, CEED_MEM_DEVICE } CeedMemType;
typedef enum { CEED_COPY_VALUES, CEED_USE_POINTER, CEED_OWN_POINTER } CeedCopyMode;
typedef enum { CEED_NORM_1, CEED_NORM_2, CEED_NORM_MAX } CeedNormType;
typedef enum { CEED_NOTRANSPOSE, CEED_TRANSPOSE } CeedTransposeMode;
typedef enum {
  CEED_EVAL_NONE   = 0,
  CEED_EVAL_INTERP = 1,
  CEED_EVAL_GRAD   = 2,
  CEED_EVAL_DIV    = 4,
  CEED_EVAL_CURL   = 8,
  CEED_EVAL_WEIGHT = 16,
} CeedEvalMode;
typedef enum { CEED_GAUSS = 0, CEED_GAUSS_LOBATTO = 1 } CeedQuadMode;
typedef enum {
  CEED_TOPOLOGY_LINE     = 1 << 16 | 0,
  CEED_TOPOLOGY_TRIANGLE = 2 << 16 | 1,
  CEED_TOPOLOGY_QUAD     = 2 << 16 | 2,
  CEED_TOPOLOGY_TET      = 3 << 16 | 3,
  CEED_TOPOLOGY_PYRAMID  = 3 << 16 | 4,
  CEED_TOPOLOGY_PRISM    = 3 << 16 | 5,
  CEED_TOPOLOGY_HEX      = 3 << 16 | 6,
} CeedElemTopology;
#define CEED_Q_VLA Q
#define CeedPragmaSIMD
#define CEED_QFUNCTION_HELPER static inline
#define CEED_QFUNCTION(name)                           \
  static const char name##_loc[] = __FILE__ ":" #name; \
  static int        name

#endif
