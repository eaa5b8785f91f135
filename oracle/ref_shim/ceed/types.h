/* Minimal stand-in for libCEED's <ceed/types.h> (TEST INFRASTRUCTURE ONLY).
 *
 * Lets the reference's QFunction headers (qfunctions/*.h, plain C99) compile unchanged on the host so that the
 * oracle restatement can be checked against them.  Only the names those headers use are defined: the scalar and
 * integer types, the QFunction declaration macros, the vector-length placeholder, the SIMD pragma, the transpose
 * enum, the success code, the eval-mode constant referenced in comments/asserts and the machine epsilon.
 * CEED_QFUNCTION(name) declares `static int name` plus the `name_loc` source-location string libCEED expects. */
#ifndef HONEE_REF_SHIM_CEED_TYPES_H
#define HONEE_REF_SHIM_CEED_TYPES_H
#include <float.h>
#include <math.h>
#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>

typedef double  CeedScalar;
typedef int32_t CeedInt;
typedef enum { CEED_NOTRANSPOSE = 0, CEED_TRANSPOSE = 1 } CeedTransposeMode;
typedef enum { CEED_EVAL_NONE = 0, CEED_EVAL_INTERP = 1, CEED_EVAL_GRAD = 2, CEED_EVAL_WEIGHT = 16 } CeedEvalMode;

#define CEED_ERROR_SUCCESS 0
#define CEED_EPSILON DBL_EPSILON
#define CEED_Q_VLA Q
#define CeedPragmaSIMD
#define CEED_QFUNCTION_HELPER static inline
#define CEED_QFUNCTION(name)                         \
  static const char name##_loc[] = __FILE__ ":" #name; \
  static int        name
#endif
