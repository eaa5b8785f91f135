/* ref_qfunctions_train.c -- exports the reference's SGS training-data QFunction, compiled unchanged, for the oracle
 * checks (TEST INFRASTRUCTURE ONLY).  A translation unit of its own because differential_filter_enums.h, which both
 * sgs_dd_training.h and differential_filter.h include, has no include guard. */
#include <ceed/types.h>

#include "sgs_dd_training.h"

#define EXPORT __attribute__((visibility("default")))

EXPORT int ref_ComputeSGS_DDAnisotropicTrainingDataNodal_Conserv(void *c, CeedInt Q, const CeedScalar *const *in, CeedScalar *const *out) {
  return ComputeSGS_DDAnisotropicTrainingDataNodal(c, Q, in, out, STATEVAR_CONSERVATIVE);
}
