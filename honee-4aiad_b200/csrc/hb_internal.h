/* hb_internal.h -- the device helpers (vector algebra, generic restriction and basis) are part of the public kernel
 * ABI in include/honee_b200.h; this header only gathers the includes the host layer uses. */
#ifndef HB_INTERNAL_H
#define HB_INTERNAL_H
#include "honee_b200.h"
#endif
