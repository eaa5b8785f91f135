/* hb_internal.h -- the device helpers (vector algebra, generic restriction and basis) are part of the public kernel
 * ABI in include/honee_b200.h; this header only gathers the includes the host layer uses. */
#ifndef HB_INTERNAL_H
#define HB_INTERNAL_H
#include "honee_b200.h"

#ifdef __cplusplus
extern "C" {
#endif
/* Greedy colouring of elements (or faces) by the L-vector entries they touch: elements of one colour share no entry.
 * Refuses an element that lists an entry twice.  color_ptr [num_colors + 1] and color_elem [num_elem] are malloc'd. */
int hb_internal_color_elements(int num_elem, int elem_size, const int32_t *offsets, int64_t l_size, int32_t **color_ptr, int32_t **color_elem,
                               int *num_colors);
#ifdef __cplusplus
}
#endif
#endif
