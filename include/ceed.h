/* ceed.h -- HONEE includes <ceed.h>; the B200 backend's declarations live in ceed/ceed.h. */
#ifndef CEED_B200_TOP_H
#define CEED_B200_TOP_H
#include "ceed/ceed.h"
#endif
