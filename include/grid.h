/* Compatibility header carrying the reference's header name (grid.h) so that
 * code written against the reference includes it unchanged.  All types and
 * functions are declared in gli_b200.h. */
#ifndef GLI_B200_COMPAT_GRID_H
#define GLI_B200_COMPAT_GRID_H
#include "gli_b200.h"
#endif
