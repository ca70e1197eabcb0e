/* Compatibility header carrying the reference's header name (symmetry.h) so that
 * code written against the reference includes it unchanged.  All types and
 * functions are declared in gli_b200.h. evaluate_octahedral_grid_permutations() is the symbol of that header provided here. */
#ifndef GLI_B200_COMPAT_SYMMETRY_H
#define GLI_B200_COMPAT_SYMMETRY_H
#include "gli_b200.h"
#endif
