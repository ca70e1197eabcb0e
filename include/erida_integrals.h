/* Compatibility header carrying the reference's header name (erida_integrals.h) so that
 * code written against the reference includes it unchanged.  All types and
 * functions are declared in gli_b200.h. */
#ifndef GLI_B200_COMPAT_ERIDA_INTEGRALS_H
#define GLI_B200_COMPAT_ERIDA_INTEGRALS_H
#include "gli_b200.h"
#endif
