/* mdcore.h -- the umbrella header name of the reference library (src/mdcore.h), so that a
 * driver written for mdcore, with its `#include "mdcore.h"`, compiles unchanged against
 * libmdcore_b200: put this directory first on the include path (-I include) and link
 * -lmdcore_b200 instead of -lmdcore_single.  Everything is declared in mdcore_b200.h. */
#ifndef MDCORE_H_B200
#define MDCORE_H_B200
#include "mdcore_b200.h"
#endif
