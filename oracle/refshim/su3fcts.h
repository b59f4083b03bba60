/* su3fcts.h -- openQCD-1.4 header name used by the wloop modules; everything is
 * declared in shim.h (one process, compile-time lattice). */
#ifndef SU3FCTS_H
#define SU3FCTS_H
#include "shim.h"
#endif
