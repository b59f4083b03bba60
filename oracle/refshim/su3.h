/* su3.h -- openQCD-1.4 header name used by the wloop modules; everything is
 * declared in shim.h (one process, compile-time lattice). */
#ifndef SU3_H
#define SU3_H
#include "shim.h"
#endif
