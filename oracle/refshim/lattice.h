/* lattice.h -- openQCD-1.4 header name used by the wloop modules; everything is
 * declared in shim.h (one process, compile-time lattice). */
#ifndef LATTICE_H
#define LATTICE_H
#include "shim.h"
#endif
