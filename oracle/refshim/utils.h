/* utils.h -- openQCD-1.4 header name used by the wloop modules; everything is
 * declared in shim.h (one process, compile-time lattice). */
#ifndef UTILS_H
#define UTILS_H
#include "shim.h"
#endif
