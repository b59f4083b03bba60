/* uflds.h -- openQCD-1.4 header name used by the wloop modules; everything is
 * declared in shim.h (one process, compile-time lattice). */
#ifndef UFLDS_H
#define UFLDS_H
#include "shim.h"
#endif
