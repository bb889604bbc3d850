#ifndef REF_HOST_CUCOMPLEX_SHIM_H
#define REF_HOST_CUCOMPLEX_SHIM_H
#include "cuda.h"
typedef double2 cuDoubleComplex;
static inline cuDoubleComplex make_cuDoubleComplex(double r, double i) { return make_double2(r, i); }
#endif
