/* The comparison libraries only call deterministic kernels; the random-number entry points
 * are declared so that the sources compile, and abort if reached. */
#ifndef REF_HOST_CURAND_SHIM_H
#define REF_HOST_CURAND_SHIM_H
#include <stdlib.h>
#include "cuda.h"
struct curandState_t { unsigned long long s; };
typedef curandState_t curandState;
static inline double curand_uniform_double(curandState_t*) { abort(); return 0.0; }
static inline double curand_normal_double(curandState_t*) { abort(); return 0.0; }
static inline double2 curand_normal2_double(curandState_t*) { abort(); return make_double2(0, 0); }
static inline void curand_init(unsigned long long, unsigned long long, unsigned long long, curandState_t*) { abort(); }
#endif
