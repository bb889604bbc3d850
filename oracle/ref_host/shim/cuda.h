/* Host-side stand-ins for the CUDA types and qualifiers used by the CUDADSMC sources, so
 * that its per-atom __device__ functions and grid-stride kernels compile with g++ and run
 * serially on the CPU (blockIdx = threadIdx = 0, blockDim = gridDim = 1).  Used only to
 * build the reference comparison libraries under oracle/_ref/. */
#ifndef REF_HOST_CUDA_SHIM_H
#define REF_HOST_CUDA_SHIM_H
#include <math.h>
#include <stdio.h>

struct double2 { double x, y; };
struct double3 { double x, y, z; };
struct double4 { double x, y, z, w; };
struct float3 { float x, y, z; };
struct int2 { int x, y; };
struct int3 { int x, y, z; };
static inline double2 make_double2(double x, double y) { double2 r = {x, y}; return r; }
static inline double3 make_double3(double x, double y, double z) { double3 r = {x, y, z}; return r; }
static inline double4 make_double4(double x, double y, double z, double w) { double4 r = {x, y, z, w}; return r; }
static inline float3 make_float3(float x, float y, float z) { float3 r = {x, y, z}; return r; }
static inline int2 make_int2(int x, int y) { int2 r = {x, y}; return r; }
static inline int3 make_int3(int x, int y, int z) { int3 r = {x, y, z}; return r; }
static inline double rsqrt(double x) { return 1.0 / sqrt(x); }
static inline int __double2int_rd(double x) { return (int)floor(x); }

struct ref_dim3 { unsigned x, y, z; };
extern ref_dim3 blockIdx, blockDim, gridDim, threadIdx;
#endif
