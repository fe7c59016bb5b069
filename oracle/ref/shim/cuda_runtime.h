/* Host stand-in for <cuda_runtime.h>, used only to compile the reference's
 * unmodified device sources (geom.cu, utility.cu, relax.cu and the stage
 * kernels) as host C++ for the reference-pinning harness (test
 * infrastructure). It supplies the CUDA qualifiers as no-ops, the vector
 * types, a one-thread launch context, and the atomics and warp votes of a
 * single thread. The transcendental functions are bound in ref_math.h. */
#ifndef GEGS_REF_SHIM_CUDA_RUNTIME_H
#define GEGS_REF_SHIM_CUDA_RUNTIME_H

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#define __device__
#define __host__
#define __global__
#define __constant__
#define __shared__
#define __forceinline__ inline
#define __noinline__
#define __align__(n) alignas(n)

struct float2 { float x, y; };
struct float3 { float x, y, z; };
struct float4 { float x, y, z, w; };
struct int2 { int x, y; };
struct int3 { int x, y, z; };
struct int4 { int x, y, z, w; };
struct uint2 { unsigned x, y; };
struct uint3 { unsigned x, y, z; };
struct uint4 { unsigned x, y, z, w; };
struct dim3 { unsigned x, y, z; };

static inline float2 make_float2(float x, float y) { float2 r = {x, y}; return r; }
static inline float3 make_float3(float x, float y, float z) { float3 r = {x, y, z}; return r; }
static inline float4 make_float4(float x, float y, float z, float w) { float4 r = {x, y, z, w}; return r; }
static inline int2 make_int2(int x, int y) { int2 r = {x, y}; return r; }
static inline int3 make_int3(int x, int y, int z) { int3 r = {x, y, z}; return r; }
static inline uint3 make_uint3(unsigned x, unsigned y, unsigned z) { uint3 r = {x, y, z}; return r; }
static inline uint4 make_uint4(unsigned x, unsigned y, unsigned z, unsigned w) { uint4 r = {x, y, z, w}; return r; }

/* one-thread launch: every kernel runs as thread 0 of block 0 of a 1x1 grid */
static const uint3 threadIdx = {0, 0, 0};
static const uint3 blockIdx = {0, 0, 0};
static const dim3 blockDim = {1, 1, 1};
static const dim3 gridDim = {1, 1, 1};

static inline void __syncthreads(void) {}
static inline void __threadfence(void) {}
static inline int __all(int p) { return p; }
static inline int __any(int p) { return p; }
static inline unsigned __ballot(int p) { return p ? 1u : 0u; }
static inline int __popc(unsigned x) { return __builtin_popcount(x); }

static inline int atomicAdd(int *a, int v) { int o = *a; *a = o + v; return o; }
static inline unsigned atomicAdd(unsigned *a, unsigned v) { unsigned o = *a; *a = o + v; return o; }
static inline float atomicAdd(float *a, float v) { float o = *a; *a = o + v; return o; }
static inline int atomicSub(int *a, int v) { int o = *a; *a = o - v; return o; }
static inline unsigned long long atomicCAS(unsigned long long *a, unsigned long long cmp, unsigned long long v)
{
    unsigned long long o = *a;
    if (o == cmp) *a = v;
    return o;
}
static inline long long __double_as_longlong(double d) { long long r; std::memcpy(&r, &d, 8); return r; }
static inline double __longlong_as_double(long long l) { double r; std::memcpy(&r, &l, 8); return r; }
static inline int __float_as_int(float f) { int r; std::memcpy(&r, &f, 4); return r; }
static inline float __int_as_float(int i) { float r; std::memcpy(&r, &i, 4); return r; }

/* mixed-type min/max, which CUDA's device math provides (promoting to double) */
static inline double max(double a, float b) { return a > (double)b ? a : (double)b; }
static inline double max(float a, double b) { return (double)a > b ? (double)a : b; }
static inline double min(double a, float b) { return a < (double)b ? a : (double)b; }
static inline double min(float a, double b) { return (double)a < b ? (double)a : b; }

/* host-API names that appear in the reference's declarations */
typedef int cudaError_t;
typedef void *cudaStream_t;
typedef void *cudaEvent_t;

/* The host set-up routines (init.cu) move their results with these. Device
 * memory is host memory here, and a __constant__ symbol a plain global. */
enum cudaMemcpyKind { cudaMemcpyHostToHost, cudaMemcpyHostToDevice, cudaMemcpyDeviceToHost, cudaMemcpyDeviceToDevice };
template <class T> static inline cudaError_t cudaMalloc(T **p, size_t n) { *p = (T *)std::malloc(n); return 0; }
static inline cudaError_t cudaMemcpy(void *d, const void *s, size_t n, cudaMemcpyKind) { std::memcpy(d, s, n); return 0; }
template <class T> static inline cudaError_t cudaMemcpyToSymbol(T &sym, const void *s, size_t n)
{
    std::memcpy((void *)&sym, s, n);
    return 0;
}
static inline cudaError_t cudaSetDevice(int) { return 0; }

#endif
