// Comparisons of a float with a double constant, exact, in float arithmetic.
//
// The reference compares float variables with unsuffixed (double) literals,
// e.g. `xi < 0.1` (electron.cu:1806): C converts the float to double and
// compares in double. Let f = (float)D, the constant rounded to nearest.
// No float lies strictly between D and f, so for every float x (NaN included,
// for which both sides are false):
//   x <  D  <=>  (f < D ? x <= f : x <  f)
//   x <= D  <=>  (f > D ? x <  f : x <= f)
//   x >  D  <=>  (f > D ? x >= f : x >  f)
//   x >= D  <=>  (f < D ? x >  f : x >= f)
// With D a literal the condition on f folds at compile time, leaving one
// float compare instead of a conversion and a double compare. Shared by host
// and device code; tests/test_gx_cmp.py checks every case against the double
// comparison on the floats around each constant the kernels use.
#pragma once

#if defined(__CUDACC__)
#define GX_HD __host__ __device__ __forceinline__
#else
#define GX_HD static inline
#endif

GX_HD bool gx_lt(float x, double d) { const float f = (float)d; return ((double)f < d) ? (x <= f) : (x < f); }
GX_HD bool gx_le(float x, double d) { const float f = (float)d; return ((double)f > d) ? (x < f) : (x <= f); }
GX_HD bool gx_gt(float x, double d) { const float f = (float)d; return ((double)f > d) ? (x >= f) : (x > f); }
GX_HD bool gx_ge(float x, double d) { const float f = (float)d; return ((double)f < d) ? (x > f) : (x >= f); }
