/* Transcendental functions of the reference's device code, bound to the
 * oracle's (reference-pinning harness, test infrastructure).
 *
 * The reference calls CUDA's logf/expf/__sincosf/rsqrtf (and log/exp/cos/sin
 * on float arguments, which CUDA resolves to the float versions). The oracle
 * and the CUDA library use their own log/exp/sincos, built from IEEE basic
 * operations, so that GPU and CPU agree bit for bit. Binding the reference's
 * calls to those same functions holds the math library fixed, so that a
 * comparison of the reference's routines with the oracle's tests the
 * routines themselves: their branches, their operation order and their
 * use of the random numbers. rsqrtf becomes 1/sqrtf and powf(x, y)
 * exp(y log x), the oracle's forms.
 * Double-precision calls keep the host's double functions, as in CUDA. */
#ifndef GEGS_REF_MATH_H
#define GEGS_REF_MATH_H

#include <cmath>

extern "C" {
float gx_log(float x);
float gx_exp(float x);
void gx_sincos(float a, float *s, float *c);
}

static inline float ref_logf(float x) { return gx_log(x); }
static inline float ref_expf(float x) { return gx_exp(x); }
static inline void ref_sincosf(float a, float *s, float *c) { gx_sincos(a, s, c); }
static inline float ref_rsqrtf(float x) { return 1.0f / sqrtf(x); }

static inline float ref_log(float x) { return gx_log(x); }
static inline double ref_log(double x) { return std::log(x); }
static inline float ref_exp(float x) { return gx_exp(x); }
static inline double ref_exp(double x) { return std::exp(x); }
/* powf(x, y) as the oracle forms it, exp(y * log(x)) with its own log/exp */
static inline float ref_pow(float x, float y) { return gx_exp(gx_log(x) * y); }
static inline double ref_pow(double x, double y) { return std::pow(x, y); }
static inline float ref_cos(float x) { float s, c; gx_sincos(x, &s, &c); return c; }
static inline double ref_cos(double x) { return std::cos(x); }
static inline float ref_sin(float x) { float s, c; gx_sincos(x, &s, &c); return s; }
static inline double ref_sin(double x) { return std::sin(x); }

#define logf ref_logf
#define expf ref_expf
#define __logf ref_logf
#define __expf ref_expf
#define __sincosf ref_sincosf
#define sincosf ref_sincosf
#define rsqrtf ref_rsqrtf
#define log ref_log
#define exp ref_exp
#define cos ref_cos
#define pow ref_pow
#define powf ref_pow
#define sin ref_sin

#endif
