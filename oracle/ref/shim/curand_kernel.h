/* Host stand-in for <curand_kernel.h> (reference-pinning harness, test
 * infrastructure). The reference draws uniforms with curand_uniform on a
 * per-thread XORWOW state (random.cu:3-17). Here every draw replays the next
 * value of a stream the harness supplies -- the uniforms the oracle drew for
 * the same particle -- so the reference's routines and the oracle's see the
 * same random numbers in the order each of them asks for them. */
#ifndef GEGS_REF_SHIM_CURAND_KERNEL_H
#define GEGS_REF_SHIM_CURAND_KERNEL_H

#include "cuda_runtime.h"

struct curandState { int unused; };
typedef struct curandState curandStateXORWOW_t;

struct ref_uniform_stream {
    const float *u;    /* values to replay */
    unsigned n;        /* how many */
    unsigned next;     /* next to hand out */
    unsigned overrun;  /* draws asked for past the end (each returns 0.5) */
};
extern ref_uniform_stream g_ref_uniforms;

static inline float curand_uniform(curandState *) {
    ref_uniform_stream &s = g_ref_uniforms;
    if (s.next < s.n) return s.u[s.next++];
    s.overrun++;
    return 0.5f;
}

static inline void curand_init(unsigned long long, unsigned long long, unsigned long long, curandState *) {}

#endif
