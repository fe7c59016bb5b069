/* Host stand-in for <curand_kernel.h> (reference-pinning harness, test
 * infrastructure). The reference draws uniforms with curand_uniform on a
 * per-thread XORWOW state (random.cu:3-17). Here every draw replays the next
 * value of a stream the harness supplies -- the uniforms the oracle drew for
 * the same particle -- so the reference's routines and the oracle's see the
 * same random numbers in the order each of them asks for them. For a whole
 * transport run by the reference's kernels the draws come from a seeded
 * generator instead, independent of the oracle's and the GPU's streams. */
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
    int generate;      /* instead: draw from a SplitMix64 sequence (whole transports) */
    unsigned long long gen;
};
extern ref_uniform_stream g_ref_uniforms;

/* A uniform in (0, 1], the range of curand_uniform: the top 24 bits of a
 * SplitMix64 output (Steele, Lea and Flood 2014), plus one, times 2^-24. */
static inline float ref_generated_uniform(unsigned long long &x) {
    unsigned long long z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (float)((z >> 40) + 1) * (1.0f / 16777216.0f);
}

static inline float curand_uniform(curandState *) {
    ref_uniform_stream &s = g_ref_uniforms;
    if (s.generate) return ref_generated_uniform(s.gen);
    if (s.next < s.n) return s.u[s.next++];
    s.overrun++;
    return 0.5f;
}

static inline void curand_init(unsigned long long, unsigned long long, unsigned long long, curandState *) {}

#endif
