/* C entry points of the CPU oracle (test infrastructure only; see ora_internal.h). */
#ifndef GEGS_ORACLE_H
#define GEGS_ORACLE_H

#include <stdint.h>
#include <stddef.h>
#include "../include/gegs_physics.h"
#include "../include/gegs_scene.h"

typedef struct ora_stats {
    uint64_t counts[10];          /* particles processed per stage (photon .. annih) */
    uint64_t steps_photon, steps_electron;
    double e_escaped;             /* energy scored to regions 0..5 (not tallied) */
    int32_t error;
    int32_t pad_;
    uint64_t cnt[10][3];   /* per stage: region records read, tally updates, float2 table reads */
} ora_stats;

size_t ora_sizeof_physics(void);
size_t ora_sizeof_scene(void);
size_t ora_sizeof_field(void);
float ora_log(float x);
float ora_exp(float x);
void ora_sincos_turns(float t, float *s, float *c);
uint32_t ora_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1, int lane);

/* Debug trace of pushes (kind 0) and consumed particles (kind 1); forces one thread. */
void ora_set_trace(void *buf, uint32_t cap);
uint32_t ora_trace_count(void);

/* Run histories [h0, h1); adds the int64 energy tally (MeV * 2^30) into `tally`. */
int ora_run(const gegs_physics *P, const gegs_scene *S, uint64_t h0, uint64_t h1, int nthreads,
            int64_t *tally, ora_stats *stats);

/* Known-answer probes (ora_probe.c). */
int ora_probe_compton(const gegs_physics *P, int medium, uint32_t flags, float energy, uint32_t n, uint64_t seed,
                      float *e_out, float *cos_out);
int ora_probe_photo(const gegs_physics *P, int medium, uint32_t flags, float energy, uint32_t n, uint64_t seed,
                    float *ekin_out, float *cos_out);
int ora_probe_moller(const gegs_physics *P, int medium, float ekin, uint32_t n, uint64_t seed, float *frac_out,
                     float *cos_out);
void ora_probe_rotate(uint32_t n, uint64_t seed, float *norm_err, float *cos_err);
uint32_t ora_probe_walk(const gegs_physics *P, const gegs_scene *S, int field, uint32_t region, const float pos[3],
                        const float dir[3], uint32_t maxn, uint32_t *regions, float *steps);
#endif
