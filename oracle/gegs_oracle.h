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

/* One particle as the reference-pinning probes exchange it (same layout in
 * oracle/ref/ref_api.h): the reference's particle_t fields that the routines
 * read or write, plus the history index that keys the oracle's random stream. */
typedef struct gegs_probe_particle {
    uint32_t region;
    int8_t charge, leafIndex, bank;
    uint8_t module, field, status, pad0, pad1;
    float wt, e, x, y, z, u, v, w, dnear;
    uint32_t hist, pad2;
} gegs_probe_particle;

/* Geometry of n particles (ora_pin.c): howfar with step t_in[i] gives
 * far_region[i], the step far_t[i] and the particle after the call
 * (far_out[i]: leafIndex, bank, module may change); hownear gives near_t[i]. */
void ora_probe_geom(const gegs_physics *P, const gegs_scene *S, uint32_t n, const gegs_probe_particle *in,
                    const float *t_in, uint32_t *far_region, float *far_t, gegs_probe_particle *far_out,
                    float *near_t);

/* One pass of stage `stage` (the reference's kernel of that stack) for each of
 * n particles, each on its own random stream: per particle i, the uniforms
 * drawn (urec[i*ucap..], count un[i]), the particles pushed in push order
 * (out[i*ocap..], count on[i], status = stack), and every escore call
 * (dreg/de[i*dcap..], count dn[i]). Counts may exceed the capacities; only
 * what fits is written. Returns the oracle's error bits. */
int ora_probe_stage(const gegs_physics *P, const gegs_scene *S, int stage, uint32_t n, const gegs_probe_particle *in,
                    float *urec, uint32_t ucap, uint32_t *un, gegs_probe_particle *out, uint32_t ocap, uint32_t *on,
                    uint32_t *dreg, float *de, uint32_t dcap, uint32_t *dn);

/* uphi21 / uphi32 / uphi11 (utility.cu:94-218) on one particle: which = 21,
 * 32 or 11; a = costhe (21, 32) or theta (11), b = sinthe (21, 32); cs[0..1]
 * = cosphi, sinphi (in for 32, out for 21 and 11); cs[2..3] = costhe, sinthe
 * out for 11. Draws its uniform from the particle's stream (hist). */
void ora_probe_uphi(int which, float a, float b, gegs_probe_particle *p, float *cs, float *u_drawn);

/* Particles entering each stage in a run of histories [h0, h1): every k-th
 * particle taken by stage s is copied to cap[s*cap_n ..] (count ncap[s]), with
 * hist = its history index. Single thread. */
int ora_capture(const gegs_physics *P, const gegs_scene *S, uint64_t h0, uint64_t h1, uint32_t every,
                gegs_probe_particle *cap, uint32_t cap_n, uint32_t *ncap);
#endif
