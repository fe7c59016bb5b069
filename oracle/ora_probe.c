/* Probes of single oracle routines on controlled inputs, for the project's
 * known-answer tests: the Compton sampler against the analytic Klein-Nishina
 * cross section, the photoelectron direction against the Sauter
 * distribution, the Moller sampler against the Moller cross section,
 * direction rotations against orthonormality, and the voxel walk of
 * howfar_phantom against an analytic ray traversal.
 * Test infrastructure only (see ora_internal.h). */
#include <stdlib.h>
#include <string.h>
#include "ora_internal.h"
#include "gegs_oracle.h"

static void probe_ctx(ora_ctx *C, ora_stack *stk, ora_region *reg, int64_t *tally, const gegs_physics *P,
                      const gegs_scene *S, uint64_t seed)
{
    memset(C, 0, sizeof(*C));
    C->P = P;
    C->S = S;
    C->reg = reg;
    C->nvox = 1;
    C->seed_lo = (uint32_t)seed;
    C->seed_hi = (uint32_t)(seed >> 32);
    C->tally = tally;
    C->stk = stk;
}

/* n Compton events of photons of `energy` along +z in one region of `medium`
 * with region `flags`; the scattered photon's energy and cosine (2 when none
 * was emitted) per event. */
int ora_probe_compton(const gegs_physics *P, int medium, uint32_t flags, float energy, uint32_t n, uint64_t seed,
                      float *e_out, float *cos_out)
{
    ora_region reg[VAC_AND_OTH + 1];
    memset(reg, 0, sizeof reg);
    reg[VAC_AND_OTH].med = (uint16_t)medium;
    reg[VAC_AND_OTH].flags = (uint16_t)flags;
    reg[VAC_AND_OTH].rhof = 1.0f;
    reg[VAC_AND_OTH].pcut = P->ap[medium];
    reg[VAC_AND_OTH].ecut = P->ae[medium];
    ora_stack stk = {0, 0, 0};
    int64_t tally[1] = {0};
    ora_ctx C;
    probe_ctx(&C, &stk, reg, tally, P, NULL, seed);
    for (uint32_t i = 0; i < n; i++) {
        ora_particle p;
        memset(&p, 0, sizeof p);
        p.e = energy;
        p.wt = 1.0f;
        p.region = VAC_AND_OTH;
        p.w = 1.0f;
        p.status = p_compton;
        p.rng.hist_lo = i;
        stk.n = 0;
        ora_compton(&C, &p);
        e_out[i] = 0.0f;
        cos_out[i] = 2.0f;
        for (size_t k = 0; k < stk.n; k++)
            if (stk.a[k].charge == 0) { e_out[i] = stk.a[k].e; cos_out[i] = stk.a[k].w; }
    }
    free(stk.a);
    return C.error;
}

/* n photoelectric events of photons of `energy` along +z in one region of
 * `medium` with region `flags` (cuts at 0): per event the photoelectron's
 * kinetic energy and direction cosine (2 when no electron left the event). */
int ora_probe_photo(const gegs_physics *P, int medium, uint32_t flags, float energy, uint32_t n, uint64_t seed,
                    float *ekin_out, float *cos_out)
{
    ora_region reg[VAC_AND_OTH + 1];
    memset(reg, 0, sizeof reg);
    reg[VAC_AND_OTH].med = (uint16_t)medium;
    reg[VAC_AND_OTH].flags = (uint16_t)flags;
    reg[VAC_AND_OTH].rhof = 1.0f;
    ora_stack stk = {0, 0, 0};
    int64_t tally[1] = {0};
    ora_ctx C;
    probe_ctx(&C, &stk, reg, tally, P, NULL, seed);
    for (uint32_t i = 0; i < n; i++) {
        ora_particle p;
        memset(&p, 0, sizeof p);
        p.e = energy;
        p.wt = 1.0f;
        p.region = VAC_AND_OTH;
        p.w = 1.0f;
        p.status = p_photo;
        p.rng.hist_lo = i;
        stk.n = 0;
        ora_photo(&C, &p);
        ekin_out[i] = 0.0f;
        cos_out[i] = 2.0f;
        for (size_t k = 0; k < stk.n; k++)
            if (stk.a[k].charge == -1) { ekin_out[i] = stk.a[k].e - P->prm; cos_out[i] = stk.a[k].w; }
    }
    free(stk.a);
    return C.error;
}

/* n Moller events of electrons of kinetic energy `ekin` along +z in one
 * region of `medium` (cuts of the region at 0, so both electrons leave the
 * event): per event the kinetic energy of the slower electron over ekin and
 * the cosine of its direction. Returns the oracle's error bits. */
int ora_probe_moller(const gegs_physics *P, int medium, float ekin, uint32_t n, uint64_t seed, float *frac_out,
                     float *cos_out)
{
    ora_region reg[VAC_AND_OTH + 1];
    memset(reg, 0, sizeof reg);
    reg[VAC_AND_OTH].med = (uint16_t)medium;
    reg[VAC_AND_OTH].rhof = 1.0f;
    ora_stack stk = {0, 0, 0};
    int64_t tally[1] = {0};
    ora_ctx C;
    probe_ctx(&C, &stk, reg, tally, P, NULL, seed);
    for (uint32_t i = 0; i < n; i++) {
        ora_particle p;
        memset(&p, 0, sizeof p);
        p.e = ekin + P->prm;
        p.charge = -1;
        p.wt = 1.0f;
        p.region = VAC_AND_OTH;
        p.w = 1.0f;
        p.status = e_moller;
        p.rng.hist_lo = i;
        stk.n = 0;
        ora_moller(&C, &p);
        frac_out[i] = -1.0f;
        cos_out[i] = 2.0f;
        float emin = 3.0e38f;
        for (size_t k = 0; k < stk.n; k++)
            if (stk.a[k].charge == -1 && stk.a[k].e < emin) {
                emin = stk.a[k].e;
                frac_out[i] = (stk.a[k].e - P->prm) / ekin;
                cos_out[i] = stk.a[k].w;
            }
    }
    free(stk.a);
    return C.error;
}

/* n rotations by uphi21 of random unit directions by random polar angles;
 * per rotation |d'|^2 - 1 and d.d' - cos(theta). */
void ora_probe_rotate(uint32_t n, uint64_t seed, float *norm_err, float *cos_err)
{
    ora_ctx C;
    probe_ctx(&C, NULL, NULL, NULL, NULL, NULL, seed);
    for (uint32_t i = 0; i < n; i++) {
        ora_particle p;
        memset(&p, 0, sizeof p);
        p.rng.hist_lo = i;
        float cz = 2.0f * ora_rng_uniform(&C, &p.rng) - 1.0f;
        float sz = sqrtf(1.0f - cz * cz);
        float s, c;
        gx_sincos_turns(ora_rng_uniform(&C, &p.rng), &s, &c);
        p.u = sz * c; p.v = sz * s; p.w = cz;
        float u0 = p.u, v0 = p.v, w0 = p.w;
        float costhe = 2.0f * ora_rng_uniform(&C, &p.rng) - 1.0f;
        float sinthe = sqrtf((1.0f - costhe) * (1.0f + costhe));
        float cphi, sphi;
        uphi21(&C, costhe, sinthe, &cphi, &sphi, &p, &p.rng);
        norm_err[i] = p.u * p.u + p.v * p.v + p.w * p.w - 1.0f;
        cos_err[i] = u0 * p.u + v0 * p.v + w0 * p.w - costhe;
    }
}

/* The voxel walk of howfar_phantom for one straight ray in the beam frame of
 * field `field`, starting in `region` (1 = outside the phantom): the regions
 * entered and the step lengths, up to maxn steps; returns the count. */
uint32_t ora_probe_walk(const gegs_physics *P, const gegs_scene *S, int field, uint32_t region, const float pos[3],
                        const float dir[3], uint32_t maxn, uint32_t *regions, float *steps)
{
    ora_ctx C;
    probe_ctx(&C, NULL, NULL, NULL, P, S, 0);
    ora_particle p;
    memset(&p, 0, sizeof p);
    p.field = (uint8_t)field;
    p.module = GEGS_M_PHANTOM;
    p.region = region;
    p.x = pos[0]; p.y = pos[1]; p.z = pos[2];
    p.u = dir[0]; p.v = dir[1]; p.w = dir[2];
    uint32_t k = 0;
    while (k < maxn) {
        float t = 1e9f;
        uint32_t r = howfar_phantom(&C, &p, &t);
        regions[k] = r;
        steps[k] = t;
        k++;
        if (r == VACUUM_REG || t >= 1e9f) break;
        p.x = p.x + p.u * t;
        p.y = p.y + p.v * t;
        p.z = p.z + p.w * t;
        p.region = r;
    }
    return k;
}
