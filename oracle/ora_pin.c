/* Probes that let the reference's own routines be compared with the oracle's
 * on identical inputs (the reference-pinning tests). The reference side runs
 * in oracle/ref (the reference's device sources compiled as host code, fed
 * the uniforms recorded here). Test infrastructure only (see ora_internal.h). */
#include <stdlib.h>
#include <string.h>
#include "ora_internal.h"
#include "gegs_oracle.h"

static void to_ora(const gegs_probe_particle *a, ora_particle *p)
{
    memset(p, 0, sizeof(*p));
    p->status = a->status;
    p->charge = a->charge;
    p->leafIndex = a->leafIndex;
    p->bank = a->bank;
    p->module = a->module;
    p->field = a->field;
    p->region = a->region;
    p->wt = a->wt; p->e = a->e;
    p->x = a->x; p->y = a->y; p->z = a->z;
    p->u = a->u; p->v = a->v; p->w = a->w;
    p->dnear = a->dnear;
    p->rng.hist_lo = a->hist;
}

static void from_ora(const ora_particle *p, gegs_probe_particle *a)
{
    memset(a, 0, sizeof(*a));
    a->status = p->status;
    a->charge = p->charge;
    a->leafIndex = p->leafIndex;
    a->bank = p->bank;
    a->module = p->module;
    a->field = p->field;
    a->region = p->region;
    a->wt = p->wt; a->e = p->e;
    a->x = p->x; a->y = p->y; a->z = p->z;
    a->u = p->u; a->v = p->v; a->w = p->w;
    a->dnear = p->dnear;
    a->hist = p->rng.hist_lo;
}

static void pin_ctx(ora_ctx *C, const gegs_physics *P, const gegs_scene *S, ora_region *reg, uint32_t nvox,
                    ora_stack *stk, int64_t *tally)
{
    memset(C, 0, sizeof(*C));
    C->P = P;
    C->S = S;
    C->reg = reg;
    C->nvox = nvox;
    C->seed_lo = (uint32_t)S->seed;
    C->seed_hi = (uint32_t)(S->seed >> 32);
    C->stk = stk;
    C->tally = tally;
}

void ora_probe_geom(const gegs_physics *P, const gegs_scene *S, uint32_t n, const gegs_probe_particle *in,
                    const float *t_in, uint32_t *far_region, float *far_t, gegs_probe_particle *far_out,
                    float *near_t)
{
    ora_ctx C;
    pin_ctx(&C, P, S, NULL, 0, NULL, NULL);
    for (uint32_t i = 0; i < n; i++) {
        ora_particle p;
        int ok;
        to_ora(&in[i], &p);
        float t = t_in[i];
        far_region[i] = ora_howfar(&C, &p, &t, &ok);
        far_t[i] = t;
        from_ora(&p, &far_out[i]);
        to_ora(&in[i], &p);
        float tp = 0.0f;
        ora_hownear(&C, &p, &tp, &ok);
        near_t[i] = tp;
    }
}

int ora_probe_stage(const gegs_physics *P, const gegs_scene *S, int stage, uint32_t n, const gegs_probe_particle *in,
                    float *urec, uint32_t ucap, uint32_t *un, gegs_probe_particle *out, uint32_t ocap, uint32_t *on,
                    uint32_t *dreg, float *de, uint32_t dcap, uint32_t *dn)
{
    uint32_t nvox = (uint32_t)S->nx * (uint32_t)S->ny * (uint32_t)S->nz;
    ora_region *reg = ora_build_regions(P, S, nvox);
    int64_t *tally = (int64_t *)calloc(nvox, sizeof(int64_t));
    ora_stack stk = {0, 0, 0};
    ora_ctx C;
    pin_ctx(&C, P, S, reg, nvox, &stk, tally);
    int err = 0;
    for (uint32_t i = 0; i < n; i++) {
        ora_particle p;
        to_ora(&in[i], &p);
        p.status = (uint8_t)stage;
        stk.n = 0;
        C.urec = urec + (size_t)i * ucap; C.urec_cap = ucap; C.urec_n = 0;
        C.drec_region = dreg + (size_t)i * dcap; C.drec_e = de + (size_t)i * dcap; C.drec_cap = dcap; C.drec_n = 0;
        C.error = 0;
        ora_run_particle(&C, &p);
        err |= C.error;
        un[i] = C.urec_n;
        dn[i] = C.drec_n;
        on[i] = (uint32_t)stk.n;
        for (size_t k = 0; k < stk.n && k < ocap; k++) from_ora(&stk.a[k], &out[(size_t)i * ocap + k]);
    }
    free(stk.a);
    free(tally);
    free(reg);
    return err;
}

void ora_probe_uphi(int which, float a, float b, gegs_probe_particle *pp, float *cs, float *u_drawn)
{
    ora_ctx C;
    memset(&C, 0, sizeof C);
    float u = 0.0f;
    C.urec = &u; C.urec_cap = 1;
    ora_particle p;
    to_ora(pp, &p);
    if (which == 21) uphi21(&C, a, b, &cs[0], &cs[1], &p, &p.rng);
    else if (which == 32) uphi32(a, b, cs[0], cs[1], &p);
    else uphi11(&C, a, &cs[2], &cs[3], &cs[0], &cs[1], &p, &p.rng);
    *u_drawn = u;
    from_ora(&p, pp);
}

int ora_capture(const gegs_physics *P, const gegs_scene *S, uint64_t h0, uint64_t h1, uint32_t every,
                gegs_probe_particle *cap, uint32_t cap_n, uint32_t *ncap)
{
    uint32_t nvox = (uint32_t)S->nx * (uint32_t)S->ny * (uint32_t)S->nz;
    ora_region *reg = ora_build_regions(P, S, nvox);
    int64_t *tally = (int64_t *)calloc(nvox, sizeof(int64_t));
    ora_stack stk = {0, 0, 0};
    ora_ctx C;
    pin_ctx(&C, P, S, reg, nvox, &stk, tally);
    uint64_t seen[ORA_NSTAGE] = {0};
    for (int s = 0; s < ORA_NSTAGE; s++) ncap[s] = 0;
    if (every == 0) every = 1;
    for (uint64_t h = h0; h < h1; h++) {
        ora_particle p;
        if (!ora_make_primary(S, h, &p)) { C.error |= 4; continue; }
        stk.n = 0;
        ora_push(&C, &p, p.status);
        while (stk.n > 0) {
            ora_particle q = stk.a[--stk.n];
            int s = q.status;
            if (s < ORA_NSTAGE && (seen[s]++ % every) == 0 && ncap[s] < cap_n) {
                from_ora(&q, &cap[(size_t)s * cap_n + ncap[s]]);
                cap[(size_t)s * cap_n + ncap[s]].hist = (uint32_t)h;
                ncap[s]++;
            }
            ora_run_particle(&C, &q);
        }
    }
    free(stk.a);
    free(tally);
    free(reg);
    return C.error;
}
