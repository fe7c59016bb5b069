/* Oracle driver: builds the region table, turns phase-space records into
 * primaries (CUDA_EGS.cu:40-158) and runs histories one by one with a LIFO
 * particle stack.  Test infrastructure only (see ora_internal.h).
 * Exported C entry points are declared in gegs_oracle.h. */
#include <stdlib.h>
#include <string.h>
#include "ora_internal.h"
#include "gegs_oracle.h"
#ifdef _OPENMP
#include <omp.h>
#endif

size_t ora_sizeof_physics(void) { return sizeof(gegs_physics); }
size_t ora_sizeof_scene(void) { return sizeof(gegs_scene); }
size_t ora_sizeof_field(void) { return sizeof(gegs_field); }

float ora_log(float x) { return gx_log(x); }
float ora_exp(float x) { return gx_exp(x); }
void ora_sincos_turns(float t, float *s, float *c) { gx_sincos_turns(t, s, c); }
uint32_t ora_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1, int lane)
{
    return ora_philox_word(c0, c1, c2, c3, k0, k1, lane);
}

ora_region *ora_build_regions(const gegs_physics *P, const gegs_scene *S, uint32_t nvox)
{
    ora_region *reg = (ora_region *)calloc((size_t)nvox + VAC_AND_OTH, sizeof(ora_region));
    reg[0].med = VACUUM;
    for (int i = 1; i < VAC_AND_OTH; i++) {
        int med = S->other_med[i - 1];
        if (med < 0) med = S->other_med[0];
        reg[i].med = (uint16_t)med;
        reg[i].flags = (uint16_t)S->region_flags;
        reg[i].rhof = 1.0f;
        reg[i].pcut = P->ap[med];
        reg[i].ecut = P->ae[med];
    }
    for (uint32_t v = 0; v < nvox; v++) {
        ora_region *r = &reg[v + VAC_AND_OTH];
        uint16_t med = S->voxel_med[v];
        r->med = med;
        if (med == VACUUM) continue;
        r->flags = (uint16_t)S->region_flags;
        r->rhof = S->voxel_rhof[v];
        r->pcut = P->ap[med];
        r->ecut = P->ae[med];
    }
    return reg;
}

/* history index -> primary particle (CUDA_EGS.cu:52-131) */
int ora_make_primary(const gegs_scene *S, uint64_t h, ora_particle *p)
{
    int f;
    for (f = 0; f < S->nfields; f++)
        if (h >= S->fields[f].hist_begin && h < S->fields[f].hist_end) break;
    if (f == S->nfields) return 0;
    const gegs_field *F = &S->fields[f];
    uint64_t j = (h - F->hist_begin) / (uint64_t)(F->nrepeat + 1);
    const gegs_phsp_record *rec = &S->phsp[j % S->nphsp];
    memset(p, 0, sizeof(*p));
    int q;
    if (rec->latch & 0x40000000u) q = -1;
    else if (rec->latch & 0x20000000u) q = 1;
    else q = 0;
    float w2 = 1.0f - rec->u * rec->u - rec->v * rec->v;
    float w = sqrtf(w2 > 0.0f ? w2 : 0.0f);
    float wt = rec->wt;
    if (wt < 0.0f) { w = -w; wt = -wt; }
    p->charge = (int8_t)q;
    p->e = rec->e < 0.0f ? -rec->e : rec->e;
    p->wt = wt;
    p->region = 0;
    p->leafIndex = OUTMLC;
    p->bank = -1;
    p->module = (uint8_t)S->module_order[0];
    p->field = (uint8_t)f;
    p->x = rec->x;
    p->y = rec->y;
    p->z = S->z_phsp;
    p->u = rec->u;
    p->v = rec->v;
    p->w = w;
    p->dnear = INFI_DIST;
    /* beamlet fluence weight (no counterpart in the reference): the bixel of the
     * isocentre plane on the primary's straight line; same arithmetic as the GPU */
    if (S->bl_nx > 0 && w > 0.0f) {
        float t = (S->source_to_isocenter - S->z_phsp) / w;
        float xi = rec->x + rec->u * t, yi = rec->y + rec->v * t;
        float fx = (xi - S->bl_x0) / S->bl_dx, fy = (yi - S->bl_y0) / S->bl_dy;
        if (fx >= 0.0f && fy >= 0.0f && fx < (float)S->bl_nx && fy < (float)S->bl_ny) {
            int b = f * S->bl_nx * S->bl_ny + (int)fy * S->bl_nx + (int)fx;
            if (S->bl_weight) p->wt = wt * S->bl_weight[b];
        }
    }
    p->rng.hist_lo = (uint32_t)h;
    p->rng.hist_hi = (uint32_t)(h >> 32);
    p->status = q == 0 ? p_photon_step : e_electron_step;
    return 1;
}

void ora_run_particle(ora_ctx *C, ora_particle *p)
{
    C->counts[p->status]++;
    C->cur_stage = p->status;
    ora_trace(C, 1u, p->status, p);
    switch (p->status) {
    case p_photon_step: ora_photon(C, p); break;
    case p_compton: ora_compton(C, p); break;
    case p_photo: ora_photo(C, p); break;
    case p_rayleigh: ora_rayleigh(C, p); break;
    case p_pair: ora_pair(C, p); break;
    case e_electron_step: ora_electron(C, p); break;
    case e_moller: ora_moller(C, p); break;
    case e_brems: ora_brems(C, p); break;
    case e_bhabha: ora_bhabha(C, p); break;
    case e_annih: ora_annih(C, p); break;
    default: C->error |= 2; break;
    }
}

static ora_trace_rec *g_trace;
static uint32_t g_trace_cap, g_trace_n;

void ora_set_trace(void *buf, uint32_t cap) { g_trace = (ora_trace_rec *)buf; g_trace_cap = cap; g_trace_n = 0; }
uint32_t ora_trace_count(void) { return g_trace_n; }

int ora_run(const gegs_physics *P, const gegs_scene *S, uint64_t h0, uint64_t h1, int nthreads,
            int64_t *tally, ora_stats *stats)
{
    if (g_trace) nthreads = 1;
    uint32_t nvox = (uint32_t)S->nx * (uint32_t)S->ny * (uint32_t)S->nz;
    ora_region *reg = ora_build_regions(P, S, nvox);
    ora_stats tot;
    memset(&tot, 0, sizeof(tot));
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    int err = 0;
#pragma omp parallel
    {
        ora_stack stk = {0, 0, 0};
        ora_ctx C;
        memset(&C, 0, sizeof(C));
        C.P = P;
        C.S = S;
        C.reg = reg;
        C.nvox = nvox;
        C.seed_lo = (uint32_t)S->seed;
        C.seed_hi = (uint32_t)(S->seed >> 32);
        C.stk = &stk;
        C.trace = g_trace;
        C.trace_cap = g_trace_cap;
        C.trace_n = g_trace_n;
        int64_t *loc = (int64_t *)calloc(nvox, sizeof(int64_t));
        C.tally = loc;
#pragma omp for schedule(dynamic, 64)
        for (int64_t h = (int64_t)h0; h < (int64_t)h1; h++) {
            ora_particle p;
            if (!ora_make_primary(S, (uint64_t)h, &p)) { C.error |= 4; continue; }
            stk.n = 0;
            ora_push(&C, &p, p.status);
            while (stk.n > 0) {
                ora_particle q = stk.a[--stk.n];
                ora_run_particle(&C, &q);
            }
        }
#pragma omp critical
        {
            for (uint32_t v = 0; v < nvox; v++) tally[v] += loc[v];
            for (int i = 0; i < ORA_NSTAGE; i++) tot.counts[i] += C.counts[i];
            tot.steps_photon += C.steps_photon;
            tot.steps_electron += C.steps_electron;
            tot.e_escaped += C.e_escaped;
            for (int i = 0; i < ORA_NSTAGE; i++)
                for (int k = 0; k < 3; k++) tot.cnt[i][k] += C.cnt[i][k];
            err |= C.error;
            if (g_trace) g_trace_n = C.trace_n;
        }
        free(loc);
        free(stk.a);
    }
    free(reg);
    tot.error = err;
    if (stats) *stats = tot;
    return err;
}
