/* Oracle: counter-based RNG, transcendental functions, scoring and direction
 * rotation.  Test infrastructure only (see ora_internal.h). */
#include <string.h>
#include <stdlib.h>
#include "ora_internal.h"

/* ---- Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) ------------------- */
#define PHILOX_M0 0xD2511F53u
#define PHILOX_M1 0xCD9E8D57u
#define PHILOX_W0 0x9E3779B9u
#define PHILOX_W1 0xBB67AE85u

void ora_philox4(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; r++) {
        if (r) { k0 += PHILOX_W0; k1 += PHILOX_W1; }
        uint64_t p0 = (uint64_t)PHILOX_M0 * c0;
        uint64_t p1 = (uint64_t)PHILOX_M1 * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        uint32_t n1 = (uint32_t)p1;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        uint32_t n3 = (uint32_t)p0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

uint32_t ora_philox_word(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1, int lane)
{
    uint32_t c[4] = {c0, c1, c2, c3}, k[2] = {k0, k1}, o[4];
    ora_philox4(c, k, o);
    return o[lane & 3];
}

uint32_t ora_rng_u32(ora_ctx *C, ora_rng *r)
{
    uint32_t b = r->ctr >> 2;
    if (r->blk != b + 1u) {
        uint32_t c[4] = {b, r->sid_lo, r->sid_hi, r->hist_lo};
        uint32_t k[2] = {C->seed_lo, C->seed_hi + r->hist_hi};
        ora_philox4(c, k, r->buf);
        r->blk = b + 1u;
    }
    uint32_t x = r->buf[r->ctr & 3u];
    r->ctr++;
    return x;
}

float ora_rng_uniform(ora_ctx *C, ora_rng *r)
{
    uint32_t x = ora_rng_u32(C, r);
    float u = (float)((x >> 8) + 1u) * 5.9604644775390625e-08f;   /* 2^-24 */
    if (C && C->urec) {
        if (C->urec_n < C->urec_cap) C->urec[C->urec_n] = u;
        C->urec_n++;
    }
    return u;
}

void ora_rng_spawn(ora_ctx *C, ora_rng *parent, ora_rng *child)
{
    uint32_t lo = ora_rng_u32(C, parent);
    uint32_t hi = ora_rng_u32(C, parent);
    child->hist_lo = parent->hist_lo;
    child->hist_hi = parent->hist_hi;
    child->sid_lo = lo;
    child->sid_hi = hi;
    child->ctr = 0;
    child->blk = 0;
}

/* ---- transcendental functions from IEEE basic operations ----------------
 * log: x = 2^k m, m in [sqrt(1/2), sqrt(2)), s = (m-1)/(m+1),
 *      ln m = 2 atanh(s) = 2s + 2s^3/3 + ... + 2s^11/11 (Taylor series),
 *      ln 2 split Cody-Waite style so k*LN2_HI is exact.
 * exp: k = floor(x log2 e + 1/2), r = x - k ln2 (Cody & Waite 1980),
 *      e^r by its Taylor series to r^8/8!, scaled by 2^k from the bit pattern.
 * sincos of 2*pi*t: quarter-turn reduction (exact), Taylor series on
 *      [-pi/4, pi/4] to degree 9 (sin) / 8 (cos), quadrant swap.        */
static inline uint32_t f2u(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static inline float u2f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }

#define GX_LN2_HI 0.693145751953125f
#define GX_LN2_LO 1.42860682030941723212e-06f
#define GX_LOG2E 1.44269502162933349609f

float gx_log(float x)
{
    if (!(x > 0.0f)) return x == 0.0f ? -INFINITY : NAN;
    if (x == INFINITY) return x;
    uint32_t ix = f2u(x);
    int k = 0;
    if (ix < 0x00800000u) { x = x * 33554432.0f; ix = f2u(x); k = -25; }
    k += (int)(ix >> 23) - 127;
    uint32_t im = (ix & 0x007fffffu) | 0x3f800000u;
    if (im > 0x3fb504f3u) { im -= 0x00800000u; k += 1; }
    float m = u2f(im);
    float f = m - 1.0f;
    float s = f / (2.0f + f);
    float z = s * s;
    float R = z * (0.666666686534881591796875f + z * (0.4000000059604644775390625f
              + z * (0.2857142984867095947265625f + z * (0.2222222238779067993164063f
              + z * 0.1818181872367858886718750f))));
    float logm = 2.0f * s + s * R;
    float kf = (float)k;
    return kf * GX_LN2_HI + (kf * GX_LN2_LO + logm);
}

float gx_exp(float x)
{
    if (x != x) return x;
    if (x > 88.7228394f) return INFINITY;
    if (x < -103.972084f) return 0.0f;
    float kf = floorf(x * GX_LOG2E + 0.5f);
    int k = (int)kf;
    float r = (x - kf * GX_LN2_HI) - kf * GX_LN2_LO;
    float p = 1.0f + r * (1.0f + r * (0.5f + r * (0.16666667163372039794921875f
              + r * (0.041666667908430099487304688f + r * (0.0083333337679505348205566406f
              + r * (0.0013888889225199818611145020f + r * (0.00019841270113829523324966431f
              + r * 2.4801587642286904156208038e-05f)))))));
    if (k > 127) { p = p * 1.7014118346046923e+38f; k -= 127; }
    if (k < -126) { p = p * 5.42101086242752217e-20f; k += 64; }   /* 2^-64 */
    return p * u2f((uint32_t)(k + 127) << 23);
}

void gx_sincos_turns(float t, float *s, float *c)
{
    float t4 = t * 4.0f;
    float q = floorf(t4 + 0.5f);
    float f = t4 - q;
    float a = f * 1.57079637050628662109375f;
    float a2 = a * a;
    float sn = a + a * a2 * (-0.16666667163372039794921875f + a2 * (0.0083333337679505348205566406f
               + a2 * (-0.00019841270113829523324966431f + a2 * 2.7557319224737625e-06f)));
    float cs = 1.0f + a2 * (-0.5f + a2 * (0.041666667908430099487304688f
               + a2 * (-0.0013888889225199818611145020f + a2 * 2.4801587642286904156208038e-05f)));
    int iq = ((int)(q - 4.0f * floorf(q * 0.25f))) & 3;
    switch (iq) {
    case 0: *s = sn; *c = cs; break;
    case 1: *s = cs; *c = -sn; break;
    case 2: *s = -sn; *c = -cs; break;
    default: *s = -cs; *c = sn; break;
    }
}

void gx_sincos(float a, float *s, float *c)
{
    gx_sincos_turns(a * 0.15915493667125701904296875f, s, c);
}

/* ---- scoring (scoring.cu:14-26) with an int64 fixed-point tally ---------- */
void ora_escore(ora_ctx *C, uint32_t region, float energy)
{
    if (C->drec_region) {
        if (C->drec_n < C->drec_cap) { C->drec_region[C->drec_n] = region; C->drec_e[C->drec_n] = energy; }
        C->drec_n++;
    }
    if (region < VAC_AND_OTH) { C->e_escaped += (double)energy; return; }
    C->cnt[C->cur_stage][1]++;
    C->tally[region - VAC_AND_OTH] += (int64_t)llrintf(energy * 1073741824.0f);
}

void ora_trace(ora_ctx *C, uint32_t kind, int stage, const ora_particle *p)
{
    if (!C->trace) return;
    uint32_t i = C->trace_n++;
    if (i >= C->trace_cap) return;
    ora_trace_rec *t = &C->trace[i];
    t->kind_stage = kind | ((uint32_t)stage << 8);
    t->hist_lo = p->rng.hist_lo; t->sid_lo = p->rng.sid_lo; t->sid_hi = p->rng.sid_hi; t->ctr = p->rng.ctr;
    t->e = p->e; t->x = p->x; t->region = p->region;
}

void ora_push(ora_ctx *C, const ora_particle *p, int status)
{
    ora_trace(C, 0u, status, p);
    ora_stack *s = C->stk;
    if (s->n == s->cap) {
        s->cap = s->cap ? 2 * s->cap : 256;
        s->a = (ora_particle *)realloc(s->a, s->cap * sizeof(ora_particle));
    }
    s->a[s->n] = *p;
    s->a[s->n].status = (uint8_t)status;
    s->n++;
}

/* Push a particle created by an interaction: it gets a child stream of the
 * interaction's stream `parent`. */
void ora_spawn(ora_ctx *C, ora_rng *parent, ora_particle *child, int status)
{
    ora_rng_spawn(C, parent, &child->rng);
    ora_push(C, child, status);
}

/* ---- direction rotation (utility.cu:94-218) ------------------------------ */
static void rotate(float costhe, float sinthe, float cosphi, float sinphi, ora_particle *p)
{
    float A = p->u, B = p->v, Cc = p->w;
    float sinps2 = A * A + B * B;
    if (sinps2 < SMALL_POLAR_ANGLE_THRESHOLD) {
        p->u = sinthe * cosphi;
        p->v = sinthe * sinphi;
        p->w = Cc * costhe;
    } else {
        float sinpsi_i = 1.0f / sqrtf(sinps2);
        float us = sinthe * cosphi;
        float vs = sinthe * sinphi;
        float sindel = B * sinpsi_i;
        float cosdel = A * sinpsi_i;
        p->u = Cc * cosdel * us - sindel * vs + A * costhe;
        p->v = Cc * sindel * us + cosdel * vs + B * costhe;
        p->w = -us / sinpsi_i + Cc * costhe;
    }
}

void uphi21(ora_ctx *C, float costhe, float sinthe, float *cosphi, float *sinphi, ora_particle *p, ora_rng *r)
{
    float r1 = ora_rng_uniform(C, r);
    float phi = 2.0f * 3.14159265f * r1;              /* utility.cu:99-100 */
    gx_sincos(phi, sinphi, cosphi);
    rotate(costhe, sinthe, *cosphi, *sinphi, p);
}

void uphi32(float costhe, float sinthe, float cosphi, float sinphi, ora_particle *p)
{
    rotate(costhe, sinthe, cosphi, sinphi, p);
}

void uphi11(ora_ctx *C, float theta, float *costhe, float *sinthe, float *cosphi, float *sinphi, ora_particle *p, ora_rng *r)
{
    float r1 = ora_rng_uniform(C, r);
    gx_sincos(theta, sinthe, costhe);
    float phi = 2.0f * 3.14159265f * r1;              /* utility.cu:190-191 */
    gx_sincos(phi, sinphi, cosphi);
    rotate(*costhe, *sinthe, *cosphi, *sinphi, p);
}
