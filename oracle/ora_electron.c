/* Oracle: condensed-history electron/positron transport and discrete
 * electron interactions.  Test infrastructure only.
 *   ora_electron    electron.cu:888-2622  (ELECTR; PRESTA-I, spin off)
 *   msdist_pI       electron.cu:618-882
 *   mscat / sscat   electron.cu:77-279    (screened Rutherford GS sampling)
 *   ora_moller      moller.cu:16-210, eii_sample.cu:4-96
 *   ora_brems       brems.cu:36-308
 *   ora_bhabha      bhabha.cu:12-173
 *   ora_annih       annih.cu:16-207
 * Guards that the reference lacks (identical on the GPU):
 *   - mscat with lambda > LAMBMAX_MS returns no deflection (the reference
 *     leaves cos/sin unset), table indices are clamped when U == 1 exactly;
 *   - sqrt arguments of the Moller/EII kinematics are clamped at 0;
 *   - open rejection loops are capped at ORA_LOOP_CAP iterations. */
#include "ora_internal.h"

#define ORA_LOOP_CAP 1000

static inline float U(ora_ctx *C, ora_rng *r) { return ora_rng_uniform(C, r); }

static _Thread_local uint64_t *g_table_counter;   /* electron-stage table-read counter of the running thread */
static inline float ev2(const float *t, float x) { if (g_table_counter) (*g_table_counter)++; return t[0] + t[1] * x; }

static void box_phi(ora_ctx *C, ora_rng *r, float *cphi, float *sphi)
{
    float xphi, yphi, rhophi2;
    int n = 0;
    do {
        xphi = U(C, r);
        xphi = 2.0f * xphi - 1.0f;
        yphi = U(C, r);
        rhophi2 = xphi * xphi + yphi * yphi;
    } while (rhophi2 > 1.0f && ++n < ORA_LOOP_CAP);
    rhophi2 = 1.0f / rhophi2;
    *cphi = (xphi * xphi - yphi * yphi) * rhophi2;
    *sphi = 2.0f * xphi * yphi * rhophi2;
}

static void mscat(ora_ctx *C, float lambda, float chia2, float q1, float *cost, float *sint, ora_rng *r)
{
    const gegs_physics *P = C->P;
    if (lambda <= 13.8) {
        float sprob = U(C, r);
        float explambda = gx_exp(-lambda);
        if (sprob < explambda) { *cost = 1.0f; *sint = 0.0f; return; }
        float wsum = (1.0f + lambda) * explambda;
        if (sprob < wsum) {
            float xi = U(C, r);
            xi = 2.0f * chia2 * xi / (1.0f - xi + chia2);
            *cost = 1.0f - xi;
            *sint = sqrtf(xi * (2.0f - xi));
            return;
        }
        if (lambda <= 1.0f) {
            float wprob = explambda;
            wsum = explambda;
            *cost = 1.0f;
            *sint = 0.0f;
            int icount = 0;
            do {
                icount = icount + 1;
                if (icount > 20) break;
                wprob = wprob * lambda / (float)icount;
                wsum = wsum + wprob;
                float xi = U(C, r);
                xi = 2.0f * chia2 * xi / (1.0f - xi + chia2);
                float cosz = 1.0f - xi;
                float sinz = xi * (2.0f - xi);
                if (sinz > 1.0e-20) {
                    sinz = sqrtf(sinz);
                    xi = U(C, r);
                    float phi = xi * 6.2831853;
                    float sp, cp;
                    gx_sincos(phi, &sp, &cp);
                    *cost = *cost * cosz - *sint * sinz * cp;
                    *sint = (float)sqrt(fmax(0.0, (double)((1.0f - *cost) * (1.0f + *cost))));
                }
            } while (wsum <= sprob);
            return;
        }
    }
    if (lambda <= LAMBMAX_MS) {
        float llmbda = gx_log(lambda);
        float ai = llmbda * P->dllambi;
        int msi = (int)ai;
        ai = ai - (float)msi;
        float xi = U(C, r);
        if (xi < ai) msi = msi + 1;
        if (msi > MAXL_MS) msi = MAXL_MS;
        int msj;
        if (q1 < QMIN_MS) msj = 0;
        else if (q1 < QMAX_MS) {
            float aj = q1 * P->dqmsi;
            msj = (int)aj;
            aj = aj - (float)msj;
            xi = U(C, r);
            if (xi < aj) msj = msj + 1;
        } else msj = MAXQ_MS;
        float omega2;
        if (llmbda < 2.2299)
            omega2 = chia2 * (lambda + 4) * (1.347006 + llmbda * (0.209364 - llmbda * (0.45525 - llmbda * (0.50142 - 0.081234 * llmbda))));
        else
            omega2 = chia2 * (lambda + 4) * (-2.77164 + llmbda * (2.94874 - llmbda * (0.1535754 - llmbda * 0.00552888)));
        xi = U(C, r);
        float ak = xi * (float)MAXU_MS;
        int msk = (int)ak;
        ak = ak - (float)msk;
        if (msk > MAXU_MS - 1) { msk = MAXU_MS - 1; ak = 1.0f; }
        int idx = (msk * MAXQ_MS_PLUS_1 + msj) * MAXL_MS_PLUS_1 + msi;
        if (ak > P->wms_array[idx]) {
            msk = P->ims_array[idx];
            idx = (msk * MAXQ_MS_PLUS_1 + msj) * MAXL_MS_PLUS_1 + msi;
        }
        float a = P->fms_array[idx];
        float u = P->ums_array[idx];
        float du = P->ums_array[((msk + 1) * MAXQ_MS_PLUS_1 + msj) * MAXL_MS_PLUS_1 + msi] - u;
        xi = U(C, r);
        if (fabsf(a) < 0.2) {
            float x1 = 0.5 * (1 - xi) * a;
            u = u + xi * du * (1.0f + x1 * (1.0f - xi * a));
        } else
            u = u - du / a * (1.0f - sqrtf(1.0f + xi * a * (2.0f + a)));
        xi = omega2 * u / (1 + 0.5 * omega2 - u);
        if (xi > 1.99999) xi = 1.99999;
        *cost = 1.0f - xi;
        *sint = sqrtf(xi * (2.0f - xi));
        return;
    }
    *cost = 1.0f;
    *sint = 0.0f;
}

static void sscat(ora_ctx *C, float chia2, float *cost, float *sint, ora_rng *r)
{
    float xi = U(C, r);
    xi = 2.0f * chia2 * xi / (1.0f - xi + chia2);
    *cost = 1.0f - xi;
    *sint = sqrtf(xi * (2.0f - xi));
}

static void msdist_pI(ora_ctx *C, float eloss, float tustep, ora_particle *p0, float *ustep, const ora_region *rd, ora_rng *r)
{
    const gegs_physics *P = C->P;
    unsigned medium = rd->med;
    float e0 = p0->e - P->rm;
    float blccc = P->blcc[medium];
    float xcccc = P->xcc[medium];
    float e = e0 - 0.5 * eloss;
    float p2 = e * (e + P->rmt2);
    float chia2 = xcccc / p2 / (4.0f * blccc);
    float beta2 = p2 / (p2 + P->rmsq);
    float lambda = tustep * rd->rhof * blccc / beta2;
    float factor = 1 / (1 + 0.9784671 * e);
    float epsilon = eloss / e0;
    epsilon = epsilon / (1 - 0.5 * epsilon);
    float temp = 0.25 * (1 - factor * (1 - 0.333333 * factor)) * epsilon * epsilon;
    lambda = lambda * (1.0f + temp);
    lambda = lambda / (1.0f + chia2);
    float chilog = gx_log(1.0f + 1.0f / chia2);
    float q1 = 2.0f * chia2 * (chilog * (1.0f + chia2) - 1.0f);
    float xi = q1 * lambda;
    float ws, sint;
    mscat(C, lambda, chia2, xi, &ws, &sint, r);
    float cphi, sphi;
    box_phi(C, r, &cphi, &sphi);
    float us = sint * cphi;
    float vs = sint * sphi;
    float z, rr, r2, z2, r2max;
    if (xi < 0.1) z = 1 - xi * (0.5 - xi * (0.166666667 - 0.041666667 * xi));
    else z = (1.0f - gx_exp(-xi)) / xi;
    rr = 0.5 * sint;
    r2 = rr * rr;
    z2 = z * z;
    r2max = 1.0f - z2;
    if (r2max < r2) { r2 = r2max; rr = sqrtf(r2); }
    float ut = rr * cphi, vt = rr * sphi, wt = z;
    *ustep = sqrtf(z2 + r2) * tustep;
    float sint02 = p0->u * p0->u + p0->v * p0->v;
    if (sint02 > 1e-20) {
        float sint0 = sqrtf(sint02);
        float cphi0 = p0->u / sint0;
        float sphi0 = p0->v / sint0;
        float u2p = p0->w * us + sint0 * ws;
        ws = p0->w * ws - sint0 * us;
        us = u2p * cphi0 - vs * sphi0;
        vs = u2p * sphi0 + vs * cphi0;
        u2p = p0->w * ut + sint0 * wt;
        wt = p0->w * wt - sint0 * ut;
        ut = u2p * cphi0 - vt * sphi0;
        vt = u2p * sphi0 + vt * cphi0;
    } else {
        wt = p0->w * wt;
        ws = p0->w * ws;
    }
    p0->x = p0->x + tustep * ut;
    p0->y = p0->y + tustep * vt;
    p0->z = p0->z + tustep * wt;
    p0->u = us;
    p0->v = vs;
    p0->w = ws;
}

/* dE/dx at the midpoint of a sub-step (the $CALCULATE-TSTEP / $COMPUTE-RANGE pattern) */
static float range_piece(const gegs_physics *P, int qel, unsigned medium, int lel, float elk_a, float elk_b, float e_hi, float fedep)
{
    float elktmp = 0.5 * (elk_a + elk_b + 0.25 * fedep * fedep * (1 + fedep * (1 + 0.875 * fedep)));
    if (g_table_counter) (*g_table_counter)++;
    const float *d = P->dedx[qel * MXEKE * MXMED + medium * MXEKE + lel - 1];
    float dedxmid = d[0] + d[1] * elktmp;
    dedxmid = 1.0f / dedxmid;
    float aux = d[1] * dedxmid;
    float temp = fedep / (2.0f - fedep);
    aux = aux * (1.0f + 2.0f * aux) * temp * temp / 6.0f;
    return fedep * e_hi * dedxmid * (1.0f + aux);
}

/* $COMPUTE-ELOSS-G */
static float compute_eloss(const gegs_physics *P, int qel, unsigned medium, float step, float range, float rhof,
                           float eke_val, float elke, int lelke)
{
    const float *ex = P->eke01[medium];
    float de;
    float tuss = range - P->range_ep[(medium * MXEKE + lelke - 1) * 2 + qel] / rhof;
    if (tuss >= step) {
        const float *d = P->dedx[qel * MXEKE * MXMED + medium * MXEKE + lelke - 1];
        float dedxmid = d[0] + d[1] * elke;
        float aux = d[1] / dedxmid;
        de = dedxmid * step * rhof;
        float fedep = de / eke_val;
        de = de * (1 - 0.5 * fedep * aux * (1 - 0.333333 * fedep * (aux - 1 - 0.25 * fedep * (2 - aux * (4 - aux)))));
    } else {
        int lelktmp = lelke;
        tuss = (range - step) * rhof;
        if (tuss <= 0.0f) de = eke_val - P->te[medium] * 0.99;
        else {
            while (lelktmp > 1 && tuss < P->range_ep[(medium * MXEKE + lelktmp - 1) * 2 + qel]) lelktmp = lelktmp - 1;
            float elktmp = ((float)(lelktmp + 1) - ex[0]) / ex[1];
            float eketmp = P->e_array[medium * MXEKE + lelktmp];
            tuss = (P->range_ep[(medium * MXEKE + lelktmp) * 2 + qel] - tuss) / rhof;
            const float *d = P->dedx[qel * MXEKE * MXMED + medium * MXEKE + lelktmp - 1];
            float dedxmid = d[0] + d[1] * elktmp;
            float aux = d[1] / dedxmid;
            de = dedxmid * tuss * rhof;
            float fedep = de / eketmp;
            de = de * (1 - 0.5 * fedep * aux * (1 - 0.333333 * fedep * (aux - 1 - 0.25 * fedep * (2 - aux * (4 - aux)))));
            de = de + eke_val - eketmp;
        }
    }
    return de;
}

static void e_discard_below_cut(ora_ctx *C, ora_particle *p, const ora_region *rd)
{
    ora_escore(C, p->region, (p->e - C->P->prm) * p->wt);
    if (p->charge > 0) {
        /* the annihilation photons are spawned from the positron's stream: keep
         * that stream in its own variable, the spawns overwrite p->rng */
        ora_rng r = p->rng;
        ora_annih_at_rest(C, p, rd, &r);
    }
}

void ora_electron(ora_ctx *C, ora_particle *p)
{
    g_table_counter = &C->cnt[e_electron_step][2];
    const gegs_physics *P = C->P;
    const float rm = P->rm, prm = P->prm, rmt2 = P->rmt2, rmsq = P->rmsq;
    float elke = 0.0f, demfp = 0.0f, sig0 = 0.0f, total_tstep = 0.0f;
    int lelke = 0, compute_tstep = 1, is_tstep = 1;
    for (;;) {
        C->steps_electron++;
        C->cnt[e_electron_step][0]++;
        uint32_t irold = p->region, irl = irold;
        const ora_region *rd = &C->reg[irl];
        unsigned medium = rd->med;
        float rhof = rd->rhof;
        int lelec = p->charge;
        int qel = (1 + lelec) / 2;
        float eie = p->e;
        if (eie <= rd->ecut) { e_discard_below_cut(C, p, rd); return; }
        if (p->wt <= 0.0f) return;
        float eke_val = eie - rm;
        if (is_tstep) {
            compute_tstep = 1;
            if (medium != VACUUM) {
                float rnne1 = U(C, &p->rng);
                if (rnne1 == 0.0f) rnne1 = 1.0E-30f;
                demfp = fmaxf_(-gx_log(rnne1), EPSEMFP);
                elke = gx_log(eke_val);
                lelke = (int)(P->eke01[medium][0] + P->eke01[medium][1] * elke);
                if (P->sig_ismonotone[medium * 2 + qel]) {
                    float sigf = ev2(P->sig[qel * MXEKE * MXMED + medium * MXEKE + lelke - 1], elke);
                    float dedx0 = ev2(P->dedx[qel * MXEKE * MXMED + medium * MXEKE + lelke - 1], elke);
                    sigf = sigf / dedx0;
                    sig0 = sigf;
                } else sig0 = P->sig_e[qel * MXMED + medium];
            }
        }
        float sig_val = 0.0f, dedx_val = 0.0f, tstep = 0.0f, ustep = 0.0f, tustep = 0.0f, tvstep = 0.0f, vstep = 0.0f;
        float range = 0.0f, de = 0.0f, blccl = 0.0f, xccl = 0.0f, beta2 = 0.0f, chia2 = 0.0f, xi = 0.0f, tperp = 0.0f;
        int callhowfar = 0, domultiple = 0, dosingle = 0, callmsdist = 0;
        if (medium == VACUUM) {
            tstep = VACUUM_STEP;
            ustep = tstep;
            tustep = ustep;
            callhowfar = 1;
        } else {
            sig_val = sig0;
            if (sig_val <= 0.0f) { tstep = VACUUM_STEP; sig0 = 1.0E-15f; }
            else {
                if (compute_tstep) {
                    float total_de = demfp / sig_val;
                    float ekef = eke_val - total_de;
                    if (ekef <= P->e_array[medium * MXEKE + 0]) tstep = VACUUM_STEP;
                    else {
                        float elkef = gx_log(ekef);
                        int lelkef = (int)(P->eke01[medium][0] + P->eke01[medium][1] * elkef);
                        if (lelkef == lelke) {
                            float fedep = 1.0f - ekef / eke_val;
                            tstep = range_piece(P, qel, medium, lelke, elke, elkef, eke_val, fedep);
                        } else {
                            float ekei = P->e_array[medium * MXEKE + lelke - 1];
                            float elkei = ((float)lelke - P->eke01[medium][0]) / P->eke01[medium][1];
                            float fedep = 1.0f - ekei / eke_val;
                            float tuss = range_piece(P, qel, medium, lelke, elke, elkei, eke_val, fedep);
                            ekei = P->e_array[medium * MXEKE + lelkef];
                            elkei = ((float)(lelkef + 1) - P->eke01[medium][0]) / P->eke01[medium][1];
                            fedep = 1.0f - ekef / ekei;
                            tstep = range_piece(P, qel, medium, lelkef, elkei, elkef, ekei, fedep);
                            tstep = tstep + tuss + P->range_ep[(medium * MXEKE + lelke - 1) * 2 + qel]
                                    - P->range_ep[(medium * MXEKE + lelkef) * 2 + qel];
                        }
                    }
                    total_tstep = tstep;
                    compute_tstep = 0;
                }
                tstep = total_tstep / rhof;
            }
            float dedx0 = ev2(P->dedx[qel * MXEKE * MXMED + medium * MXEKE + lelke - 1], elke);
            dedx_val = rhof * dedx0;
            float tmxs_val = ev2(P->tmxs[medium * MXEKE + lelke - 1], elke);
            tmxs_val = tmxs_val / rhof;
            {
                float ekei = P->e_array[medium * MXEKE + lelke - 1];
                float elkei = ((float)lelke - P->eke01[medium][0]) / P->eke01[medium][1];
                float fedep = 1.0f - ekei / eke_val;
                range = range_piece(P, qel, medium, lelke, elke, elkei, eke_val, fedep);
                range = (range + P->range_ep[(medium * MXEKE + lelke - 1) * 2 + qel]) / rhof;
            }
            tmxs_val = fminf_(tmxs_val, P->smaxir[medium]);
            tustep = fminf_(tstep, fminf_(tmxs_val, range));
            int ok;
            ora_hownear(C, p, &tperp, &ok);
            if (!ok) { C->error |= 1; return; }
            p->dnear = tperp;
            if (P->i_do_rr[medium] == 1 && p->e < P->e_max_rr[medium]) {
                if (tperp >= range) { e_discard_below_cut(C, p, rd); return; }
            }
            blccl = rhof * P->blcc[medium];
            xccl = rhof * P->xcc[medium];
            float p2 = eke_val * (eke_val + rmt2);
            beta2 = p2 / (p2 + rmsq);
            float ssmfp = beta2 / blccl;
            float skindepth = P->skindepth_for_bca * ssmfp;
            tustep = fminf_(tustep, fmaxf_(tperp, skindepth));
            if (tustep <= tperp && (!P->exact_bca || tustep > skindepth)) {
                callmsdist = 1;
                de = compute_eloss(P, qel, medium, tustep, range, rhof, eke_val, elke, lelke);
                tvstep = tustep;
                msdist_pI(C, de, tustep, p, &ustep, rd, &p->rng);
            } else {
                if (P->exact_bca) {
                    float rnnoss = U(C, &p->rng);
                    float lambda = -gx_log(1.0f - rnnoss);
                    float tmp = (eke_val / rm + 1.0f);
                    float lambda_max = 0.5 * blccl * rm / dedx_val * tmp * tmp * tmp;
                    if (lambda >= 0.0f && lambda_max > 0.0f) {
                        float tuss;
                        if (lambda < lambda_max) tuss = lambda * ssmfp * (1 - 0.5 * lambda / lambda_max);
                        else tuss = 0.5 * lambda * ssmfp;
                        if (tuss < tustep) { tustep = tuss; dosingle = 1; } else dosingle = 0;
                    } else return;
                    ustep = tustep;
                } else {
                    domultiple = 1;
                    float ekems = eke_val - 0.5 * tustep * dedx_val;
                    p2 = ekems * (ekems + rmt2);
                    beta2 = p2 / (p2 + rmsq);
                    chia2 = xccl / (4.0f * blccl * p2);
                    xi = 0.5 * xccl / p2 / beta2 * tustep;
                    xi = xi * (gx_log((float)(1 + 1.0 / chia2)) - 1 / (1 + chia2));
                    if (xi < 0.1) ustep = tustep * (1 - xi * (0.5 - xi * 0.166667));
                    else ustep = tustep * (1.0f - gx_exp(-xi)) / xi;
                }
                callhowfar = (ustep < tperp) ? 0 : 1;
            }
        }
        uint32_t irnew = p->region;
        int idisc = 0;
        float ustep0 = ustep;
        if (callhowfar || p->wt <= 0.0f) {
            int ok;
            irnew = ora_howfar(C, p, &ustep, &ok);
            if (!ok) { C->error |= 1; return; }
        }
        if (irnew == 0) {
            if (rd->med == VACUUM || p->leafIndex == PASSMLC) idisc = 1; else idisc = -1;
        }
        if (idisc > 0) {
            p->region = 0;
            ora_escore(C, 0, (p->e + (float)p->charge * prm) * p->wt);
            return;
        }
        if (ustep <= 0.0f) ustep = 0.0f;
        if (ustep == 0.0f || medium == VACUUM) {
            if (ustep != 0.0f) {
                vstep = ustep;
                p->x = p->x + p->u * vstep;
                p->y = p->y + p->v * vstep;
                p->z = p->z + p->w * vstep;
                p->dnear = p->dnear - vstep;
            }
            p->region = irnew;
            rd = &C->reg[irnew];
            if (eie <= rd->ecut) { e_discard_below_cut(C, p, rd); return; }
            if (ustep != 0.0f && idisc < 0) {
                ora_escore(C, p->region, (p->e + (float)p->charge * prm) * p->wt);
                return;
            }
            is_tstep = 1;
            continue;
        }
        vstep = ustep;
        if (callhowfar) {
            if (P->exact_bca) {
                tvstep = vstep;
                if (tvstep != tustep) dosingle = 0;
            } else {
                if (vstep < ustep0) {
                    float ekems = eke_val - 0.5 * tustep * vstep / ustep0 * dedx_val;
                    float p2 = ekems * (ekems + rmt2);
                    beta2 = p2 / (p2 + rmsq);
                    chia2 = xccl / (4.0f * blccl * p2);
                    xi = 0.5 * xccl / p2 / beta2 * vstep;
                    xi = xi * (gx_log((float)(1 + 1.0 / chia2)) - 1 / (1 + chia2));
                    if (xi < 0.1) tvstep = vstep * (1 + xi * (0.5 + xi * 0.333333));
                    else {
                        if (xi < 0.999999) tvstep = -vstep * gx_log(1 - xi) / xi;
                        else return;
                    }
                } else tvstep = tustep;
            }
            de = compute_eloss(P, qel, medium, tvstep, range, rhof, eke_val, elke, lelke);
        } else {
            tvstep = tustep;
            if (!callmsdist) de = compute_eloss(P, qel, medium, tvstep, range, rhof, eke_val, elke, lelke);
        }
        float save_de = de;
        float edep = de;
        float ekef = eke_val - de;
        if (!callmsdist) {
            float sinthe = 0.0f, costhe = 0.0f;
            if (domultiple) {
                float lambda = blccl * tvstep / beta2 / 1.0f / (1.0f + chia2);
                mscat(C, lambda, chia2, xi, &costhe, &sinthe, &p->rng);
            } else if (dosingle) {
                float ekems = fmaxf_(ekef, rd->ecut - rm);
                float p2 = ekems * (ekems + rmt2);
                beta2 = p2 / (p2 + rmsq);
                chia2 = P->xcc[medium] / (4.0f * P->blcc[medium] * p2);
                sscat(C, chia2, &costhe, &sinthe, &p->rng);
            } else { sinthe = 0.0f; costhe = 1.0f; }
            p->x = p->x + p->u * vstep;
            p->y = p->y + p->v * vstep;
            p->z = p->z + p->w * vstep;
            if (domultiple || dosingle) {
                float sinphi, cosphi;
                uphi21(C, costhe, sinthe, &cosphi, &sinphi, p, &p->rng);
            }
        }
        p->dnear = p->dnear - vstep;
        irold = p->region;
        eie = eie - edep;
        p->e = eie;
        ora_escore(C, irold, edep * p->wt);
        if (irnew == irl && eie <= rd->ecut) { e_discard_below_cut(C, p, rd); return; }
        unsigned medold = medium;
        if (medium != VACUUM) {
            eke_val = eie - rm;
            elke = gx_log(eke_val);
            lelke = (int)(P->eke01[medium][0] + P->eke01[medium][1] * elke);
        }
        if (irnew != irold) {
            p->region = irnew;
            irl = irnew;
            rd = &C->reg[irl];
            medium = rd->med;
            C->cnt[e_electron_step][0]++;
        }
        if (eie <= rd->ecut) { e_discard_below_cut(C, p, rd); return; }
        if (idisc < 0) {
            ora_escore(C, p->region, (p->e + (float)p->charge * prm) * p->wt);
            return;
        }
        if (medium != medold) { is_tstep = 1; continue; }
        demfp = demfp - save_de * sig_val;
        total_tstep = total_tstep - tvstep * rhof;
        if (total_tstep < 1e-9) demfp = 0.0f;
        if (demfp >= EPSEMFP) { is_tstep = 0; continue; }
        float sigf = ev2(P->sig[qel * MXEKE * MXMED + medium * MXEKE + lelke - 1], elke);
        float dedx0 = ev2(P->dedx[qel * MXEKE * MXMED + medium * MXEKE + lelke - 1], elke);
        sigf = sigf / dedx0;
        float sigratio = sigf / sig0;
        float rfict = U(C, &p->rng);
        if (rfict > sigratio) { is_tstep = 1; continue; }
        if (lelec < 0) {
            float ebr1_val = ev2(P->ebr1[medium * MXEKE + lelke - 1], elke);
            float rnno24 = U(C, &p->rng);
            if (rnno24 <= ebr1_val) { ora_push(C, p, e_brems); return; }
            if (p->e <= P->thmoll[medium] && P->eii_flag == 0) {
                if (ebr1_val <= 0.0f) { is_tstep = 1; continue; }
                ora_push(C, p, e_brems);
                return;
            }
            ora_push(C, p, e_moller);
            return;
        }
        float pbr1_val = ev2(P->pbr1[medium * MXEKE + lelke - 1], elke);
        float rnno25 = U(C, &p->rng);
        if (rnno25 < pbr1_val) { ora_push(C, p, e_brems); return; }
        float pbr2_val = ev2(P->pbr2[medium * MXEKE + lelke - 1], elke);
        if (rnno25 < pbr2_val) ora_push(C, p, e_bhabha);
        else ora_push(C, p, e_annih);
        return;
    }
}

static void eii_sample(ora_ctx *C, int ish, int iz, float uj, ora_particle *p, const ora_region *rd, ora_rng *r, float *edep)
{
    const gegs_physics *P = C->P;
    const float rm = P->rm, prm = P->prm, rmt2 = P->rmt2;
    unsigned medium = rd->med;
    ora_particle p1 = *p;
    float eie = p->e;
    float t = eie - rm;
    float tau = t / rm;
    float tau12 = (tau + 1.0f) * (tau + 1.0f);
    float p2 = tau * tau + 2.0f * tau;
    float beta2 = p2 / tau12;
    float wmax = 0.5 * (t + uj);
    float xmax = uj / wmax;
    float c1 = (wmax / eie) * (wmax / eie);
    float c2 = (2.0f * tau + 1.0f) / tau12;
    float fm_s = gx_log(rmt2 * p2 / uj) - beta2 - 0.5f;
    float prob_s = 0.66666667 * fm_s * (1 + xmax + xmax * xmax);
    float fm_h = 2.0f + c1 - c2;
    if (fm_h < 1.0f) fm_h = 1.0f;
    float prob = fm_h + prob_s;
    float r1, frej, wx;
    int n = 0;
    do {
        r1 = U(C, r);
        if ((r1 * prob) < fm_h) {
            r1 = U(C, r);
            wx = 1.0f / (r1 * xmax + 1.0f - r1);
            float wxx = wx * xmax;
            float aux = wxx / (2.0f - wxx);
            frej = (1.0f + aux * (aux - c2) + c1 * wxx * wxx) / fm_h;
        } else {
            r1 = U(C, r);
            wx = 1.0f / gx_exp(gx_log(r1 * xmax * xmax * xmax + 1.0f - r1) * 0.333333333f);
            frej = 1.0f - gx_log(wx) / fm_s;
        }
        r1 = U(C, r);
    } while (r1 >= frej && ++n < ORA_LOOP_CAP);
    wx = wx * uj;
    float h1 = (eie + prm) / t;
    float ese1 = eie - wx;
    p->e = ese1;
    float dcosth = h1 * (ese1 - prm) / (ese1 + prm);
    float sinthe = sqrtf(fmaxf_(0.0f, 1.0f - dcosth));
    float costhe = sqrtf(dcosth);
    float sinphi, cosphi;
    uphi21(C, costhe, sinthe, &cosphi, &sinphi, p, r);
    float ese2 = wx - uj + prm;
    if (ese2 > P->ae[medium]) {
        p1.e = ese2;
        dcosth = h1 * (ese2 - prm) / (ese2 + prm);
        sinthe = -sqrtf(fmaxf_(0.0f, 1.0f - dcosth));
        costhe = sqrtf(dcosth);
        uphi32(costhe, sinthe, cosphi, sinphi, &p1);
        ora_spawn(C, r, &p1, e_electron_step);
        *edep = 0.0f;
    } else {
        *edep = wx - uj;
    }
    ora_relax(C, uj, ish, iz, edep, *p, rd, r);
}

void ora_moller(ora_ctx *C, ora_particle *p)
{
    const gegs_physics *P = C->P;
    const float rm = P->rm, prm = P->prm;
    ora_rng r = p->rng;
    const ora_region *rd = &C->reg[p->region];
    float edep = 0.0f;
    ora_particle p1 = *p;
    unsigned medium = rd->med;
    float eie = p->e;
    float ekin = eie - prm;
    float elke = gx_log(ekin);
    if ((P->eii_flag > 0) && (P->eii_nsh[medium] > 0)) {
        int lelke = (int)(P->eke01[medium][1] * elke + P->eke01[medium][0]);
        float sigm = P->sig[medium * MXEKE + lelke - 1][1] * elke + P->sig[medium * MXEKE + lelke - 1][0];
        float pbrem = P->ebr1[medium * MXEKE + lelke - 1][1] * elke + P->ebr1[medium * MXEKE + lelke - 1][0];
        sigm = sigm * (1.0f - pbrem);
        float rsh = U(C, &r);
        rsh = sigm * rsh;
        for (int iele = 0; iele < P->nne[medium]; iele++) {
            int iz = (int)(P->zelem[iele * MXMED + medium] + 0.5);
            int nsh = P->eii_no[iele * MXMED + medium];
            if (nsh > 0) {
                int ifirst = P->eii_first[iele * MXMED + medium];
                for (int ish = 1; ish <= nsh; ish++) {
                    float uj = P->binding_energies[(iz - 1) * MXSHELL + ish - 1];
                    if ((ekin > uj) && (uj > P->te[medium] || uj > P->ap[medium])) {
                        int jj = ifirst + ish - 1;
                        int i = (int)(P->eii[jj - 1][0] * elke + P->eii[jj - 1][1] + (float)((jj - 1) * N_EII_BINS));
                        if (i < 1 + (jj - 1) * N_EII_BINS) i = 1 + (jj - 1) * N_EII_BINS;
                        if (i > jj * N_EII_BINS) i = jj * N_EII_BINS;
                        float sig_j = P->eii_xsection[i - 1][0] * elke + P->eii_xsection[i - 1][1];
                        sig_j = sig_j * P->pz[MXMED * iele + medium] * P->eii_cons[medium];
                        rsh -= sig_j;
                        if (rsh < 0.0f) {
                            eii_sample(C, ish, iz, uj, p, rd, &r, &edep);
                            if (p->e < rd->ecut) edep += p->e - prm;
                            else ora_spawn(C, &r, p, e_electron_step);
                            ora_escore(C, p->region, edep * p->wt);
                            return;
                        }
                    }
                }
            }
        }
    }
    float te = P->te[medium];
    if (ekin <= 2.0f * te) { ora_escore(C, p->region, (p->e - prm) * p->wt); return; }
    float t0 = ekin / rm;
    float e0 = t0 + 1.0f;
    float extrae = eie - P->thmoll[medium];
    float e02 = e0 * e0;
    float g2 = t0 * t0 / e02;
    float g3 = (2.0f * t0 + 1.0f) / e02;
    float gmax = (1.0f + 1.25 * g2);
    float rnno27, rejf4, br, rr;
    int n = 0;
    do {
        rnno27 = U(C, &r);
        br = te / (ekin - extrae * rnno27);
        rr = br / (1.0f - br);
        rnno27 = U(C, &r);
        rejf4 = (1.0f + g2 * br * br + rr * (rr - g3));
        rnno27 = gmax * rnno27;
    } while (rnno27 > rejf4 && ++n < ORA_LOOP_CAP);
    float ekse2 = br * ekin;
    float ese1 = eie - ekse2;
    float ese2 = ekse2 + prm;
    p->e = ese1;
    p1.e = ese2;
    float h1 = (eie + prm) / ekin;
    float dcosth = h1 * (ese1 - prm) / (ese1 + prm);
    float sinthe = sqrtf(fmaxf_(0.0f, 1.0f - dcosth));
    float costhe = sqrtf(dcosth);
    float sinphi, cosphi;
    uphi21(C, costhe, sinthe, &cosphi, &sinphi, p, &r);
    if (p->e < rd->ecut) edep += p->e - prm;
    else ora_spawn(C, &r, p, e_electron_step);
    dcosth = h1 * (ese2 - prm) / (ese2 + prm);
    sinthe = -sqrtf(fmaxf_(0.0f, 1.0f - dcosth));
    costhe = sqrtf(dcosth);
    uphi32(costhe, sinthe, cosphi, sinphi, &p1);
    if (p1.e < rd->ecut) edep += p1.e - prm;
    else ora_spawn(C, &r, &p1, e_electron_step);
    ora_escore(C, p->region, edep * p->wt);
}

void ora_brems(ora_ctx *C, ora_particle *p)
{
    const gegs_physics *P = C->P;
    const float rm = P->rm, prm = P->prm;
    ora_rng r = p->rng;
    const ora_region *rd = &C->reg[p->region];
    float edep = 0.0f;
    ora_particle p1 = *p;
    unsigned m = rd->med;
    int nbr = P->nbr_split;
    if (nbr < 1) return;
    float eie = p->e;
    int l = (eie < 50.0) ? 1 : 3;
    int l1 = l + 1;
    float ekin = eie - prm;
    float elke = gx_log(ekin);
    float brmin = P->ap[m] / ekin;
    float waux = elke - P->log_ap[m];
    float a = 0.0f, b = 0.0f, c = 0.0f, sinpsi = 0.0f, sindel = 0.0f, cosdel = 0.0f;
    float ztarg = 0.0f, tteie = 0.0f, y2maxi = 0.0f, z2maxi = 0.0f;
    int ibrdst = P->ibrdst;
    if (ibrdst >= 0) {
        a = p->u; b = p->v; c = p->w;
        sinpsi = a * a + b * b;
        if (sinpsi > 1e-20) {
            sinpsi = sqrtf(sinpsi);
            sindel = b / sinpsi;
            cosdel = a / sinpsi;
        }
        ztarg = P->zbrang[m];
        tteie = eie / rm;
        float beta = sqrtf((tteie - 1.0f) * (tteie + 1.0f)) / tteie;
        float y2max = 2.0f * beta * (1.0f + beta) * tteie * tteie;
        y2maxi = 1.0f / y2max;
        if (ibrdst == 1) {
            float z2max = y2max + 1.0f;
            z2maxi = sqrtf(z2max);
        }
    }
    float ese = eie;
    for (int ibr = 1; ibr <= nbr; ibr++) {
        float rnno06, rejf, esg;
        int n = 0;
        do {
            rnno06 = U(C, &r);
            float br = brmin * gx_exp(rnno06 * waux);
            esg = ekin * br;
            ese = eie - esg;
            float delta = esg / eie / ese * P->delcm[m];
            float aux = ese / eie;
            float phi1, phi2;
            if (delta < 1.0f) {
                phi1 = P->dl1[m * 8 + l - 1] + delta * (P->dl2[m * 8 + l - 1] + delta * P->dl3[m * 8 + l - 1]);
                phi2 = P->dl1[m * 8 + l1 - 1] + delta * (P->dl2[m * 8 + l1 - 1] + delta * P->dl3[m * 8 + l1 - 1]);
            } else {
                phi1 = P->dl4[m * 8 + l - 1] + P->dl5[m * 8 + l - 1] * gx_log(delta + P->dl6[m * 8 + l - 1]);
                phi2 = phi1;
            }
            rejf = (1.0f + aux * aux) * phi1 - 2.0f * aux * phi2 / 3.0f;
            rnno06 = U(C, &r);
        } while (rnno06 >= rejf && ++n < ORA_LOOP_CAP);
        p1.e = esg;
        p1.charge = 0;
        p1.wt = p->wt / (float)nbr;
        if (ibrdst >= 0) {
            float y2tst;
            if (ibrdst == 1) {
                float esedei = ese / rm / tteie;
                float rjarg1 = 1.0f + esedei * esedei;
                float rjarg2 = rjarg1 + 2.0f * esedei;
                float aux = 2.0f * ese * tteie / esg;
                aux = aux * aux;
                float aux1 = aux * ztarg;
                float rjarg3;
                if (aux1 > 10.0f) rjarg3 = P->lzbrang[m] + (1.0f - aux1) / (aux1 * aux1);
                else rjarg3 = gx_log(aux / (1.0f + aux1));
                float rejmax = rjarg1 * rjarg3 - rjarg2;
                float rtest, rejtst;
                int nn = 0;
                do {
                    y2tst = U(C, &r);
                    rtest = U(C, &r);
                    float aux3 = z2maxi / (y2tst + (1.0f - y2tst) * z2maxi);
                    rtest = rtest * aux3 * rejmax;
                    y2tst = aux3 * aux3 - 1.0f;
                    float y2tst1 = esedei * y2tst / (aux3 * aux3 * aux3 * aux3);
                    float aux4 = 16.0f * y2tst1 - rjarg2;
                    float aux5 = rjarg1 - 4.0f * y2tst1;
                    if (rtest < (aux4 + aux5 * rjarg3)) break;
                    float aux2 = gx_log(aux / (1.0f + aux1 / (aux3 * aux3 * aux3 * aux3)));
                    rejtst = aux4 + aux5 * aux2;
                } while (rtest >= rejtst && ++nn < ORA_LOOP_CAP);
            } else {
                y2tst = U(C, &r);
                y2tst = y2tst / (1.0f - y2tst + y2maxi);
            }
            float costhe = 1.0f - 2.0f * y2tst * y2maxi;
            float sinthe = sqrtf(fmaxf_((1.0f - costhe) * (1.0f + costhe), 0.0f));
            float cphi, sphi;
            box_phi(C, &r, &cphi, &sphi);
            if (sinpsi >= 1e-10) {
                float us = sinthe * cphi;
                float vs = sinthe * sphi;
                p1.u = c * cosdel * us - sindel * vs + a * costhe;
                p1.v = c * sindel * us + cosdel * vs + b * costhe;
                p1.w = c * costhe - sinpsi * us;
            } else {
                p1.u = sinthe * cphi;
                p1.v = sinthe * sphi;
                p1.w = c * costhe;
            }
        }
        if (p1.e < rd->pcut) edep += p1.e;
        else ora_spawn(C, &r, &p1, p_photon_step);
    }
    p->e = ese;
    if (p->e < rd->ecut) edep += p->e - prm;
    else ora_spawn(C, &r, p, e_electron_step);
    ora_escore(C, p->region, edep * p->wt);
}

void ora_bhabha(ora_ctx *C, ora_particle *p)
{
    const gegs_physics *P = C->P;
    const float rm = P->rm, prm = P->prm;
    ora_rng r = p->rng;
    const ora_region *rd = &C->reg[p->region];
    float edep = 0.0f;
    ora_particle p1 = *p;
    unsigned m = rd->med;
    float eip = p->e;
    float ekin = eip - prm;
    float t0 = ekin / rm;
    float e0 = t0 + 1.0f;
    float yy = 1.0f / (t0 + 2.0f);
    float e02 = e0 * e0;
    float beta2 = (e02 - 1.0f) / e02;
    float ep0 = P->te[m] / ekin;
    float ep0c = 1.0f - ep0;
    float y2 = yy * yy;
    float yp = 1.0f - 2.0f * yy;
    float yp2 = yp * yp;
    float b4 = yp2 * yp;
    float b3 = b4 + yp2;
    float b2 = yp * (3.0f + y2);
    float b1 = 2.0f - y2;
    float rnno03, rejf2, br;
    int n = 0;
    do {
        rnno03 = U(C, &r);
        br = ep0 / (1.0f - ep0c * rnno03);
        rnno03 = U(C, &r);
        rejf2 = (1.0f - beta2 * br * (b1 - br * (b2 - br * (b3 - br * b4))));
    } while (rnno03 > rejf2 && ++n < ORA_LOOP_CAP);
    if (br < 0.5f) p1.charge = -1;
    else { p->charge = -1; p1.charge = 1; br = 1.0f - br; }
    br = fmaxf_(br, 0.0f);
    float ekse2 = br * ekin;
    float ese1 = eip - ekse2;
    float ese2 = ekse2 + prm;
    p->e = ese1;
    p1.e = ese2;
    float h1 = (eip + prm) / ekin;
    float dcosth = fminf_(1.0f, h1 * (ese1 - prm) / (ese1 + prm));
    float sinthe = sqrtf(1.0f - dcosth);
    float costhe = sqrtf(dcosth);
    float sinphi, cosphi;
    uphi21(C, costhe, sinthe, &cosphi, &sinphi, p, &r);
    if (p->e < rd->ecut) {
        edep += p->e - prm;
        if (p->charge > 0) ora_annih_at_rest(C, p, rd, &r);
    } else ora_spawn(C, &r, p, e_electron_step);
    dcosth = h1 * (ese2 - prm) / (ese2 + prm);
    sinthe = -sqrtf(fmaxf_(0.0f, 1.0f - dcosth));
    costhe = sqrtf(dcosth);
    uphi32(costhe, sinthe, cosphi, sinphi, &p1);
    if (p1.e < rd->ecut) {
        edep += p1.e - prm;
        if (p1.charge > 0) ora_annih_at_rest(C, &p1, rd, &r);
    } else ora_spawn(C, &r, &p1, e_electron_step);
    ora_escore(C, p->region, edep * p->wt);
}

void ora_annih(ora_ctx *C, ora_particle *p)
{
    const gegs_physics *P = C->P;
    const float rm = P->rm, prm = P->prm;
    ora_rng r = p->rng;
    const ora_region *rd = &C->reg[p->region];
    float edep = 0.0f;
    int nbr = P->nbr_split;
    if (nbr <= 0) return;
    float avip = p->e + prm;
    float a = avip / rm;
    float g = a - 1.0f;
    float t = g - 1.0f;
    float pp = sqrtf(a * t);
    float pot = pp / t;
    float ep0 = 1.0f / (a + pp);
    float wsamp = gx_log((1.0f - ep0) / ep0);
    float aa = p->u, bb = p->v, cc = p->w;
    float sinpsi = aa * aa + bb * bb, sindel = 0.0f, cosdel = 0.0f;
    if (sinpsi > 1e-20) {
        sinpsi = sqrtf(sinpsi);
        sindel = bb / sinpsi;
        cosdel = aa / sinpsi;
    }
    if (nbr > 1) p->wt = p->wt / (float)nbr;
    for (int ibr = 1; ibr <= nbr; ibr++) {
        float rnno01, rejf, ep;
        int n = 0;
        do {
            rnno01 = U(C, &r);
            ep = ep0 * gx_exp(rnno01 * wsamp);
            rnno01 = U(C, &r);
            rejf = 1.0f - (ep * a - 1.0f) * (ep * a - 1.0f) / (ep * (a * a - 2.0f));
        } while (rnno01 > rejf && ++n < ORA_LOOP_CAP);
        float esg1 = avip * ep;
        p->e = esg1;
        p->charge = 0;
        float costhe = fminf_(1.0f, (esg1 - rm) * pot / esg1);
        float sinthe = sqrtf(1.0f - costhe * costhe);
        float cphi, sphi;
        box_phi(C, &r, &cphi, &sphi);
        if (sinpsi >= 1e-10) {
            float us = sinthe * cphi, vs = sinthe * sphi;
            p->u = cc * cosdel * us - sindel * vs + aa * costhe;
            p->v = cc * sindel * us + cosdel * vs + bb * costhe;
            p->w = cc * costhe - sinpsi * us;
        } else {
            p->u = sinthe * cphi; p->v = sinthe * sphi; p->w = cc * costhe;
        }
        if (p->e < rd->pcut) edep += p->e;
        else ora_spawn(C, &r, p, p_photon_step);
        float esg2 = avip - esg1;
        p->e = esg2;
        costhe = fminf_(1.0f, (esg2 - rm) * pot / esg2);
        sinthe = -sqrtf(1.0f - costhe * costhe);
        if (sinpsi >= 1e-10) {
            float us = sinthe * cphi, vs = sinthe * sphi;
            p->u = cc * cosdel * us - sindel * vs + aa * costhe;
            p->v = cc * sindel * us + cosdel * vs + bb * costhe;
            p->w = cc * costhe - sinpsi * us;
        } else {
            p->u = sinthe * cphi; p->v = sinthe * sphi; p->w = cc * costhe;
        }
        if (p->e < rd->pcut) edep += p->e;
        else ora_spawn(C, &r, p, p_photon_step);
    }
    ora_escore(C, p->region, edep * p->wt);
}
