/* Oracle: photon transport and photon interactions.  Test infrastructure only.
 *   ora_photon       photon.cu:6-292      (PHOTON step loop)
 *   ora_compton      compton.cu:17-492    (Klein-Nishina + bound Compton)
 *   ora_photo        photo.cu:1-279
 *   ora_rayleigh     rayleigh.cu:4-157
 *   ora_pair         pair.cu:14-431
 *   ora_relax        relax.cu:14-238
 *   ora_annih_at_rest annihatrest.cu:10-68
 * Rejection loops without an iteration cap in the reference get a cap of
 * ORA_LOOP_CAP (never reached with these tables; identical on the GPU). */
#include "ora_internal.h"

#define ORA_LOOP_CAP 1000

static const short first_transition[5] = {1, 20, 27, 33, 38};
static const short last_transition[5] = {19, 26, 32, 37, 39};
static const short final_state[39] = {4, 3, 5, 6, 202, 302, 402, 404, 403, 303, 502, 503, 504, 602, 603, 604, 505, 605, 606,
                                      13, 14, 5, 6, 505, 605, 606, 14, 5, 6, 505, 605, 606, 5, 6, 505, 605, 606, 6, 606};

static inline float U(ora_ctx *C, ora_rng *r) { return ora_rng_uniform(C, r); }

/* a point of the unit disc by rejection; returns 1 / (x^2 + y^2) */
static float box_xy(ora_ctx *C, ora_rng *r, float *xphi, float *yphi)
{
    float rhophi2;
    int n = 0;
    do {
        *xphi = U(C, r);
        *xphi = 2.0f * *xphi - 1.0f;
        *yphi = U(C, r);
        rhophi2 = *xphi * *xphi + *yphi * *yphi;
    } while (rhophi2 > 1.0f && ++n < ORA_LOOP_CAP);
    return 1.0f / rhophi2;
}

/* azimuth by the box method ($SELECT-AZIMUTHAL-ANGLE) */
static void box_phi(ora_ctx *C, ora_rng *r, float *cphi, float *sphi)
{
    float xphi, yphi;
    float rhophi2 = box_xy(C, r, &xphi, &yphi);
    *cphi = (xphi * xphi - yphi * yphi) * rhophi2;
    *sphi = 2.0f * xphi * yphi * rhophi2;
}

/* isotropic direction used by RELAX for fluorescence/Auger particles
 * (relax.cu:187-217; products in the reference's order) */
static void relax_direction(ora_ctx *C, ora_rng *r, ora_particle *p)
{
    float eta = U(C, r);
    eta = 2.0f * eta - 1.0f;
    p->w = eta;
    eta = (1.0f - eta) * (1.0f + eta);
    if (eta > SMALL_POLAR_ANGLE_THRESHOLD) {
        eta = sqrtf(eta);
        float xphi, yphi;
        float rhophi2 = box_xy(C, r, &xphi, &yphi);
        p->u = eta * (xphi * xphi - yphi * yphi) * rhophi2;
        p->v = eta * 2.0f * xphi * yphi * rhophi2;
    } else {
        p->u = 0.0f; p->v = 0.0f; p->w = 1.0f;
    }
}

void ora_photon(ora_ctx *C, ora_particle *p)
{
    const gegs_physics *P = C->P;
    const float rm2 = 2.0f * P->rm;
    for (;;) {
        C->steps_photon++;
        C->cnt[p_photon_step][0]++;
        const ora_region *rd = &C->reg[p->region];
        if (p->e <= rd->pcut) { ora_escore(C, p->region, p->e * p->wt); return; }
        if (p->wt <= 0.0f) return;
        float r1 = U(C, &p->rng);
        float dpmfp = -gx_log(r1);
        float gle = gx_log(p->e);
        int lgle = 0;
        float tstep, gmfp_val = 0.0f, cohfac = 0.0f;
        unsigned med = rd->med;
        if (med == VACUUM) tstep = VACUUM_STEP;
        else {
            lgle = (int)(P->ge[med][0] + P->ge[med][1] * gle);
            C->cnt[p_photon_step][2] += 2 + ((rd->flags & GEGS_F_RAYLEIGH) ? 1 : 0);
            const float *g = P->gmfp[med * MXGE + lgle];
            float gmfpr0 = g[0] + g[1] * gle;
            gmfp_val = gmfpr0 / rd->rhof;
            if (rd->flags & GEGS_F_RAYLEIGH) {
                const float *c = P->cohe[med * MXGE + lgle];
                cohfac = c[0] + c[1] * gle;
                gmfp_val = gmfp_val * cohfac;
            }
            tstep = gmfp_val * dpmfp;
        }
        int ok;
        uint32_t new_region = ora_howfar(C, p, &tstep, &ok);
        if (!ok) { C->error |= 1; return; }
        int idisc = 0;
        if (new_region == 0) {
            if (med == VACUUM || p->leafIndex == PASSMLC) idisc = 1; else idisc = -1;
        }
        if (idisc > 0) { p->region = 0; ora_escore(C, 0, p->e * p->wt); return; }
        p->x = p->x + p->u * tstep;
        p->y = p->y + p->v * tstep;
        p->z = p->z + p->w * tstep;
        if (med != VACUUM) dpmfp = fmaxf_(0.0f, dpmfp - tstep / gmfp_val);
        unsigned old_medium = med;
        if (new_region != p->region) { p->region = new_region; rd = &C->reg[new_region]; C->cnt[p_photon_step][0]++; }
        if (p->e <= rd->pcut || idisc < 0) { ora_escore(C, p->region, p->e * p->wt); return; }
        if ((rd->med != old_medium) || (rd->med == VACUUM) || (dpmfp >= EPSGMFP)) continue;
        if (rd->flags & GEGS_F_RAYLEIGH) {
            r1 = U(C, &p->rng);
            if (r1 < 1.0f - cohfac) { ora_push(C, p, p_rayleigh); return; }
        }
        C->cnt[p_photon_step][2] += 2;
        const float *b1 = P->gbr1[rd->med * MXGE + lgle];
        const float *b2 = P->gbr2[rd->med * MXGE + lgle];
        float gbr1_val = b1[0] + b1[1] * gle;
        float gbr2_val = b2[0] + b2[1] * gle;
        r1 = U(C, &p->rng);
        if ((r1 <= gbr1_val) && (p->e > rm2)) ora_push(C, p, p_pair);
        else if (r1 < gbr2_val) ora_push(C, p, p_compton);
        else ora_push(C, p, p_photo);
        return;
    }
}

void ora_relax(ora_ctx *C, float energy, int n, int iz, float *edep, ora_particle p, const ora_region *rd, ora_rng *r)
{
    const gegs_physics *P = C->P;
    const float rm = P->rm, prm = P->prm;
    int vac_array[MXVAC];
    float e_arr[MXVAC];
    if ((n < 1) || (n > MXSHELL)) return;
    float e_cut = fminf_(rd->ecut - rm, rd->pcut);
    e_cut = fmaxf_(RELAX_CUTOFF, e_cut);
    if (energy <= e_cut) { *edep += energy; return; }
    int n_vac = 1;
    vac_array[0] = n;
    e_arr[0] = energy;
    for (;;) {
        int shell = vac_array[n_vac - 1];
        float ei = e_arr[n_vac - 1];
        n_vac -= 1;
        if (ei <= e_cut) {
            *edep += ei;
            if (n_vac > 0) continue;
            break;
        }
        if (shell == MXSHELL) {
            p.e = ei + prm;
            p.charge = -1;
            relax_direction(C, r, &p);
            if (p.e < rd->ecut) *edep += p.e - prm;
            else ora_spawn(C, r, &p, e_electron_step);
            if (n_vac > 0) continue;
            break;
        }
        if (n_vac + 2 > MXVAC) { *edep += ei; if (n_vac > 0) continue; break; }
        float eta = U(C, r);
        int k;
        for (k = first_transition[shell - 1]; k <= last_transition[shell - 1] - 1; k++) {
            eta = eta - P->relaxation_prob[MXTRANS * (iz - 1) + k - 1];
            if (eta <= 0.0f) break;
        }
        int fin = final_state[k - 1];
        int iql;
        float elcut, ex;
        if (fin < 100) {
            if (fin < 10) { iql = 0; elcut = rd->pcut; }
            else { fin = fin - 10; iql = -1; elcut = rd->ecut - rm; }
            float ef = P->binding_energies[MXSHELL * (iz - 1) + fin - 1];
            ex = ei - ef;
            n_vac += 1;
            vac_array[n_vac - 1] = fin;
            e_arr[n_vac - 1] = ef;
        } else {
            int f1 = fin / 100;
            int f2 = fin - f1 * 100;
            n_vac += 1;
            vac_array[n_vac - 1] = f1;
            e_arr[n_vac - 1] = P->binding_energies[MXSHELL * (iz - 1) + f1 - 1];
            n_vac += 1;
            vac_array[n_vac - 1] = f2;
            e_arr[n_vac - 1] = P->binding_energies[MXSHELL * (iz - 1) + f2 - 1];
            iql = -1;
            ex = ei - e_arr[n_vac - 1] - e_arr[n_vac - 2];
            elcut = rd->ecut - rm;
        }
        if (ex <= elcut) *edep += ex;
        else {
            p.charge = (int8_t)iql;
            if (iql == 0) p.e = ex; else p.e = ex + rm;
            relax_direction(C, r, &p);
            if (iql == 0) {
                if (p.e < rd->pcut) *edep += p.e;
                else ora_spawn(C, r, &p, p_photon_step);
            } else {
                if (p.e < rd->ecut) *edep += p.e - prm;
                else ora_spawn(C, r, &p, e_electron_step);
            }
        }
    }
}

void ora_compton(ora_ctx *C, ora_particle *p)
{
    const gegs_physics *P = C->P;
    const float rm = P->rm, prm = P->prm;
    ora_rng r = p->rng;
    const ora_region *rd = &C->reg[p->region];
    float edep = 0.0f;
    ora_particle p1 = *p;
    unsigned medium = rd->med;
    float peig = p->e;
    float ko = peig / rm;
    float broi = 1.0f + 2.0f * ko;
    int ibcmpl;
    switch (rd->flags & 0x000Eu) {
    case 0x2u: ibcmpl = 1; break;
    case 0x6u: ibcmpl = 2; break;
    case 0xAu: ibcmpl = 3; break;
    default: ibcmpl = 0;
    }
    for (int compton_loops = 0;; compton_loops++) {
        if (compton_loops > 100) break;
        float uj = 0.0f, jo = 0.0f;
        int j = 0;
        if (ibcmpl > 0) {
            float rnno17 = U(C, &r);
            int nsh = P->n_shell[medium];
            rnno17 = 1.0f + rnno17 * (float)nsh;
            int i = (int)rnno17;
            if (i > nsh) i = nsh;                       /* U = 1 exactly */
            if (rnno17 > P->eno_array[medium * MXMDSH + i - 1]) i = P->eno_atbin_array[medium * MXMDSH + i - 1];
            j = P->shell_array[medium * MXMDSH + i - 1];
            uj = P->be_array[j - 1];
            if (ko <= uj) {
                if (ibcmpl == 1) { p->rng = r; ora_push(C, p, p_photon_step); break; }
                else continue;
            }
            jo = P->jo_array[j - 1];
        }
        /* Klein-Nishina (always); alph1/alpha/bro/rejmax recomputed every pass */
        float bro = 1.0 / broi, br, temp = 0.0f, sinthe = 0.0f, costhe;
        int br_loops = 0;
        do {
            if (ko > 2.0f) {
                float alph1 = gx_log(broi);
                float alph2 = ko * (broi + 1.0f) * bro * bro;
                float alpha = alph1 + alph2;
                float aux, rejf3, rnno19;
                int n19 = 0;
                do {
                    float rnno15 = U(C, &r);
                    float rnno16 = U(C, &r);
                    if ((rnno15 * alpha) < alph1) br = gx_exp(alph1 * rnno16) * bro;
                    else br = sqrtf(rnno16 * broi * broi + (1.0f - rnno16)) * bro;
                    temp = (1.0f - br) / (ko * br);
                    sinthe = fmaxf_(0.0f, temp * (2.0f - temp));
                    aux = 1.0f + br * br;
                    rejf3 = aux - br * sinthe;
                    rnno19 = U(C, &r);
                    n19++;
                    if (n19 > 100) break;
                } while (rnno19 * aux > rejf3);
            } else {
                float rejmax = broi + bro;
                float rnno16, rejf3;
                int n16 = 0;
                do {
                    float rnno15 = U(C, &r);
                    rnno16 = U(C, &r);
                    br = bro + (1.0f - bro) * rnno15;
                    temp = (1.0f - br) / (ko * br);
                    sinthe = fmaxf_(0.0f, temp * (2.0f - temp));
                    rejf3 = 1.0f + br * br - br * sinthe;
                    if (n16++ > 100) break;
                } while (rnno16 * br * rejmax > rejf3);
            }
        } while ((br < bro || br > 1.0f) && ++br_loops < ORA_LOOP_CAP);
        costhe = 1.0f - temp;
        if (ibcmpl == 0) {
            uj = 0.0f;
        } else {
            float aux = ko * (ko - uj) * temp;
            float aux1 = 2.0f * aux + uj * uj;
            float pzmax = aux - uj;
            if ((pzmax < 0.0f) && (pzmax * pzmax >= aux1)) {
                if (ibcmpl == 1) { p->rng = r; ora_push(C, p, p_photon_step); break; }
                else continue;
            }
            pzmax = pzmax / sqrtf(aux1);
            float qc2 = 1.0f + br * br - 2.0f * br * costhe;
            float qc = sqrtf(qc2);
            float af, fmax1, fpz;
            if (pzmax > 1.0f) {
                pzmax = 1.0f; af = 0.0f; fmax1 = 1.0f; fpz = 1.0f;
            } else {
                float aux3 = 1.0f + 2.0f * jo * fabsf(pzmax);
                float aux4 = 0.5 * (1 - aux3 * aux3);
                fpz = 0.5 * gx_exp(aux4);
                af = qc * (1.0f + br * (br - costhe) / qc2);
                if (af < 0.0f) {
                    if (pzmax > 0.0f) fpz = 1.0f - fpz;
                    float eta_incoh = U(C, &r);
                    if (eta_incoh > fpz) {
                        if (ibcmpl == 1) { p->rng = r; ora_push(C, p, p_photon_step); break; }
                        else continue;
                    }
                    af = 0.0f; fmax1 = 1.0f;
                } else {
                    float fpz1;
                    if (pzmax < -0.15) { fmax1 = 1 - af * 0.15; fpz1 = fpz * fmax1 * jo; }
                    else if (pzmax < 0.15) {
                        fmax1 = 1.0f + af * pzmax;
                        aux3 = 1 / (1 + 0.33267252734 * aux3);
                        aux4 = fpz * aux3 * (0.3480242 + aux3 * (-0.0958798 + aux3 * 0.7478556)) + P->erfjo_array[j - 1];
                        if (pzmax > 0.0f) { fpz1 = (1 - fmax1 * fpz) * jo - 0.62665706866 * af * aux4; fpz = 1.0f - fpz; }
                        else fpz1 = fmax1 * fpz * jo - 0.62665706866 * af * aux4;
                    } else { fmax1 = 1 + af * 0.15; fpz1 = (1.0f - fmax1 * fpz) * jo; fpz = 1.0f - fpz; }
                    float eta_incoh = U(C, &r);
                    if (eta_incoh * jo > fpz1) {
                        if (ibcmpl == 1) { p->rng = r; ora_push(C, p, p_photon_step); break; }
                        else continue;
                    }
                }
            }
            float pz = 0.0f;
            for (int pz_loops = 0;; pz_loops++) {
                if (pz_loops > 100) { pz = 0.0f; break; }
                if (ibcmpl != 2) {
                    float rnno18 = U(C, &r);
                    rnno18 = rnno18 * fpz;
                    if (rnno18 < 0.5) {
                        rnno18 = fmax(1e-30, (double)(2.0f * rnno18));
                        pz = 0.5 * (1 - sqrtf(1 - 2 * gx_log(rnno18))) / jo;
                    } else {
                        rnno18 = 2.0f * (1.0f - rnno18);
                        pz = 0.5 * (sqrtf(1 - 2 * gx_log(rnno18)) - 1) / jo;
                    }
                    if (fabsf(pz) > 1.0f) continue;
                    if (pz < 0.15) {
                        float frej;
                        if (pz < -0.15) frej = 1 - af * 0.15; else frej = 1.0f + af * pz;
                        float eta = U(C, &r);
                        if (eta * fmax1 > frej) continue;
                    }
                } else { pz = 0.0f; uj = 0.0f; }
                break;
            }
            if (fabsf(pz) < 0.01) br = br * (1.0f + pz * (qc + (br * br - costhe) * pz));
            else {
                float a1 = 1.0f - pz * pz * br * costhe;
                float a2 = 1.0f - pz * pz * br * br;
                float a3 = qc2 - br * br * pz * pz * sinthe;
                if (a3 > 1e-10) br = br / a2 * (a1 + pz * sqrtf(a3));
            }
            uj = uj * prm;
        }
        float pesg = br * peig;
        float pese = peig - pesg - uj + prm;
        sinthe = sqrtf(sinthe);
        p->e = pesg;
        float sinphi, cosphi;
        uphi21(C, costhe, sinthe, &cosphi, &sinphi, p, &r);
        if (p->e < rd->pcut) edep += p->e;
        else ora_spawn(C, &r, p, p_photon_step);
        float aux = 1.0f + br * br - 2.0f * br * costhe;
        if (aux > 1e-8) {
            costhe = (1.0f - br * costhe) / sqrtf(aux);
            sinthe = (1.0f - costhe) * (1.0f + costhe);
            if (sinthe > 0.0f) sinthe = -sqrtf(sinthe); else sinthe = 0.0f;
        } else { costhe = 0.0f; sinthe = -1.0f; }
        p1.e = pese;
        p1.charge = -1;
        uphi32(costhe, sinthe, cosphi, sinphi, &p1);
        if (p1.e < rd->ecut) edep += p1.e - prm;
        else ora_spawn(C, &r, &p1, e_electron_step);
        if ((ibcmpl == 1) || (ibcmpl == 3)) {
            if (uj > RELAX_CUTOFF)
                ora_relax(C, uj, P->shn_array[j - 1], P->iz_array[j - 1], &edep, *p, rd, &r);
            else edep += uj;
        }
        break;
    }
    ora_escore(C, p->region, edep * p->wt);
}

void ora_photo(ora_ctx *C, ora_particle *p)
{
    const gegs_physics *P = C->P;
    const float rm = P->rm, prm = P->prm;
    ora_rng r = p->rng;
    const ora_region *rd = &C->reg[p->region];
    float probs[MXEL];
    int ints[MXEL];
    float edep = 0.0f;
    unsigned medium = rd->med;
    float peig = p->e;
    unsigned iedgfl = rd->flags & GEGS_F_ATOMIC_RELAXATION;
    unsigned iphter = rd->flags & GEGS_F_PHOTO_ANGULAR;
    if (peig < P->edge_energies[1]) {
        p->charge = -1;
        p->e = peig + prm;
        if (p->e < rd->ecut) ora_escore(C, p->region, (p->e - prm) * p->wt);
        else ora_spawn(C, &r, p, e_electron_step);
        return;
    }
    float gle = gx_log(p->e);
    int do_relax = 0;
    float e_vac = 0.0f;
    int iz = 1, j = 0, k = 0;
    if (iedgfl != 0) {
        int nne = P->nne[medium];
        if (nne == 1) {
            iz = (int)(P->zelem[medium] + 0.5);
            for (j = 0; j < P->edge_number[iz - 1]; j++)
                if (peig >= P->edge_energies[MXEDGE * (iz - 1) + j]) break;
        } else {
            float aux = peig * peig;
            float aux1 = aux * peig;
            aux = aux * sqrtf(peig);
            float sigtot = 0.0f;
            for (k = 0; k < nne; k++) {
                iz = (int)(P->zelem[MXMED * k + medium] + 0.5);
                int b = MXEDGE * (iz - 1);
                float sigma;
                if (peig > P->edge_energies[b]) {
                    j = 1;
                    sigma = (P->edge_a[b] + P->edge_b[b] / peig + P->edge_c[b] / aux + P->edge_d[b] / aux1) / peig;
                } else {
                    for (j = 2; j <= P->edge_number[iz - 1]; j++)
                        if (peig >= P->edge_energies[b + j - 1]) break;
                    sigma = P->edge_a[b + j - 1] + gle * (P->edge_b[b + j - 1] + gle * (P->edge_c[b + j - 1] + gle * P->edge_d[b + j - 1]));
                    sigma = gx_exp(sigma);
                }
                sigma = sigma * P->pz[MXMED * k + medium];
                sigtot = sigtot + sigma;
                probs[k] = sigma;
                ints[k] = j;
            }
            float br = U(C, &r);
            br = br * sigtot;
            for (k = 0; k < nne; k++) {
                br = br - probs[k];
                if (br <= 0.0f) break;
            }
            if (k >= nne) k = nne - 1;                  /* rounding left br > 0 */
            iz = (int)(P->zelem[MXMED * k + medium] + 0.5);
            j = ints[k];
        }
        if (peig <= P->binding_energies[MXSHELL * (iz - 1) + 5]) {
            edep += peig;
        } else {
            float br = U(C, &r);
            for (k = 1; k <= 5; k++) {
                if (peig > P->binding_energies[MXSHELL * (iz - 1) + k - 1]) {
                    float tmp = P->interaction_prob[MXSHELL * (iz - 1) + k - 1];
                    if (br < tmp) break;
                    br = (br - tmp) / (1.0f - tmp);
                }
            }
            e_vac = P->binding_energies[MXSHELL * (iz - 1) + k - 1];
            p->e = peig - e_vac + prm;
            do_relax = 1;
            p->charge = -1;
        }
    } else {
        p->e = peig + prm;
        p->charge = -1;
    }
    if (p->charge == -1) {
        if (p->e > rd->ecut) {
            if (iphter) {
                float beta = sqrtf((p->e - rm) * (p->e + rm)) / p->e;
                float gamma = p->e / rm;
                float alpha = 0.5 * gamma - 0.5 + 1.0f / gamma;
                float ratio = beta / alpha;
                float xi, rnpht2, sinth2, costhe;
                int nl = 0;
                do {
                    float rnpht = U(C, &r);
                    rnpht = 2.0f * rnpht - 1.0f;
                    if (ratio <= 0.2) {
                        float fkappa = rnpht + 0.5 * ratio * (1.0f - rnpht) * (1 + rnpht);
                        if (gamma < 100.0f) costhe = (beta + fkappa) / (1.0f + beta * fkappa);
                        else {
                            if (fkappa > 0.0f)
                                costhe = 1.0f - (1.0f - fkappa) * (gamma - 3.0f) / (2.0f * (1.0f + fkappa) * (gamma - 1.0f) * (gamma - 1.0f) * (gamma - 1.0f));
                            else costhe = (beta + fkappa) / (1.0f + beta * fkappa);
                        }
                        xi = (1.0f + beta * fkappa) * gamma * gamma;
                    } else {
                        xi = gamma * gamma * (1.0f + alpha * (sqrtf(1.0f + ratio * (2.0f * rnpht + ratio)) - 1.0f));
                        costhe = (1.0f - 1.0f / xi) / beta;
                    }
                    sinth2 = fmaxf_(0.0f, (1.0f - costhe) * (1.0f + costhe));
                    rnpht2 = U(C, &r);
                } while (rnpht2 > (0.5 * (1.0f + gamma) * sinth2 * xi / gamma) && ++nl < ORA_LOOP_CAP);
                float sinthe = sqrtf(sinth2);
                float sinphi, cosphi;
                uphi21(C, costhe, sinthe, &cosphi, &sinphi, p, &r);
            }
            ora_spawn(C, &r, p, e_electron_step);
        } else {
            edep += p->e - prm;
        }
    }
    if (do_relax) ora_relax(C, e_vac, k, iz, &edep, *p, rd, &r);
    ora_escore(C, p->region, edep * p->wt);
}

void ora_rayleigh(ora_ctx *C, ora_particle *p)
{
    const gegs_physics *P = C->P;
    ora_rng r = p->rng;
    const ora_region *rd = &C->reg[p->region];
    unsigned med = rd->med;
    float gle = gx_log(p->e);
    int lgle = (int)(P->ge[med][0] + P->ge[med][1] * gle);
    const float *pm = P->pmax[med * MXGE + lgle];
    float pmax_val = pm[0] + pm[1] * gle;
    float xmax = HC_INVERSE * p->e;
    float costhe = 0.0f, costhe2 = 0.0f;
    int accept = 0, nouter = 0;
    do {
        float xv = 0.0f;
        int ninner = 0;
        do {
            float r1 = U(C, &r);
            float temp = r1 * pmax_val;
            int ibin = (int)(temp * (float)(RAYCDFSIZE - 1));
            if (ibin > RAYCDFSIZE - 2) ibin = RAYCDFSIZE - 2;  /* temp = 1 exactly */
            int ib = (int)P->i_array[med * RAYCDFSIZE + ibin] - 1;
            int next_ib = (int)P->i_array[med * RAYCDFSIZE + ibin + 1] - 1;
            if (next_ib > ib) {
                for (;;) {
                    const float *rdat = P->rayleigh_data[med * MXRAYFF + ib + 1];
                    if ((temp < rdat[1]) || (ib >= RAYCDFSIZE - 2)) break;
                    ib++;
                }
            }
            const float *rdat = P->rayleigh_data[med * MXRAYFF + ib];
            temp = (temp - rdat[1]) * rdat[3];
            xv = rdat[0] * gx_exp(gx_log(1.0f + temp) * rdat[2]);
        } while (!(xv < xmax) && ++ninner < ORA_LOOP_CAP);
        float r2 = U(C, &r);
        xv = xv / p->e;
        costhe = 1.0f - TWICE_HC2 * xv * xv;
        costhe2 = costhe * costhe;
        if (2.0f * r2 < 1.0f + costhe2) accept = 1;
    } while (!accept && ++nouter < ORA_LOOP_CAP);
    float sinthe = sqrtf(1.0f - costhe2);
    float cosphi, sinphi;
    uphi21(C, costhe, sinthe, &cosphi, &sinphi, p, &r);
    if (p->e < rd->pcut) ora_escore(C, p->region, p->e * p->wt);
    else ora_spawn(C, &r, p, p_photon_step);
}

void ora_annih_at_rest(ora_ctx *C, ora_particle *p, const ora_region *rd, ora_rng *r)
{
    const gegs_physics *P = C->P;
    float edep = 0.0f;
    int nbr = P->nbr_split;
    if (nbr > 1) p->wt = p->wt / (float)nbr;
    p->e = P->prm;
    p->charge = 0;
    for (int ibr = 1; ibr <= nbr; ibr++) {
        float costhe = U(C, r);
        costhe = 2.0f * costhe - 1.0f;
        float sinthe = sqrtf(fmaxf_(0.0f, (1.0f - costhe) * (1.0f + costhe)));
        float cphi, sphi;
        box_phi(C, r, &cphi, &sphi);
        p->u = sinthe * cphi;
        p->v = sinthe * sphi;
        p->w = costhe;
        if (p->e < rd->pcut) edep += p->e;
        else ora_spawn(C, r, p, p_photon_step);
        p->u = -p->u; p->v = -p->v; p->w = -p->w;
        if (p->e < rd->pcut) edep += p->e;
        else ora_spawn(C, r, p, p_photon_step);
    }
    ora_escore(C, p->region, edep * p->wt);
}

/* lowest-order pair angle (iprdst_use == 1) and the other iprdst options */
static void pair_angle(ora_ctx *C, ora_rng *r, int use, float ese, float eig, unsigned medium, float *costhe, float *sinthe)
{
    const gegs_physics *P = C->P;
    const float rm = P->rm;
    if (use == 1) {
        float pse = sqrtf(fmaxf_(0.0f, (ese - rm) * (ese + rm)));
        float c = U(C, r);
        c = 1.0f - 2.0 * c;
        *sinthe = rm * sqrtf((1.0f - c) * (1.0f + c)) / (pse * c + ese);
        *costhe = (ese * c + pse) / (pse * c + ese);
    } else if (use == 2) {
        float ztarg = P->zbrang[medium];
        float tteig = eig / rm, ttese = ese / rm;
        float esedei = ttese / (tteig - ttese);
        float eseder = 1.0f / esedei;
        float ximin = 1.0f / (1.0f + (3.141593 * ttese) * (3.141593 * ttese));
        float g1 = ((1.0f + eseder) * (1.0f + esedei) / (2.0f * tteig));
        float rejmin = 2.0f + 3.0f * (esedei + eseder) - 4.00 * (esedei + eseder + 1.0f - 4.0f * (ximin - 0.5f) * (ximin - 0.5f))
                       * (1.0f + 0.25f * gx_log(g1 * g1 + ztarg * ximin * ximin));
        float ya = (2.0f / tteig) * (2.0f / tteig);
        float xitry = fmaxf_(0.01f, fmaxf_(ximin, fminf_(0.5f, sqrtf(ya / ztarg))));
        float galpha = 1.0f + 0.25 * gx_log(ya + ztarg * xitry * xitry);
        float gbeta = 0.5f * ztarg * xitry / (ya + ztarg * xitry * xitry);
        galpha = galpha - gbeta * (xitry - 0.5f);
        float ximid = galpha / (3.0f * gbeta);
        if (galpha >= 0.0f) ximid = 0.5f - ximid + sqrtf(ximid * ximid + 0.25);
        else ximid = 0.5f - ximid - sqrtf(ximid * ximid + 0.25);
        ximid = fmaxf_(0.01f, fmaxf_(ximin, fminf_(0.5f, ximid)));
        float rejmid = 2.0f + 3.0f * (esedei + eseder) - 4.0f * (esedei + eseder + 1.0f - 4.0 * (ximid - 0.5f) * (ximid - 0.5f))
                       * (1.0f + 0.25 * gx_log(g1 * g1 + ztarg * ximid * ximid));
        float rejtop = 1.02 * fmaxf_(rejmin, rejmid);
        float rtest, rtst, theta;
        int n = 0;
        do {
            float xitst = U(C, r);
            float rejtst = 2.0f + 3.0f * (esedei + eseder) - 4.0f * (esedei + eseder + 1.0f - 4.0f * (xitst - 0.5) * (xitst - 0.5))
                           * (1.0f + 0.25 * gx_log(g1 * g1 + ztarg * xitst * xitst));
            rtest = U(C, r);
            theta = sqrtf(1.0f / xitst - 1.0f) / ttese;
            rtst = rejtst / rejtop;
        } while (((rtest > rtst) || (theta >= 3.1415926535f)) && ++n < ORA_LOOP_CAP);
        gx_sincos(theta, sinthe, costhe);
    } else if (use == 3) {
        float c = U(C, r);
        c = 1.0f - 2.0f * c;
        float s = (1.0f - c) * (1.0f + c);
        *costhe = c;
        *sinthe = s > 0.0f ? sqrtf(s) : 0.0f;
    } else {
        float c = U(C, r);
        c = 1.0f - 2.0f * sqrtf(c);
        float s = (1.0f - c) * (1.0f + c);
        *costhe = c;
        *sinthe = s > 0.0f ? sqrtf(s) : 0.0f;
    }
}

void ora_pair(ora_ctx *C, ora_particle *p)
{
    const gegs_physics *P = C->P;
    const float rm = P->rm, prm = P->prm, rmt2 = P->rmt2;
    ora_rng r = p->rng;
    const ora_region *rd = &C->reg[p->region];
    float edep = 0.0f;
    ora_particle p1 = *p;
    unsigned m = rd->med;
    float eig = p->e;
    float ese1, ese2;
    int iq1, iq2;
    if (eig <= 2.1) {
        float rnno30 = U(C, &r);
        ese2 = prm + 0.5 * rnno30 * (eig - 2 * prm);
        rnno30 = U(C, &r);
        ese1 = eig - ese2;
        if (rnno30 < 0.5) { iq1 = -1; iq2 = 1; } else { iq1 = 1; iq2 = -1; }
    } else {
        float amax, bmax, aux1;
        int l, l1;
        if (eig < 50.0f) {
            l = 5; l1 = l + 1;
            float delta = 4.0f * P->delcm[m] / eig;
            if (delta < 1.0f) {
                amax = P->dl1[8 * m + l - 1] + delta * (P->dl2[8 * m + l - 1] + delta * P->dl3[8 * m + l - 1]);
                bmax = P->dl1[8 * m + l1 - 1] + delta * (P->dl2[8 * m + l1 - 1] + delta * P->dl3[8 * m + l1 - 1]);
            } else {
                float aux2 = gx_log(delta + P->dl6[8 * m + l - 1]);
                amax = P->dl4[8 * m + l - 1] + P->dl5[8 * m + l - 1] * aux2;
                bmax = P->dl4[8 * m + l1 - 1] + P->dl5[8 * m + l1 - 1] * aux2;
            }
            aux1 = 1.0f - rmt2 / eig;
            aux1 = aux1 * aux1;
            aux1 = aux1 * amax / 3.0f;
            aux1 = aux1 / (bmax + aux1);
        } else {
            l = 7;
            amax = P->dl1[m * 8 + l - 1];
            bmax = P->dl1[m * 8 + l];
            aux1 = P->bpar[m * 2 + 1] * (1.0f - P->bpar[m * 2] * rm / eig);
        }
        float del0 = eig * P->delcm[m];
        float eavail = eig - rmt2;
        float rnno30, rejmax, rejf, eminus;
        int n = 0;
        do {
            rnno30 = U(C, &r);
            float rnno31 = U(C, &r);
            float br;
            if (rnno30 > aux1) { br = 0.5 * rnno31; rejmax = bmax; l1 = l + 1; }
            else {
                rnno30 = U(C, &r);
                rnno30 = fmaxf_(rnno30, rnno31);
                rnno31 = U(C, &r);
                float b1 = fmaxf_(rnno30, rnno31);
                br = 0.5 * (1 - b1);
                rejmax = amax;
                l1 = l;
            }
            eminus = br * eavail + rm;
            float eplus = eig - eminus;
            float delta = del0 / (eminus * eplus);
            if (delta < 1.0f)
                rejf = P->dl1[m * 8 + l1 - 1] + delta * (P->dl2[m * 8 + l1 - 1] + delta * P->dl3[m * 8 + l1 - 1]);
            else
                rejf = P->dl4[m * 8 + l1 - 1] + P->dl5[m * 8 + l1 - 1] * gx_log(delta + P->dl6[m * 8 + l1 - 1]);
            rnno30 = U(C, &r);
        } while ((rnno30 * rejmax) > rejf && ++n < ORA_LOOP_CAP);
        ese2 = eminus;
        ese1 = eig - ese2;
        rnno30 = U(C, &r);
        if (rnno30 < 0.5) { iq1 = -1; iq2 = 1; } else { iq1 = 1; iq2 = -1; }
    }
    p->e = ese1;
    p1.e = ese2;
    p->charge = (int8_t)iq1;
    p1.charge = (int8_t)iq2;
    float costhe = 1.0f, sinthe = 0.0f, sinphi, cosphi;
    int iprdst = P->iprdst;
    if (iprdst > 0) {
        int use;
        if (iprdst == 4) {
            float rtest = U(C, &r);
            float gbeta = ese1 / (ese1 + 10.0f);
            use = (rtest < gbeta) ? 1 : 4;
        } else if ((iprdst == 2) && (eig < 4.14)) use = 1;
        else use = iprdst;
        for (int ichrg = 1; ichrg <= 2; ichrg++) {
            float ese;
            if (ichrg == 1) ese = ese1;
            else {
                ese = ese2;
                if (iprdst == 4) {
                    float gbeta = ese / (ese + 10.0f);
                    float rtest = U(C, &r);
                    use = (rtest < gbeta) ? 1 : 4;
                }
            }
            pair_angle(C, &r, use, ese, eig, m, &costhe, &sinthe);
            if (ichrg == 1) {
                uphi21(C, costhe, sinthe, &cosphi, &sinphi, p, &r);
                if (p->e < rd->ecut) {
                    edep += p->e - prm;
                    if (p->charge > 0) ora_annih_at_rest(C, p, rd, &r);
                } else ora_spawn(C, &r, p, e_electron_step);
            } else {
                sinthe = -sinthe;
                uphi32(costhe, sinthe, cosphi, sinphi, &p1);
                if (p1.e < rd->ecut) {
                    edep += p1.e - prm;
                    if (p1.charge > 0) ora_annih_at_rest(C, &p1, rd, &r);
                } else ora_spawn(C, &r, &p1, e_electron_step);
            }
        }
        ora_escore(C, p->region, edep * p->wt);
        return;
    }
    uphi11(C, 0.0f, &costhe, &sinthe, &cosphi, &sinphi, p, &r);
    if (p->e < rd->ecut) {
        edep += p->e - prm;
        if (p->charge > 0) ora_annih_at_rest(C, p, rd, &r);
    } else ora_spawn(C, &r, p, e_electron_step);
    sinthe = -sinthe;
    uphi32(costhe, sinthe, cosphi, sinphi, &p1);
    if (p1.e < rd->ecut) {
        edep += p1.e - prm;
        if (p1.charge > 0) ora_annih_at_rest(C, &p1, rd, &r);
    } else ora_spawn(C, &r, &p1, e_electron_step);
    ora_escore(C, p->region, edep * p->wt);
}
