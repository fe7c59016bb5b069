// Device photon transport and photon interactions.
//   photon_step     photon.cu:6-292 (one PHOTON loop iteration per call)
//   compton         compton.cu:17-492
//   photo           photo.cu:1-279
//   rayleigh        rayleigh.cu:4-157
//   pair            pair.cu:14-431
//   relax           relax.cu:14-238
//   annih_at_rest   annihatrest.cu:10-68
// Each routine samples with the incoming particle's stream `r`; particles it
// creates get child streams (push_spawn).  Rejection loops the reference leaves
// open are capped at GX_LOOP_CAP iterations.
#pragma once
#include "dev_geom.cuh"

__device__ __forceinline__ float U(const DevCtx &C, Rng &r) { return rng_uniform(C, r); }

__device__ __forceinline__ void rotate_dir(float costhe, float sinthe, float cosphi, float sinphi, Part &p)
{
    float A = p.u, B = p.v, Cc = p.w;
    float sinps2 = A * A + B * B;
    if (sinps2 < 1E-20f) {
        p.u = sinthe * cosphi;
        p.v = sinthe * sinphi;
        p.w = Cc * costhe;
    } else {
        float sinpsi_i = 1.0f / sqrtf(sinps2);
        float us = sinthe * cosphi;
        float vs = sinthe * sinphi;
        float sindel = B * sinpsi_i;
        float cosdel = A * sinpsi_i;
        p.u = Cc * cosdel * us - sindel * vs + A * costhe;
        p.v = Cc * sindel * us + cosdel * vs + B * costhe;
        p.w = -us / sinpsi_i + Cc * costhe;
    }
}

// UPHI(2,1) (utility.cu:94-142)
__device__ __forceinline__ void uphi21(const DevCtx &C, float costhe, float sinthe, float &cosphi, float &sinphi, Part &p, Rng &r)
{
    float r1 = U(C, r);
    float phi = 2.0f * 3.14159265f * r1;      // utility.cu:99-100
    gx_sincos(phi, &sinphi, &cosphi);
    rotate_dir(costhe, sinthe, cosphi, sinphi, p);
}

// UPHI(3,2) (utility.cu:144-179)
__device__ __forceinline__ void uphi32(float costhe, float sinthe, float cosphi, float sinphi, Part &p)
{
    rotate_dir(costhe, sinthe, cosphi, sinphi, p);
}

// a point of the unit disc by rejection; returns 1 / (x^2 + y^2)
__device__ __forceinline__ float box_xy(const DevCtx &C, Rng &r, float &xphi, float &yphi)
{
    float rhophi2;
    int n = 0;
    do {
        xphi = U(C, r);
        xphi = 2.0f * xphi - 1.0f;
        yphi = U(C, r);
        rhophi2 = xphi * xphi + yphi * yphi;
    } while (rhophi2 > 1.0f && ++n < GX_LOOP_CAP);
    return 1.0f / rhophi2;
}

__device__ __forceinline__ void box_phi(const DevCtx &C, Rng &r, float &cphi, float &sphi)
{
    float xphi, yphi;
    const float rhophi2 = box_xy(C, r, xphi, yphi);
    cphi = (xphi * xphi - yphi * yphi) * rhophi2;
    sphi = 2.0f * xphi * yphi * rhophi2;
}

// isotropic direction of a fluorescence or Auger particle (relax.cu:187-217;
// the products in the reference's order: sin(theta) times the box terms first)
__device__ __forceinline__ void relax_direction(const DevCtx &C, Rng &r, Part &p)
{
    float eta = U(C, r);
    eta = 2.0f * eta - 1.0f;
    p.w = eta;
    eta = (1.0f - eta) * (1.0f + eta);
    if (eta > 1E-20f) {
        eta = sqrtf(eta);
        float xphi, yphi;
        const float rhophi2 = box_xy(C, r, xphi, yphi);
        p.u = eta * (xphi * xphi - yphi * yphi) * rhophi2;
        p.v = eta * 2.0f * xphi * yphi * rhophi2;
    } else {
        p.u = 0.0f; p.v = 0.0f; p.w = 1.0f;
    }
}

__constant__ short c_first_transition[5] = {1, 20, 27, 33, 38};
__constant__ short c_last_transition[5] = {19, 26, 32, 37, 39};
__constant__ short c_final_state[39] = {4, 3, 5, 6, 202, 302, 402, 404, 403, 303, 502, 503, 504, 602, 603, 604, 505, 605, 606,
                                        13, 14, 5, 6, 505, 605, 606, 14, 5, 6, 505, 605, 606, 5, 6, 505, 605, 606, 6, 606};

// Fluorescence / Auger / Coster-Kronig cascade for a vacancy in shell n of element iz.
__device__ void relax(const DevCtx &C, float energy, int n, int iz, float &edep, Part p, const RegInfo &rd, Rng &r)
{
    const gegs_physics *P = C.P;
    const float rm = P->rm, prm = P->prm;
    int vac_array[10];
    float e_arr[10];
    if ((n < 1) || (n > GEGS_MXSHELL)) return;
    float e_cut = fminf_(rd.ecut - rm, rd.pcut);
    e_cut = fmaxf_(0.001f, e_cut);
    if (energy <= e_cut) { edep += energy; return; }
    int n_vac = 1;
    vac_array[0] = n;
    e_arr[0] = energy;
    for (;;) {
        int shell = vac_array[n_vac - 1];
        float ei = e_arr[n_vac - 1];
        n_vac -= 1;
        if (ei <= e_cut) {
            edep += ei;
            if (n_vac > 0) continue;
            break;
        }
        if (shell == GEGS_MXSHELL) {
            p.e = ei + prm;
            p.charge = -1;
            relax_direction(C, r, p);
            if (p.e < rd.ecut) edep += p.e - prm;
            else push_spawn(C, ST_ELECTRON, p, r);
            if (n_vac > 0) continue;
            break;
        }
        if (n_vac + 2 > 10) { edep += ei; if (n_vac > 0) continue; break; }
        float eta = U(C, r);
        int k;
        for (k = c_first_transition[shell - 1]; k <= c_last_transition[shell - 1] - 1; k++) {
            eta = eta - __ldg(&P->relaxation_prob[GEGS_MXTRANS * (iz - 1) + k - 1]);
            if (eta <= 0.0f) break;
        }
        int fin = c_final_state[k - 1];
        int iql;
        float elcut, ex;
        if (fin < 100) {
            if (fin < 10) { iql = 0; elcut = rd.pcut; }
            else { fin = fin - 10; iql = -1; elcut = rd.ecut - rm; }
            float ef = __ldg(&P->binding_energies[GEGS_MXSHELL * (iz - 1) + fin - 1]);
            ex = ei - ef;
            n_vac += 1;
            vac_array[n_vac - 1] = fin;
            e_arr[n_vac - 1] = ef;
        } else {
            int f1 = fin / 100;
            int f2 = fin - f1 * 100;
            n_vac += 1;
            vac_array[n_vac - 1] = f1;
            e_arr[n_vac - 1] = __ldg(&P->binding_energies[GEGS_MXSHELL * (iz - 1) + f1 - 1]);
            n_vac += 1;
            vac_array[n_vac - 1] = f2;
            e_arr[n_vac - 1] = __ldg(&P->binding_energies[GEGS_MXSHELL * (iz - 1) + f2 - 1]);
            iql = -1;
            ex = ei - e_arr[n_vac - 1] - e_arr[n_vac - 2];
            elcut = rd.ecut - rm;
        }
        if (ex <= elcut) edep += ex;
        else {
            p.charge = (int8_t)iql;
            if (iql == 0) p.e = ex; else p.e = ex + rm;
            relax_direction(C, r, p);
            if (iql == 0) {
                if (p.e < rd.pcut) edep += p.e;
                else push_spawn(C, ST_PHOTON, p, r);
            } else {
                if (p.e < rd.ecut) edep += p.e - prm;
                else push_spawn(C, ST_ELECTRON, p, r);
            }
        }
    }
}

// With C.stage_tables (run option GEGS_RUN_STAGE_TABLES) the photon consumers
// stage the {gmfp, cohe} table of the plan's media (C.ptab, nmed * MXGE
// float4, 19.2 KB for six media) in dynamic shared memory once per block, and
// a step reads its mean free path and Rayleigh factor from there; otherwise
// from the physics block through L1/L2. Same values either way. On the CT
// 5-field plan the staged form is 1.2 % slower (the slice is L1-resident and
// the carve-out shrinks L1 for the region gathers), so it is an option the
// batch autotuner can pick per plan.
extern __shared__ float4 g_smem_ptab[];

__host__ __device__ constexpr size_t photon_smem_bytes(int nmed) { return (size_t)nmed * GX_MXGE * sizeof(float4); }

__device__ __forceinline__ void stage_photon_tables(const DevCtx &C)
{
    if (!C.stage_tables) return;
    const int n = C.nmed * GX_MXGE;
    for (int i = threadIdx.x; i < n; i += blockDim.x) g_smem_ptab[i] = __ldg(&C.ptab[i]);
    __syncthreads();
}

// One iteration of the PHOTON loop.  Returns true when the photon has left
// the photon stage (absorbed, escaped or queued for an interaction).
// SH: the {gmfp, cohe} table is staged in shared memory (stage_photon_tables).
template <int G = GX_GEOM_ALL, bool SH = false>
__device__ bool photon_step(const DevCtx &C, Part &p, Rng &r)
{
    const gegs_physics *P = C.P;
    RegInfo rd = region_info(C, p.region);
    if (p.e <= rd.pcut) { escore(C, p, p.region, p.e * p.wt); return true; }
    if (p.wt <= 0.0f) return true;
    float r1 = U(C, r);
    float dpmfp = -gx_log(r1);
    float gle = gx_log(p.e);
    int lgle = 0;
    float tstep, gmfp_val = 0.0f, cohfac = 0.0f;
    unsigned med = rd.med;
    if (med == GX_VACUUM) tstep = GX_VACUUM_STEP;
    else {
        float2 ge = __ldg(reinterpret_cast<const float2 *>(P->ge[med]));
        lgle = (int)(ge.x + ge.y * gle);
        float4 t;
        if (SH && C.stage_tables) t = g_smem_ptab[med * GX_MXGE + lgle];
        else {
            const float2 g = __ldg(reinterpret_cast<const float2 *>(P->gmfp[med * GX_MXGE + lgle]));
            t.x = g.x; t.y = g.y;
        }
        float gmfpr0 = t.x + t.y * gle;
        gmfp_val = gmfpr0 / rd.rhof;
        if (rd.flags & GEGS_F_RAYLEIGH) {
            if (!(SH && C.stage_tables)) {
                const float2 c = __ldg(reinterpret_cast<const float2 *>(P->cohe[med * GX_MXGE + lgle]));
                t.z = c.x; t.w = c.y;
            }
            cohfac = t.z + t.w * gle;
            gmfp_val = gmfp_val * cohfac;
        }
        tstep = gmfp_val * dpmfp;
    }
    bool ok;
    uint32_t new_region = howfar_g<G>(C, p, tstep, ok);
    if (!ok) { atomicOr(C.err, GX_ERR_MODULE); return true; }
    int idisc = 0;
    if (new_region == 0) {
        if (med == GX_VACUUM || p.leafIndex == GX_PASSMLC) idisc = 1; else idisc = -1;
    }
    if (idisc > 0) { p.region = 0; escore(C, p, 0, p.e * p.wt); return true; }
    p.x = p.x + p.u * tstep;
    p.y = p.y + p.v * tstep;
    p.z = p.z + p.w * tstep;
    if (med != GX_VACUUM) dpmfp = fmaxf_(0.0f, dpmfp - tstep / gmfp_val);
    unsigned old_medium = med;
    if (new_region != p.region) { p.region = new_region; rd = region_info(C, new_region); }
    if (p.e <= rd.pcut || idisc < 0) { escore(C, p, p.region, p.e * p.wt); return true; }
    if ((rd.med != old_medium) || (rd.med == GX_VACUUM) || gx_ge(dpmfp, GX_EPSGMFP)) return false;
    if (rd.flags & GEGS_F_RAYLEIGH) {
        r1 = U(C, r);
        if (r1 < 1.0f - cohfac) { push_move(C, ST_RAYLEIGH, p, r); return true; }
    }
    float2 b1 = __ldg(reinterpret_cast<const float2 *>(P->gbr1[rd.med * GX_MXGE + lgle]));
    float2 b2 = __ldg(reinterpret_cast<const float2 *>(P->gbr2[rd.med * GX_MXGE + lgle]));
    float gbr1_val = b1.x + b1.y * gle;
    float gbr2_val = b2.x + b2.y * gle;
    r1 = U(C, r);
    if ((r1 <= gbr1_val) && (p.e > 2.0f * P->rm)) push_move(C, ST_PAIR, p, r);
    else if (r1 < gbr2_val) push_move(C, ST_COMPTON, p, r);
    else push_move(C, ST_PHOTO, p, r);
    return true;
}

__device__ void compton(const DevCtx &C, Part p, Rng &r)
{
    const gegs_physics *P = C.P;
    const float rm = P->rm, prm = P->prm;
    RegInfo rd = region_info(C, p.region);
    float edep = 0.0f;
    Part p1 = p;
    unsigned medium = rd.med;
    float peig = p.e;
    float ko = peig / rm;
    float broi = 1.0f + 2.0f * ko;
    int ibcmpl;
    switch (rd.flags & 0x000Eu) {
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
            float rnno17 = U(C, r);
            int nsh = P->n_shell[medium];
            rnno17 = 1.0f + rnno17 * (float)nsh;
            int i = (int)rnno17;
            if (i > nsh) i = nsh;
            if (rnno17 > __ldg(&P->eno_array[medium * GEGS_MXMDSH + i - 1])) i = __ldg(&P->eno_atbin_array[medium * GEGS_MXMDSH + i - 1]);
            j = __ldg(&P->shell_array[medium * GEGS_MXMDSH + i - 1]);
            uj = __ldg(&P->be_array[j - 1]);
            if (ko <= uj) {
                if (ibcmpl == 1) { push_move(C, ST_PHOTON, p, r); break; }
                else continue;
            }
            jo = __ldg(&P->jo_array[j - 1]);
        }
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
                    float rnno15 = U(C, r);
                    float rnno16 = U(C, r);
                    if ((rnno15 * alpha) < alph1) br = gx_exp(alph1 * rnno16) * bro;
                    else br = sqrtf(rnno16 * broi * broi + (1.0f - rnno16)) * bro;
                    temp = (1.0f - br) / (ko * br);
                    sinthe = fmaxf_(0.0f, temp * (2.0f - temp));
                    aux = 1.0f + br * br;
                    rejf3 = aux - br * sinthe;
                    rnno19 = U(C, r);
                    n19++;
                    if (n19 > 100) break;
                } while (rnno19 * aux > rejf3);
            } else {
                float rejmax = broi + bro;
                float rnno16, rejf3;
                int n16 = 0;
                do {
                    float rnno15 = U(C, r);
                    rnno16 = U(C, r);
                    br = bro + (1.0f - bro) * rnno15;
                    temp = (1.0f - br) / (ko * br);
                    sinthe = fmaxf_(0.0f, temp * (2.0f - temp));
                    rejf3 = 1.0f + br * br - br * sinthe;
                    if (n16++ > 100) break;
                } while (rnno16 * br * rejmax > rejf3);
            }
        } while ((br < bro || br > 1.0f) && ++br_loops < GX_LOOP_CAP);
        costhe = 1.0f - temp;
        if (ibcmpl == 0) {
            uj = 0.0f;
        } else {
            float aux = ko * (ko - uj) * temp;
            float aux1 = 2.0f * aux + uj * uj;
            float pzmax = aux - uj;
            if ((pzmax < 0.0f) && (pzmax * pzmax >= aux1)) {
                if (ibcmpl == 1) { push_move(C, ST_PHOTON, p, r); break; }
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
                    float eta_incoh = U(C, r);
                    if (eta_incoh > fpz) {
                        if (ibcmpl == 1) { push_move(C, ST_PHOTON, p, r); break; }
                        else continue;
                    }
                    af = 0.0f; fmax1 = 1.0f;
                } else {
                    float fpz1;
                    if (gx_lt(pzmax, -0.15)) { fmax1 = 1 - af * 0.15; fpz1 = fpz * fmax1 * jo; }
                    else if (gx_lt(pzmax, 0.15)) {
                        fmax1 = 1.0f + af * pzmax;
                        aux3 = 1 / (1 + 0.33267252734 * aux3);
                        aux4 = fpz * aux3 * (0.3480242 + aux3 * (-0.0958798 + aux3 * 0.7478556)) + __ldg(&P->erfjo_array[j - 1]);
                        if (pzmax > 0.0f) { fpz1 = (1 - fmax1 * fpz) * jo - 0.62665706866 * af * aux4; fpz = 1.0f - fpz; }
                        else fpz1 = fmax1 * fpz * jo - 0.62665706866 * af * aux4;
                    } else { fmax1 = 1 + af * 0.15; fpz1 = (1.0f - fmax1 * fpz) * jo; fpz = 1.0f - fpz; }
                    float eta_incoh = U(C, r);
                    if (eta_incoh * jo > fpz1) {
                        if (ibcmpl == 1) { push_move(C, ST_PHOTON, p, r); break; }
                        else continue;
                    }
                }
            }
            float pz = 0.0f;
            for (int pz_loops = 0;; pz_loops++) {
                if (pz_loops > 100) { pz = 0.0f; break; }
                if (ibcmpl != 2) {
                    float rnno18 = U(C, r);
                    rnno18 = rnno18 * fpz;
                    if (rnno18 < 0.5) {
                        rnno18 = fmax(1e-30, (double)(2.0f * rnno18));
                        pz = 0.5 * (1 - sqrtf(1 - 2 * gx_log(rnno18))) / jo;
                    } else {
                        rnno18 = 2.0f * (1.0f - rnno18);
                        pz = 0.5 * (sqrtf(1 - 2 * gx_log(rnno18)) - 1) / jo;
                    }
                    if (fabsf(pz) > 1.0f) continue;
                    if (gx_lt(pz, 0.15)) {
                        float frej;
                        if (gx_lt(pz, -0.15)) frej = 1 - af * 0.15; else frej = 1.0f + af * pz;
                        float eta = U(C, r);
                        if (eta * fmax1 > frej) continue;
                    }
                } else { pz = 0.0f; uj = 0.0f; }
                break;
            }
            if (gx_lt(fabsf(pz), 0.01)) br = br * (1.0f + pz * (qc + (br * br - costhe) * pz));
            else {
                float a1 = 1.0f - pz * pz * br * costhe;
                float a2 = 1.0f - pz * pz * br * br;
                float a3 = qc2 - br * br * pz * pz * sinthe;
                if (gx_gt(a3, 1e-10)) br = br / a2 * (a1 + pz * sqrtf(a3));
            }
            uj = uj * prm;
        }
        float pesg = br * peig;
        float pese = peig - pesg - uj + prm;
        sinthe = sqrtf(sinthe);
        p.e = pesg;
        float sinphi, cosphi;
        uphi21(C, costhe, sinthe, cosphi, sinphi, p, r);
        if (p.e < rd.pcut) edep += p.e;
        else push_spawn(C, ST_PHOTON, p, r);
        float aux = 1.0f + br * br - 2.0f * br * costhe;
        if (gx_gt(aux, 1e-8)) {
            costhe = (1.0f - br * costhe) / sqrtf(aux);
            sinthe = (1.0f - costhe) * (1.0f + costhe);
            if (sinthe > 0.0f) sinthe = -sqrtf(sinthe); else sinthe = 0.0f;
        } else { costhe = 0.0f; sinthe = -1.0f; }
        p1.e = pese;
        p1.charge = -1;
        uphi32(costhe, sinthe, cosphi, sinphi, p1);
        if (p1.e < rd.ecut) edep += p1.e - prm;
        else push_spawn(C, ST_ELECTRON, p1, r);
        if ((ibcmpl == 1) || (ibcmpl == 3)) {
            if (gx_gt(uj, 0.001))
                relax(C, uj, __ldg(&P->shn_array[j - 1]), __ldg(&P->iz_array[j - 1]), edep, p, rd, r);
            else edep += uj;
        }
        break;
    }
    escore(C, p, p.region, edep * p.wt);
}

__device__ void photo(const DevCtx &C, Part p, Rng &r)
{
    const gegs_physics *P = C.P;
    const float rm = P->rm, prm = P->prm;
    RegInfo rd = region_info(C, p.region);
    float probs[GEGS_MXEL];
    int ints[GEGS_MXEL];
    float edep = 0.0f;
    unsigned medium = rd.med;
    float peig = p.e;
    unsigned iedgfl = rd.flags & GEGS_F_ATOMIC_RELAXATION;
    unsigned iphter = rd.flags & GEGS_F_PHOTO_ANGULAR;
    if (peig < __ldg(&P->edge_energies[1])) {
        p.charge = -1;
        p.e = peig + prm;
        if (p.e < rd.ecut) escore(C, p, p.region, (p.e - prm) * p.wt);
        else push_spawn(C, ST_ELECTRON, p, r);
        return;
    }
    float gle = gx_log(p.e);
    bool do_relax = false;
    float e_vac = 0.0f;
    int iz = 1, j = 0, k = 0;
    if (iedgfl != 0) {
        int nne = P->nne[medium];
        if (nne == 1) {
            iz = (int)(__ldg(&P->zelem[medium]) + 0.5);
            for (j = 0; j < __ldg(&P->edge_number[iz - 1]); j++)
                if (peig >= __ldg(&P->edge_energies[GEGS_MXEDGE * (iz - 1) + j])) break;
        } else {
            float aux = peig * peig;
            float aux1 = aux * peig;
            aux = aux * sqrtf(peig);
            float sigtot = 0.0f;
            for (k = 0; k < nne; k++) {
                iz = (int)(__ldg(&P->zelem[GX_MXMED * k + medium]) + 0.5);
                int b = GEGS_MXEDGE * (iz - 1);
                float sigma;
                if (peig > __ldg(&P->edge_energies[b])) {
                    j = 1;
                    sigma = (__ldg(&P->edge_a[b]) + __ldg(&P->edge_b[b]) / peig + __ldg(&P->edge_c[b]) / aux + __ldg(&P->edge_d[b]) / aux1) / peig;
                } else {
                    int ne = __ldg(&P->edge_number[iz - 1]);
                    for (j = 2; j <= ne; j++)
                        if (peig >= __ldg(&P->edge_energies[b + j - 1])) break;
                    sigma = __ldg(&P->edge_a[b + j - 1]) + gle * (__ldg(&P->edge_b[b + j - 1]) + gle * (__ldg(&P->edge_c[b + j - 1]) + gle * __ldg(&P->edge_d[b + j - 1])));
                    sigma = gx_exp(sigma);
                }
                sigma = sigma * __ldg(&P->pz[GX_MXMED * k + medium]);
                sigtot = sigtot + sigma;
                probs[k] = sigma;
                ints[k] = j;
            }
            float br = U(C, r);
            br = br * sigtot;
            for (k = 0; k < nne; k++) {
                br = br - probs[k];
                if (br <= 0.0f) break;
            }
            if (k >= nne) k = nne - 1;
            iz = (int)(__ldg(&P->zelem[GX_MXMED * k + medium]) + 0.5);
            j = ints[k];
        }
        if (peig <= __ldg(&P->binding_energies[GEGS_MXSHELL * (iz - 1) + 5])) {
            edep += peig;
        } else {
            float br = U(C, r);
            for (k = 1; k <= 5; k++) {
                if (peig > __ldg(&P->binding_energies[GEGS_MXSHELL * (iz - 1) + k - 1])) {
                    float tmp = __ldg(&P->interaction_prob[GEGS_MXSHELL * (iz - 1) + k - 1]);
                    if (br < tmp) break;
                    br = (br - tmp) / (1.0f - tmp);
                }
            }
            e_vac = __ldg(&P->binding_energies[GEGS_MXSHELL * (iz - 1) + k - 1]);
            p.e = peig - e_vac + prm;
            do_relax = true;
            p.charge = -1;
        }
    } else {
        p.e = peig + prm;
        p.charge = -1;
    }
    if (p.charge == -1) {
        if (p.e > rd.ecut) {
            if (iphter) {
                float beta = sqrtf((p.e - rm) * (p.e + rm)) / p.e;
                float gamma = p.e / rm;
                float alpha = 0.5 * gamma - 0.5 + 1.0f / gamma;
                float ratio = beta / alpha;
                float xi, rnpht2, sinth2, costhe;
                int nl = 0;
                do {
                    float rnpht = U(C, r);
                    rnpht = 2.0f * rnpht - 1.0f;
                    if (gx_le(ratio, 0.2)) {
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
                    rnpht2 = U(C, r);
                } while (rnpht2 > (0.5 * (1.0f + gamma) * sinth2 * xi / gamma) && ++nl < GX_LOOP_CAP);
                float sinthe = sqrtf(sinth2);
                float sinphi, cosphi;
                uphi21(C, costhe, sinthe, cosphi, sinphi, p, r);
            }
            push_spawn(C, ST_ELECTRON, p, r);
        } else {
            edep += p.e - prm;
        }
    }
    if (do_relax) relax(C, e_vac, k, iz, edep, p, rd, r);
    escore(C, p, p.region, edep * p.wt);
}

__device__ void rayleigh(const DevCtx &C, Part p, Rng &r)
{
    const gegs_physics *P = C.P;
    RegInfo rd = region_info(C, p.region);
    unsigned med = rd.med;
    float gle = gx_log(p.e);
    float2 ge = __ldg(reinterpret_cast<const float2 *>(P->ge[med]));
    int lgle = (int)(ge.x + ge.y * gle);
    float2 pm = __ldg(reinterpret_cast<const float2 *>(P->pmax[med * GX_MXGE + lgle]));
    float pmax_val = pm.x + pm.y * gle;
    float xmax = 80.65506856998f * p.e;
    float costhe = 0.0f, costhe2 = 0.0f;
    bool accept = false;
    int nouter = 0;
    const float4 *rdat = reinterpret_cast<const float4 *>(P->rayleigh_data[med * GEGS_MXRAYFF]);
    do {
        float xv = 0.0f;
        int ninner = 0;
        do {
            float r1 = U(C, r);
            float temp = r1 * pmax_val;
            int ibin = (int)(temp * (float)(GEGS_RAYCDFSIZE - 1));
            if (ibin > GEGS_RAYCDFSIZE - 2) ibin = GEGS_RAYCDFSIZE - 2;
            int ib = __ldg(&P->i_array[med * GEGS_RAYCDFSIZE + ibin]) - 1;
            int next_ib = __ldg(&P->i_array[med * GEGS_RAYCDFSIZE + ibin + 1]) - 1;
            if (next_ib > ib) {
                for (;;) {
                    float4 d = __ldg(&rdat[ib + 1]);
                    if ((temp < d.y) || (ib >= GEGS_RAYCDFSIZE - 2)) break;
                    ib++;
                }
            }
            float4 d = __ldg(&rdat[ib]);
            temp = (temp - d.y) * d.w;
            xv = d.x * gx_exp(gx_log(1.0f + temp) * d.z);
        } while (!(xv < xmax) && ++ninner < GX_LOOP_CAP);
        float r2 = U(C, r);
        xv = xv / p.e;
        costhe = 1.0f - 0.000307444456f * xv * xv;
        costhe2 = costhe * costhe;
        if (2.0f * r2 < 1.0f + costhe2) accept = true;
    } while (!accept && ++nouter < GX_LOOP_CAP);
    float sinthe = sqrtf(1.0f - costhe2);
    float cosphi, sinphi;
    uphi21(C, costhe, sinthe, cosphi, sinphi, p, r);
    if (p.e < rd.pcut) escore(C, p, p.region, p.e * p.wt);
    else push_spawn(C, ST_PHOTON, p, r);
}

__device__ void annih_at_rest(const DevCtx &C, Part &p, const RegInfo &rd, Rng &r)
{
    const gegs_physics *P = C.P;
    float edep = 0.0f;
    int nbr = P->nbr_split;
    if (nbr > 1) p.wt = p.wt / (float)nbr;
    p.e = P->prm;
    p.charge = 0;
    for (int ibr = 1; ibr <= nbr; ibr++) {
        float costhe = U(C, r);
        costhe = 2.0f * costhe - 1.0f;
        float sinthe = sqrtf(fmaxf_(0.0f, (1.0f - costhe) * (1.0f + costhe)));
        float cphi, sphi;
        box_phi(C, r, cphi, sphi);
        p.u = sinthe * cphi;
        p.v = sinthe * sphi;
        p.w = costhe;
        if (p.e < rd.pcut) edep += p.e;
        else push_spawn(C, ST_PHOTON, p, r);
        p.u = -p.u; p.v = -p.v; p.w = -p.w;
        if (p.e < rd.pcut) edep += p.e;
        else push_spawn(C, ST_PHOTON, p, r);
    }
    escore(C, p, p.region, edep * p.wt);
}

__device__ void pair_angle(const DevCtx &C, Rng &r, int use, float ese, float eig, unsigned medium, float &costhe, float &sinthe)
{
    const gegs_physics *P = C.P;
    const float rm = P->rm;
    if (use == 1) {
        float pse = sqrtf(fmaxf_(0.0f, (ese - rm) * (ese + rm)));
        float c = U(C, r);
        c = 1.0f - 2.0 * c;
        sinthe = rm * sqrtf((1.0f - c) * (1.0f + c)) / (pse * c + ese);
        costhe = (ese * c + pse) / (pse * c + ese);
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
        } while (((rtest > rtst) || (theta >= 3.1415926535f)) && ++n < GX_LOOP_CAP);
        gx_sincos(theta, &sinthe, &costhe);
    } else if (use == 3) {
        float c = U(C, r);
        c = 1.0f - 2.0f * c;
        float s = (1.0f - c) * (1.0f + c);
        costhe = c;
        sinthe = s > 0.0f ? sqrtf(s) : 0.0f;
    } else {
        float c = U(C, r);
        c = 1.0f - 2.0f * sqrtf(c);
        float s = (1.0f - c) * (1.0f + c);
        costhe = c;
        sinthe = s > 0.0f ? sqrtf(s) : 0.0f;
    }
}

__device__ void pair(const DevCtx &C, Part p, Rng &r)
{
    const gegs_physics *P = C.P;
    const float rm = P->rm, prm = P->prm, rmt2 = P->rmt2;
    RegInfo rd = region_info(C, p.region);
    float edep = 0.0f;
    Part p1 = p;
    unsigned m = rd.med;
    float eig = p.e;
    float ese1, ese2;
    int iq1, iq2;
    if (gx_le(eig, 2.1)) {
        float rnno30 = U(C, r);
        ese2 = prm + 0.5 * rnno30 * (eig - 2 * prm);
        rnno30 = U(C, r);
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
            rnno30 = U(C, r);
            float rnno31 = U(C, r);
            float br;
            if (rnno30 > aux1) { br = 0.5 * rnno31; rejmax = bmax; l1 = l + 1; }
            else {
                rnno30 = U(C, r);
                rnno30 = fmaxf_(rnno30, rnno31);
                rnno31 = U(C, r);
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
            rnno30 = U(C, r);
        } while ((rnno30 * rejmax) > rejf && ++n < GX_LOOP_CAP);
        ese2 = eminus;
        ese1 = eig - ese2;
        rnno30 = U(C, r);
        if (rnno30 < 0.5) { iq1 = -1; iq2 = 1; } else { iq1 = 1; iq2 = -1; }
    }
    p.e = ese1;
    p1.e = ese2;
    p.charge = (int8_t)iq1;
    p1.charge = (int8_t)iq2;
    float costhe = 1.0f, sinthe = 0.0f, sinphi, cosphi;
    int iprdst = P->iprdst;
    if (iprdst > 0) {
        int use;
        if (iprdst == 4) {
            float rtest = U(C, r);
            float gbeta = ese1 / (ese1 + 10.0f);
            use = (rtest < gbeta) ? 1 : 4;
        } else if ((iprdst == 2) && gx_lt(eig, 4.14)) use = 1;
        else use = iprdst;
        for (int ichrg = 1; ichrg <= 2; ichrg++) {
            float ese;
            if (ichrg == 1) ese = ese1;
            else {
                ese = ese2;
                if (iprdst == 4) {
                    float gbeta = ese / (ese + 10.0f);
                    float rtest = U(C, r);
                    use = (rtest < gbeta) ? 1 : 4;
                }
            }
            pair_angle(C, r, use, ese, eig, m, costhe, sinthe);
            if (ichrg == 1) {
                uphi21(C, costhe, sinthe, cosphi, sinphi, p, r);
                if (p.e < rd.ecut) {
                    edep += p.e - prm;
                    if (p.charge > 0) annih_at_rest(C, p, rd, r);
                } else push_spawn(C, ST_ELECTRON, p, r);
            } else {
                sinthe = -sinthe;
                uphi32(costhe, sinthe, cosphi, sinphi, p1);
                if (p1.e < rd.ecut) {
                    edep += p1.e - prm;
                    if (p1.charge > 0) annih_at_rest(C, p1, rd, r);
                } else push_spawn(C, ST_ELECTRON, p1, r);
            }
        }
        escore(C, p, p.region, edep * p.wt);
        return;
    }
    {
        float r1 = U(C, r);
        gx_sincos(0.0f, &sinthe, &costhe);
        float phi = 2.0f * 3.14159265f * r1;  // uphi11 (utility.cu:190-191)
        gx_sincos(phi, &sinphi, &cosphi);
        rotate_dir(costhe, sinthe, cosphi, sinphi, p);
    }
    if (p.e < rd.ecut) {
        edep += p.e - prm;
        if (p.charge > 0) annih_at_rest(C, p, rd, r);
    } else push_spawn(C, ST_ELECTRON, p, r);
    sinthe = -sinthe;
    uphi32(costhe, sinthe, cosphi, sinphi, p1);
    if (p1.e < rd.ecut) {
        edep += p1.e - prm;
        if (p1.charge > 0) annih_at_rest(C, p1, rd, r);
    } else push_spawn(C, ST_ELECTRON, p1, r);
    escore(C, p, p.region, edep * p.wt);
}
