// Device electron/positron transport (ELECTR, electron.cu:888-2622; PRESTA-I,
// spin off) and the discrete electron interactions:
//   mscat / sscat / msdist_pI   electron.cu:77-279, 618-882
//   moller (+ eii_sample)       moller.cu:16-210, eii_sample.cu:4-96
//   brems                       brems.cu:36-308
//   bhabha                      bhabha.cu:12-173
//   annih                       annih.cu:16-207
#pragma once
#include "dev_photon.cuh"

__device__ __forceinline__ float2 tab2(const float (*t)[2], int i) { return __ldg(reinterpret_cast<const float2 *>(t[i])); }
__device__ __forceinline__ float ev2(float2 t, float x) { return t.x + t.y * x; }

__device__ void mscat(const DevCtx &C, float lambda, float chia2, float q1, float &cost, float &sint, Rng &r)
{
    const gegs_physics *P = C.P;
    if (gx_le(lambda, 13.8)) {
        float sprob = U(C, r);
        float explambda = gx_exp(-lambda);
        if (sprob < explambda) { cost = 1.0f; sint = 0.0f; return; }
        float wsum = (1.0f + lambda) * explambda;
        if (sprob < wsum) {
            float xi = U(C, r);
            xi = 2.0f * chia2 * xi / (1.0f - xi + chia2);
            cost = 1.0f - xi;
            sint = sqrtf(xi * (2.0f - xi));
            return;
        }
        if (lambda <= 1.0f) {
            float wprob = explambda;
            wsum = explambda;
            cost = 1.0f;
            sint = 0.0f;
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
                if (gx_gt(sinz, 1.0e-20)) {
                    sinz = sqrtf(sinz);
                    xi = U(C, r);
                    float phi = xi * 6.2831853;
                    float sp, cp;
                    gx_sincos(phi, &sp, &cp);
                    cost = cost * cosz - sint * sinz * cp;
                    // sqrt(max(0.0, x)) in double (electron.cu:160), rounded to float:
                    // +0 for x <= 0, else the correctly rounded square root of x
                    const float sx = (1.0f - cost) * (1.0f + cost);
                    sint = sx > 0.0f ? sqrtf(sx) : 0.0f;
                }
            } while (wsum <= sprob);
            return;
        }
    }
    if (gx_le(lambda, 1e5)) {
        float llmbda = gx_log(lambda);
        float ai = llmbda * P->dllambi;
        int msi = (int)ai;
        ai = ai - (float)msi;
        float xi = U(C, r);
        if (xi < ai) msi = msi + 1;
        if (msi > GEGS_MAXL_MS) msi = GEGS_MAXL_MS;
        int msj;
        if (gx_lt(q1, 1e-3)) msj = 0;
        else if (q1 < 0.5f) {
            float aj = q1 * P->dqmsi;
            msj = (int)aj;
            aj = aj - (float)msj;
            xi = U(C, r);
            if (xi < aj) msj = msj + 1;
        } else msj = GEGS_MAXQ_MS;
        float omega2;
        if (gx_lt(llmbda, 2.2299))
            omega2 = chia2 * (lambda + 4) * (1.347006 + llmbda * (0.209364 - llmbda * (0.45525 - llmbda * (0.50142 - 0.081234 * llmbda))));
        else
            omega2 = chia2 * (lambda + 4) * (-2.77164 + llmbda * (2.94874 - llmbda * (0.1535754 - llmbda * 0.00552888)));
        xi = U(C, r);
        float ak = xi * (float)GEGS_MAXU_MS;
        int msk = (int)ak;
        ak = ak - (float)msk;
        if (msk > GEGS_MAXU_MS - 1) { msk = GEGS_MAXU_MS - 1; ak = 1.0f; }
        const int sj = (GEGS_MAXQ_MS + 1), sl = (GEGS_MAXL_MS + 1);
        int idx = (msk * sj + msj) * sl + msi;
        if (ak > __ldg(&P->wms_array[idx])) {
            msk = __ldg(&P->ims_array[idx]);
            idx = (msk * sj + msj) * sl + msi;
        }
        float a = __ldg(&P->fms_array[idx]);
        float u = __ldg(&P->ums_array[idx]);
        float du = __ldg(&P->ums_array[((msk + 1) * sj + msj) * sl + msi]) - u;
        xi = U(C, r);
        if (gx_lt(fabsf(a), 0.2)) {
            float x1 = 0.5 * (1 - xi) * a;
            u = u + xi * du * (1.0f + x1 * (1.0f - xi * a));
        } else
            u = u - du / a * (1.0f - sqrtf(1.0f + xi * a * (2.0f + a)));
        xi = omega2 * u / (1 + 0.5 * omega2 - u);
        if (gx_gt(xi, 1.99999)) xi = (float)1.99999;
        cost = 1.0f - xi;
        sint = sqrtf(xi * (2.0f - xi));
        return;
    }
    cost = 1.0f;
    sint = 0.0f;
}

__device__ __forceinline__ void sscat(const DevCtx &C, float chia2, float &cost, float &sint, Rng &r)
{
    float xi = U(C, r);
    xi = 2.0f * chia2 * xi / (1.0f - xi + chia2);
    cost = 1.0f - xi;
    sint = sqrtf(xi * (2.0f - xi));
}

__device__ void msdist_pI(const DevCtx &C, float eloss, float tustep, Part &p0, float &ustep, const RegInfo &rd, Rng &r)
{
    const gegs_physics *P = C.P;
    unsigned medium = rd.med;
    float e0 = p0.e - P->rm;
    float blccc = P->blcc[medium];
    float xcccc = P->xcc[medium];
    float e = e0 - 0.5 * eloss;
    float p2 = e * (e + P->rmt2);
    float chia2 = xcccc / p2 / (4.0f * blccc);
    float beta2 = p2 / (p2 + P->rmsq);
    float lambda = tustep * rd.rhof * blccc / beta2;
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
    mscat(C, lambda, chia2, xi, ws, sint, r);
    float cphi, sphi;
    box_phi(C, r, cphi, sphi);
    float us = sint * cphi;
    float vs = sint * sphi;
    float z, rr, r2, z2, r2max;
    if (gx_lt(xi, 0.1)) z = 1 - xi * (0.5 - xi * (0.166666667 - 0.041666667 * xi));
    else z = (1.0f - gx_exp(-xi)) / xi;
    rr = 0.5 * sint;
    r2 = rr * rr;
    z2 = z * z;
    r2max = 1.0f - z2;
    if (r2max < r2) { r2 = r2max; rr = sqrtf(r2); }
    float ut = rr * cphi, vt = rr * sphi, wt = z;
    ustep = sqrtf(z2 + r2) * tustep;
    float sint02 = p0.u * p0.u + p0.v * p0.v;
    if (gx_gt(sint02, 1e-20)) {
        float sint0 = sqrtf(sint02);
        float cphi0 = p0.u / sint0;
        float sphi0 = p0.v / sint0;
        float u2p = p0.w * us + sint0 * ws;
        ws = p0.w * ws - sint0 * us;
        us = u2p * cphi0 - vs * sphi0;
        vs = u2p * sphi0 + vs * cphi0;
        u2p = p0.w * ut + sint0 * wt;
        wt = p0.w * wt - sint0 * ut;
        ut = u2p * cphi0 - vt * sphi0;
        vt = u2p * sphi0 + vt * cphi0;
    } else {
        wt = p0.w * wt;
        ws = p0.w * ws;
    }
    p0.x = p0.x + tustep * ut;
    p0.y = p0.y + tustep * vt;
    p0.z = p0.z + tustep * wt;
    p0.u = us;
    p0.v = vs;
    p0.w = ws;
}

__device__ __forceinline__ float range_piece(const gegs_physics *P, int qel, unsigned medium, int lel, float elk_a, float elk_b,
                                             float e_hi, float fedep)
{
    float elktmp = 0.5 * (elk_a + elk_b + 0.25 * fedep * fedep * (1 + fedep * (1 + 0.875 * fedep)));
    float2 d = tab2(P->dedx, qel * GX_MXEKE * GX_MXMED + medium * GX_MXEKE + lel - 1);
    float dedxmid = d.x + d.y * elktmp;
    dedxmid = 1.0f / dedxmid;
    float aux = d.y * dedxmid;
    float temp = fedep / (2.0f - fedep);
    aux = aux * (1.0f + 2.0f * aux) * temp * temp / 6.0f;
    return fedep * e_hi * dedxmid * (1.0f + aux);
}

__device__ float compute_eloss(const gegs_physics *P, int qel, unsigned medium, float step, float range, float rhof,
                               float eke_val, float elke, int lelke)
{
    float2 ex = tab2(P->eke01, medium);
    float de;
    float tuss = range - __ldg(&P->range_ep[(medium * GX_MXEKE + lelke - 1) * 2 + qel]) / rhof;
    if (tuss >= step) {
        float2 d = tab2(P->dedx, qel * GX_MXEKE * GX_MXMED + medium * GX_MXEKE + lelke - 1);
        float dedxmid = d.x + d.y * elke;
        float aux = d.y / dedxmid;
        de = dedxmid * step * rhof;
        float fedep = de / eke_val;
        de = de * (1 - 0.5 * fedep * aux * (1 - 0.333333 * fedep * (aux - 1 - 0.25 * fedep * (2 - aux * (4 - aux)))));
    } else {
        int lelktmp = lelke;
        tuss = (range - step) * rhof;
        if (tuss <= 0.0f) de = eke_val - P->te[medium] * 0.99;
        else {
            while (lelktmp > 1 && tuss < __ldg(&P->range_ep[(medium * GX_MXEKE + lelktmp - 1) * 2 + qel])) lelktmp = lelktmp - 1;
            float elktmp = ((float)(lelktmp + 1) - ex.x) / ex.y;
            float eketmp = __ldg(&P->e_array[medium * GX_MXEKE + lelktmp]);
            tuss = (__ldg(&P->range_ep[(medium * GX_MXEKE + lelktmp) * 2 + qel]) - tuss) / rhof;
            float2 d = tab2(P->dedx, qel * GX_MXEKE * GX_MXMED + medium * GX_MXEKE + lelktmp - 1);
            float dedxmid = d.x + d.y * elktmp;
            float aux = d.y / dedxmid;
            de = dedxmid * tuss * rhof;
            float fedep = de / eketmp;
            de = de * (1 - 0.5 * fedep * aux * (1 - 0.333333 * fedep * (aux - 1 - 0.25 * fedep * (2 - aux * (4 - aux)))));
            de = de + eke_val - eketmp;
        }
    }
    return de;
}

// state an electron carries between steps inside the electron stage
struct EState {
    float elke, demfp, sig0, total_tstep;
    int lelke;
    bool compute_tstep, is_tstep;
};

__device__ __forceinline__ void estate_init(EState &s)
{
    s.elke = 0.0f; s.demfp = 0.0f; s.sig0 = 0.0f; s.total_tstep = 0.0f;
    s.lelke = 0; s.compute_tstep = true; s.is_tstep = true;
}

// A positron at rest handed to the annihilation kernel carries energy 0 (one
// annihilating in flight carries its total energy, above the rest mass).
__device__ __forceinline__ bool at_rest_mark(const Part &p) { return p.e == 0.0f; }

__device__ __forceinline__ void e_discard_below_cut(const DevCtx &C, Part &p, const RegInfo &rd, Rng &r)
{
    escore(C, p, p.region, (p.e - C.P->prm) * p.wt);
    if (p.charge > 0) {
        if (C.pipelined) {
            // the photon transport of this wave runs beside this kernel and takes
            // no new photons: the annihilation kernel, after both transports,
            // makes them from the same random stream (region_info(p.region) is rd)
            p.e = 0.0f;
            push_move(C, ST_ANNIH, p, r);
        } else annih_at_rest(C, p, rd, r);
    }
}

// One iteration of the ELECTR loop.  Returns true when the particle has left
// the electron stage.
// Returns 0 while the particle stays in the electron stage, 1 when it has
// left it, (DEFER only) 2 when the step needs howfar and (ONLY_NEAR only) 3
// when it does not, before the step changes the particle: the caller then
// re-queues the particle as it stood at the start of the step (howfar is the
// first thing in the step that changes the particle; the step state and the
// random counter are restored by the caller), and the step runs again, whole,
// in a pass whose warps hold only such particles.
template <int G = GX_GEOM_ALL, bool DEFER = false, bool ONLY_NEAR = false>
__device__ int electron_step(const DevCtx &C, Part &p, Rng &r, EState &s)
{
    const gegs_physics *P = C.P;
    const float rm = P->rm, prm = P->prm, rmt2 = P->rmt2, rmsq = P->rmsq;
    uint32_t irold = p.region, irl = irold;
    RegInfo rd = region_info(C, irl);
    unsigned medium = rd.med;
    float rhof = rd.rhof;
    int lelec = p.charge;
    int qel = (1 + lelec) / 2;
    float eie = p.e;
    if (eie <= rd.ecut) { e_discard_below_cut(C, p, rd, r); return true; }
    if (p.wt <= 0.0f) return true;
    float eke_val = eie - rm;
    if (s.is_tstep) {
        s.compute_tstep = true;
        if (medium != GX_VACUUM) {
            float rnne1 = U(C, r);
            if (rnne1 == 0.0f) rnne1 = 1.0E-30f;
            s.demfp = fmaxf_(-gx_log(rnne1), GX_EPSEMFP);
            s.elke = gx_log(eke_val);
            float2 e01 = tab2(P->eke01, medium);
            s.lelke = (int)(e01.x + e01.y * s.elke);
            if (__ldg(&P->sig_ismonotone[medium * 2 + qel])) {
                float sigf = ev2(tab2(P->sig, qel * GX_MXEKE * GX_MXMED + medium * GX_MXEKE + s.lelke - 1), s.elke);
                float dedx0 = ev2(tab2(P->dedx, qel * GX_MXEKE * GX_MXMED + medium * GX_MXEKE + s.lelke - 1), s.elke);
                sigf = sigf / dedx0;
                s.sig0 = sigf;
            } else s.sig0 = __ldg(&P->sig_e[qel * GX_MXMED + medium]);
        }
    }
    const float elke = s.elke;
    const int lelke = s.lelke;
    float sig_val = 0.0f, dedx_val = 0.0f, tstep = 0.0f, ustep = 0.0f, tustep = 0.0f, tvstep = 0.0f, vstep = 0.0f;
    float range = 0.0f, de = 0.0f, blccl = 0.0f, xccl = 0.0f, beta2 = 0.0f, chia2 = 0.0f, xi = 0.0f, tperp = 0.0f;
    bool callhowfar = false, domultiple = false, dosingle = false, callmsdist = false;
    if (medium == GX_VACUUM) {
        tstep = GX_VACUUM_STEP;
        ustep = tstep;
        tustep = ustep;
        callhowfar = true;
    } else {
        float2 e01 = tab2(P->eke01, medium);
        sig_val = s.sig0;
        if (sig_val <= 0.0f) { tstep = GX_VACUUM_STEP; s.sig0 = 1.0E-15f; }
        else {
            if (s.compute_tstep) {
                float total_de = s.demfp / sig_val;
                float ekef = eke_val - total_de;
                if (ekef <= __ldg(&P->e_array[medium * GX_MXEKE + 0])) tstep = GX_VACUUM_STEP;
                else {
                    float elkef = gx_log(ekef);
                    int lelkef = (int)(e01.x + e01.y * elkef);
                    if (lelkef == lelke) {
                        float fedep = 1.0f - ekef / eke_val;
                        tstep = range_piece(P, qel, medium, lelke, elke, elkef, eke_val, fedep);
                    } else {
                        float ekei = __ldg(&P->e_array[medium * GX_MXEKE + lelke - 1]);
                        float elkei = ((float)lelke - e01.x) / e01.y;
                        float fedep = 1.0f - ekei / eke_val;
                        float tuss = range_piece(P, qel, medium, lelke, elke, elkei, eke_val, fedep);
                        ekei = __ldg(&P->e_array[medium * GX_MXEKE + lelkef]);
                        elkei = ((float)(lelkef + 1) - e01.x) / e01.y;
                        fedep = 1.0f - ekef / ekei;
                        tstep = range_piece(P, qel, medium, lelkef, elkei, elkef, ekei, fedep);
                        tstep = tstep + tuss + __ldg(&P->range_ep[(medium * GX_MXEKE + lelke - 1) * 2 + qel])
                                - __ldg(&P->range_ep[(medium * GX_MXEKE + lelkef) * 2 + qel]);
                    }
                }
                s.total_tstep = tstep;
                s.compute_tstep = false;
            }
            tstep = s.total_tstep / rhof;
        }
        float dedx0 = ev2(tab2(P->dedx, qel * GX_MXEKE * GX_MXMED + medium * GX_MXEKE + lelke - 1), elke);
        dedx_val = rhof * dedx0;
        float tmxs_val = ev2(tab2(P->tmxs, medium * GX_MXEKE + lelke - 1), elke);
        tmxs_val = tmxs_val / rhof;
        {
            float ekei = __ldg(&P->e_array[medium * GX_MXEKE + lelke - 1]);
            float elkei = ((float)lelke - e01.x) / e01.y;
            float fedep = 1.0f - ekei / eke_val;
            range = range_piece(P, qel, medium, lelke, elke, elkei, eke_val, fedep);
            range = (range + __ldg(&P->range_ep[(medium * GX_MXEKE + lelke - 1) * 2 + qel])) / rhof;
        }
        tmxs_val = fminf_(tmxs_val, P->smaxir[medium]);
        tustep = fminf_(tstep, fminf_(tmxs_val, range));
        const bool do_rr = P->i_do_rr[medium] == 1 && p.e < P->e_max_rr[medium];
        // In the jaws, a lower bound of hownear above the thresholds it is
        // compared with (range for range rejection, else tustep) decides every
        // comparison below as the exact value would, and then tustep is left
        // unchanged: the bound stands in for the value.
        float lb = -1.0f;
        if (G == GX_GEOM_JAWS && (p.module == GEGS_M_SECJAWY || p.module == GEGS_M_SECJAWX))
            lb = jaws_near_lower_bound(C, p);
        if (lb > (do_rr ? range : tustep)) tperp = lb;
        else {
            bool ok;
            hownear_g<G>(C, p, tperp, ok);
            if (!ok) { atomicOr(C.err, GX_ERR_MODULE); return true; }
        }
        if (do_rr) {
            if (tperp >= range) { e_discard_below_cut(C, p, rd, r); return true; }
        }
        blccl = rhof * P->blcc[medium];
        xccl = rhof * P->xcc[medium];
        float p2 = eke_val * (eke_val + rmt2);
        beta2 = p2 / (p2 + rmsq);
        float ssmfp = beta2 / blccl;
        float skindepth = P->skindepth_for_bca * ssmfp;
        tustep = fminf_(tustep, fmaxf_(tperp, skindepth));
        if (tustep <= tperp && (!P->exact_bca || tustep > skindepth)) {
            callmsdist = true;
            de = compute_eloss(P, qel, medium, tustep, range, rhof, eke_val, elke, lelke);
            tvstep = tustep;
            if (ONLY_NEAR) return 3;
            msdist_pI(C, de, tustep, p, ustep, rd, r);
        } else {
            if (P->exact_bca) {
                float rnnoss = U(C, r);
                float lambda = -gx_log(1.0f - rnnoss);
                float tmp = (eke_val / rm + 1.0f);
                float lambda_max = 0.5 * blccl * rm / dedx_val * tmp * tmp * tmp;
                if (lambda >= 0.0f && lambda_max > 0.0f) {
                    float tuss;
                    if (lambda < lambda_max) tuss = lambda * ssmfp * (1 - 0.5 * lambda / lambda_max);
                    else tuss = 0.5 * lambda * ssmfp;
                    if (tuss < tustep) { tustep = tuss; dosingle = true; } else dosingle = false;
                } else return true;
                ustep = tustep;
            } else {
                domultiple = true;
                float ekems = eke_val - 0.5 * tustep * dedx_val;
                p2 = ekems * (ekems + rmt2);
                beta2 = p2 / (p2 + rmsq);
                chia2 = xccl / (4.0f * blccl * p2);
                xi = 0.5 * xccl / p2 / beta2 * tustep;
                xi = xi * (gx_log((float)(1 + 1.0 / chia2)) - 1 / (1 + chia2));
                if (gx_lt(xi, 0.1)) ustep = tustep * (1 - xi * (0.5 - xi * 0.166667));
                else ustep = tustep * (1.0f - gx_exp(-xi)) / xi;
            }
            callhowfar = !(ustep < tperp);
            if (ONLY_NEAR && !callhowfar) return 3;
        }
    }
    uint32_t irnew = p.region;
    int idisc = 0;
    float ustep0 = ustep;
    if (callhowfar || p.wt <= 0.0f) {
        if (DEFER) return 2;
        bool ok;
        irnew = howfar_g<G>(C, p, ustep, ok);
        if (!ok) { atomicOr(C.err, GX_ERR_MODULE); return true; }
    }
    if (irnew == 0) {
        if (rd.med == GX_VACUUM || p.leafIndex == GX_PASSMLC) idisc = 1; else idisc = -1;
    }
    if (idisc > 0) {
        p.region = 0;
        escore(C, p, 0, (p.e + (float)p.charge * prm) * p.wt);
        return true;
    }
    if (ustep <= 0.0f) ustep = 0.0f;
    if (ustep == 0.0f || medium == GX_VACUUM) {
        if (ustep != 0.0f) {
            vstep = ustep;
            p.x = p.x + p.u * vstep;
            p.y = p.y + p.v * vstep;
            p.z = p.z + p.w * vstep;
        }
        p.region = irnew;
        rd = region_info(C, irnew);
        if (eie <= rd.ecut) { e_discard_below_cut(C, p, rd, r); return true; }
        if (ustep != 0.0f && idisc < 0) {
            escore(C, p, p.region, (p.e + (float)p.charge * prm) * p.wt);
            return true;
        }
        s.is_tstep = true;
        return false;
    }
    vstep = ustep;
    if (callhowfar) {
        if (P->exact_bca) {
            tvstep = vstep;
            if (tvstep != tustep) dosingle = false;
        } else {
            if (vstep < ustep0) {
                float ekems = eke_val - 0.5 * tustep * vstep / ustep0 * dedx_val;
                float p2 = ekems * (ekems + rmt2);
                beta2 = p2 / (p2 + rmsq);
                chia2 = xccl / (4.0f * blccl * p2);
                xi = 0.5 * xccl / p2 / beta2 * vstep;
                xi = xi * (gx_log((float)(1 + 1.0 / chia2)) - 1 / (1 + chia2));
                if (gx_lt(xi, 0.1)) tvstep = vstep * (1 + xi * (0.5 + xi * 0.333333));
                else {
                    if (gx_lt(xi, 0.999999)) tvstep = -vstep * gx_log(1 - xi) / xi;
                    else return true;
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
            mscat(C, lambda, chia2, xi, costhe, sinthe, r);
        } else if (dosingle) {
            float ekems = fmaxf_(ekef, rd.ecut - rm);
            float p2 = ekems * (ekems + rmt2);
            beta2 = p2 / (p2 + rmsq);
            chia2 = P->xcc[medium] / (4.0f * P->blcc[medium] * p2);
            sscat(C, chia2, costhe, sinthe, r);
        } else { sinthe = 0.0f; costhe = 1.0f; }
        p.x = p.x + p.u * vstep;
        p.y = p.y + p.v * vstep;
        p.z = p.z + p.w * vstep;
        if (domultiple || dosingle) {
            float sinphi, cosphi;
            uphi21(C, costhe, sinthe, cosphi, sinphi, p, r);
        }
    }
    irold = p.region;
    eie = eie - edep;
    p.e = eie;
    escore(C, p, irold, edep * p.wt);
    if (irnew == irl && eie <= rd.ecut) { e_discard_below_cut(C, p, rd, r); return true; }
    unsigned medold = medium;
    if (medium != GX_VACUUM) {
        eke_val = eie - rm;
        s.elke = gx_log(eke_val);
        float2 e01 = tab2(P->eke01, medium);
        s.lelke = (int)(e01.x + e01.y * s.elke);
    }
    if (irnew != irold) {
        p.region = irnew;
        irl = irnew;
        rd = region_info(C, irl);
        medium = rd.med;
    }
    if (eie <= rd.ecut) { e_discard_below_cut(C, p, rd, r); return true; }
    if (idisc < 0) {
        escore(C, p, p.region, (p.e + (float)p.charge * prm) * p.wt);
        return true;
    }
    if (medium != medold) { s.is_tstep = true; return false; }
    s.demfp = s.demfp - save_de * sig_val;
    s.total_tstep = s.total_tstep - tvstep * rhof;
    if (gx_lt(s.total_tstep, 1e-9)) s.demfp = 0.0f;
    if (gx_ge(s.demfp, GX_EPSEMFP)) { s.is_tstep = false; return false; }
    float sigf = ev2(tab2(P->sig, qel * GX_MXEKE * GX_MXMED + medium * GX_MXEKE + s.lelke - 1), s.elke);
    float dedx0 = ev2(tab2(P->dedx, qel * GX_MXEKE * GX_MXMED + medium * GX_MXEKE + s.lelke - 1), s.elke);
    sigf = sigf / dedx0;
    float sigratio = sigf / s.sig0;
    float rfict = U(C, r);
    if (rfict > sigratio) { s.is_tstep = true; return false; }
    if (lelec < 0) {
        float ebr1_val = ev2(tab2(P->ebr1, medium * GX_MXEKE + s.lelke - 1), s.elke);
        float rnno24 = U(C, r);
        if (rnno24 <= ebr1_val) { push_move(C, ST_BREMS, p, r); return true; }
        if (p.e <= P->thmoll[medium] && P->eii_flag == 0) {
            if (ebr1_val <= 0.0f) { s.is_tstep = true; return false; }
            push_move(C, ST_BREMS, p, r);
            return true;
        }
        push_move(C, ST_MOLLER, p, r);
        return true;
    }
    float pbr1_val = ev2(tab2(P->pbr1, medium * GX_MXEKE + s.lelke - 1), s.elke);
    float rnno25 = U(C, r);
    if (rnno25 < pbr1_val) { push_move(C, ST_BREMS, p, r); return true; }
    float pbr2_val = ev2(tab2(P->pbr2, medium * GX_MXEKE + s.lelke - 1), s.elke);
    if (rnno25 < pbr2_val) push_move(C, ST_BHABHA, p, r);
    else push_move(C, ST_ANNIH, p, r);
    return true;
}

__device__ void eii_sample(const DevCtx &C, int ish, int iz, float uj, Part &p, const RegInfo &rd, Rng &r, float &edep)
{
    const gegs_physics *P = C.P;
    const float rm = P->rm, prm = P->prm, rmt2 = P->rmt2;
    unsigned medium = rd.med;
    Part p1 = p;
    float eie = p.e;
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
    } while (r1 >= frej && ++n < GX_LOOP_CAP);
    wx = wx * uj;
    float h1 = (eie + prm) / t;
    float ese1 = eie - wx;
    p.e = ese1;
    float dcosth = h1 * (ese1 - prm) / (ese1 + prm);
    float sinthe = sqrtf(fmaxf_(0.0f, 1.0f - dcosth));
    float costhe = sqrtf(dcosth);
    float sinphi, cosphi;
    uphi21(C, costhe, sinthe, cosphi, sinphi, p, r);
    float ese2 = wx - uj + prm;
    if (ese2 > P->ae[medium]) {
        p1.e = ese2;
        dcosth = h1 * (ese2 - prm) / (ese2 + prm);
        sinthe = -sqrtf(fmaxf_(0.0f, 1.0f - dcosth));
        costhe = sqrtf(dcosth);
        uphi32(costhe, sinthe, cosphi, sinphi, p1);
        push_spawn(C, ST_ELECTRON, p1, r);
        edep = 0.0f;
    } else {
        edep = wx - uj;
    }
    relax(C, uj, ish, iz, edep, p, rd, r);
}

__device__ void moller(const DevCtx &C, Part p, Rng &r)
{
    const gegs_physics *P = C.P;
    const float rm = P->rm, prm = P->prm;
    RegInfo rd = region_info(C, p.region);
    float edep = 0.0f;
    Part p1 = p;
    unsigned medium = rd.med;
    float eie = p.e;
    float ekin = eie - prm;
    float elke = gx_log(ekin);
    if ((P->eii_flag > 0) && (P->eii_nsh[medium] > 0)) {
        float2 e01 = tab2(P->eke01, medium);
        int lelke = (int)(e01.y * elke + e01.x);
        float2 sg = tab2(P->sig, medium * GX_MXEKE + lelke - 1);
        float2 eb = tab2(P->ebr1, medium * GX_MXEKE + lelke - 1);
        float sigm = sg.y * elke + sg.x;
        float pbrem = eb.y * elke + eb.x;
        sigm = sigm * (1.0f - pbrem);
        float rsh = U(C, r);
        rsh = sigm * rsh;
        int nne = P->nne[medium];
        for (int iele = 0; iele < nne; iele++) {
            int iz = (int)(__ldg(&P->zelem[iele * GX_MXMED + medium]) + 0.5);
            int nsh = __ldg(&P->eii_no[iele * GX_MXMED + medium]);
            if (nsh > 0) {
                int ifirst = __ldg(&P->eii_first[iele * GX_MXMED + medium]);
                for (int ish = 1; ish <= nsh; ish++) {
                    float uj = __ldg(&P->binding_energies[(iz - 1) * GEGS_MXSHELL + ish - 1]);
                    if ((ekin > uj) && (uj > P->te[medium] || uj > P->ap[medium])) {
                        int jj = ifirst + ish - 1;
                        float2 ej = tab2(P->eii, jj - 1);
                        int i = (int)(ej.x * elke + ej.y + (float)((jj - 1) * GEGS_N_EII_BINS));
                        if (i < 1 + (jj - 1) * GEGS_N_EII_BINS) i = 1 + (jj - 1) * GEGS_N_EII_BINS;
                        if (i > jj * GEGS_N_EII_BINS) i = jj * GEGS_N_EII_BINS;
                        float2 ex = tab2(P->eii_xsection, i - 1);
                        float sig_j = ex.x * elke + ex.y;
                        sig_j = sig_j * __ldg(&P->pz[GX_MXMED * iele + medium]) * P->eii_cons[medium];
                        rsh -= sig_j;
                        if (rsh < 0.0f) {
                            eii_sample(C, ish, iz, uj, p, rd, r, edep);
                            if (p.e < rd.ecut) edep += p.e - prm;
                            else push_spawn(C, ST_ELECTRON, p, r);
                            escore(C, p, p.region, edep * p.wt);
                            return;
                        }
                    }
                }
            }
        }
    }
    float te = P->te[medium];
    if (ekin <= 2.0f * te) { escore(C, p, p.region, (p.e - prm) * p.wt); return; }
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
        rnno27 = U(C, r);
        br = te / (ekin - extrae * rnno27);
        rr = br / (1.0f - br);
        rnno27 = U(C, r);
        rejf4 = (1.0f + g2 * br * br + rr * (rr - g3));
        rnno27 = gmax * rnno27;
    } while (rnno27 > rejf4 && ++n < GX_LOOP_CAP);
    float ekse2 = br * ekin;
    float ese1 = eie - ekse2;
    float ese2 = ekse2 + prm;
    p.e = ese1;
    p1.e = ese2;
    float h1 = (eie + prm) / ekin;
    float dcosth = h1 * (ese1 - prm) / (ese1 + prm);
    float sinthe = sqrtf(fmaxf_(0.0f, 1.0f - dcosth));
    float costhe = sqrtf(dcosth);
    float sinphi, cosphi;
    uphi21(C, costhe, sinthe, cosphi, sinphi, p, r);
    if (p.e < rd.ecut) edep += p.e - prm;
    else push_spawn(C, ST_ELECTRON, p, r);
    dcosth = h1 * (ese2 - prm) / (ese2 + prm);
    sinthe = -sqrtf(fmaxf_(0.0f, 1.0f - dcosth));
    costhe = sqrtf(dcosth);
    uphi32(costhe, sinthe, cosphi, sinphi, p1);
    if (p1.e < rd.ecut) edep += p1.e - prm;
    else push_spawn(C, ST_ELECTRON, p1, r);
    escore(C, p, p.region, edep * p.wt);
}

__device__ void brems(const DevCtx &C, Part p, Rng &r)
{
    const gegs_physics *P = C.P;
    const float rm = P->rm, prm = P->prm;
    RegInfo rd = region_info(C, p.region);
    float edep = 0.0f;
    Part p1 = p;
    unsigned m = rd.med;
    int nbr = P->nbr_split;
    if (nbr < 1) return;
    float eie = p.e;
    int l = gx_lt(eie, 50.0) ? 1 : 3;
    int l1 = l + 1;
    float ekin = eie - prm;
    float elke = gx_log(ekin);
    float brmin = P->ap[m] / ekin;
    float waux = elke - P->log_ap[m];
    float a = 0.0f, b = 0.0f, c = 0.0f, sinpsi = 0.0f, sindel = 0.0f, cosdel = 0.0f;
    float ztarg = 0.0f, tteie = 0.0f, y2maxi = 0.0f, z2maxi = 0.0f;
    int ibrdst = P->ibrdst;
    if (ibrdst >= 0) {
        a = p.u; b = p.v; c = p.w;
        sinpsi = a * a + b * b;
        if (gx_gt(sinpsi, 1e-20)) {
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
            rnno06 = U(C, r);
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
            rnno06 = U(C, r);
        } while (rnno06 >= rejf && ++n < GX_LOOP_CAP);
        p1.e = esg;
        p1.charge = 0;
        p1.wt = p.wt / (float)nbr;
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
                    y2tst = U(C, r);
                    rtest = U(C, r);
                    float aux3 = z2maxi / (y2tst + (1.0f - y2tst) * z2maxi);
                    rtest = rtest * aux3 * rejmax;
                    y2tst = aux3 * aux3 - 1.0f;
                    float y2tst1 = esedei * y2tst / (aux3 * aux3 * aux3 * aux3);
                    float aux4 = 16.0f * y2tst1 - rjarg2;
                    float aux5 = rjarg1 - 4.0f * y2tst1;
                    if (rtest < (aux4 + aux5 * rjarg3)) break;
                    float aux2 = gx_log(aux / (1.0f + aux1 / (aux3 * aux3 * aux3 * aux3)));
                    rejtst = aux4 + aux5 * aux2;
                } while (rtest >= rejtst && ++nn < GX_LOOP_CAP);
            } else {
                y2tst = U(C, r);
                y2tst = y2tst / (1.0f - y2tst + y2maxi);
            }
            float costhe = 1.0f - 2.0f * y2tst * y2maxi;
            float sinthe = sqrtf(fmaxf_((1.0f - costhe) * (1.0f + costhe), 0.0f));
            float cphi, sphi;
            box_phi(C, r, cphi, sphi);
            if (gx_ge(sinpsi, 1e-10)) {
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
        if (p1.e < rd.pcut) edep += p1.e;
        else push_spawn(C, ST_PHOTON, p1, r);
    }
    p.e = ese;
    if (p.e < rd.ecut) edep += p.e - prm;
    else push_spawn(C, ST_ELECTRON, p, r);
    escore(C, p, p.region, edep * p.wt);
}

__device__ void bhabha(const DevCtx &C, Part p, Rng &r)
{
    const gegs_physics *P = C.P;
    const float rm = P->rm, prm = P->prm;
    RegInfo rd = region_info(C, p.region);
    float edep = 0.0f;
    Part p1 = p;
    unsigned m = rd.med;
    float eip = p.e;
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
        rnno03 = U(C, r);
        br = ep0 / (1.0f - ep0c * rnno03);
        rnno03 = U(C, r);
        rejf2 = (1.0f - beta2 * br * (b1 - br * (b2 - br * (b3 - br * b4))));
    } while (rnno03 > rejf2 && ++n < GX_LOOP_CAP);
    if (br < 0.5f) p1.charge = -1;
    else { p.charge = -1; p1.charge = 1; br = 1.0f - br; }
    br = fmaxf_(br, 0.0f);
    float ekse2 = br * ekin;
    float ese1 = eip - ekse2;
    float ese2 = ekse2 + prm;
    p.e = ese1;
    p1.e = ese2;
    float h1 = (eip + prm) / ekin;
    float dcosth = fminf_(1.0f, h1 * (ese1 - prm) / (ese1 + prm));
    float sinthe = sqrtf(1.0f - dcosth);
    float costhe = sqrtf(dcosth);
    float sinphi, cosphi;
    uphi21(C, costhe, sinthe, cosphi, sinphi, p, r);
    if (p.e < rd.ecut) {
        edep += p.e - prm;
        if (p.charge > 0) annih_at_rest(C, p, rd, r);
    } else push_spawn(C, ST_ELECTRON, p, r);
    dcosth = h1 * (ese2 - prm) / (ese2 + prm);
    sinthe = -sqrtf(fmaxf_(0.0f, 1.0f - dcosth));
    costhe = sqrtf(dcosth);
    uphi32(costhe, sinthe, cosphi, sinphi, p1);
    if (p1.e < rd.ecut) {
        edep += p1.e - prm;
        if (p1.charge > 0) annih_at_rest(C, p1, rd, r);
    } else push_spawn(C, ST_ELECTRON, p1, r);
    escore(C, p, p.region, edep * p.wt);
}

__device__ void annih(const DevCtx &C, Part p, Rng &r)
{
    const gegs_physics *P = C.P;
    const float rm = P->rm, prm = P->prm;
    RegInfo rd = region_info(C, p.region);
    float edep = 0.0f;
    int nbr = P->nbr_split;
    if (nbr <= 0) return;
    float avip = p.e + prm;
    float a = avip / rm;
    float g = a - 1.0f;
    float t = g - 1.0f;
    float pp = sqrtf(a * t);
    float pot = pp / t;
    float ep0 = 1.0f / (a + pp);
    float wsamp = gx_log((1.0f - ep0) / ep0);
    float aa = p.u, bb = p.v, cc = p.w;
    float sinpsi = aa * aa + bb * bb, sindel = 0.0f, cosdel = 0.0f;
    if (gx_gt(sinpsi, 1e-20)) {
        sinpsi = sqrtf(sinpsi);
        sindel = bb / sinpsi;
        cosdel = aa / sinpsi;
    }
    if (nbr > 1) p.wt = p.wt / (float)nbr;
    for (int ibr = 1; ibr <= nbr; ibr++) {
        float rnno01, rejf, ep;
        int n = 0;
        do {
            rnno01 = U(C, r);
            ep = ep0 * gx_exp(rnno01 * wsamp);
            rnno01 = U(C, r);
            rejf = 1.0f - (ep * a - 1.0f) * (ep * a - 1.0f) / (ep * (a * a - 2.0f));
        } while (rnno01 > rejf && ++n < GX_LOOP_CAP);
        float esg1 = avip * ep;
        p.e = esg1;
        p.charge = 0;
        float costhe = fminf_(1.0f, (esg1 - rm) * pot / esg1);
        float sinthe = sqrtf(1.0f - costhe * costhe);
        float cphi, sphi;
        box_phi(C, r, cphi, sphi);
        if (gx_ge(sinpsi, 1e-10)) {
            float us = sinthe * cphi, vs = sinthe * sphi;
            p.u = cc * cosdel * us - sindel * vs + aa * costhe;
            p.v = cc * sindel * us + cosdel * vs + bb * costhe;
            p.w = cc * costhe - sinpsi * us;
        } else {
            p.u = sinthe * cphi; p.v = sinthe * sphi; p.w = cc * costhe;
        }
        if (p.e < rd.pcut) edep += p.e;
        else push_spawn(C, ST_PHOTON, p, r);
        float esg2 = avip - esg1;
        p.e = esg2;
        costhe = fminf_(1.0f, (esg2 - rm) * pot / esg2);
        sinthe = -sqrtf(1.0f - costhe * costhe);
        if (gx_ge(sinpsi, 1e-10)) {
            float us = sinthe * cphi, vs = sinthe * sphi;
            p.u = cc * cosdel * us - sindel * vs + aa * costhe;
            p.v = cc * sindel * us + cosdel * vs + bb * costhe;
            p.w = cc * costhe - sinpsi * us;
        } else {
            p.u = sinthe * cphi; p.v = sinthe * sphi; p.w = cc * costhe;
        }
        if (p.e < rd.pcut) edep += p.e;
        else push_spawn(C, ST_PHOTON, p, r);
    }
    escore(C, p, p.region, edep * p.wt);
}
