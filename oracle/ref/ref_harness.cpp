/* Reference-pinning harness -- TEST INFRASTRUCTURE ONLY.
 *
 * Compiles the reference's own device sources, unmodified, from where they
 * lie (the recipe in oracle/ref/Makefile passes their directory with -I), as
 * host C++: geom.cu (howfar/hownear of the phantom, the DYNVMLC and the
 * secondary jaws), utility.cu (uphi21/32/11, the particle stacks), relax.cu,
 * and the ten stage kernels (photon.cu, compton.cu, photo.cu, rayleigh.cu,
 * pair.cu, electron.cu, moller.cu, brems.cu, bhabha.cu, annih.cu, with
 * eii_sample.cu and annihatrest.cu). The stand-in headers in shim/ turn the
 * CUDA qualifiers into no-ops and run every kernel as one thread; ref_math.h
 * binds the transcendental functions to the oracle's own; curand_uniform
 * replays a supplied stream. The exported ref_* functions below fill the
 * reference's device globals from a gegs_physics block and a gegs_scene and
 * run one routine on given particles, so tests can compare the reference's
 * results with the oracle's, bit for bit, on the same inputs and the same
 * random numbers.
 *
 * Nothing here is shipped or linked by the CUDA library. */
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iostream>
#include <string>
#include <sys/types.h>
#include <vector>

// The reference's CUDA_EGS.h types `ulong` itself; glibc already has one.
#define ulong gegs_ref_ulong

#include "CUDA_EGS.h"
#include "EGSnrc_Parameters.h"
#include "commonBlocks dev.h"

#include "ref_api.h"

// The photon tables are device pointers declared in media.cu (media.cu:72-100),
// which is host code the harness does not compile; the same names here.
typedef struct __align__(16) rayleigh_data_t {
    float xgrid;
    float fcum;
    float b_array;
    float c_array;
} rayleigh_data_t;
float2 *ge, *gmfp, *gbr1, *gbr2, *cohe, *pmax;
rayleigh_data_t *rayleigh_data;
uint *i_array;

ref_uniform_stream g_ref_uniforms;

#include "ref_math.h"

// ---- escore (scoring.cu:14-26) as a recorder of every call, or, during a
// whole transport (ref_transport), the reference's own sum per phantom voxel
struct ref_deposit { uint32_t region; float energy; };
static std::vector<ref_deposit> g_deposits;
static double *g_transport_tally = nullptr;

__device__ void escore(uint region, float energy)
{
    if (g_transport_tally) {
        if (region >= vac_and_oth) g_transport_tally[region - vac_and_oth] += (double)energy;
        return;
    }
    g_deposits.push_back(ref_deposit{region, energy});
}

#include "geom.cu"
#include "utility.cu"
#include "annihatrest.cu"
#include "pair.cu"
#include "relax.cu"
#include "eii_sample.cu"
#include "moller.cu"
#include "compton.cu"
#include "photo.cu"
#include "rayleigh.cu"
#include "photon.cu"
#include "brems.cu"
#include "bhabha.cu"
#include "annih.cu"
#include "electron.cu"

// ---------------------------------------------------------------------------
// state filled from the caller's gegs_physics / gegs_scene
// ---------------------------------------------------------------------------
static std::vector<float2> g_tab_ge, g_tab_gmfp, g_tab_gbr1, g_tab_gbr2, g_tab_cohe, g_tab_pmax;
static std::vector<rayleigh_data_t> g_tab_rayleigh;
static std::vector<uint> g_tab_i_array;
static std::vector<region_data_t> g_regions;
static std::vector<float> g_xb, g_yb, g_zb;
static std::vector<gegs_field> g_fields;
static const gegs_phsp_record *g_phsp = nullptr;   // the caller's scene keeps it alive
static uint64_t g_nphsp = 0;
static curandState g_state;
static std::vector<particle_t> g_stack_mem[NUM_SIMU_CAT];
static const int kStackCap = 4096;

template <typename D, typename S>
static void copy_n(D *dst, const S *src, size_t n)
{
    for (size_t i = 0; i < n; i++) dst[i] = (D)src[i];
}

static void copy_f2(float2 *dst, const float (*src)[2], size_t n)
{
    for (size_t i = 0; i < n; i++) dst[i] = make_float2(src[i][0], src[i][1]);
}

extern "C" int ref_load(const gegs_physics *P, const gegs_scene *S)
{
    if (!P || !S) return 1;
    // ---- physics tables: the reference's globals (commonBlocks dev.h, media.cu)
    copy_n(dl1, P->dl1, 48); copy_n(dl2, P->dl2, 48); copy_n(dl3, P->dl3, 48);
    copy_n(dl4, P->dl4, 48); copy_n(dl5, P->dl5, 48); copy_n(dl6, P->dl6, 48);
    copy_n(bpar, P->bpar, 12);
    copy_n(wa, P->wa, 60); copy_n(pz, P->pz, 60); copy_n(zelem, P->zelem, 60);
    copy_n(delcm, P->delcm, 6); copy_n(zbrang, P->zbrang, 6); copy_n(lzbrang, P->lzbrang, 6);
    copy_n(nne, P->nne, 6);
    ibrdst = P->ibrdst; iprdst = P->iprdst;
    copy_n(log_ap, P->log_ap, 6);
    copy_n(iz_array, P->iz_array, MXTOTSH); copy_n(be_array, P->be_array, MXTOTSH);
    copy_n(jo_array, P->jo_array, MXTOTSH); copy_n(erfjo_array, P->erfjo_array, MXTOTSH);
    copy_n(ne_array, P->ne_array, MXTOTSH); copy_n(shn_array, P->shn_array, MXTOTSH);
    copy_n(shell_array, P->shell_array, MXMDSH * MXMED); copy_n(eno_array, P->eno_array, MXMDSH * MXMED);
    copy_n(eno_atbin_array, P->eno_atbin_array, MXMDSH * MXMED); copy_n(n_shell, P->n_shell, MXMED);
    copy_n(binding_energies, P->binding_energies, MXSHELL * MXELEMENT);
    copy_n(interaction_prob, P->interaction_prob, MXSHELL * MXELEMENT);
    copy_n(relaxation_prob, P->relaxation_prob, MXTRANS * MXELEMENT);
    copy_n(edge_energies, P->edge_energies, MXEDGE * MXELEMENT);
    copy_n(edge_number, P->edge_number, MXELEMENT);
    copy_n(edge_a, P->edge_a, MXEDGE * MXELEMENT); copy_n(edge_b, P->edge_b, MXEDGE * MXELEMENT);
    copy_n(edge_c, P->edge_c, MXEDGE * MXELEMENT); copy_n(edge_d, P->edge_d, MXEDGE * MXELEMENT);
    copy_n(range_ep, P->range_ep, 2 * MXEKE * MXMED); copy_n(e_array, P->e_array, MXEKE * MXMED);
    copy_n(sig_e, P->sig_e, 2 * MXMED);
    copy_f2(eke01, P->eke01, MXMED);
    copy_n(blcc, P->blcc, MXMED); copy_n(xcc, P->xcc, MXMED);
    copy_f2(ebr1, P->ebr1, MXEKE * MXMED); copy_f2(pbr1, P->pbr1, MXEKE * MXMED);
    copy_f2(pbr2, P->pbr2, MXEKE * MXMED); copy_f2(tmxs, P->tmxs, MXEKE * MXMED);
    copy_f2(sig, P->sig, 2 * MXEKE * MXMED); copy_f2(dedx, P->dedx, 2 * MXEKE * MXMED);
    copy_n(expeke1, P->expeke1, MXMED);
    for (int i = 0; i < 2 * MXMED; i++) sig_ismonotone[i] = P->sig_ismonotone[i] != 0;
    copy_f2(eii_xsection, P->eii_xsection, MAX_EII_BINS);
    copy_n(eii_cons, P->eii_cons, MXMED);
    copy_f2(eii, P->eii, MAX_EII_SHELLS);
    copy_n(eii_z, P->eii_z, MAX_EII_SHELLS); copy_n(eii_sh, P->eii_sh, MAX_EII_SHELLS);
    copy_n(eii_nshells, P->eii_nshells, MXELEMENT); copy_n(eii_nsh, P->eii_nsh, MXMED);
    copy_n(eii_first, P->eii_first, MXMED * MXEL); copy_n(eii_no, P->eii_no, MXMED * MXEL);
    eii_flag = P->eii_flag;
    copy_n(smaxir, P->smaxir, MXMED);
    estepe = P->estepe; ximax = P->ximax; skindepth_for_bca = P->skindepth_for_bca;
    transport_algorithm = P->transport_algorithm;
    exact_bca = P->exact_bca != 0; spin_effects = P->spin_effects != 0;
    const size_t nms = (size_t)MAXL_MS_PLUS_1 * MAXQ_MS_PLUS_1 * MAXU_MS_PLUS_1;
    copy_n(ums_array, P->ums_array, nms); copy_n(fms_array, P->fms_array, nms);
    copy_n(wms_array, P->wms_array, nms); copy_n(ims_array, P->ims_array, nms);
    llammin = P->llammin; llammax = P->llammax; dllamb = P->dllamb; dllambi = P->dllambi;
    dqms = P->dqms; dqmsi = P->dqmsi;
    copy_n(rlc, P->rlc, MXMED);
    rmt2 = P->rmt2; rmsq = P->rmsq;
    copy_n(ap, P->ap, MXMED); copy_n(ae, P->ae, MXMED); copy_n(up, P->up, MXMED); copy_n(ue, P->ue, MXMED);
    copy_n(te, P->te, MXMED); copy_n(thmoll, P->thmoll, MXMED);
    prm = P->prm; rm = P->rm; prmt2 = 2.0f * P->prm;
    copy_n(e_max_rr, P->e_max_rr, MXMED); copy_n(i_do_rr, P->i_do_rr, MXMED);
    nbr_split = P->nbr_split;
    g_tab_ge.resize(MXMED); copy_f2(g_tab_ge.data(), P->ge, MXMED);
    const size_t ng = (size_t)MXMED * MXGE;
    g_tab_gmfp.resize(ng); copy_f2(g_tab_gmfp.data(), P->gmfp, ng);
    g_tab_gbr1.resize(ng); copy_f2(g_tab_gbr1.data(), P->gbr1, ng);
    g_tab_gbr2.resize(ng); copy_f2(g_tab_gbr2.data(), P->gbr2, ng);
    g_tab_cohe.resize(ng); copy_f2(g_tab_cohe.data(), P->cohe, ng);
    g_tab_pmax.resize(ng); copy_f2(g_tab_pmax.data(), P->pmax, ng);
    g_tab_rayleigh.resize((size_t)MXMED * MXRAYFF);
    for (size_t i = 0; i < g_tab_rayleigh.size(); i++)
        g_tab_rayleigh[i] = rayleigh_data_t{P->rayleigh_data[i][0], P->rayleigh_data[i][1], P->rayleigh_data[i][2],
                                            P->rayleigh_data[i][3]};
    g_tab_i_array.resize((size_t)MXMED * RAYCDFSIZE);
    copy_n(g_tab_i_array.data(), P->i_array, g_tab_i_array.size());
    ge = g_tab_ge.data(); gmfp = g_tab_gmfp.data(); gbr1 = g_tab_gbr1.data(); gbr2 = g_tab_gbr2.data();
    cohe = g_tab_cohe.data(); pmax = g_tab_pmax.data();
    rayleigh_data = g_tab_rayleigh.data(); i_array = g_tab_i_array.data();

    // ---- regions (init_regions, init.cu:909-1052): 0 vacuum, 1-5 beam line, 6+ voxels
    const uint64_t nvox = (uint64_t)S->nx * S->ny * S->nz;
    g_regions.assign(nvox + vac_and_oth, region_data_t{});
    g_regions[0].med = VACUUM;
    for (int i = 1; i < vac_and_oth; i++) {
        int med = S->other_med[i - 1];
        if (med < 0) med = S->other_med[0];
        region_data_t &r = g_regions[i];
        r.med = (ushort)med; r.flags = (ushort)S->region_flags; r.rhof = 1.0f;
        r.pcut = P->ap[med]; r.ecut = P->ae[med];
    }
    for (uint64_t v = 0; v < nvox; v++) {
        region_data_t &r = g_regions[v + vac_and_oth];
        r.med = S->voxel_med[v];
        if (r.med == VACUUM) continue;
        r.flags = (ushort)S->region_flags;
        r.rhof = S->voxel_rhof[v];
        r.pcut = P->ap[r.med];
        r.ecut = P->ae[r.med];
    }
    region_data = g_regions.data();

    // ---- phantom (init_phantom_and_MLC, init.cu:1164-1275)
    g_xb.assign(S->x_bounds, S->x_bounds + S->nx + 1);
    g_yb.assign(S->y_bounds, S->y_bounds + S->ny + 1);
    g_zb.assign(S->z_bounds, S->z_bounds + S->nz + 1);
    phantom_N = make_uint3((unsigned)S->nx, (unsigned)S->ny, (unsigned)S->nz);
    phantom_x_bounds = g_xb.data(); phantom_y_bounds = g_yb.data(); phantom_z_bounds = g_zb.data();
    size_phantom = (uint)nvox;

    // ---- beam line: isocentre, source distance, module order, MLC constants
    SourceToIsocenter = S->source_to_isocenter;
    Change_xyz = S->change_xyz != 0;
    isocenter_location = make_float3(S->iso[0], S->iso[1], S->iso[2]);
    for (int i = 0; i < MAX_MODULE_PLUS_1; i++) module_order[i] = (char)S->module_order[i];
    MLC_rmax = S->mlc_rmax; MLC_zmin = S->mlc_zmin; MLC_zthick = S->mlc_zthick;
    MLC_x_start = S->mlc_x_start; MLC_x_end = S->mlc_x_end; MLC_x_mid_1 = S->mlc_x_mid_1;
    MLC_x_mid_2 = S->mlc_x_mid_2; MLC_air_gap = S->mlc_air_gap; MLC_wl_full = S->mlc_wl_full;
    MLC_wl_target = S->mlc_wl_target; MLC_wl_isocenter = S->mlc_wl_isocenter; MLC_wt = S->mlc_wt;
    for (int i = 0; i < 960; i++) crossXZ[i] = make_float2(S->crossXZ[i][0], S->crossXZ[i][1]);
    for (int i = 0; i < 4; i++) {
        boundaryXZ[i] = make_float2(S->boundaryXZ[i][0], S->boundaryXZ[i][1]);
        boundaryYZ[i] = make_float2(S->boundaryYZ[i][0], S->boundaryYZ[i][1]);
    }
    g_fields.assign(S->fields, S->fields + S->nfields);
    g_phsp = S->phsp;
    g_nphsp = S->nphsp;
    z_phsp = S->z_phsp;

    // ---- stacks and the random-number state
    devStates = &g_state;
    for (int s = 0; s < NUM_SIMU_CAT; s++) {
        g_stack_mem[s].assign(kStackCap, particle_t{});
        stack[s] = g_stack_mem[s].data();
        np[s] = -1;
        np_max[s] = kStackCap;
    }
    return ref_select_field(0);
}

// per-field set-up (setup_secjaws, init.cu:1504-1592; init_leaf_pos, init.cu:1594-1662;
// the gantry angle upload, CUDA_EGS.cu:426-434)
extern "C" int ref_select_field(int f)
{
    if (f < 0 || f >= (int)g_fields.size()) return 1;
    const gegs_field &F = g_fields[(size_t)f];
    cosAngle = F.cos_angle;
    sinAngle = F.sin_angle;
    for (int i = 0; i < 4; i++) {
        boundMinY[i] = make_float2(F.boundMinY[i][0], F.boundMinY[i][1]);
        boundMinX[i] = make_float2(F.boundMinX[i][0], F.boundMinX[i][1]);
        boundMaxY[i] = make_float2(F.boundMaxY[i][0], F.boundMaxY[i][1]);
        boundMaxX[i] = make_float2(F.boundMaxX[i][0], F.boundMaxX[i][1]);
    }
    for (int i = 0; i < 8; i++) {
        jawsGeomY[i] = make_float2(F.jawsGeomY[i][0], F.jawsGeomY[i][1]);
        jawsGeomX[i] = make_float2(F.jawsGeomX[i][0], F.jawsGeomX[i][1]);
    }
    for (int i = 0; i < TOTAL_MLC_LEAF / 2; i++) endnode[i] = (point2D *)&g_fields[(size_t)f].endnode[i][0][0];
    return 0;
}

// ---------------------------------------------------------------------------
// probes: one routine of the reference on given particles
// ---------------------------------------------------------------------------
static int g_field = -1;

static void to_ref(const gegs_probe_particle &a, particle_t &p)
{
    std::memset(&p, 0, sizeof p);
    p.status = a.status;
    p.nRepeat = 0;
    p.charge = a.charge;
    p.process = true;
    p.region = a.region;
    p.leafIndex = a.leafIndex;
    p.bank = a.bank;
    p.module = a.module;
    p.latch = 0;
    p.wt = a.wt; p.e = a.e;
    p.x = a.x; p.y = a.y; p.z = a.z;
    p.u = a.u; p.v = a.v; p.w = a.w;
    p.dnear = a.dnear;
}

static void from_ref(const particle_t &p, uint8_t field, uint32_t hist, gegs_probe_particle &a)
{
    std::memset(&a, 0, sizeof a);
    a.status = p.status;
    a.charge = p.charge;
    a.region = p.region;
    a.leafIndex = p.leafIndex;
    a.bank = p.bank;
    a.module = p.module;
    a.field = field;
    a.wt = p.wt; a.e = p.e;
    a.x = p.x; a.y = p.y; a.z = p.z;
    a.u = p.u; a.v = p.v; a.w = p.w;
    a.dnear = p.dnear;
    a.hist = hist;
}

static bool use_field(int f)
{
    if (f == g_field) return true;
    if (ref_select_field(f) != 0) return false;
    g_field = f;
    return true;
}

// howfar / hownear dispatch by module (photon.cu:142-158, electron.cu:1491-1508)
static uint ref_howfar_one(particle_t &p, float &t, int &ok)
{
    ok = 1;
    if (p.module == m_SecJawY) return howfar_SecJawsY(p, t);
    if (p.module == m_SecJawX) return howfar_SecJawsX(p, t);
    if (p.module == m_VarMLCs) return howfar_MLC(p, t);
    if (p.module == m_Phantom) return howfar_phantom(p, t);
    ok = 0;
    return 0;
}

static void ref_hownear_one(particle_t &p, float &tperp, int &ok)
{
    ok = 1;
    if (p.module == m_SecJawY) hownear_SecJawsY(p, tperp);
    else if (p.module == m_SecJawX) hownear_SecJawsX(p, tperp);
    else if (p.module == m_VarMLCs) hownear_MLC(p, tperp);
    else if (p.module == m_Phantom) hownear_phantom(p, tperp);
    else { ok = 0; tperp = 0.0f; }
}

extern "C" int ref_probe_geom(uint32_t n, const gegs_probe_particle *in, const float *t_in, uint32_t *far_region,
                              float *far_t, gegs_probe_particle *far_out, float *near_t)
{
    int bad = 0;
    for (uint32_t i = 0; i < n; i++) {
        if (!use_field(in[i].field)) return -1;
        particle_t p;
        int ok;
        to_ref(in[i], p);
        float t = t_in[i];
        far_region[i] = ref_howfar_one(p, t, ok);
        far_t[i] = t;
        from_ref(p, in[i].field, in[i].hist, far_out[i]);
        bad += !ok;
        to_ref(in[i], p);
        float tp = 0.0f;
        ref_hownear_one(p, tp, ok);
        near_t[i] = tp;
    }
    return bad;
}

extern "C" int ref_probe_uphi(int which, float a, float b, gegs_probe_particle *pp, float *cs, float u)
{
    particle_t p;
    to_ref(*pp, p);
    g_ref_uniforms = ref_uniform_stream{&u, 1u, 0u, 0u};
    curandState st;
    if (which == 21) uphi21(a, b, cs[0], cs[1], p, &st);
    else if (which == 32) uphi32(a, b, cs[0], cs[1], p);
    else uphi11(a, cs[2], cs[3], cs[0], cs[1], p, &st);
    from_ref(p, pp->field, pp->hist, *pp);
    return (int)g_ref_uniforms.overrun;
}

// stage number -> the reference's kernel draining that stack
static void run_kernel(int stage)
{
    switch (stage) {
    case p_photon_step: photon_step(); break;
    case p_compton: compton(); break;
    case p_photo: photo(); break;
    case p_rayleigh: rayleigh(); break;
    case p_pair: pair_production(); break;
    case e_electron_step: electr_step(); break;
    case e_moller: moller(); break;
    case e_brems: brems(); break;
    case e_bhabha: bhabha(); break;
    case e_annih: annih(); break;
    default: break;
    }
}

// One pop of the stage's kernel per particle: the particle alone on its stack,
// the uniforms to replay, then the other stacks' contents (push order within
// each stack) and the escore calls. Returns the number of particles for which
// the kernel asked for more uniforms than supplied (each such draw gave 0.5).
extern "C" int ref_probe_stage(int stage, uint32_t n, const gegs_probe_particle *in, const float *u,
                               const uint32_t *un, uint32_t ucap, gegs_probe_particle *out, uint32_t ocap,
                               uint32_t *on, uint32_t *dreg, float *de, uint32_t dcap, uint32_t *dn, uint32_t *used)
{
    int overruns = 0;
    for (uint32_t i = 0; i < n; i++) {
        if (!use_field(in[i].field)) return -1;
        for (int s = 0; s < NUM_SIMU_CAT; s++) np[s] = -1;
        particle_t p;
        to_ref(in[i], p);
        p.status = (uchar)stage;
        np[stage] = 0;
        stack[stage][0] = p;
        g_ref_uniforms = ref_uniform_stream{u + (size_t)i * ucap, un[i] < ucap ? un[i] : ucap, 0u, 0u};
        g_deposits.clear();
        run_kernel(stage);
        used[i] = g_ref_uniforms.next + g_ref_uniforms.overrun;
        if (g_ref_uniforms.overrun) overruns++;
        uint32_t k = 0;
        for (int s = 0; s < NUM_SIMU_CAT; s++)
            for (int j = 0; j <= np[s]; j++) {
                if (k < ocap) from_ref(stack[s][j], in[i].field, in[i].hist, out[(size_t)i * ocap + k]);
                if (k < ocap) out[(size_t)i * ocap + k].status = (uint8_t)s;
                k++;
            }
        on[i] = k;
        dn[i] = (uint32_t)g_deposits.size();
        for (uint32_t j = 0; j < dn[i] && j < dcap; j++) {
            dreg[(size_t)i * dcap + j] = g_deposits[j].region;
            de[(size_t)i * dcap + j] = g_deposits[j].energy;
        }
    }
    return overruns;
}

// ---------------------------------------------------------------------------
// Host set-up: the reference's own readers and geometry set-up (init.cu),
// run on plan files, so tests can compare the scene this package builds from
// the same files. The media tables and the region set-up are not needed for
// that: init_media and init_regions stand in for media.cu:1294 and
// init.cu:909 and keep what init_phantom_and_MLC hands them.
// ---------------------------------------------------------------------------
struct medium_t;

static std::vector<std::string> g_setup_media;
static std::vector<int> g_setup_media_idx;
static std::vector<float> g_setup_density;
static int g_setup_other[max_oth_med];
static std::string g_setup_error;

struct ref_setup_failure {};

medium_t **init_media(uint nmed, string *media_names)
{
    g_setup_media.assign(media_names, media_names + nmed);
    return (medium_t **)calloc(1, sizeof(medium_t *));
}

void init_regions(uint nreg, medium_t **, int *media_indices, float *densities, int *other_med_IDs)
{
    g_setup_media_idx.assign(media_indices, media_indices + nreg);
    g_setup_density.assign(densities, densities + nreg);
    std::memcpy(g_setup_other, other_med_IDs, sizeof g_setup_other);
}

void logstr(const char *, ...) {}

void error(int ret, const char *format, ...)
{
    char buf[512];
    va_list a;
    va_start(a, format);
    std::vsnprintf(buf, sizeof buf, format, a);
    va_end(a);
    g_setup_error = "error " + std::to_string(ret) + ": " + buf;
    throw ref_setup_failure{};
}

void ce(int) {}
void ce(int, const char *, ...) {}

#include "commonBlocks host.h"   // h_nmed and the range-rejection arrays that init_phantom_and_MLC sets
#include "ref_setup.inc"

static void ref_gantry_one(uint iField, float *c, float *s)
{
#include "ref_gantry.inc"
    *c = h_cosAngle;
    *s = h_sinAngle;
}

struct ref_setup_field {
    float angle, x1, x2, y1, y2, mu, output_factor, cos_angle, sin_angle, angle_rad;
    float pos[TOTAL_MLC_LEAF];
    point2D jaws[32];            // boundMinY, boundMinX, boundMaxY, boundMaxX (4 each), jawsGeomY, jawsGeomX (8 each)
    point2D endnode[TOTAL_MLC_LEAF / 2][34];
};
static std::vector<ref_setup_field> g_setup_fields;
static std::vector<float> g_setup_bounds[3];
static std::vector<float> g_setup_mass;

extern "C" int ref_setup_run(const char *egsphant, const char *mlc_egsinp, const char *jaws_egsinp,
                             const char *mlcinfo, const char *data_directory, const char *outfac_file, float sid,
                             const char *default_medium, char *msg, size_t msg_len)
{
    static std::string s_phant, s_mlc, s_jaws, s_info, s_dir, s_of;
    s_phant = egsphant; s_mlc = mlc_egsinp; s_jaws = jaws_egsinp; s_info = mlcinfo; s_dir = data_directory;
    s_of = outfac_file ? outfac_file : "";
    egsphant_file = s_phant.c_str();
    egsinp_file = s_mlc.c_str();
    secjaws_file = s_jaws.c_str();
    mlcinfo_file = s_info.c_str();
    data_dir = s_dir.c_str();
    output_factor_file = s_of.c_str();
    outfac_on = outfac_file != nullptr;
    h_SourceToIsocenter = sid;
    Block_on = false;
    Wedge_on = false;
    GPUNo = 1;
    g_setup_error.clear();
    g_setup_fields.clear();
    try {
        init_phantom_and_MLC(string(default_medium));
        for (int k = 0; k < 3; k++) {
            const float *b = k == 0 ? d_phantom_x_bounds[0] : k == 1 ? d_phantom_y_bounds[0] : d_phantom_z_bounds[0];
            const uint n = (k == 0 ? h_phantom_N.x : k == 1 ? h_phantom_N.y : h_phantom_N.z) + 1;
            g_setup_bounds[k].assign(b, b + n);
        }
        g_setup_mass.assign(voxel_mass, voxel_mass + h_size_phantom);
        read_mlcinp();
        for (int i = 0; i < N_Field; i++) {
            ref_setup_field F;
            F.angle = field[i].angle; F.x1 = field[i].x1; F.x2 = field[i].x2; F.y1 = field[i].y1;
            F.y2 = field[i].y2; F.mu = (float)field[i].MU; F.output_factor = field[i].output_factor;
            std::memcpy(F.pos, field[i].pos, sizeof F.pos);
            setup_secjaws(i);
            std::memcpy(F.jaws + 0, boundMinY, sizeof boundMinY);
            std::memcpy(F.jaws + 4, boundMinX, sizeof boundMinX);
            std::memcpy(F.jaws + 8, boundMaxY, sizeof boundMaxY);
            std::memcpy(F.jaws + 12, boundMaxX, sizeof boundMaxX);
            std::memcpy(F.jaws + 16, jawsGeomY, sizeof jawsGeomY);
            std::memcpy(F.jaws + 24, jawsGeomX, sizeof jawsGeomX);
            init_leaf_pos(i);
            for (int j = 0; j < TOTAL_MLC_LEAF / 2; j++) std::memcpy(F.endnode[j], endnode[j], 34 * sizeof(point2D));
            ref_gantry_one(i, &F.cos_angle, &F.sin_angle);     // turns field[i].angle into radians, as the reference does
            F.angle_rad = field[i].angle;
            g_setup_fields.push_back(F);
        }
    } catch (const ref_setup_failure &) {
        if (msg && msg_len) std::snprintf(msg, msg_len, "%s", g_setup_error.c_str());
        return 1;
    }
    return 0;
}

// Copy one named result of ref_setup_run into dst (at most `bytes`); returns
// the size of the result in bytes, or -1 for an unknown name or field.
extern "C" long ref_setup_get(const char *name, int f, void *dst, size_t bytes)
{
    std::string n(name);
    const void *src = nullptr;
    size_t size = 0;
    std::string names;
    float mlc[12];
    int dims[3];
    float jaws[5];
    if (n == "dims") { dims[0] = h_phantom_N.x; dims[1] = h_phantom_N.y; dims[2] = h_phantom_N.z; src = dims; size = sizeof dims; }
    else if (n == "x_bounds" || n == "y_bounds" || n == "z_bounds") {
        const auto &v = g_setup_bounds[n[0] - 'x'];
        src = v.data(); size = v.size() * sizeof(float);
    }
    else if (n == "voxel_mass") { src = g_setup_mass.data(); size = g_setup_mass.size() * sizeof(float); }
    else if (n == "media_index") { src = g_setup_media_idx.data(); size = g_setup_media_idx.size() * sizeof(int); }
    else if (n == "density") { src = g_setup_density.data(); size = g_setup_density.size() * sizeof(float); }
    else if (n == "other_med") { src = g_setup_other; size = sizeof g_setup_other; }
    else if (n == "media") {
        for (auto &m : g_setup_media) names += m + "\n";
        src = names.data(); size = names.size();
    }
    else if (n == "mlc") {
        const float v[12] = {MLC_rmax, MLC_zmin, MLC_zthick, MLC_x_start, MLC_x_end, MLC_x_mid_1, MLC_x_mid_2,
                             MLC_air_gap, MLC_wl_full, MLC_wl_target, MLC_wl_isocenter, MLC_wt};
        std::memcpy(mlc, v, sizeof mlc); src = mlc; size = sizeof mlc;
    }
    else if (n == "crossXZ") { src = crossXZ; size = sizeof crossXZ; }
    else if (n == "boundaryXZ") { src = boundaryXZ; size = sizeof boundaryXZ; }
    else if (n == "boundaryYZ") { src = boundaryYZ; size = sizeof boundaryYZ; }
    else if (n == "crossYZ") { src = h_crossYZ; size = sizeof h_crossYZ; }
    else if (n == "secjaws") {
        jaws[0] = SecJaws.rmax; jaws[1] = SecJaws.zminy; jaws[2] = SecJaws.zmaxy; jaws[3] = SecJaws.zminx;
        jaws[4] = SecJaws.zmaxx; src = jaws; size = sizeof jaws;
    }
    else if (n == "nfields") { dims[0] = (int)g_setup_fields.size(); src = dims; size = sizeof(int); }
    else if (n == "field" || n == "pos" || n == "jaws" || n == "endnode") {
        if (f < 0 || f >= (int)g_setup_fields.size()) return -1;
        const ref_setup_field &F = g_setup_fields[f];
        if (n == "field") { src = &F.angle; size = 10 * sizeof(float); }
        else if (n == "pos") { src = F.pos; size = sizeof F.pos; }
        else if (n == "jaws") { src = F.jaws; size = sizeof F.jaws; }
        else { src = F.endnode; size = sizeof F.endnode; }
    }
    else return -1;
    if (dst) std::memcpy(dst, src, size < bytes ? size : bytes);
    return (long)size;
}


// ---------------------------------------------------------------------------
// A whole transport by the reference's own kernels: histories [h0, h1) of the
// loaded scene, field by field. Each batch of primaries goes onto the photon
// stack as load_stack_from_phspfile puts them there (CUDA_EGS.cu:54-136), and
// the ten stage kernels run, each draining its stack, until every stack is
// empty. The random numbers come from a seeded generator (shim/curand_kernel.h),
// so the result is an independent sample of the reference's transport, for
// statistical comparison with the package's dose. tally: energy per voxel in
// MeV, added to. Returns the number of stack overflows seen (0 expected).
// ---------------------------------------------------------------------------
extern "C" long ref_transport(uint64_t h0, uint64_t h1, uint64_t seed, double *tally, uint64_t nvox)
{
    if (!g_phsp || g_nphsp == 0 || !tally || nvox != (uint64_t)size_phantom) return -1;
    const int kBatch = 256;
    long overflows = 0;
    g_transport_tally = tally;
    g_ref_uniforms = ref_uniform_stream{nullptr, 0u, 0u, 0u, 1, seed * 0x2545F4914F6CDD1Dull + 1u};
    for (int f = 0; f < (int)g_fields.size(); f++) {
        const gegs_field &F = g_fields[(size_t)f];
        const uint64_t a = std::max<uint64_t>(h0, F.hist_begin), b = std::min<uint64_t>(h1, F.hist_end);
        if (a >= b) continue;
        ref_select_field(f);
        g_field = f;
        for (uint64_t h = a; h < b; h += kBatch) {
            const uint64_t e = std::min<uint64_t>(b, h + kBatch);
            for (uint64_t k = h; k < e; k++) {
                const gegs_phsp_record &r = g_phsp[((k - F.hist_begin) / (uint64_t)(F.nrepeat + 1)) % g_nphsp];
                particle_t p;
                std::memset(&p, 0, sizeof p);
                char q = (r.latch & 0x40000000u) ? -1 : ((r.latch & 0x20000000u) ? 1 : 0);
                float w = std::sqrt(1 - r.u * r.u - r.v * r.v);
                float wt = r.wt;
                if (wt < 0) { w = -w; wt = -wt; }
                p.status = q == 0 ? p_new_particle : e_new_particle;
                p.nRepeat = 0;
                p.charge = q;
                p.process = 1;
                p.e = r.e < 0 ? -r.e : r.e;
                p.wt = wt;
                p.region = 0;
                p.leafIndex = INIT_MLC_STAT;
                p.bank = -1;
                p.module = module_order[m_FirstMd];
                p.latch = 0;
                p.x = r.x; p.y = r.y; p.z = z_phsp;
                p.u = r.u; p.v = r.v; p.w = w;
                p.dnear = INFI_DIST;
                stack[p_photon_step][++np[p_photon_step]] = p;
            }
            bool busy = true;
            while (busy) {
                busy = false;
                for (int s = 0; s < NUM_SIMU_CAT; s++) {
                    if (np[s] < 0) continue;
                    run_kernel(s);
                    busy = true;
                    for (int q2 = 0; q2 < NUM_SIMU_CAT; q2++)
                        if (np[q2] >= np_max[q2] - 1) overflows++;
                }
            }
        }
    }
    g_transport_tally = nullptr;
    g_ref_uniforms = ref_uniform_stream{nullptr, 0u, 0u, 0u, 0, 0ull};
    return overflows;
}
