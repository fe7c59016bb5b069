/* Generated from gegs_b200/physics_layout.py -- edit the field list there.
 *
 * Physics-table block read by the transport kernels.  Same content and
 * index conventions as the reference's __device__ globals
 * (commonBlocks dev.h:11-262, media.cu:96-100); float2 pairs are float[2].
 * Every member is 4 bytes wide; _padN members put every array on a
 * 16-byte boundary so the kernels can use float2/float4 loads. */
#ifndef GEGS_PHYSICS_H
#define GEGS_PHYSICS_H

#include <stdint.h>

#define GEGS_MXMED 6
#define GEGS_MXGE 200
#define GEGS_MXEKE 150
#define GEGS_MXEL 10
#define GEGS_MXRAYFF 100
#define GEGS_RAYCDFSIZE 100
#define GEGS_MXELEMENT 100
#define GEGS_MXSHELL 6
#define GEGS_MXTRANS 39
#define GEGS_MXEDGE 16
#define GEGS_MXTOTSH 1538
#define GEGS_MXMDSH 50
#define GEGS_MAX_EII_SHELLS 40
#define GEGS_N_EII_BINS 250
#define GEGS_MAXL_MS 63
#define GEGS_MAXQ_MS 7
#define GEGS_MAXU_MS 31
#define GEGS_MS_SIZE 16384
#define GEGS_MAX_EII_BINS 10000

typedef struct gegs_physics {
    int32_t nmed;
    float rm;
    float prm;
    float rmt2;
    float rmsq;
    float estepe;
    float ximax;
    float skindepth_for_bca;
    int32_t transport_algorithm;
    int32_t exact_bca;
    int32_t spin_effects;
    int32_t ibrdst;
    int32_t iprdst;
    int32_t nbr_split;
    int32_t eii_flag;
    int32_t _pad0[1];
    float rho[6];
    int32_t _pad1[2];
    float ae[6];
    int32_t _pad2[2];
    float ap[6];
    int32_t _pad3[2];
    float ue[6];
    int32_t _pad4[2];
    float up[6];
    int32_t _pad5[2];
    float te[6];
    int32_t _pad6[2];
    float thmoll[6];
    int32_t _pad7[2];
    float rlc[6];
    int32_t _pad8[2];
    float delcm[6];
    int32_t _pad9[2];
    float zbrang[6];
    int32_t _pad10[2];
    float lzbrang[6];
    int32_t _pad11[2];
    float log_ap[6];
    int32_t _pad12[2];
    float blcc[6];
    int32_t _pad13[2];
    float xcc[6];
    int32_t _pad14[2];
    float expeke1[6];
    int32_t _pad15[2];
    float smaxir[6];
    int32_t _pad16[2];
    float e_max_rr[6];
    int32_t _pad17[2];
    int32_t i_do_rr[6];
    int32_t _pad18[2];
    int32_t nne[6];
    int32_t _pad19[2];
    float zelem[60];
    float pz[60];
    float wa[60];
    float dl1[48];
    float dl2[48];
    float dl3[48];
    float dl4[48];
    float dl5[48];
    float dl6[48];
    float bpar[12];
    float ge[6][2];
    float gmfp[1200][2];
    float gbr1[1200][2];
    float gbr2[1200][2];
    float cohe[1200][2];
    float pmax[1200][2];
    float rayleigh_data[600][4];
    int32_t i_array[600];
    float eke01[6][2];
    float sig[1800][2];
    float dedx[1800][2];
    float ebr1[900][2];
    float pbr1[900][2];
    float pbr2[900][2];
    float tmxs[900][2];
    float range_ep[1800];
    float e_array[900];
    float sig_e[12];
    int32_t sig_ismonotone[12];
    float binding_energies[600];
    float interaction_prob[600];
    float relaxation_prob[3900];
    float edge_energies[1600];
    float edge_a[1600];
    float edge_b[1600];
    float edge_c[1600];
    float edge_d[1600];
    int32_t edge_number[100];
    int32_t iz_array[1538];
    int32_t _pad20[2];
    int32_t shn_array[1538];
    int32_t _pad21[2];
    int32_t ne_array[1538];
    int32_t _pad22[2];
    float be_array[1538];
    int32_t _pad23[2];
    float jo_array[1538];
    int32_t _pad24[2];
    float erfjo_array[1538];
    int32_t _pad25[2];
    int32_t shell_array[300];
    float eno_array[300];
    int32_t eno_atbin_array[300];
    int32_t n_shell[6];
    float llammin;
    float llammax;
    float dllamb;
    float dllambi;
    float dqms;
    float dqmsi;
    float ums_array[16384];
    float fms_array[16384];
    float wms_array[16384];
    int32_t ims_array[16384];
    float eii_xsection[10000][2];
    float eii_cons[6];
    int32_t _pad26[2];
    float eii[40][2];
    int32_t eii_z[40];
    int32_t eii_sh[40];
    int32_t eii_nshells[100];
    int32_t eii_nsh[6];
    int32_t _pad27[2];
    int32_t eii_first[60];
    int32_t eii_no[60];
} gegs_physics;

/* X-macro over the float members (every value must be finite; checked by
 * gegs_check_physics before a block is used). */
#define GEGS_PHYSICS_FLOAT_MEMBERS(X) \
    X(rm) \
    X(prm) \
    X(rmt2) \
    X(rmsq) \
    X(estepe) \
    X(ximax) \
    X(skindepth_for_bca) \
    X(rho) \
    X(ae) \
    X(ap) \
    X(ue) \
    X(up) \
    X(te) \
    X(thmoll) \
    X(rlc) \
    X(delcm) \
    X(zbrang) \
    X(lzbrang) \
    X(log_ap) \
    X(blcc) \
    X(xcc) \
    X(expeke1) \
    X(smaxir) \
    X(e_max_rr) \
    X(zelem) \
    X(pz) \
    X(wa) \
    X(dl1) \
    X(dl2) \
    X(dl3) \
    X(dl4) \
    X(dl5) \
    X(dl6) \
    X(bpar) \
    X(ge) \
    X(gmfp) \
    X(gbr1) \
    X(gbr2) \
    X(cohe) \
    X(pmax) \
    X(rayleigh_data) \
    X(eke01) \
    X(sig) \
    X(dedx) \
    X(ebr1) \
    X(pbr1) \
    X(pbr2) \
    X(tmxs) \
    X(range_ep) \
    X(e_array) \
    X(sig_e) \
    X(binding_energies) \
    X(interaction_prob) \
    X(relaxation_prob) \
    X(edge_energies) \
    X(edge_a) \
    X(edge_b) \
    X(edge_c) \
    X(edge_d) \
    X(be_array) \
    X(jo_array) \
    X(erfjo_array) \
    X(eno_array) \
    X(llammin) \
    X(llammax) \
    X(dllamb) \
    X(dllambi) \
    X(dqms) \
    X(dqmsi) \
    X(ums_array) \
    X(fms_array) \
    X(wms_array) \
    X(eii_xsection) \
    X(eii_cons) \
    X(eii)

#endif /* GEGS_PHYSICS_H */
