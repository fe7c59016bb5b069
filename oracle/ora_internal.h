/* CPU oracle for the GEGS transport hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * This is a plain-C restatement of the reference's device routines
 * (photon.cu, compton.cu, photo.cu, rayleigh.cu, pair.cu, relax.cu,
 * electron.cu, moller.cu, eii_sample.cu, brems.cu, bhabha.cu, annih.cu,
 * annihatrest.cu, utility.cu, geom.cu, scoring.cu), run history by history
 * with a per-history particle stack.  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg load it, as the checker; the CUDA library
 * never links or calls it.
 *
 * Parity contract with the CUDA path (both sides implement it independently):
 *   - RNG: Philox4x32-10 (Salmon et al., SC'11).  key = (seed_lo, seed_hi + hist_hi),
 *     counter = (draw>>2, sid_lo, sid_hi, hist_lo); draw n uses output word n&3.
 *     uniform = ((x>>8)+1) * 2^-24 in (0,1], the range of curand_uniform.
 *   - A particle that only changes stage keeps its stream; every particle an
 *     interaction pushes gets a child stream (sid = next two raw words).
 *   - Transcendentals: own log/exp/sincos built from IEEE + - * / sqrt only,
 *     compiled without FMA contraction on both sides.
 *   - Energy tally: int64 fixed point, llrint(edep*wt * 2^30) per escore call.
 * Parity against EGSnrc data is unpinned (the reference's data files are absent);
 * parity against cuRAND streams is unpinned by design (counter-based RNG).
 */
#ifndef ORA_INTERNAL_H
#define ORA_INTERNAL_H

#include <stdint.h>
#include <stddef.h>
#include <math.h>
#include "../include/gegs_physics.h"
#include "../include/gegs_scene.h"

#define MXMED GEGS_MXMED
#define MXGE GEGS_MXGE
#define MXEKE GEGS_MXEKE
#define MXEL GEGS_MXEL
#define MXRAYFF GEGS_MXRAYFF
#define RAYCDFSIZE GEGS_RAYCDFSIZE
#define MXSHELL GEGS_MXSHELL
#define MXTRANS GEGS_MXTRANS
#define MXEDGE GEGS_MXEDGE
#define MXMDSH GEGS_MXMDSH
#define N_EII_BINS GEGS_N_EII_BINS
#define MAXL_MS GEGS_MAXL_MS
#define MAXQ_MS GEGS_MAXQ_MS
#define MAXU_MS GEGS_MAXU_MS
#define MAXL_MS_PLUS_1 (MAXL_MS + 1)
#define MAXQ_MS_PLUS_1 (MAXQ_MS + 1)
#define LAMBMAX_MS 1e5
#define QMIN_MS 1e-3
#define QMAX_MS 0.5
#define MXVAC 10
#define RELAX_CUTOFF 0.001
#define EPSEMFP 1.e-5
#define EPSGMFP 1.e-5
#define EPSTEP 0.0005
#define INFI_DIST 1e5
#define OUTMLC (-99)
#define PASSMLC (-98)
#define VACUUM 0xFFFFu
#define VACUUM_STEP 1E8f
#define SMALL_POLAR_ANGLE_THRESHOLD 1E-20f
/* The reference's constants keep its types: these are double literals
 * (EGSnrc_Parameters.h:78-127, CUDA_EGS.h:34,80), so an expression that uses
 * one is evaluated in double, as in the reference. */
#define HC_INVERSE 80.65506856998f
#define TWICE_HC2 0.000307444456f
#define PRESTA_II 0

/* region layout (CUDA_EGS.h:369-385) */
#define VAC_AND_OTH 6
#define VACUUM_REG 0
#define DEFAULT_REG 1
#define SECJAWS_REG 2
#define MLC_REGION 3

enum {
    p_photon_step = 0, p_compton = 1, p_photo = 2, p_rayleigh = 3, p_pair = 4,
    e_electron_step = 5, e_moller = 6, e_brems = 7, e_bhabha = 8, e_annih = 9,
    ORA_NSTAGE = 10
};

typedef struct {
    uint32_t hist_lo, hist_hi, sid_lo, sid_hi, ctr;
    uint32_t blk;          /* cached block index + 1 (0 = none) */
    uint32_t buf[4];
} ora_rng;

typedef struct {
    uint8_t status;
    int8_t charge;
    int8_t leafIndex, bank;
    uint8_t module, field;
    uint32_t region;
    float wt, e, x, y, z, u, v, w, dnear;
    ora_rng rng;
} ora_particle;

typedef struct {
    uint16_t med, flags;
    float rhof, pcut, ecut;
} ora_region;

typedef struct {
    ora_particle *a;
    size_t n, cap;
} ora_stack;

typedef struct {
    uint32_t kind_stage, hist_lo, sid_lo, sid_hi, ctr;
    float e, x;
    uint32_t region;
} ora_trace_rec;

typedef struct {
    const gegs_physics *P;
    const gegs_scene *S;
    ora_region *reg;         /* nvox + 6 */
    uint32_t nvox;
    uint32_t seed_lo, seed_hi;
    int64_t *tally;          /* nvox */
    ora_stack *stk;
    uint64_t counts[ORA_NSTAGE];
    uint64_t steps_photon, steps_electron;
    double e_escaped;        /* energy leaving through region 0 (for conservation audits) */
    int error;
    /* algorithmic-traffic counters per stage: [0] region records read,
     * [1] tally updates, [2] float2 table reads */
    uint64_t cnt[ORA_NSTAGE][3];
    int cur_stage;
    ora_trace_rec *trace;    /* debug trace (single-threaded runs only) */
    uint32_t trace_n, trace_cap;
    /* probes: record every uniform drawn and every escore call (null: off) */
    float *urec;
    uint32_t urec_n, urec_cap;
    uint32_t *drec_region;
    float *drec_e;
    uint32_t drec_n, drec_cap;
} ora_ctx;

void ora_trace(ora_ctx *C, uint32_t kind, int stage, const ora_particle *p);

/* rng + math (ora_base.c) */
uint32_t ora_philox_word(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1, int lane);
void ora_philox4(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
uint32_t ora_rng_u32(ora_ctx *C, ora_rng *r);
float ora_rng_uniform(ora_ctx *C, ora_rng *r);
void ora_rng_spawn(ora_ctx *C, ora_rng *parent, ora_rng *child);
float gx_log(float x);
float gx_exp(float x);
void gx_sincos_turns(float t, float *s, float *c);
void gx_sincos(float a, float *s, float *c);

void ora_escore(ora_ctx *C, uint32_t region, float energy);
void ora_push(ora_ctx *C, const ora_particle *p, int status);
void ora_spawn(ora_ctx *C, ora_rng *parent, ora_particle *child, int status);

void uphi21(ora_ctx *C, float costhe, float sinthe, float *cosphi, float *sinphi, ora_particle *p, ora_rng *r);
void uphi32(float costhe, float sinthe, float cosphi, float sinphi, ora_particle *p);
void uphi11(ora_ctx *C, float theta, float *costhe, float *sinthe, float *cosphi, float *sinphi, ora_particle *p, ora_rng *r);

/* driver (ora_driver.c) */
ora_region *ora_build_regions(const gegs_physics *P, const gegs_scene *S, uint32_t nvox);
void ora_run_particle(ora_ctx *C, ora_particle *p);
int ora_make_primary(const gegs_scene *S, uint64_t h, ora_particle *p);

/* geometry (ora_geom.c) */
uint32_t ora_howfar(ora_ctx *C, ora_particle *p, float *t, int *ok);
void ora_hownear(ora_ctx *C, ora_particle *p, float *tperp, int *ok);
uint32_t howfar_phantom(ora_ctx *C, const ora_particle *p0, float *t);
void hownear_phantom(ora_ctx *C, const ora_particle *p0, float *tperp);

/* interactions (ora_photon.c, ora_electron.c) */
void ora_photon(ora_ctx *C, ora_particle *p);
void ora_compton(ora_ctx *C, ora_particle *p);
void ora_photo(ora_ctx *C, ora_particle *p);
void ora_rayleigh(ora_ctx *C, ora_particle *p);
void ora_pair(ora_ctx *C, ora_particle *p);
void ora_relax(ora_ctx *C, float energy, int n, int iz, float *edep, ora_particle p, const ora_region *rd, ora_rng *r);
void ora_electron(ora_ctx *C, ora_particle *p);
void ora_moller(ora_ctx *C, ora_particle *p);
void ora_brems(ora_ctx *C, ora_particle *p);
void ora_bhabha(ora_ctx *C, ora_particle *p);
void ora_annih(ora_ctx *C, ora_particle *p);
void ora_annih_at_rest(ora_ctx *C, ora_particle *p, const ora_region *rd, ora_rng *r);

static inline float fmaxf_(float a, float b) { return a > b ? a : b; }
static inline float fminf_(float a, float b) { return a < b ? a : b; }

#endif
