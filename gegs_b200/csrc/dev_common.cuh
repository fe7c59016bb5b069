// Device-side building blocks of the transport kernels: particle record,
// per-launch context, counter-based RNG, IEEE-only transcendentals, event
// queues with warp-aggregated pushes, and the int64 energy tally.
//
// Determinism contract (shared with the CPU oracle, implemented separately):
//  * RNG: Philox4x32-10 (Salmon et al., SC'11).  key = (seed_lo, seed_hi + hist_hi),
//    counter = (draw>>2, sid_lo, sid_hi, hist_lo), draw n -> word n&3,
//    uniform = ((x>>8)+1) * 2^-24 in (0,1] (the range curand_uniform has).
//  * A particle that only changes stage keeps its stream; every particle an
//    interaction creates gets a child stream (sid = next two raw words).
//  * log/exp/sincos are built from IEEE + - * / only; the library is compiled
//    with -fmad=false so no FMA contraction changes a rounding.
//  * Energy is tallied as int64 fixed point: rint(edep*wt*2^30) per deposit,
//    so the sum is exact and independent of the order of atomics.
#pragma once
#include <stddef.h>
#include <stdint.h>
#include <cooperative_groups.h>
#include "../../include/gegs_physics.h"
#include "../../include/gegs_scene.h"
#include "gx_cmp.h"

namespace cg = cooperative_groups;

// The kernels read table entries as float2 / float4: those members must sit on
// 16-byte (physics block) and 8-byte (field polygons) boundaries.
#define GX_ALIGNED(T, m, a) static_assert(offsetof(T, m) % (a) == 0, #m " misaligned")
GX_ALIGNED(gegs_physics, ge, 16); GX_ALIGNED(gegs_physics, gmfp, 16); GX_ALIGNED(gegs_physics, gbr1, 16);
GX_ALIGNED(gegs_physics, gbr2, 16); GX_ALIGNED(gegs_physics, cohe, 16); GX_ALIGNED(gegs_physics, pmax, 16);
GX_ALIGNED(gegs_physics, rayleigh_data, 16); GX_ALIGNED(gegs_physics, eke01, 16); GX_ALIGNED(gegs_physics, sig, 16);
GX_ALIGNED(gegs_physics, dedx, 16); GX_ALIGNED(gegs_physics, ebr1, 16); GX_ALIGNED(gegs_physics, pbr1, 16);
GX_ALIGNED(gegs_physics, pbr2, 16); GX_ALIGNED(gegs_physics, tmxs, 16); GX_ALIGNED(gegs_physics, eii_xsection, 16);
GX_ALIGNED(gegs_physics, eii, 16);
static_assert(sizeof(gegs_physics) % 16 == 0, "physics block size");
GX_ALIGNED(gegs_field, boundMinY, 8); GX_ALIGNED(gegs_field, boundMaxY, 8); GX_ALIGNED(gegs_field, boundMinX, 8);
GX_ALIGNED(gegs_field, boundMaxX, 8); GX_ALIGNED(gegs_field, jawsGeomY, 8); GX_ALIGNED(gegs_field, jawsGeomX, 8);
GX_ALIGNED(gegs_field, endnode, 8);
static_assert(sizeof(gegs_field) % 16 == 0, "field record size");

#define GX_MXMED GEGS_MXMED
#define GX_MXGE GEGS_MXGE
#define GX_MXEKE GEGS_MXEKE
#define GX_NSTAGE 10
// queues: 10 event stages, then per particle type one ping-pong pair of
// continuation queues for each geometry class in beam order (0 jaws, 1 MLC,
// 2 phantom): photons 10..15, electrons 16..21 (pair = type base + 2 * class).
// The step-budgeted consumers re-queue into them; electron continuations carry
// their step state (estate[qid - GX_Q_ECONT]). Queues 22 (jaws) and 23 (MLC)
// hold the electron steps that need a boundary search (howfar), as they stood
// at their start, for the near-boundary pass of the same wave. Queue 24 holds
// the jaws photons past their step limit, for the long-track kernel that runs
// beside the electron phase.
#define GX_NCLASS 3
#define GX_Q_PCONT 10
#define GX_Q_ECONT 16
#define GX_Q_ENEAR 22
#define GX_Q_PLONG 24
#define GX_NQ 25
#define GX_NESTATE 8
#define GX_TL_KERNELS 32   // wave timeline slots per wave
#define GX_LOOP_CAP 1000
// The reference's step constants are double literals (EGSnrc_Parameters.h:91-92,
// CUDA_EGS.h:34): a step that adds EPSTEP, and a comparison with EPSGMFP or
// EPSEMFP, is evaluated in double, as there. (INFI_DIST, 1e5, is exact in float.)
#define GX_EPSGMFP 1.e-5
#define GX_EPSEMFP 1.e-5
#define GX_EPSTEP 0.0005
#define GX_INFI_DIST 1e5f
#define GX_OUTMLC (-99)
#define GX_PASSMLC (-98)
#define GX_VACUUM 0xFFFFu
#define GX_VACUUM_STEP 1E8f
#define GX_VAC_AND_OTH 6

enum : int {
    ST_PHOTON = 0, ST_COMPTON = 1, ST_PHOTO = 2, ST_RAYLEIGH = 3, ST_PAIR = 4,
    ST_ELECTRON = 5, ST_MOLLER = 6, ST_BREMS = 7, ST_BHABHA = 8, ST_ANNIH = 9
};

// error bits reported back to the host
enum : uint32_t {
    GX_ERR_QUEUE_FULL = 1u, GX_ERR_MODULE = 2u, GX_ERR_SOURCE = 4u, GX_ERR_STEP_BUDGET = 8u
};

// 64-byte particle record (4 x 16 B) -- the queues are arrays of these.
struct __align__(16) Part {
    float e, wt, x, y;
    float z, u, v, w;
    uint32_t region, hist_lo, hist_hi, ctr;
    uint32_t sid_lo, sid_hi;
    int8_t charge, leafIndex, bank;
    uint8_t module;
    uint8_t field, status;
    uint16_t beamlet;       // beamlet of the history's primary (GX_NO_BEAMLET: none)
};
static_assert(sizeof(Part) == 64, "particle record must be 64 bytes");
#define GX_NO_BEAMLET 0xFFFFu
// copies of the beamlet gradient accumulator (lane-indexed, summed on the host)
#define GX_GRAD_COPIES 32

// 8-byte region record (medium, flags, density ratio); cuts come from the medium.
struct __align__(8) Vox {
    uint16_t med, flags;
    float rhof;
};

// Debug trace record: one per queue push (kind 0) and per particle taken by a
// consumer (kind 1); the oracle writes the same records.
struct TraceRec {
    uint32_t kind_stage;       // kind | stage << 8
    uint32_t hist_lo, sid_lo, sid_hi, ctr;
    float e, x;
    uint32_t region;
};

// electron step state carried by a continued electron (EState, packed)
struct __align__(16) EStatePk {
    float elke, demfp, sig0, total_tstep;
    int lelke;
    uint32_t flags;       // bit0 compute_tstep, bit1 is_tstep
    uint32_t pad0, pad1;
};

struct QueueSet {
    Part *buf[GX_NQ];
    uint32_t cap[GX_NQ];
    EStatePk *estate[GX_NESTATE];  // state of the electron continuation queues
    uint32_t *peak;                // per queue the most records it held in one cycle (null: not recorded)
    uint32_t *count;      // [GX_NQ] items queued
    uint32_t *head;       // [GX_NQ] items taken by the running consumer
    uint32_t *done;       // [GX_NQ] finished blocks of the running consumer
};

// Unsigned division by a divisor fixed for the run, as a multiply-high and
// shifts (Granlund and Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994, fig. 4.1): exact for every 32-bit dividend.
struct FastDiv {
    uint32_t m, sh, one;
};

__host__ __device__ inline FastDiv make_fastdiv(uint32_t d)
{
    FastDiv f = {0u, 0u, d == 1u ? 1u : 0u};
    if (d > 1u) {
        uint32_t l = 0;
        while ((1ull << l) < d) l++;                     // l = ceil(log2 d), 1..31 here
        f.m = (uint32_t)((((1ull << 32) * ((1ull << l) - d)) / d) + 1ull);
        f.sh = l - 1u;
    }
    return f;
}

__device__ __forceinline__ uint32_t fastdiv(const FastDiv &f, uint32_t n)
{
    if (f.one) return n;
    const uint32_t t = __umulhi(f.m, n);
    return (t + ((n - t) >> 1)) >> f.sh;
}

// Everything a transport kernel needs; passed by value as a kernel parameter.
struct DevCtx {
    const gegs_physics *P;
    // Tables re-laid out on the device from P (same values, read together):
    //   ptab[med*MXGE + lgle] = {gmfp.a, gmfp.b, cohe.a, cohe.b}: the photon mean
    //     free path and Rayleigh factor of one step, the slice the photon
    //     consumers stage in shared memory when stage_tables is set.
    const float4 *ptab;
    int nmed;
    uint32_t stage_tables;          // GEGS_RUN_STAGE_TABLES of the run
    const Vox *reg;                 // nvox + 6 regions
    const float *xb, *yb, *zb;
    const gegs_field *fields;
    const float2 *crossXZ;          // 960
    const float4 *jaw_lines;        // [field][jaw][8] edge lines of the jaws hownear polygons
    const gegs_phsp_record *phsp;
    unsigned long long *tally;      // int64 MeV*2^30 per voxel
    uint32_t *err;
    unsigned long long *stats;      // per-stage processed counts [GX_NSTAGE], steps [2]
    TraceRec *trace;                // debug trace (null = off)
    uint32_t *trace_n;
    uint32_t trace_cap;
    const uint32_t *wave;           // wave counter (parity selects the continuation buffers)
    const uint32_t *budget_shift;   // step budgets shifted left by this (the planner's tail setting)
    uint32_t *photon_done;          // photon MLC and phantom consumers finished in this wave
    uint32_t *electron_done;        // electron branches (jaws, MLC, phantom) finished in this wave
    uint32_t overlap;               // 1: a phase's class consumers run as concurrent graph branches
    uint32_t pipelined;             // 1: a wave runs both transport phases at once, then both interaction
                                    // phases (persistent form); a positron that stops in the electron
                                    // transport annihilates at rest in the annihilation kernel
    uint32_t photon_budget, electron_budget;   // steps per particle per launch before continuation
    unsigned long long *timeline;   // [timeline_waves][16][2] first start / last end (ns) per kernel; null: off
    uint32_t timeline_waves;
    QueueSet q;
    uint64_t nphsp;
    int nx, ny, nz, nfields;
    FastDiv div_nx, div_nxny;       // voxel index decode: / nx, / (nx * ny)
    int change_xyz, hownear_off;
    float sid, iso0, iso1, iso2, z_phsp;
    float mlc_rmax, mlc_zmin, mlc_zthick, mlc_x_start, mlc_x_end, mlc_x_mid_1, mlc_x_mid_2;
    float mlc_air_gap, mlc_wl_full, mlc_wl_target, mlc_wl_isocenter, mlc_wt;
    float2 boundaryXZ[4], boundaryYZ[4];
    int8_t module_order[8];
    uint32_t seed_lo, seed_hi;
    // beamlets: tagging grid, fluence weights (null: 1) and, in a gradient
    // replay, d(objective)/d(energy) per voxel and the per-beamlet accumulator
    int bl_nx, bl_ny, nbeamlets;
    float bl_x0, bl_y0, bl_dx, bl_dy;
    const float *bl_weight;
    const double *gvm;
    double *grad;           // [GX_GRAD_COPIES][nbeamlets]; null: energy tally
};

// ---------------------------------------------------------------------------
// Philox4x32-10
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint4 gx_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                           uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; r++) {
        if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
        uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    }
    return make_uint4(c0, c1, c2, c3);
}

// Per-particle stream with a window of two Philox blocks (8 words). The window
// is refilled at one converged point per transport step (rng_window), so the
// sampling code that draws numbers holds no inlined copy of Philox; a draw past
// the window (rare: a step uses 5 words typically, 8 or fewer in 98 %) takes an
// out-of-line refill. Any word is a pure function of (key, counter), so where a
// block is computed does not change the numbers.
struct Rng {
    uint32_t hist_lo, hist_hi, sid_lo, sid_hi, ctr;
    uint32_t wb;    // block index of w0 plus one; 0 = empty window
    uint4 w0, w1;   // blocks wb-1 and wb
};

__device__ __forceinline__ void rng_load(Rng &r, const Part &p)
{
    r.hist_lo = p.hist_lo; r.hist_hi = p.hist_hi; r.sid_lo = p.sid_lo; r.sid_hi = p.sid_hi;
    r.ctr = p.ctr; r.wb = 0;
}

__device__ __forceinline__ void rng_store(const Rng &r, Part &p)
{
    p.hist_lo = r.hist_lo; p.hist_hi = r.hist_hi; p.sid_lo = r.sid_lo; p.sid_hi = r.sid_hi; p.ctr = r.ctr;
}

__device__ __noinline__ uint4 rng_block(uint32_t b, uint32_t sid_lo, uint32_t sid_hi, uint32_t hist_lo,
                                        uint32_t k0, uint32_t k1)
{
    return gx_philox(b, sid_lo, sid_hi, hist_lo, k0, k1);
}

// Make the window start at the block of the next draw (call where the warp is converged).
__device__ __forceinline__ void rng_window(const DevCtx &C, Rng &r)
{
    const uint32_t b = r.ctr >> 2;
    if (r.wb == b + 1u) return;
    if (r.wb != 0u && r.wb == b) r.w0 = r.w1;
    else r.w0 = gx_philox(b, r.sid_lo, r.sid_hi, r.hist_lo, C.seed_lo, C.seed_hi + r.hist_hi);
    r.w1 = gx_philox(b + 1u, r.sid_lo, r.sid_hi, r.hist_lo, C.seed_lo, C.seed_hi + r.hist_hi);
    r.wb = b + 1u;
}

__device__ __forceinline__ uint32_t rng_u32(const DevCtx &C, Rng &r)
{
    uint32_t k = r.ctr - ((r.wb - 1u) << 2);
    if (r.wb == 0u || k >= 8u) {
        const uint32_t b = r.ctr >> 2;
        r.w0 = rng_block(b, r.sid_lo, r.sid_hi, r.hist_lo, C.seed_lo, C.seed_hi + r.hist_hi);
        r.w1 = rng_block(b + 1u, r.sid_lo, r.sid_hi, r.hist_lo, C.seed_lo, C.seed_hi + r.hist_hi);
        r.wb = b + 1u;
        k = r.ctr & 3u;
    }
    const uint4 w = k < 4u ? r.w0 : r.w1;
    const uint32_t j = k & 3u;
    const uint32_t x = j == 0 ? w.x : (j == 1 ? w.y : (j == 2 ? w.z : w.w));
    r.ctr++;
    return x;
}

__device__ __forceinline__ float rng_uniform(const DevCtx &C, Rng &r)
{
    uint32_t x = rng_u32(C, r);
    return __uint2float_rn((x >> 8) + 1u) * 5.9604644775390625e-08f;
}

// child stream for a particle created by an interaction
__device__ __forceinline__ void rng_spawn(const DevCtx &C, Rng &parent, Part &child)
{
    uint32_t lo = rng_u32(C, parent);
    uint32_t hi = rng_u32(C, parent);
    child.hist_lo = parent.hist_lo;
    child.hist_hi = parent.hist_hi;
    child.sid_lo = lo;
    child.sid_hi = hi;
    child.ctr = 0;
}

// ---------------------------------------------------------------------------
// transcendentals from IEEE basic operations (Cody-Waite reduction, Taylor series)
// ---------------------------------------------------------------------------
#define GX_LN2_HI 0.693145751953125f
#define GX_LN2_LO 1.42860682030941723212e-06f
#define GX_LOG2E 1.44269502162933349609f

__device__ __forceinline__ float gx_log(float x)
{
    if (!(x > 0.0f)) return x == 0.0f ? __int_as_float(0xff800000) : __int_as_float(0x7fc00000);
    if (x == __int_as_float(0x7f800000)) return x;
    uint32_t ix = __float_as_uint(x);
    int k = 0;
    if (ix < 0x00800000u) { x = __fmul_rn(x, 33554432.0f); ix = __float_as_uint(x); k = -25; }
    k += (int)(ix >> 23) - 127;
    uint32_t im = (ix & 0x007fffffu) | 0x3f800000u;
    if (im > 0x3fb504f3u) { im -= 0x00800000u; k += 1; }
    float m = __uint_as_float(im);
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

__device__ __forceinline__ float gx_exp(float x)
{
    if (x != x) return x;
    if (x > 88.7228394f) return __int_as_float(0x7f800000);
    if (x < -103.972084f) return 0.0f;
    float kf = floorf(x * GX_LOG2E + 0.5f);
    int k = (int)kf;
    float r = (x - kf * GX_LN2_HI) - kf * GX_LN2_LO;
    float p = 1.0f + r * (1.0f + r * (0.5f + r * (0.16666667163372039794921875f
              + r * (0.041666667908430099487304688f + r * (0.0083333337679505348205566406f
              + r * (0.0013888889225199818611145020f + r * (0.00019841270113829523324966431f
              + r * 2.4801587642286904156208038e-05f)))))));
    if (k > 127) { p = p * 1.7014118346046923e+38f; k -= 127; }
    if (k < -126) { p = p * 5.42101086242752217e-20f; k += 64; }
    return p * __uint_as_float((uint32_t)(k + 127) << 23);
}

__device__ __forceinline__ void gx_sincos_turns(float t, float *s, float *c)
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
    if (iq == 0) { *s = sn; *c = cs; }
    else if (iq == 1) { *s = cs; *c = -sn; }
    else if (iq == 2) { *s = -sn; *c = -cs; }
    else { *s = -cs; *c = sn; }
}

__device__ __forceinline__ void gx_sincos(float a, float *s, float *c)
{
    gx_sincos_turns(a * 0.15915493667125701904296875f, s, c);
}

__device__ __forceinline__ float fmaxf_(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float fminf_(float a, float b) { return a < b ? a : b; }

// ---------------------------------------------------------------------------
// region table, scoring, queues
// ---------------------------------------------------------------------------
struct RegInfo {
    unsigned med, flags;
    float rhof, pcut, ecut;
};

__device__ __forceinline__ RegInfo region_info(const DevCtx &C, uint32_t region)
{
    Vox v = C.reg[region];
    RegInfo r;
    r.med = v.med;
    r.flags = v.flags;
    r.rhof = v.rhof;
    if (v.med == GX_VACUUM) { r.pcut = 0.0f; r.ecut = 0.0f; }
    else { r.pcut = __ldg(&C.P->ap[v.med]); r.ecut = __ldg(&C.P->ae[v.med]); }
    return r;
}

// Gradient replay: d(objective)/d(beamlet weight) += energy * d(objective)/d(energy in the voxel).
// Out of line: only the replay reaches it, and inlined at every scoring site it
// would enlarge the forward kernels.
__device__ __noinline__ void escore_grad(const DevCtx &C, uint32_t beamlet, uint32_t region, float energy)
{
    if (beamlet == GX_NO_BEAMLET) return;
    double g = (double)energy * __ldg(&C.gvm[region - GX_VAC_AND_OTH]);
    if (g != 0.0) atomicAdd(&C.grad[(size_t)(threadIdx.x & (GX_GRAD_COPIES - 1)) * C.nbeamlets + beamlet], g);
}

__device__ __forceinline__ void escore(const DevCtx &C, const Part &p, uint32_t region, float energy)
{
    if (region < GX_VAC_AND_OTH) return;
    if (C.grad) {
        escore_grad(C, p.beamlet, region, energy);
        return;
    }
    long long q = __float2ll_rn(energy * 1073741824.0f);
    if (q != 0) atomicAdd(&C.tally[region - GX_VAC_AND_OTH], (unsigned long long)q);
}

__device__ __forceinline__ void store_part(Part *dst, const Part &p)
{
    const uint4 *s = reinterpret_cast<const uint4 *>(&p);
    uint4 *d = reinterpret_cast<uint4 *>(dst);
    d[0] = s[0]; d[1] = s[1]; d[2] = s[2]; d[3] = s[3];
}

__device__ __forceinline__ Part load_part(const Part *src)
{
    Part p;
    const uint4 *s = reinterpret_cast<const uint4 *>(src);
    uint4 *d = reinterpret_cast<uint4 *>(&p);
    d[0] = s[0]; d[1] = s[1]; d[2] = s[2]; d[3] = s[3];
    return p;
}

__device__ __forceinline__ void trace_event(const DevCtx &C, uint32_t kind, int stage, const Part &p)
{
    if (!C.trace) return;
    uint32_t i = atomicAdd(C.trace_n, 1u);
    if (i >= C.trace_cap) return;
    TraceRec t;
    t.kind_stage = kind | ((uint32_t)stage << 8);
    t.hist_lo = p.hist_lo; t.sid_lo = p.sid_lo; t.sid_hi = p.sid_hi; t.ctr = p.ctr;
    t.e = p.e; t.x = p.x; t.region = p.region;
    C.trace[i] = t;
}

// Append one record to queue `qid`; lanes of the warp that push to the same
// queue at the same time share one atomic.
__device__ __forceinline__ void push(const DevCtx &C, int qid, const Part &p)
{
    cg::coalesced_group g = cg::coalesced_threads();
    cg::coalesced_group sub = cg::labeled_partition(g, qid);
    uint32_t base = 0;
    if (sub.thread_rank() == 0) base = atomicAdd(&C.q.count[qid], (uint32_t)sub.size());
    base = sub.shfl(base, 0);
    uint32_t idx = base + sub.thread_rank();
    if (idx < C.q.cap[qid]) {
        Part r = p;
        r.status = (uint8_t)qid;
        store_part(&C.q.buf[qid][idx], r);
        trace_event(C, 0u, qid, r);
    } else {
        atomicOr(C.err, GX_ERR_QUEUE_FULL);
    }
}

// push of a particle that keeps its stream (stage change)
__device__ __forceinline__ void push_move(const DevCtx &C, int qid, Part p, const Rng &r)
{
    rng_store(r, p);
    push(C, qid, p);
}

// push of a particle created by an interaction (child stream)
__device__ __forceinline__ void push_spawn(const DevCtx &C, int qid, Part p, Rng &parent)
{
    rng_spawn(C, parent, p);
    push(C, qid, p);
}
