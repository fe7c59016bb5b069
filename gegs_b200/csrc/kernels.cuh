// Transport kernels.  One consumer kernel per event queue (the reference's
// ten stacks, CUDA_EGS.h:362-367), fed by a source kernel that turns
// phase-space records into primaries on the device.
//
// Persistent form: the photon and electron consumers keep every lane busy by
// refilling idle lanes from the queue with one warp-aggregated atomic per
// refill (persistent threads with regeneration), and a one-thread planner
// kernel decides the next wave and sets the CUDA-graph loop condition, so a
// whole run is a single graph launch with no host round trip.
// Plain form: the reference's structure -- each thread pops its own particle
// with a global atomic, and the host synchronises and reads the queue counters
// back after every launch (CUDA_EGS.cu:226-365, 498-799).
#pragma once
#include "dev_electron.cuh"
#include "../../include/gegs.h"     // gegs_probe_state

// Step budgets in the tail of a run (fewer than batch / GX_TAIL_DIV particles
// in flight and no history left to inject) are GX_TAIL_SHIFT doublings larger.
// On the CT 5-field plan (40M-history runs, 24M in flight) this takes 180
// waves down to about 105 and the run 1.8 % faster; shifts of 3 to 6 and
// thresholds from batch/16 to batch/4096 measured the same within 0.2 %.
#ifndef GX_TAIL_SHIFT
#define GX_TAIL_SHIFT 2u
#endif
#ifndef GX_TAIL_DIV
#define GX_TAIL_DIV 256u
#endif

// steps one particle may take inside one consumer launch before it is dropped
// and GX_ERR_STEP_BUDGET is raised (guards the persistent loops against a
// particle that stops making progress)
#define GX_STEP_BUDGET 4000000u

struct SchedState {
    unsigned long long next, end;     // history cursor
    unsigned long long h0, h1;        // histories injected by the current wave
    uint32_t batch, waves, max_waves, pending;
    uint32_t refill_below;
    uint32_t photon_done;             // photon MLC and phantom consumers finished in this wave
    uint32_t electron_done;           // electron branches finished in this wave
    uint32_t budget_shift;            // step budgets of the next wave are shifted left by this (tail of a run)
};

// ---- wave timeline (tracing; off unless DevCtx::timeline is set) ------------
// Kernel ids: 0 source; 1-3 photon jaws / MLC / phantom; 4-7 Compton, photo,
// Rayleigh, pair; 8-10 electron jaws / MLC / phantom; 11-14 Moller, brems,
// Bhabha, annihilation. Each block's thread 0 lowers the kernel's start stamp
// of this wave when the block begins and raises its end stamp once the block
// is done (after the block's barrier).
enum : int { TL_SOURCE = 0, TL_PHOTON = 1, TL_PINT = 4, TL_ELECTRON = 8, TL_EINT = 11, TL_ENEAR = 15, TL_PLONG = 16 };

__device__ __forceinline__ void timeline_mark(const DevCtx &C, int kernel, bool end)
{
    if (C.timeline == nullptr || threadIdx.x != 0) return;
    uint32_t w = *((volatile const uint32_t *)C.wave);
    if (w >= C.timeline_waves) return;
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    unsigned long long *slot = C.timeline + ((size_t)w * GX_TL_KERNELS + (size_t)kernel) * 2;
    if (end) atomicMax(slot + 1, t);
    else atomicMin(slot, t);
}

__device__ __forceinline__ void consumer_done(const DevCtx &C, int q, int q2 = -1, uint32_t *finished = nullptr)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        uint32_t prev = atomicAdd(&C.q.done[q], 1u);
        if (prev == gridDim.x - 1) {
            if (C.q.peak) {
                atomicMax(&C.q.peak[q], *((volatile uint32_t *)&C.q.count[q]));
                if (q2 >= 0) atomicMax(&C.q.peak[q2], *((volatile uint32_t *)&C.q.count[q2]));
            }
            C.q.count[q] = 0;
            C.q.head[q] = 0;
            C.q.done[q] = 0;
            if (q2 >= 0) C.q.count[q2] = 0;
            __threadfence();
            if (finished) atomicAdd(finished, 1u);
        }
    }
}

// Re-queue a particle whose per-launch step budget ran out (same stream, same
// state: the result does not depend on where a track is split).
__device__ __forceinline__ void push_cont(const DevCtx &C, int qid, Part p, const Rng &r, const EStatePk *st)
{
    rng_store(r, p);
    // lanes of a warp may push to different queues here: one atomic per queue
    cg::coalesced_group g = cg::labeled_partition(cg::coalesced_threads(), qid);
    uint32_t base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(&C.q.count[qid], (uint32_t)g.size());
    base = g.shfl(base, 0);
    uint32_t idx = base + g.thread_rank();
    if (idx < C.q.cap[qid]) {
        store_part(&C.q.buf[qid][idx], p);
        if (st) C.q.estate[qid - GX_Q_ECONT][idx] = *st;
    } else {
        atomicOr(C.err, GX_ERR_QUEUE_FULL);
    }
}

__device__ __forceinline__ EStatePk pack_estate(const EState &s)
{
    EStatePk k;
    k.elke = s.elke; k.demfp = s.demfp; k.sig0 = s.sig0; k.total_tstep = s.total_tstep;
    k.lelke = s.lelke;
    k.flags = (s.compute_tstep ? 1u : 0u) | (s.is_tstep ? 2u : 0u);
    k.pad0 = 0; k.pad1 = 0;
    return k;
}

__device__ __forceinline__ void unpack_estate(const EStatePk &k, EState &s)
{
    s.elke = k.elke; s.demfp = k.demfp; s.sig0 = k.sig0; s.total_tstep = k.total_tstep;
    s.lelke = k.lelke;
    s.compute_tstep = (k.flags & 1u) != 0;
    s.is_tstep = (k.flags & 2u) != 0;
}

__device__ __forceinline__ uint32_t queue_len(const DevCtx &C, int q)
{
    uint32_t n = *((volatile uint32_t *)&C.q.count[q]);
    return n < C.q.cap[q] ? n : C.q.cap[q];
}

__device__ __forceinline__ void block_stat_add(const DevCtx &C, int slot, unsigned long long v)
{
    // warp reduction then one atomic per warp
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(&C.stats[slot], v);
}

// ---- source: history index -> primary (CUDA_EGS.cu:52-131) -----------------
__device__ bool make_primary(const DevCtx &C, unsigned long long h, Part &p)
{
    int f;
    for (f = 0; f < C.nfields; f++) {
        unsigned long long hb = C.fields[f].hist_begin, he = C.fields[f].hist_end;
        if (h >= hb && h < he) break;
    }
    if (f == C.nfields) return false;
    const gegs_field *F = &C.fields[f];
    unsigned long long j = (h - F->hist_begin) / (unsigned long long)(F->nrepeat + 1);
    const gegs_phsp_record *rec = &C.phsp[j % C.nphsp];
    uint32_t latch = __ldg(&rec->latch);
    float re = __ldg(&rec->e), rx = __ldg(&rec->x), ry = __ldg(&rec->y);
    float ru = __ldg(&rec->u), rv = __ldg(&rec->v), rwt = __ldg(&rec->wt);
    int q;
    if (latch & 0x40000000u) q = -1;
    else if (latch & 0x20000000u) q = 1;
    else q = 0;
    float w2 = 1.0f - ru * ru - rv * rv;
    float w = sqrtf(w2 > 0.0f ? w2 : 0.0f);
    float wt = rwt;
    if (wt < 0.0f) { w = -w; wt = -wt; }
    p.charge = (int8_t)q;
    p.e = re < 0.0f ? -re : re;
    p.wt = wt;
    p.region = 0;
    p.leafIndex = GX_OUTMLC;
    p.bank = -1;
    p.module = (uint8_t)C.module_order[0];
    p.field = (uint8_t)f;
    p.x = rx; p.y = ry; p.z = C.z_phsp;
    p.u = ru; p.v = rv; p.w = w;
    p.hist_lo = (uint32_t)h;
    p.hist_hi = (uint32_t)(h >> 32);
    p.sid_lo = 0; p.sid_hi = 0; p.ctr = 0;
    p.status = 0;
    // beamlet: the bixel of the isocentre plane on the primary's straight line
    p.beamlet = GX_NO_BEAMLET;
    if (C.bl_nx > 0 && w > 0.0f) {
        float t = (C.sid - C.z_phsp) / w;
        float xi = rx + ru * t, yi = ry + rv * t;
        float fx = (xi - C.bl_x0) / C.bl_dx, fy = (yi - C.bl_y0) / C.bl_dy;
        if (fx >= 0.0f && fy >= 0.0f && fx < (float)C.bl_nx && fy < (float)C.bl_ny) {
            int b = f * C.bl_nx * C.bl_ny + (int)fy * C.bl_nx + (int)fx;
            p.beamlet = (uint16_t)b;
            if (C.bl_weight) p.wt = wt * __ldg(&C.bl_weight[b]);
        }
    }
    return true;
}

__global__ void k_source(const __grid_constant__ DevCtx C, const SchedState *st)
{
    timeline_mark(C, TL_SOURCE, false);
    unsigned long long h0 = st->h0, h1 = st->h1;
    unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long h = h0 + blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; h < h1; h += stride) {
        Part p;
        if (!make_primary(C, h, p)) { atomicOr(C.err, GX_ERR_SOURCE); continue; }
        push(C, p.charge == 0 ? ST_PHOTON : ST_ELECTRON, p);
    }
    if (C.timeline) {
        __syncthreads();
        timeline_mark(C, TL_SOURCE, true);
    }
}

// ---- persistent consumers with warp regeneration ---------------------------
// A consumer drains the continuation queue of the previous wave (indices
// [0, n_cont)) and then its stage queue ([n_cont, n)) through one shared head
// counter `hq`; idle lanes of a warp are refilled with one atomic.
template <int Q, bool ELEC>
__device__ __forceinline__ bool refill(const DevCtx &C, int hq, uint32_t n_cont, uint32_t n, int qc, bool &exhausted,
                                       bool active, Part &p, Rng &r, EState *s, unsigned long long &taken)
{
    const uint32_t lane = threadIdx.x & 31u;
    unsigned need = __ballot_sync(0xffffffffu, !active);
    if (need == 0u || exhausted) return active;
    uint32_t cnt = __popc(need);
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(&C.q.head[hq], cnt);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base + cnt >= n) exhausted = true;
    if (!active) {
        uint32_t idx = base + __popc(need & ((1u << lane) - 1u));
        if (idx < n) {
            if (idx < n_cont) {
                p = load_part(&C.q.buf[qc][idx]);
                rng_load(r, p);
                if (ELEC) unpack_estate(C.q.estate[qc - GX_Q_ECONT][idx], *s);
            } else {
                p = load_part(&C.q.buf[Q][idx - n_cont]);
                rng_load(r, p);
                if (ELEC) estate_init(*s);
                trace_event(C, 1u, Q, p);
                taken++;
            }
            return true;
        }
    }
    return active;
}

// Register caps of the transport consumers (minimum resident 256-thread
// blocks per SM); measured best on the CT 5-field plan.
#ifndef GX_PHOTON_MIN_BLOCKS
#define GX_PHOTON_MIN_BLOCKS 4
#endif
// the near-boundary electron passes: 80 registers
#ifndef GX_ELECTRON_MIN_BLOCKS
#define GX_ELECTRON_MIN_BLOCKS 3
#endif
// the phantom electrons: 64 registers. Its step spills some 280 bytes there
// against about 100 at 80 registers, yet the fourth block per SM hides more of
// the loads' latency: 2.1 % faster on C3 (5 blocks, 48 registers: 2.2 % slower)
#ifndef GX_EPHANTOM_MIN_BLOCKS
#define GX_EPHANTOM_MIN_BLOCKS 4
#endif
// the jaws photons (and their long tracks): 48 registers, 0.3 % faster than 64
#ifndef GX_PJAWS_MIN_BLOCKS
#define GX_PJAWS_MIN_BLOCKS 5
#endif
// the MLC photon kernel, the most divergent, runs best with 80 registers (fewer spills)
#ifndef GX_PMLC_MIN_BLOCKS
#define GX_PMLC_MIN_BLOCKS 3
#endif
// the first pass of the jaws and MLC electrons, without howfar: 48 registers
// (5 blocks), 0.3 % faster than 64
#ifndef GX_EHEAD_MIN_BLOCKS
#define GX_EHEAD_MIN_BLOCKS 5
#endif

// Transport consumer for photons (ELEC false) or electrons of one geometry
// class G. The three class kernels of a particle type run concurrently; the
// phantom kernel also takes the stage queue's new particles. A particle
// outside the class, or one whose step budget for this launch is spent, is
// re-queued with its state for the next wave (into its class's continuation
// queue), so the tally does not depend on where a track is split.
//
// Electrons in the jaws and the MLC run in two passes. The first hands every
// step that needs a boundary search (howfar, the costliest routine of these
// classes, wanted by few lanes of a warp at a time) to its class's
// near-boundary queue, as the step stood at its start; the second (NEAR) runs
// those steps again, whole, and carries its particles on while their steps
// need howfar, so that its warps search boundaries with most lanes at once. A
// step that does not goes back, as it stood, to the first pass of the next
// wave. For jaws photons the second form (NEAR) is the long-track kernel:
// it takes the photons still going when the photon phase ended and steps them
// beside the electron phase.
template <bool ELEC, int G, bool NEAR = false>
__device__ __forceinline__ void transport_consumer(const DevCtx &C)
{
    constexpr int Q = ELEC ? ST_ELECTRON : ST_PHOTON;
    constexpr int base = ELEC ? GX_Q_ECONT : GX_Q_PCONT;
    constexpr int cls = G - GX_GEOM_JAWS;                // 0 jaws, 1 MLC, 2 phantom
    constexpr bool FIRST = (G == GX_GEOM_PHANTOM);        // takes the new particles
    constexpr bool DEFER = ELEC && (G == GX_GEOM_JAWS || G == GX_GEOM_MLC) && !NEAR;
    // the photon jaws kernel's second form (NEAR): the long tracks, beside the electron phase
    constexpr bool LONG = !ELEC && G == GX_GEOM_JAWS && NEAR;
    constexpr int tl = LONG ? TL_PLONG : NEAR ? TL_ENEAR : (ELEC ? TL_ELECTRON : TL_PHOTON) + cls;
    timeline_mark(C, tl, false);
    if (!ELEC) stage_photon_tables(C);
    const uint32_t par = *C.wave & 1u;
    const int qc_in = LONG ? GX_Q_PLONG : NEAR ? GX_Q_ENEAR + cls : base + 2 * cls + (int)par;
    const int qc_out = base + 2 * cls + (int)(par ^ 1u);
    const int hq = FIRST ? Q : qc_in;
    const uint32_t n_cont = queue_len(C, qc_in);
    const uint32_t n = n_cont + (FIRST ? queue_len(C, Q) : 0u);
    // per-class budgets (measured on the CT 5-field plan): photons take 8x their
    // budget in the jaws and MLC, where a few bounce along leaf gaps for many
    // steps; electrons take 2x theirs in the phantom
    const uint32_t budget = (ELEC ? (cls < 2 ? C.electron_budget : 2u * C.electron_budget)
                                  : (cls < 2 ? 8u * C.photon_budget : C.photon_budget)) << *C.budget_shift;
    // A jaws photon takes a handful of steps, except the rare one that runs
    // almost parallel to a jaw face in tens of thousands of tiny steps. Past
    // its budget such a photon keeps stepping while the other photon consumers
    // of the wave are still running (up to 64 budgets), so that its long track
    // advances with the bulk of the work instead of one budget per wave in the
    // run's tail. Only when the phase's kernels run concurrently (C.overlap).
    constexpr bool JAWS_PHOTON = !ELEC && G == GX_GEOM_JAWS;
    // In the pipelined form the jaws photons step on while any of the five
    // other transport branches of the wave (both particle types) still runs.
    const volatile uint32_t *others_done = LONG ? C.electron_done : C.photon_done;
    const volatile uint32_t *others_done2 = C.electron_done;
    const uint32_t others = LONG ? 3u : C.pipelined ? 5u : 2u;
    // in the serial persistent form, a jaws photon still going when the photon
    // phase ends moves on to the long-track kernel, which runs beside the
    // electron phase the same way
    const int q_limit = (JAWS_PHOTON && !LONG && C.overlap && !C.pipelined) ? GX_Q_PLONG : qc_out;
    Part p;
    Rng r;
    EState s;
    bool active = false, exhausted = false;
    unsigned long long taken = 0, steps = 0;
    uint32_t nst = 0;
    for (;;) {
        bool was = active;
        active = refill<Q, ELEC>(C, hq, n_cont, n, qc_in, exhausted, active, p, r, &s, taken);
        if (active && !was) nst = 0;
        if (!__any_sync(0xffffffffu, active)) break;
        if (active) {
            if (!in_geom_class<G>(p)) {
                const int tq = base + 2 * (geom_class_of(p.module) - GX_GEOM_JAWS) + (int)(par ^ 1u);
                if (ELEC) { EStatePk k = pack_estate(s); push_cont(C, tq, p, r, &k); }
                else push_cont(C, tq, p, r, nullptr);
                active = false;
            } else {
                steps++;
                rng_window(C, r);
                bool done;
                if (DEFER || (ELEC && NEAR)) {
                    const uint32_t ctr0 = r.ctr;
                    const EState s0 = s;
                    const int code = DEFER ? electron_step<G, true, false>(C, p, r, s)
                                           : electron_step<G, false, true>(C, p, r, s);
                    if (code >= 2) {
                        // needs howfar (to the near-boundary pass) or, in that pass, does
                        // not (back to the first pass of the next wave): re-queued as it stood
                        r.ctr = ctr0;
                        EStatePk k = pack_estate(s0);
                        push_cont(C, code == 2 ? GX_Q_ENEAR + cls : qc_out, p, r, &k);
                        steps--;
                    }
                    done = code != 0;                 // leaves this pass either way
                } else done = ELEC ? electron_step<G>(C, p, r, s) != 0 : photon_step<G, true>(C, p, r);
                if (done) active = false;
                else if (++nst >= budget &&
                         (!JAWS_PHOTON || !C.overlap || nst >= 64u * budget ||
                          (((nst - budget) & 15u) == 0u &&
                           *others_done + (C.pipelined && !LONG ? *others_done2 : 0u) >= others))) {
                    if (ELEC) { EStatePk k = pack_estate(s); push_cont(C, qc_out, p, r, &k); }
                    else push_cont(C, q_limit, p, r, nullptr);
                    active = false;
                }
            }
        }
    }
    if (FIRST) block_stat_add(C, Q, taken);
    block_stat_add(C, GX_NSTAGE + (ELEC ? 1 : 0), steps);
    // steps in the jaws and the MLC (slots 12-15; the phantom's are the rest)
    if (cls < 2) block_stat_add(C, GX_NSTAGE + 2 + 2 * (ELEC ? 1 : 0) + cls, steps);
    // the last kernel of each photon branch but the jaws (MLC, phantom), and of
    // each electron branch (jaws and MLC near-boundary passes, phantom)
    uint32_t *fin = (!ELEC && G != GX_GEOM_JAWS) ? C.photon_done
                  : (ELEC && (NEAR || G == GX_GEOM_PHANTOM)) ? C.electron_done : nullptr;
    if (FIRST) consumer_done(C, Q, qc_in, fin);
    else consumer_done(C, qc_in, -1, fin);
    timeline_mark(C, tl, true);
}

__global__ void __launch_bounds__(256, GX_PJAWS_MIN_BLOCKS) k_photon_jaws(const __grid_constant__ DevCtx C)
{
    transport_consumer<false, GX_GEOM_JAWS>(C);
}

__global__ void __launch_bounds__(256, GX_PJAWS_MIN_BLOCKS) k_photon_jaws_long(const __grid_constant__ DevCtx C)
{
    transport_consumer<false, GX_GEOM_JAWS, true>(C);
}

__global__ void __launch_bounds__(256, GX_PMLC_MIN_BLOCKS) k_photon_mlc(const __grid_constant__ DevCtx C)
{
    transport_consumer<false, GX_GEOM_MLC>(C);
}

__global__ void __launch_bounds__(256, GX_PHOTON_MIN_BLOCKS) k_photon(const __grid_constant__ DevCtx C)
{
    transport_consumer<false, GX_GEOM_PHANTOM>(C);
}

__global__ void __launch_bounds__(256, GX_EHEAD_MIN_BLOCKS) k_electron_jaws(const __grid_constant__ DevCtx C)
{
    transport_consumer<true, GX_GEOM_JAWS>(C);
}

__global__ void __launch_bounds__(256, GX_EHEAD_MIN_BLOCKS) k_electron_mlc(const __grid_constant__ DevCtx C)
{
    transport_consumer<true, GX_GEOM_MLC>(C);
}

__global__ void __launch_bounds__(256, GX_ELECTRON_MIN_BLOCKS) k_electron_jaws_near(const __grid_constant__ DevCtx C)
{
    transport_consumer<true, GX_GEOM_JAWS, true>(C);
}

__global__ void __launch_bounds__(256, GX_ELECTRON_MIN_BLOCKS) k_electron_mlc_near(const __grid_constant__ DevCtx C)
{
    transport_consumer<true, GX_GEOM_MLC, true>(C);
}

__global__ void __launch_bounds__(256, GX_EPHANTOM_MIN_BLOCKS) k_electron(const __grid_constant__ DevCtx C)
{
    transport_consumer<true, GX_GEOM_PHANTOM>(C);
}

template <int Q>
__device__ __forceinline__ void run_interaction(const DevCtx &C, const Part &p, Rng &r)
{
    if (Q == ST_COMPTON) compton(C, p, r);
    else if (Q == ST_PHOTO) photo(C, p, r);
    else if (Q == ST_RAYLEIGH) rayleigh(C, p, r);
    else if (Q == ST_PAIR) pair(C, p, r);
    else if (Q == ST_MOLLER) moller(C, p, r);
    else if (Q == ST_BREMS) brems(C, p, r);
    else if (Q == ST_BHABHA) bhabha(C, p, r);
    else if (Q == ST_ANNIH) {
        if (at_rest_mark(p)) {
            Part q = p;
            annih_at_rest(C, q, region_info(C, q.region), r);
        } else annih(C, p, r);
    }
}

// Entries an interaction kernel counts as processed: all but the positrons
// handed over at rest (counted nowhere in the serial form either).
template <int Q>
__device__ __forceinline__ unsigned counted(const Part &p)
{
    return (Q == ST_ANNIH && at_rest_mark(p)) ? 0u : 1u;
}

template <int Q>
__global__ void __launch_bounds__(256) k_interact(const __grid_constant__ DevCtx C)
{
    constexpr int tl = Q < ST_ELECTRON ? TL_PINT + (Q - ST_COMPTON) : TL_EINT + (Q - ST_MOLLER);
    timeline_mark(C, tl, false);
    const uint32_t n = queue_len(C, Q);
    unsigned long long taken = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        Part p = load_part(&C.q.buf[Q][i]);
        Rng r;
        rng_load(r, p);
        rng_window(C, r);
        trace_event(C, 1u, Q, p);
        run_interaction<Q>(C, p, r);
        taken += counted<Q>(p);
    }
    block_stat_add(C, Q, taken);
    consumer_done(C, Q);
    timeline_mark(C, tl, true);
}

// ---- plain form: per-thread pops, one stage per launch ---------------------
template <int Q>
__global__ void __launch_bounds__(256) k_plain(const __grid_constant__ DevCtx C)
{
    const uint32_t n = queue_len(C, Q);
    unsigned long long taken = 0, steps = 0;
    for (;;) {
        uint32_t idx = atomicAdd(&C.q.head[Q], 1u);
        if (idx >= n) break;
        Part p = load_part(&C.q.buf[Q][idx]);
        Rng r;
        rng_load(r, p);
        trace_event(C, 1u, Q, p);
        taken += counted<Q>(p);
        if (Q == ST_PHOTON) {
            uint32_t nst = 0;
            while (!photon_step(C, p, r)) {
                steps++;
                if (++nst > GX_STEP_BUDGET) { atomicOr(C.err, GX_ERR_STEP_BUDGET); break; }
            }
            steps++;
        } else if (Q == ST_ELECTRON) {
            EState s;
            estate_init(s);
            uint32_t nst = 0;
            while (!electron_step(C, p, r, s)) {
                steps++;
                if (++nst > GX_STEP_BUDGET) { atomicOr(C.err, GX_ERR_STEP_BUDGET); break; }
            }
            steps++;
        } else {
            run_interaction<Q>(C, p, r);
        }
    }
    block_stat_add(C, Q, taken);
    if (Q == ST_PHOTON) block_stat_add(C, GX_NSTAGE, steps);
    if (Q == ST_ELECTRON) block_stat_add(C, GX_NSTAGE + 1, steps);
    consumer_done(C, Q);
}

// ---- planner: next wave's injection and the loop condition -----------------
__device__ __forceinline__ uint32_t plan_wave(const DevCtx &C, SchedState *st)
{
    uint32_t inflight = 0;
    for (int q = 0; q < GX_NQ; q++) inflight += *((volatile uint32_t *)&C.q.count[q]);
    uint32_t main_q = *((volatile uint32_t *)&C.q.count[ST_PHOTON]) + *((volatile uint32_t *)&C.q.count[ST_ELECTRON]);
    for (int q = GX_Q_PCONT; q < GX_NQ; q++) main_q += *((volatile uint32_t *)&C.q.count[q]);
    // once the population falls below `refill_below`, top it up to `batch`
    unsigned long long remaining = st->end - st->next;
    unsigned long long inject = 0;
    if (remaining > 0 && main_q < st->refill_below && main_q < st->batch) {
        inject = st->batch - main_q;
        if (inject > remaining) inject = remaining;
    }
    st->h0 = st->next;
    st->h1 = st->next + inject;
    st->next += inject;
    // The tail of a run: every history injected and few particles left. The
    // waves are then short and their fixed cost (launches, the step chains of
    // single particles) dominates; larger step budgets take fewer of them.
    st->budget_shift = (st->next >= st->end && main_q < st->batch / GX_TAIL_DIV) ? GX_TAIL_SHIFT : 0u;
    st->waves++;
    st->photon_done = 0u;
    st->electron_done = 0u;
    uint32_t pending = (inflight > 0 || inject > 0 || st->next < st->end) ? 1u : 0u;
    if (pending && st->waves >= st->max_waves) {
        atomicOr(C.err, GX_ERR_STEP_BUDGET);
        pending = 0;
    }
    if (*((volatile uint32_t *)C.err) & GX_ERR_QUEUE_FULL) pending = 0;
    st->pending = pending;
    return pending;
}

__global__ void k_plan(const __grid_constant__ DevCtx C, SchedState *st)
{
    plan_wave(C, st);
}

// Planner of a host-driven loop that queues several waves between checks
// (gegs_run_noalloc): once a plan has ended the run (pending 0), later calls
// inject nothing and count no wave, so the run's wave count and injected
// histories are those of the graph form, which stops at that plan.
__global__ void k_plan_gated(const __grid_constant__ DevCtx C, SchedState *st)
{
    if (st->pending == 0u) {
        st->h0 = st->h1 = st->next;
        return;
    }
    plan_wave(C, st);
}

__global__ void k_plan_cond(const __grid_constant__ DevCtx C, SchedState *st, cudaGraphConditionalHandle handle)
{
    uint32_t pending = plan_wave(C, st);
    cudaGraphSetConditional(handle, pending);
}

// ---- geometry probe (gegs_probe_geometry) ----------------------------------
__device__ __forceinline__ Part probe_part(const gegs_probe_state &s)
{
    Part p = {};
    p.region = s.region; p.charge = s.charge; p.leafIndex = s.leafIndex; p.bank = s.bank;
    p.module = s.module; p.field = s.field; p.status = s.status;
    p.wt = s.wt; p.e = s.e; p.x = s.x; p.y = s.y; p.z = s.z; p.u = s.u; p.v = s.v; p.w = s.w;
    return p;
}

__global__ void k_probe_geometry(const __grid_constant__ DevCtx C, uint32_t n, const gegs_probe_state *in,
                                 const float *t_in, uint32_t *far_region, float *far_t, gegs_probe_state *far_out,
                                 float *near_t)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const gegs_probe_state s = in[i];
    Part p = probe_part(s);
    float t = t_in[i];
    bool ok;
    far_region[i] = howfar(C, p, t, ok);
    far_t[i] = t;
    gegs_probe_state o = s;
    o.leafIndex = p.leafIndex; o.bank = p.bank; o.module = p.module;
    far_out[i] = o;
    Part q = probe_part(s);
    float tp = 0.0f;
    hownear(C, q, tp, ok);
    near_t[i] = tp;
}

__global__ void k_dose(const unsigned long long *tally, const float *mass, double unit, double *out, uint64_t n)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        double m = (double)mass[i];
        if (m == 0.0) m = 1.0;
        out[i] = (double)(long long)tally[i] * 9.313225746154785e-10 / m * unit;
    }
}

// ---- batch statistics (the reference's GET_UNCERTAINTY, CUDA_EGS.cu:817-876) ----
// One batch ends: x = tally gained since the last fold (MeV), S1 += x, S2 += x^2.
__global__ void k_stat_fold(const unsigned long long *tally, unsigned long long *snap, double *s1, double *s2,
                            uint64_t n)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const unsigned long long t = tally[i];
        const double x = (double)(long long)(t - snap[i]) * 9.313225746154785e-10;
        snap[i] = t;
        s1[i] += x;
        s2[i] += x * x;
    }
}

// Batch mean and the relative standard error of the mean of n batches,
// sqrt((S2/n - (S1/n)^2) / (n - 1)) / (S1/n) (0 where nothing was deposited).
__global__ void k_stat_final(const double *s1, const double *s2, double n, double *mean, double *rel, uint64_t nv)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nv; i += (uint64_t)gridDim.x * blockDim.x) {
        const double m = s1[i] / n;
        const double v = s2[i] / n - m * m;
        mean[i] = m;
        rel[i] = m > 0.0 ? sqrt((v > 0.0 ? v : 0.0) / (n - 1.0)) / m : 0.0;
    }
}
