/* C ABI of the B200 transport library (libgegs_b200.so).
 *
 * Plain pointers and sizes only.  One engine = one CUDA device + one stream;
 * an engine is not thread-safe (drive it from one host thread at a time).
 * The caller owns host buffers; the engine owns its device buffers.
 *
 * Mapping to the reference (RicciWoo/GEGS), which is a monolithic program
 * whose internal seams these calls replace:
 *   gegs_create + gegs_set_physics + gegs_set_scene
 *       replace init() (init.cu:1682-1710): tables, phantom, MLC/jaws set-up
 *       and the cudaMemcpyToSymbol uploads (copy.cu:3-277).
 *   gegs_run
 *       replaces runSimulation(histories_per_MU, iField) (CUDA_EGS.cu:367-900)
 *       and its per-kernel host loop launch_kernels() (CUDA_EGS.cu:226-365);
 *       all fields of the scene run in one call.
 *   gegs_get_tally / gegs_get_dose
 *       replace the D2H copy of eng_score and the host field sum
 *       (CUDA_EGS.cu:1723-1735) and the dose conversion of write_dose()
 *       (output.c:873-918).
 * Errors are returned as status codes; the reference calls exit() instead
 * (output.c:51-90).
 */
#ifndef GEGS_H
#define GEGS_H

#include <stddef.h>
#include <stdint.h>
#include "gegs_physics.h"
#include "gegs_scene.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gegs_engine gegs_engine;

typedef enum gegs_status {
    GEGS_OK = 0,
    GEGS_ERR_ARG = 1,          /* invalid argument or call order */
    GEGS_ERR_CUDA = 2,         /* CUDA runtime error (see gegs_last_error) */
    GEGS_ERR_QUEUE_FULL = 3,   /* an event queue overflowed: particles were lost */
    GEGS_ERR_MODULE = 4,       /* particle in an unsupported beam module */
    GEGS_ERR_NOMEM = 5,        /* device allocation failed */
    GEGS_ERR_STEP_BUDGET = 6,  /* the wave budget of a run was exhausted */
    GEGS_ERR_SOURCE = 7        /* history outside every field's range */
} gegs_status;

typedef enum gegs_mode {
    GEGS_MODE_PERSISTENT = 0,  /* device-driven wave loop in one CUDA graph */
    GEGS_MODE_PLAIN = 1,       /* host loop: one kernel per event type, sync + counter read-back each launch */
    GEGS_MODE_TIMED = 2        /* persistent kernels driven wave by wave from the host with CUDA events
                                  around every launch (per-kernel device times in gegs_run_stats) */
} gegs_mode;

typedef struct gegs_run_opts {
    int32_t mode;              /* gegs_mode */
    uint32_t batch;            /* particles kept in flight (0 = 60 % of the run's histories in steps of 64K,
                                  64K to 30M, within 85 % of free device memory; queue memory ~5 KB each,
                                  ~157 GB at 30M) */
    int32_t blocks_per_sm;     /* 0 = default (6: grid = 6 x SM count) */
    int32_t threads_per_block; /* 0 = default */
    uint32_t max_waves;        /* safety budget (0 = default) */
    uint32_t step_budget;      /* steps per particle per launch before it is continued in the next wave:
                                  bits 0-15 photons, 16-31 electrons (0 = defaults 32 / 4); photons get
                                  8x theirs in the jaws and MLC, electrons 2x theirs in the phantom */
    uint32_t refill_below;     /* new histories are injected once fewer than this many particles are in
                                  flight, topping the population up to `batch` (0 = default batch / 4) */
    uint32_t queue_cap;        /* testing aid: at most this many records per event queue (0 = sized from
                                  `batch`). A queue that would overflow drops nothing silently: the run
                                  stops after the wave and returns GEGS_ERR_QUEUE_FULL (the reference
                                  drops the particle with a message, utility.cu:270-275) */
    uint32_t flags;            /* GEGS_RUN_STAGE_TABLES: photon consumers stage the mean-free-path and
                                  Rayleigh tables of the plan's media in shared memory (same results;
                                  1.2 % slower on the CT 5-field plan, an autotuner choice per plan);
                                  GEGS_RUN_SERIAL_WAVES (persistent form): each wave runs the photon
                                  transport, the photon interactions, the electron transport and the
                                  electron interactions in turn, instead of both transports at once and
                                  then all interactions (the default, pipelined: a particle made by an
                                  interaction is transported in the next wave; 1.9 % faster on the CT
                                  5-field plan). The tally is the same either way */
} gegs_run_opts;

#define GEGS_RUN_STAGE_TABLES 1u
#define GEGS_RUN_SERIAL_WAVES 2u

#define GEGS_NQUEUES 25

typedef struct gegs_run_stats {
    uint64_t processed[10];    /* particles handled per stage: photon, compton, photo, rayleigh,
                                  pair, electron, moller, brems, bhabha, annih */
    uint64_t photon_steps, electron_steps;
    uint32_t waves;
    uint32_t error_bits;
    double device_ms;          /* device time of the last gegs_run (CUDA events) */
    double stage_ms[16];       /* GEGS_MODE_TIMED: device ms per kernel kind: 10 stages (photon and electron
                                  in the phantom), source, planner, photon and electron in the jaws,
                                  photon and electron in the MLC */
    uint64_t stage_launches[16];
    uint64_t photon_steps_class[3];   /* steps in the jaws, the MLC, the phantom (persistent and timed forms) */
    uint64_t electron_steps_class[3];
    /* per event queue (10 stages, 12 continuation queues, 2 near-boundary
     * queues, 1 long-track queue): the most records it held in one cycle of
     * the persistent and timed forms, and its capacity (0 after gegs_run_noalloc) */
    uint32_t queue_peak[GEGS_NQUEUES];
    uint32_t queue_cap[GEGS_NQUEUES];
} gegs_run_stats;

/* Engine life cycle */
gegs_status gegs_create(int device, gegs_engine **out);
void gegs_destroy(gegs_engine *e);
const char *gegs_last_error(const gegs_engine *e);

/* Physics tables (struct gegs_physics, same layout the reference keeps in
 * __device__ globals); checked with gegs_check_physics, then copied to HBM. */
gegs_status gegs_set_physics(gegs_engine *e, const gegs_physics *P);

/* Host-only check of a physics block (no GPU needed): nmed in 1..GEGS_MXMED,
 * every float member finite, every used medium's density positive. Returns
 * GEGS_ERR_ARG and a message naming the first bad entry (msg may be NULL).
 * The reference has no such check: its HATCH readers trust the data files
 * (media.cu:332-830). */
gegs_status gegs_check_physics(const gegs_physics *P, char *msg, size_t msg_len);

/* Phantom, beam-line geometry, fields and phase space; all copied to HBM.
 * Resets the tally. */
gegs_status gegs_set_scene(gegs_engine *e, const gegs_scene *S);

/* Replace only the phase-space records (host memory; copied on the engine's stream). */
gegs_status gegs_set_phsp(gegs_engine *e, const gegs_phsp_record *recs, uint64_t n);

/* Transport histories [hist_begin, hist_end) of the scene; energy is added to
 * the int64 tally (MeV * 2^30 per voxel).  opts may be NULL. */
gegs_status gegs_run(gegs_engine *e, uint64_t hist_begin, uint64_t hist_end, const gegs_run_opts *opts);

/* gegs_run in two halves, for running several engines (plans) at once on one
 * GPU (no counterpart in the reference, which runs fields one after another):
 * gegs_launch queues the persistent-form run on the engine's stream and
 * returns; gegs_wait blocks until it is done and reports like gegs_run. Each
 * engine has its own stream, so runs launched on several engines overlap on
 * the device. One launched run per engine at a time. */
gegs_status gegs_launch(gegs_engine *e, uint64_t hist_begin, uint64_t hist_end, const gegs_run_opts *opts);
gegs_status gegs_wait(gegs_engine *e);

/* Replace field `index` of the scene (its gantry cosine and sine, history range,
 * recycling count, jaw and leaf-end polygons) without uploading the phantom
 * again; the tally is kept. The reference sets a field up before each field's
 * run (setup_secjaws, init_leaf_pos, CUDA_EGS.cu:416-432). */
gegs_status gegs_set_field(gegs_engine *e, int32_t index, const gegs_field *F);

/* The CUDA stream (a cudaStream_t of the engine's device, passed as a pointer)
 * on which the engine issues all of its work from now on, so that a caller can
 * order it with its own work; NULL returns to the engine's own stream. The
 * caller keeps the stream alive while the engine uses it. (The reference has
 * no streams: runSimulation synchronises after every kernel, CUDA_EGS.cu:226-365.) */
gegs_status gegs_set_stream(gegs_engine *e, void *cuda_stream);

/* Several plans in one launch: the persistent-form runs of n engines on one
 * device (engine i transports [hist_begin[i], hist_end[i]) with opts[i]; opts
 * may be NULL) as one CUDA graph, one branch per engine -- its planner, then
 * its wave loop -- launched once on the first engine's stream. Each engine is
 * then finished with gegs_wait; its device_ms is the time of the whole group.
 * The graph is kept and launched again when the same engines, in the same
 * order and state, are grouped next.
 * The reference runs plans and fields one after another (CUDA_EGS.cu:1715-1742). */
gegs_status gegs_launch_group(gegs_engine *const *engines, int32_t n, const uint64_t *hist_begin,
                              const uint64_t *hist_end, const gegs_run_opts *opts);

/* No counterpart in the reference: an addition of this library.
 *
 * gegs_run_noalloc transports histories [hist_begin, hist_end) like gegs_run
 * and adds to the same tally, but it allocates no device memory. Its event
 * queues, scheduler state and counters live in one fixed array compiled into
 * the library (about 28 MB, held on every GPU that loads the library until the
 * process exits). Use it when the caller cannot allocate at run time:
 *   - a planning system or dose server that reserved the GPU's memory when it
 *     started, where a later cudaMalloc of gegs_run's queues (several GB at
 *     the default batch) fails or breaks up its pool;
 *   - a latency-bound loop that cannot absorb cudaFree's device-wide
 *     synchronisation.
 * The scene, physics tables and tally are still the engine's, set up
 * beforehand with gegs_create, gegs_set_physics and gegs_set_scene.
 *
 * batch = particles kept in flight: 0 means GEGS_NOALLOC_MAX_BATCH. Larger
 * values return GEGS_ERR_ARG. A small batch transports far fewer histories per
 * second than gegs_run with its default batch; the tally is the same bit for
 * bit. The first call on a device looks up the array's device address and
 * loads the library's kernels on that device, so make it before any stream
 * capture on that device. Every call on a device shares the one array; the
 * call clears the counters that must start at zero, but calls that overlap on
 * the same GPU (two engines, two threads) race on it and must be serialised
 * by the caller. The call returns when the transport is done. */
#define GEGS_NOALLOC_MAX_BATCH 4096u
gegs_status gegs_run_noalloc(gegs_engine *e, uint64_t hist_begin, uint64_t hist_end, uint32_t batch);

/* Beamlets (no counterpart in the reference; the scene's bl_* fields define
 * the grid). gegs_set_beamlet_weights replaces the n = nfields*bl_nx*bl_ny
 * fluence weights that multiply the weight of each tagged primary.
 *
 * gegs_backward returns d(objective)/d(weight) for every beamlet, given
 * voxel_grad[v] = d(objective)/d(energy deposited in voxel v, MeV) on the
 * host (nvox doubles; for a dose objective: dL/dD_v * dose_unit / mass_v).
 * It replays histories [hist_begin, hist_end) from their RNG counters with
 * unit fluence weights, adding energy * voxel_grad[v] of every deposit to the
 * gradient of the deposit's beamlet, so no per-history deposit is stored. The
 * tally is not touched. opts as for gegs_run (the persistent form is used). */
gegs_status gegs_set_beamlet_weights(gegs_engine *e, const float *w, uint32_t n);
gegs_status gegs_backward(gegs_engine *e, uint64_t hist_begin, uint64_t hist_end, const double *voxel_grad,
                          double *beamlet_grad, uint32_t n, const gegs_run_opts *opts);

gegs_status gegs_reset_tally(gegs_engine *e);

/* Copy the int64 tally (nvox entries) to host memory. */
gegs_status gegs_get_tally(gegs_engine *e, int64_t *out, uint64_t nvox);

/* Load the int64 tally from host memory (no counterpart in the reference,
 * which has no checkpoint). A checkpoint is the tally and the next history
 * index: loading it and running the remaining histories gives the tally of
 * the whole run bit for bit (per-history random streams, integer sums). */
gegs_status gegs_set_tally(gegs_engine *e, const int64_t *in, uint64_t nvox);

/* dose[i] = tally[i] * 2^-30 / voxel_mass[i] * dose_unit, in double, on the device;
 * voxel_mass is a host array of nvox entries (0 treated as 1, init.cu:1256-1271). */
gegs_status gegs_get_dose(gegs_engine *e, const float *voxel_mass, double dose_unit, double *out, uint64_t nvox);

gegs_status gegs_get_stats(gegs_engine *e, gegs_run_stats *out);

/* Batch statistics on the device, the reference's GET_UNCERTAINTY batch
 * method (CUDA_EGS.cu:817-876, there on the host after every batch):
 * gegs_stat_begin starts a series at the current tally; each gegs_stat_fold
 * ends a batch -- the energy deposited since the previous fold is that batch's
 * x_b per voxel, and S1 += x_b, S2 += x_b^2 in double. gegs_stat_get returns
 * per voxel the batch mean S1/n (MeV) and the relative standard error of the
 * mean, sqrt((S2/n - (S1/n)^2) / (n - 1)) / (S1/n), the reference's formula
 * (0 where nothing was deposited); n >= 2 folds are needed. */
gegs_status gegs_stat_begin(gegs_engine *e);
gegs_status gegs_stat_fold(gegs_engine *e);
gegs_status gegs_stat_get(gegs_engine *e, double *mean, double *rel_se, uint64_t nvox, uint32_t *nbatch);

/* A particle state for gegs_probe_geometry (56 bytes). */
typedef struct gegs_probe_state {
    uint32_t region;
    int8_t charge, leafIndex, bank;
    uint8_t module, field, status, pad0, pad1;
    float wt, e, x, y, z, u, v, w, dnear;
    uint32_t hist, pad2;
} gegs_probe_state;

/* The device's geometry routines on n given states, for checking them against
 * other implementations (no counterpart in the reference): per state i, howfar
 * of the step t_in[i] gives the region entered far_region[i], the step
 * far_t[i] and the state after the call far_out[i] (its leaf index, bank and
 * module may change); hownear of the unchanged state gives near_t[i]. The
 * routines are the transport's own (geom.cu:54-1543 restated). Needs a scene;
 * allocates device memory for the call. */
gegs_status gegs_probe_geometry(gegs_engine *e, uint32_t n, const gegs_probe_state *in, const float *t_in,
                                uint32_t *far_region, float *far_t, gegs_probe_state *far_out, float *near_t);

/* Device pointer of the tally (for callers that keep results in HBM). */
gegs_status gegs_tally_device_ptr(gegs_engine *e, void **out);

/* Debug trace: record every queue push and every particle a consumer takes
 * (32-byte records: kind|stage<<8, hist_lo, sid_lo, sid_hi, ctr, e, x, region).
 * capacity 0 turns tracing off.  gegs_get_trace copies min(n, capacity)
 * records, returns the number produced in *n and clears the buffer. */
/* Wave timeline (tracing; no counterpart in the reference, which times each
 * launch with events, CUDA_EGS.cu:249-294): with max_waves > 0, every run of
 * the persistent or timed form records for waves 0..max_waves-1 and each
 * kernel the first block's start and the last block's end (%globaltimer, ns)
 * in [wave][32][2]. Kernels: 0 source; 1-3 photon jaws, MLC, phantom;
 * 4-7 Compton, photo, Rayleigh, pair; 8-10 electron jaws, MLC, phantom;
 * 11-14 Moller, brems, Bhabha, annihilation; 15 the near-boundary passes of
 * the jaws and MLC electrons (together); 16 the long jaws-photon tracks run
 * beside the electron phase; 17-31 unused. A kernel that did not
 * run in a wave keeps start = UINT64_MAX, end = 0. 0 turns it off. */
gegs_status gegs_set_timeline(gegs_engine *e, uint32_t max_waves);
gegs_status gegs_get_timeline(gegs_engine *e, uint64_t *out, uint32_t max_waves);

gegs_status gegs_set_trace(gegs_engine *e, uint32_t capacity);
gegs_status gegs_get_trace(gegs_engine *e, void *out, uint32_t capacity, uint32_t *n);

/* Library introspection */
size_t gegs_sizeof_physics(void);
size_t gegs_sizeof_scene(void);
size_t gegs_sizeof_field(void);
const char *gegs_version(void);

#ifdef __cplusplus
}
#endif
#endif /* GEGS_H */
