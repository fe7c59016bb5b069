// Host engine behind the C ABI (include/gegs.h): device buffers, the event
// queues, the persistent CUDA-graph wave loop and the plain host-driven loop.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <memory>
#include <mutex>
#include <string>
#include <vector>
#include "kernels.cuh"
#include "../../include/gegs.h"

namespace {

// queue capacity per history in flight, per stage
constexpr float kCapFactor[GX_NQ] = {6.f, 3.f, 3.f, 3.f, 3.f, 6.f, 3.f, 3.f, 3.f, 3.f,   // stages
                                     2.f, 2.f, 2.f, 2.f, 3.f, 3.f,                        // photon continuations
                                     2.f, 2.f, 2.f, 2.f, 3.f, 3.f,
                                     3.f, 3.f,                                            // jaws / MLC electrons near a boundary
                                     1.f};                                                // long jaws photon tracks

constexpr unsigned long long cap_factor_sum()
{
    unsigned long long t = 0;
    for (int q = 0; q < GX_NQ; q++) t += (unsigned long long)kCapFactor[q];
    return t;
}

constexpr unsigned long long estate_factor_sum()
{
    unsigned long long t = 0;
    for (int q = GX_Q_ECONT; q < GX_Q_ECONT + GX_NESTATE; q++) t += (unsigned long long)kCapFactor[q];
    return t;
}

}  // namespace

static_assert(GX_NQ == GEGS_NQUEUES, "gegs_run_stats reports every queue");

// side streams of the graph's parallel branches (the pipelined wave forks
// eight interaction kernels: the engine's stream and seven more)
static constexpr int kAux = 7;

struct gegs_engine {
    int device = 0;
    int nsm = 0;
    cudaStream_t stream = nullptr;     // the stream all of the engine's work goes on
    cudaStream_t own_stream = nullptr; // the engine's own (stream, unless gegs_set_stream named another)
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // side streams and events that fork the independent kernels of a wave into
    // parallel branches of the persistent graph
    cudaStream_t aux[kAux] = {};
    cudaEvent_t ev_fork = nullptr, ev_join[kAux] = {};
    std::string err;

    gegs_physics *d_P = nullptr;
    float4 *d_ptab = nullptr;          // {gmfp, cohe} per (medium, energy bin) (DevCtx::ptab)
    Vox *d_reg = nullptr;
    float *d_xb = nullptr, *d_yb = nullptr, *d_zb = nullptr;
    gegs_field *d_fields = nullptr;
    float2 *d_cross = nullptr;
    float4 *d_jaw_lines = nullptr;      // per field and jaw: 8 unit edge lines (jaws hownear bound)
    gegs_phsp_record *d_phsp = nullptr;
    uint64_t nphsp = 0, phsp_cap = 0;
    unsigned long long *d_tally = nullptr;
    uint64_t nvox = 0;
    uint32_t *d_err = nullptr;
    unsigned long long *d_stats = nullptr;
    SchedState *d_sched = nullptr;
    unsigned long long *d_timeline = nullptr;   // wave timeline (gegs_set_timeline)
    uint32_t timeline_waves = 0;
    std::vector<unsigned long long> timeline_init;
    TraceRec *d_trace = nullptr;
    uint32_t *d_trace_n = nullptr;
    uint32_t trace_cap = 0;
    uint32_t *d_qmeta = nullptr;       // count[GX_NQ], head[GX_NQ], done[GX_NQ], peak[GX_NQ]
    Part *d_qbuf[GX_NQ] = {};
    EStatePk *d_estate[GX_NESTATE] = {};
    uint32_t qcap[GX_NQ] = {};
    uint32_t batch = 0;
    uint32_t queue_cap = 0;            // gegs_run_opts::queue_cap of the current queues

    DevCtx ctx{};
    bool have_physics = false, have_scene = false;
    unsigned long long ctx_gen = 1;
    unsigned long long uid = 0;        // unique per engine of the process (group graph keys)
    std::vector<gegs_field> host_fields;   // the scene's fields as last set (gegs_set_field)
    int nfields = 0;

    // cached persistent graph
    // cached persistent graphs: slot 0 forward transport, slot 1 gradient replay
    int slot = 0;
    cudaGraphExec_t gexec[2] = {};
    unsigned long long graph_gen[2] = {};
    int graph_grid[2] = {}, graph_threads[2] = {};

    // beamlets
    float *d_blw = nullptr;            // fluence weights
    uint32_t nbeamlets = 0;
    double *d_gvm = nullptr;           // d(objective)/d(energy) per voxel, for the replay
    double *d_grad = nullptr;          // [GX_GRAD_COPIES][nbeamlets]

    gegs_run_stats last{};
    bool in_flight = false;            // gegs_launch queued a run that gegs_wait has not finished
    std::shared_ptr<struct GroupRun> group;   // the group graph this engine's launched run belongs to
    std::shared_ptr<struct GroupRun> group_cache;   // the last group graph built with this engine

    // batch statistics (gegs_stat_*): per voxel the sum and sum of squares of
    // batch energies (MeV) and the tally at the last fold
    double *d_stat_s1 = nullptr, *d_stat_s2 = nullptr;
    unsigned long long *d_stat_snap = nullptr;
    uint64_t stat_nvox = 0;
    uint32_t stat_batches = 0;
};

static gegs_status cuda_fail(gegs_engine *e, cudaError_t c, const char *what)
{
    char buf[256];
    snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(c));
    e->err = buf;
    return c == cudaErrorMemoryAllocation ? GEGS_ERR_NOMEM : GEGS_ERR_CUDA;
}

#define CK(call, what)                                        \
    do {                                                      \
        cudaError_t _c = (call);                              \
        if (_c != cudaSuccess) return cuda_fail(e, _c, what); \
    } while (0)

template <typename T>
static cudaError_t realloc_dev(T **p, size_t n)
{
    if (*p) cudaFree(*p);
    *p = nullptr;
    if (n == 0) return cudaSuccess;
    return cudaMalloc((void **)p, n * sizeof(T));
}

// Unit normal form (a, b, c), a*x + b*y = c, of the line through each edge of
// the polygons that hownear_secjaws_y / _x measure (the bounding polygon and
// the jaw opening), per field and jaw: [field][jaw: Y, X][8]. |a*x + b*y - c|
// is at most the distance to the edge, so the smallest over the eight lines
// bounds hownear from below (jaws_near_lower_bound). A zero-length edge gets
// a line through its point.
static std::vector<float4> jaw_edge_lines(const gegs_field *F, int nfields)
{
    std::vector<float4> out((size_t)(nfields > 0 ? nfields : 0) * 16);
    auto line = [](const float (*poly)[2], int i) {
        const double ax = poly[i][0], ay = poly[i][1];
        const double bx = poly[(i + 1) & 3][0], by = poly[(i + 1) & 3][1];
        double nx = -(by - ay), ny = bx - ax;
        double len = std::sqrt(nx * nx + ny * ny);
        if (len == 0.0) { nx = 1.0; ny = 0.0; len = 1.0; }
        nx /= len; ny /= len;
        return make_float4((float)nx, (float)ny, (float)(nx * ax + ny * ay), 0.0f);
    };
    for (int f = 0; f < nfields; f++) {
        float4 *o = out.data() + (size_t)f * 16;
        for (int i = 0; i < 4; i++) {
            o[i] = line(F[f].boundMaxY, i);
            o[4 + i] = line(F[f].jawsGeomY + 2, i);
            o[8 + i] = line(F[f].boundMaxX, i);
            o[12 + i] = line(F[f].jawsGeomX + 2, i);
        }
    }
    return out;
}

extern "C" {

const char *gegs_version(void) { return "gegs_b200 0.1 (sm_100a)"; }
size_t gegs_sizeof_physics(void) { return sizeof(gegs_physics); }
size_t gegs_sizeof_scene(void) { return sizeof(gegs_scene); }
size_t gegs_sizeof_field(void) { return sizeof(gegs_field); }

const char *gegs_last_error(const gegs_engine *e) { return e ? e->err.c_str() : "null engine"; }

gegs_status gegs_create(int device, gegs_engine **out)
{
    if (!out) return GEGS_ERR_ARG;
    *out = nullptr;
    gegs_engine *e = new gegs_engine();
    static std::atomic<unsigned long long> next_uid{1};
    e->uid = next_uid++;
    e->device = device;
    cudaError_t c = cudaSetDevice(device);
    if (c != cudaSuccess) { gegs_status s = cuda_fail(e, c, "cudaSetDevice"); *out = e; return s; }
    cudaDeviceGetAttribute(&e->nsm, cudaDevAttrMultiProcessorCount, device);
    CK(cudaStreamCreateWithFlags(&e->own_stream, cudaStreamNonBlocking), "stream");
    e->stream = e->own_stream;
    CK(cudaEventCreate(&e->ev0), "event");
    CK(cudaEventCreate(&e->ev1), "event");
    for (int k = 0; k < kAux; k++) {
        CK(cudaStreamCreateWithFlags(&e->aux[k], cudaStreamNonBlocking), "stream");
        CK(cudaEventCreateWithFlags(&e->ev_join[k], cudaEventDisableTiming), "event");
    }
    CK(cudaEventCreateWithFlags(&e->ev_fork, cudaEventDisableTiming), "event");
    CK(cudaMalloc(&e->d_err, sizeof(uint32_t)), "err");
    CK(cudaMalloc(&e->d_stats, sizeof(unsigned long long) * 16), "stats");
    CK(cudaMalloc(&e->d_sched, sizeof(SchedState)), "sched");
    CK(cudaMalloc(&e->d_qmeta, sizeof(uint32_t) * 4 * GX_NQ), "qmeta");
    CK(cudaMemset(e->d_qmeta, 0, sizeof(uint32_t) * 4 * GX_NQ), "qmeta");
    *out = e;
    return GEGS_OK;
}

void gegs_destroy(gegs_engine *e)
{
    if (!e) return;
    cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    for (int k = 0; k < 2; k++) if (e->gexec[k]) cudaGraphExecDestroy(e->gexec[k]);
    cudaFree(e->d_blw); cudaFree(e->d_gvm); cudaFree(e->d_grad);
    cudaFree(e->d_P); cudaFree(e->d_ptab); cudaFree(e->d_reg); cudaFree(e->d_xb); cudaFree(e->d_yb); cudaFree(e->d_zb);
    cudaFree(e->d_timeline);
    cudaFree(e->d_fields); cudaFree(e->d_cross); cudaFree(e->d_jaw_lines); cudaFree(e->d_phsp); cudaFree(e->d_tally);
    cudaFree(e->d_err); cudaFree(e->d_stats); cudaFree(e->d_sched); cudaFree(e->d_qmeta);
    cudaFree(e->d_trace); cudaFree(e->d_trace_n);
    cudaFree(e->d_stat_s1); cudaFree(e->d_stat_s2); cudaFree(e->d_stat_snap);
    for (int q = 0; q < GX_NQ; q++) cudaFree(e->d_qbuf[q]);
    for (int k = 0; k < GX_NESTATE; k++) cudaFree(e->d_estate[k]);
    if (e->ev0) cudaEventDestroy(e->ev0);
    if (e->ev1) cudaEventDestroy(e->ev1);
    for (int k = 0; k < kAux; k++) {
        if (e->aux[k]) cudaStreamDestroy(e->aux[k]);
        if (e->ev_join[k]) cudaEventDestroy(e->ev_join[k]);
    }
    if (e->ev_fork) cudaEventDestroy(e->ev_fork);
    if (e->own_stream) cudaStreamDestroy(e->own_stream);
    delete e;
}

gegs_status gegs_check_physics(const gegs_physics *P, char *msg, size_t msg_len)
{
    auto fail = [&](const char *text) {
        if (msg && msg_len) snprintf(msg, msg_len, "%s", text);
        return GEGS_ERR_ARG;
    };
    if (!P) return fail("physics block is NULL");
    if (P->nmed < 1 || P->nmed > GEGS_MXMED) return fail("physics block: nmed outside 1..GEGS_MXMED");
    char buf[160];
#define GX_CHECK_FINITE(name)                                                                        \
    {                                                                                                \
        const float *v = (const float *)((const char *)P + offsetof(gegs_physics, name));            \
        const size_t n = sizeof(((const gegs_physics *)nullptr)->name) / sizeof(float);              \
        for (size_t i = 0; i < n; i++)                                                               \
            if (!std::isfinite(v[i])) {                                                              \
                snprintf(buf, sizeof buf, "physics block: %s[%zu] is not finite", #name, i);         \
                return fail(buf);                                                                    \
            }                                                                                        \
    }
    GEGS_PHYSICS_FLOAT_MEMBERS(GX_CHECK_FINITE)
#undef GX_CHECK_FINITE
    for (int m = 0; m < P->nmed; m++)
        if (!(P->rho[m] > 0.0f)) return fail("physics block: a medium has a density that is not positive");
    for (int i = 0; i < GEGS_MS_SIZE; i++)        // alias bins of the scattering tables (the sampler reads bin + 1)
        if (P->ims_array[i] < 0 || P->ims_array[i] > GEGS_MAXU_MS - 1)
            return fail("physics block: ims_array holds a bin outside 0..GEGS_MAXU_MS-1");
    if (msg && msg_len) msg[0] = '\0';
    return GEGS_OK;
}

gegs_status gegs_set_physics(gegs_engine *e, const gegs_physics *P)
{
    if (!e || !P) return GEGS_ERR_ARG;
    {
        char msg[192];
        if (gegs_check_physics(P, msg, sizeof msg) != GEGS_OK) { e->err = msg; return GEGS_ERR_ARG; }
    }
    CK(cudaSetDevice(e->device), "cudaSetDevice");
    if (!e->d_P) CK(cudaMalloc(&e->d_P, sizeof(gegs_physics)), "physics");
    CK(cudaMemcpyAsync(e->d_P, P, sizeof(gegs_physics), cudaMemcpyHostToDevice, e->stream), "physics H2D");
    // {gmfp, cohe} interleaved, the slice a photon step reads (see DevCtx::ptab)
    const size_t ng = (size_t)GEGS_MXMED * GEGS_MXGE;
    std::vector<float4> ptab(ng);
    for (size_t i = 0; i < ng; i++)
        ptab[i] = make_float4(P->gmfp[i][0], P->gmfp[i][1], P->cohe[i][0], P->cohe[i][1]);
    if (!e->d_ptab) CK(cudaMalloc(&e->d_ptab, ng * sizeof(float4)), "photon tables");
    CK(cudaMemcpyAsync(e->d_ptab, ptab.data(), ng * sizeof(float4), cudaMemcpyHostToDevice, e->stream), "tables H2D");
    CK(cudaStreamSynchronize(e->stream), "physics sync");
    e->have_physics = true;
    e->ctx.P = e->d_P;
    e->ctx.ptab = e->d_ptab;
    e->ctx.nmed = P->nmed;
    e->ctx_gen++;
    return GEGS_OK;
}

gegs_status gegs_set_phsp(gegs_engine *e, const gegs_phsp_record *recs, uint64_t n)
{
    if (!e || !recs || n == 0) return GEGS_ERR_ARG;
    CK(cudaSetDevice(e->device), "cudaSetDevice");
    if (n > e->phsp_cap) {
        CK(realloc_dev(&e->d_phsp, n), "phsp");
        e->phsp_cap = n;
        e->ctx_gen++;
    }
    CK(cudaMemcpyAsync(e->d_phsp, recs, n * sizeof(gegs_phsp_record), cudaMemcpyHostToDevice, e->stream), "phsp H2D");
    if (e->nphsp != n) e->ctx_gen++;
    e->nphsp = n;
    e->ctx.phsp = e->d_phsp;
    e->ctx.nphsp = n;
    return GEGS_OK;
}

gegs_status gegs_set_scene(gegs_engine *e, const gegs_scene *S)
{
    if (!e || !S || !e->have_physics) return GEGS_ERR_ARG;
    if (S->nx <= 0 || S->ny <= 0 || S->nz <= 0 || S->nfields < 1 || S->nfields > GEGS_MAX_FIELDS || !S->phsp || S->nphsp == 0)
        return GEGS_ERR_ARG;
    CK(cudaSetDevice(e->device), "cudaSetDevice");
    gegs_physics Ph;
    CK(cudaMemcpy(&Ph, e->d_P, sizeof Ph, cudaMemcpyDeviceToHost), "physics D2H");
    uint64_t nvox = (uint64_t)S->nx * S->ny * S->nz;
    std::vector<Vox> reg(nvox + GX_VAC_AND_OTH);
    reg[0].med = GX_VACUUM; reg[0].flags = 0; reg[0].rhof = 0.0f;
    for (int i = 1; i < GX_VAC_AND_OTH; i++) {
        int med = S->other_med[i - 1];
        if (med < 0) med = S->other_med[0];
        if (med < 0 || med >= Ph.nmed) { e->err = "other_med outside the media list"; return GEGS_ERR_ARG; }
        reg[i].med = (uint16_t)med; reg[i].flags = (uint16_t)S->region_flags; reg[i].rhof = 1.0f;
    }
    for (uint64_t v = 0; v < nvox; v++) {
        Vox &r = reg[v + GX_VAC_AND_OTH];
        uint16_t med = S->voxel_med[v];
        r.med = med;
        if (med == GX_VACUUM) { r.flags = 0; r.rhof = 0.0f; continue; }
        if (med >= Ph.nmed) { e->err = "voxel medium outside the media list"; return GEGS_ERR_ARG; }
        r.flags = (uint16_t)S->region_flags;
        r.rhof = S->voxel_rhof[v];
    }
    CK(realloc_dev(&e->d_reg, reg.size()), "regions");
    CK(cudaMemcpy(e->d_reg, reg.data(), reg.size() * sizeof(Vox), cudaMemcpyHostToDevice), "regions H2D");
    CK(realloc_dev(&e->d_xb, (size_t)S->nx + 1), "bounds");
    CK(realloc_dev(&e->d_yb, (size_t)S->ny + 1), "bounds");
    CK(realloc_dev(&e->d_zb, (size_t)S->nz + 1), "bounds");
    CK(cudaMemcpy(e->d_xb, S->x_bounds, ((size_t)S->nx + 1) * 4, cudaMemcpyHostToDevice), "bounds H2D");
    CK(cudaMemcpy(e->d_yb, S->y_bounds, ((size_t)S->ny + 1) * 4, cudaMemcpyHostToDevice), "bounds H2D");
    CK(cudaMemcpy(e->d_zb, S->z_bounds, ((size_t)S->nz + 1) * 4, cudaMemcpyHostToDevice), "bounds H2D");
    e->host_fields.assign(S->fields, S->fields + S->nfields);
    e->nfields = S->nfields;
    CK(realloc_dev(&e->d_fields, (size_t)S->nfields), "fields");
    CK(cudaMemcpy(e->d_fields, S->fields, sizeof(gegs_field) * S->nfields, cudaMemcpyHostToDevice), "fields H2D");
    {
        std::vector<float4> lines = jaw_edge_lines(S->fields, S->nfields);
        CK(realloc_dev(&e->d_jaw_lines, lines.size()), "jaw lines");
        CK(cudaMemcpy(e->d_jaw_lines, lines.data(), lines.size() * sizeof(float4), cudaMemcpyHostToDevice),
           "jaw lines H2D");
    }
    if (!e->d_cross) CK(cudaMalloc(&e->d_cross, sizeof(float2) * 960), "crossXZ");
    CK(cudaMemcpy(e->d_cross, S->crossXZ, sizeof(float2) * 960, cudaMemcpyHostToDevice), "crossXZ H2D");
    if (nvox != e->nvox || !e->d_tally) {
        CK(realloc_dev(&e->d_tally, nvox), "tally");
        e->nvox = nvox;
    }
    CK(cudaMemset(e->d_tally, 0, nvox * sizeof(unsigned long long)), "tally reset");
    gegs_status st = gegs_set_phsp(e, S->phsp, S->nphsp);
    if (st != GEGS_OK) return st;
    CK(cudaStreamSynchronize(e->stream), "scene sync");

    DevCtx &C = e->ctx;
    C.P = e->d_P;
    C.reg = e->d_reg;
    C.xb = e->d_xb; C.yb = e->d_yb; C.zb = e->d_zb;
    C.fields = e->d_fields;
    C.crossXZ = e->d_cross;
    C.jaw_lines = e->d_jaw_lines;
    C.phsp = e->d_phsp;
    C.nphsp = e->nphsp;
    C.tally = e->d_tally;
    C.err = e->d_err;
    C.stats = e->d_stats;
    C.nx = S->nx; C.ny = S->ny; C.nz = S->nz; C.nfields = S->nfields;
    C.div_nx = make_fastdiv((uint32_t)S->nx);
    C.div_nxny = make_fastdiv((uint32_t)S->nx * (uint32_t)S->ny);
    C.change_xyz = S->change_xyz;
    C.hownear_off = S->hownear_region_offset == 6 ? 6 : 5;
    C.sid = S->source_to_isocenter;
    C.iso0 = S->iso[0]; C.iso1 = S->iso[1]; C.iso2 = S->iso[2];
    C.z_phsp = S->z_phsp;
    C.mlc_rmax = S->mlc_rmax; C.mlc_zmin = S->mlc_zmin; C.mlc_zthick = S->mlc_zthick;
    C.mlc_x_start = S->mlc_x_start; C.mlc_x_end = S->mlc_x_end; C.mlc_x_mid_1 = S->mlc_x_mid_1;
    C.mlc_x_mid_2 = S->mlc_x_mid_2; C.mlc_air_gap = S->mlc_air_gap; C.mlc_wl_full = S->mlc_wl_full;
    C.mlc_wl_target = S->mlc_wl_target; C.mlc_wl_isocenter = S->mlc_wl_isocenter; C.mlc_wt = S->mlc_wt;
    for (int i = 0; i < 4; i++) {
        C.boundaryXZ[i] = make_float2(S->boundaryXZ[i][0], S->boundaryXZ[i][1]);
        C.boundaryYZ[i] = make_float2(S->boundaryYZ[i][0], S->boundaryYZ[i][1]);
    }
    for (int i = 0; i < 8; i++) C.module_order[i] = S->module_order[i];
    C.seed_lo = (uint32_t)S->seed;
    C.seed_hi = (uint32_t)(S->seed >> 32);
    // beamlet grid and fluence weights
    uint64_t nbl = S->bl_nx > 0 && S->bl_ny > 0 ? (uint64_t)S->nfields * S->bl_nx * S->bl_ny : 0;
    if (nbl >= GX_NO_BEAMLET) { e->err = "at most 65534 beamlets"; return GEGS_ERR_ARG; }
    C.bl_nx = nbl ? S->bl_nx : 0; C.bl_ny = nbl ? S->bl_ny : 0; C.nbeamlets = (int)nbl;
    C.bl_x0 = S->bl_x0; C.bl_y0 = S->bl_y0; C.bl_dx = S->bl_dx; C.bl_dy = S->bl_dy;
    C.bl_weight = nullptr;
    C.gvm = nullptr;
    C.grad = nullptr;
    if (nbl != e->nbeamlets) {
        CK(realloc_dev(&e->d_blw, (size_t)nbl), "beamlet weights");
        CK(realloc_dev(&e->d_grad, (size_t)nbl * GX_GRAD_COPIES), "beamlet gradient");
        e->nbeamlets = (uint32_t)nbl;
    }
    if (nbl && S->bl_weight) {
        CK(cudaMemcpy(e->d_blw, S->bl_weight, nbl * sizeof(float), cudaMemcpyHostToDevice), "beamlet weights H2D");
        C.bl_weight = e->d_blw;
    }
    if (e->d_gvm) { cudaFree(e->d_gvm); e->d_gvm = nullptr; }
    e->have_scene = true;
    e->ctx_gen++;
    return GEGS_OK;
}

gegs_status gegs_reset_tally(gegs_engine *e)
{
    if (!e || !e->d_tally) return GEGS_ERR_ARG;
    CK(cudaMemsetAsync(e->d_tally, 0, e->nvox * sizeof(unsigned long long), e->stream), "tally reset");
    CK(cudaStreamSynchronize(e->stream), "tally reset sync");
    return GEGS_OK;
}

}  // extern "C"

// Queue memory per particle of the in-flight batch (records and electron state).
constexpr unsigned long long kQueueBytesPerParticle =
    cap_factor_sum() * sizeof(Part) + estate_factor_sum() * sizeof(EStatePk);

// In-flight batch when the caller leaves it at 0: 60 % of the run's histories
// in steps of 64K, between 64K and 30M (about 157 GB of queues), and within
// 85 % of the device memory that is free once this engine's current queues are
// counted as free. More particles in flight keep more lanes busy and need
// fewer waves: on the CT 5-field plan's 40M-history steps, 24M in flight is
// 2.9 % faster than 16M, 16M 7 % faster than 6M, and 26M to 30M gain nothing
// over 24M; the whole 2e8-history plan in one launch is 1.1 % faster with 30M
// in flight than with 25M (and 1.3 % slower with 20M).
static uint32_t default_batch(gegs_engine *e, uint64_t histories)
{
    const uint64_t step = 1ull << 16, most = 30ull << 20;
    uint64_t want = histories / 5 * 3;
    want = want / step * step;
    if (want < step) want = step;
    if (want > most) want = most;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
        unsigned long long have = (unsigned long long)e->batch * kQueueBytesPerParticle;
        unsigned long long fit = (unsigned long long)((double)(free_b + have) * 0.85) / kQueueBytesPerParticle;
        fit = fit / step * step;
        if (want > fit) want = fit > step ? fit : step;
    }
    return (uint32_t)want;
}

// Queue buffers for `batch` particles in flight; queue_cap > 0 caps every
// queue's capacity (a testing aid that makes a run overflow on purpose).
static gegs_status ensure_queues(gegs_engine *e, uint32_t batch, uint32_t queue_cap)
{
    if (batch == e->batch && queue_cap == e->queue_cap) return GEGS_OK;
    for (int q = 0; q < GX_NQ; q++) {
        uint64_t cap = (uint64_t)(kCapFactor[q] * (float)batch) + 4096;
        if (cap > 0xFFFFFFF0ull) cap = 0xFFFFFFF0ull;
        if (queue_cap && cap > queue_cap) cap = queue_cap;
        CK(realloc_dev(&e->d_qbuf[q], (size_t)cap), "queue buffer");
        e->qcap[q] = (uint32_t)cap;
    }
    for (int k = 0; k < GX_NESTATE; k++)
        CK(realloc_dev(&e->d_estate[k], (size_t)e->qcap[GX_Q_ECONT + k]), "electron state");
    e->batch = batch;
    e->queue_cap = queue_cap;
    e->ctx_gen++;
    return GEGS_OK;
}

static void fill_queue_ctx(gegs_engine *e)
{
    QueueSet &Q = e->ctx.q;
    for (int q = 0; q < GX_NQ; q++) { Q.buf[q] = e->d_qbuf[q]; Q.cap[q] = e->qcap[q]; }
    for (int k = 0; k < GX_NESTATE; k++) Q.estate[k] = e->d_estate[k];
    Q.count = e->d_qmeta;
    Q.head = e->d_qmeta + GX_NQ;
    Q.done = e->d_qmeta + 2 * GX_NQ;
    Q.peak = e->d_qmeta + 3 * GX_NQ;
    e->ctx.wave = &e->d_sched->waves;
    e->ctx.budget_shift = &e->d_sched->budget_shift;
    e->ctx.photon_done = &e->d_sched->photon_done;
    e->ctx.electron_done = &e->d_sched->electron_done;
    e->ctx.overlap = 1u;
}

// One wave of the persistent form, as captured into the graph body. Kernels
// with no data between them run as parallel branches: the three photon
// consumers, the four photon interactions, the three electron consumers (the
// jaws and MLC branches each followed by their near-boundary pass, which
// drains what the first pass queued) with the long jaws-photon tracks beside
// them, and the four electron interactions (each reads its own queues; the
// pushes they share are atomic appends read only by a later phase).
static void launch_wave_kernels(gegs_engine *e, int grid, int threads)
{
    const DevCtx &C = e->ctx;
    cudaStream_t s = e->stream, *a = e->aux;
    auto fork = [&](int n) {
        cudaEventRecord(e->ev_fork, s);
        for (int k = 0; k < n; k++) cudaStreamWaitEvent(a[k], e->ev_fork, 0);
    };
    auto join = [&](int n) {
        for (int k = 0; k < n; k++) {
            cudaEventRecord(e->ev_join[k], a[k]);
            cudaStreamWaitEvent(s, e->ev_join[k], 0);
        }
    };
    k_source<<<grid, threads, 0, s>>>(C, e->d_sched);
    const size_t ps = C.stage_tables ? photon_smem_bytes(C.nmed) : 0;   // the staged {gmfp, cohe} table
    if (C.pipelined) {
        // Both transport phases at once: the photon consumers read the photon
        // queues, the electron consumers the electron queues, and neither
        // pushes to a queue the other reads (a positron stopping in the
        // electron transport goes to the annihilation queue). Then all eight
        // interaction kernels, whose new particles the next wave transports.
        // The branches are created in the order in which their blocks are best
        // given the SMs: the jaws photons first (their long tracks keep
        // stepping while the other branches run), then the MLC and phantom
        // photons, then the electrons of the phantom, the MLC and the jaws.
        // Measured on the 40M-history C3 step against the order jaws, MLC,
        // phantom with photons and electrons interleaved: 1.7 % faster; the
        // jaws photons created last: 6 % slower.
        fork(5);
        k_photon_jaws<<<grid, threads, ps, a[0]>>>(C);
        k_photon_mlc<<<grid, threads, ps, a[1]>>>(C);
        k_photon<<<grid, threads, ps, s>>>(C);
        k_electron<<<grid, threads, 0, a[4]>>>(C);
        k_electron_mlc<<<grid, threads, 0, a[3]>>>(C);
        k_electron_mlc_near<<<grid, threads, 0, a[3]>>>(C);
        k_electron_jaws<<<grid, threads, 0, a[2]>>>(C);
        k_electron_jaws_near<<<grid, threads, 0, a[2]>>>(C);
        join(5);
        fork(7);
        k_interact<ST_COMPTON><<<grid, threads, 0, s>>>(C);
        k_interact<ST_PHOTO><<<grid, threads, 0, a[0]>>>(C);
        k_interact<ST_RAYLEIGH><<<grid, threads, 0, a[1]>>>(C);
        k_interact<ST_PAIR><<<grid, threads, 0, a[2]>>>(C);
        k_interact<ST_MOLLER><<<grid, threads, 0, a[3]>>>(C);
        k_interact<ST_BREMS><<<grid, threads, 0, a[4]>>>(C);
        k_interact<ST_BHABHA><<<grid, threads, 0, a[5]>>>(C);
        k_interact<ST_ANNIH><<<grid, threads, 0, a[6]>>>(C);
        join(7);
        return;
    }
    fork(2);
    k_photon_jaws<<<grid, threads, ps, a[0]>>>(C);
    k_photon_mlc<<<grid, threads, ps, a[1]>>>(C);
    k_photon<<<grid, threads, ps, s>>>(C);
    join(2);
    fork(3);
    k_interact<ST_COMPTON><<<grid, threads, 0, s>>>(C);
    k_interact<ST_PHOTO><<<grid, threads, 0, a[0]>>>(C);
    k_interact<ST_RAYLEIGH><<<grid, threads, 0, a[1]>>>(C);
    k_interact<ST_PAIR><<<grid, threads, 0, a[2]>>>(C);
    join(3);
    fork(3);
    k_photon_jaws_long<<<grid, threads, ps, a[2]>>>(C);
    k_electron_jaws<<<grid, threads, 0, a[0]>>>(C);
    k_electron_jaws_near<<<grid, threads, 0, a[0]>>>(C);
    k_electron_mlc<<<grid, threads, 0, a[1]>>>(C);
    k_electron_mlc_near<<<grid, threads, 0, a[1]>>>(C);
    k_electron<<<grid, threads, 0, s>>>(C);
    join(3);
    fork(3);
    k_interact<ST_MOLLER><<<grid, threads, 0, s>>>(C);
    k_interact<ST_BREMS><<<grid, threads, 0, a[0]>>>(C);
    k_interact<ST_BHABHA><<<grid, threads, 0, a[1]>>>(C);
    k_interact<ST_ANNIH><<<grid, threads, 0, a[2]>>>(C);
    join(3);
}

// Adds an engine's wave loop to g: a WHILE node whose body is one wave and
// whose condition k_plan_cond sets on the device. With a planner, the loop is
// preceded by the k_plan node that plans the first wave (a run launched on
// its own launches k_plan before the graph instead).
static gegs_status add_wave_loop(gegs_engine *e, cudaGraph_t g, int grid, int threads, bool with_planner)
{
    cudaGraphNode_t pnode = nullptr;
    if (with_planner) {
        void *args[] = {(void *)&e->ctx, (void *)&e->d_sched};
        cudaKernelNodeParams kp = {};
        kp.func = (void *)k_plan;
        kp.gridDim = dim3(1);
        kp.blockDim = dim3(1);
        kp.kernelParams = args;
        CK(cudaGraphAddKernelNode(&pnode, g, nullptr, 0, &kp), "planner node");
    }
    cudaGraphConditionalHandle handle;
    CK(cudaGraphConditionalHandleCreate(&handle, g, 1, cudaGraphCondAssignDefault), "conditional handle");
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t cnode;
    CK(cudaGraphAddNode(&cnode, g, pnode ? &pnode : nullptr, pnode ? 1 : 0, &cp), "conditional node");
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    CK(cudaStreamBeginCaptureToGraph(e->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal), "capture");
    launch_wave_kernels(e, grid, threads);
    k_plan_cond<<<1, 1, 0, e->stream>>>(e->ctx, e->d_sched, handle);
    cudaGraph_t captured;
    CK(cudaStreamEndCapture(e->stream, &captured), "end capture");
    return GEGS_OK;
}

static gegs_status build_graph(gegs_engine *e, int grid, int threads)
{
    const int k = e->slot;
    if (e->gexec[k] && e->graph_gen[k] == e->ctx_gen && e->graph_grid[k] == grid && e->graph_threads[k] == threads)
        return GEGS_OK;
    if (e->gexec[k]) { cudaGraphExecDestroy(e->gexec[k]); e->gexec[k] = nullptr; }
    cudaGraph_t g;
    CK(cudaGraphCreate(&g, 0), "graph create");
    gegs_status st = add_wave_loop(e, g, grid, threads, false);
    if (st != GEGS_OK) { cudaGraphDestroy(g); return st; }
    CK(cudaGraphInstantiate(&e->gexec[k], g, 0), "graph instantiate");
    cudaGraphDestroy(g);
    e->graph_gen[k] = e->ctx_gen;
    e->graph_grid[k] = grid;
    e->graph_threads[k] = threads;
    return GEGS_OK;
}

// The executable graph of a group launch, shared by the group's engines and
// destroyed when the last of them has waited for its run.
struct GroupKey {
    unsigned long long uid, gen;       // the engine (never reused) and its context generation
    int grid, threads;
    bool operator==(const GroupKey &o) const { return uid == o.uid && gen == o.gen && grid == o.grid && threads == o.threads; }
};

struct GroupRun {
    cudaGraphExec_t exec = nullptr;
    std::vector<GroupKey> key;          // the engines, in order, with the state their branches were captured from
    ~GroupRun() { if (exec) cudaGraphExecDestroy(exec); }
};

static gegs_status run_finish(gegs_engine *e);

// Everything a run needs before its kernels: options resolved into the
// context, queues sized, the scheduler state and the counters reset on the
// engine's stream.
struct RunSetup {
    gegs_run_opts o;
    int grid, threads;
    uint32_t max_waves;
};

static gegs_status prepare_run(gegs_engine *e, uint64_t hist_begin, uint64_t hist_end, const gegs_run_opts *opts,
                               RunSetup &R)
{
    if (!e || !e->have_scene || hist_end < hist_begin) return GEGS_ERR_ARG;
    if (e->in_flight) { e->err = "a launched run has not been waited for (gegs_wait)"; return GEGS_ERR_ARG; }
    CK(cudaSetDevice(e->device), "cudaSetDevice");
    gegs_run_opts &o = R.o;
    o = {};
    if (opts) o = *opts;
    uint32_t batch = o.batch ? o.batch : default_batch(e, hist_end - hist_begin);
    int threads = o.threads_per_block ? o.threads_per_block : 256;
    // 6 blocks per SM: more than the 3-4 that fit at once, so that a block that
    // finishes early is replaced while a consumer's queue still has work (C3: -0.8 %)
    int bps = o.blocks_per_sm ? o.blocks_per_sm : 6;
    int grid = e->nsm * bps;
    uint32_t max_waves = o.max_waves ? o.max_waves : 200000u;
    const uint32_t stage = (o.flags & GEGS_RUN_STAGE_TABLES) ? 1u : 0u;
    if (stage != e->ctx.stage_tables) { e->ctx.stage_tables = stage; e->ctx_gen++; }
    const uint32_t pipe = (o.mode == GEGS_MODE_PERSISTENT && !(o.flags & GEGS_RUN_SERIAL_WAVES)) ? 1u : 0u;
    if (pipe != e->ctx.pipelined) { e->ctx.pipelined = pipe; e->ctx_gen++; }
    uint32_t pb = (o.step_budget & 0xFFFFu) ? (o.step_budget & 0xFFFFu) : 32u;
    uint32_t eb = (o.step_budget >> 16) ? (o.step_budget >> 16) : 4u;
    if (pb != e->ctx.photon_budget || eb != e->ctx.electron_budget) {
        e->ctx.photon_budget = pb;
        e->ctx.electron_budget = eb;
        e->ctx_gen++;
    }
    gegs_status st = ensure_queues(e, batch, o.queue_cap);
    if (st != GEGS_OK) return st;
    fill_queue_ctx(e);

    SchedState hs = {};
    hs.next = hist_begin;
    hs.end = hist_end;
    hs.batch = batch;
    hs.max_waves = max_waves;
    hs.refill_below = o.refill_below ? o.refill_below : (batch / 4u > 0u ? batch / 4u : 1u);
    CK(cudaMemcpyAsync(e->d_sched, &hs, sizeof hs, cudaMemcpyHostToDevice, e->stream), "sched H2D");
    CK(cudaMemsetAsync(e->d_qmeta, 0, sizeof(uint32_t) * 4 * GX_NQ, e->stream), "qmeta reset");
    CK(cudaMemsetAsync(e->d_err, 0, sizeof(uint32_t), e->stream), "err reset");
    CK(cudaMemsetAsync(e->d_stats, 0, sizeof(unsigned long long) * 16, e->stream), "stats reset");
    if (e->d_timeline) {
        // start stamps at the maximum, end stamps at 0 (each wave x kernel pair)
        e->timeline_init.resize((size_t)e->timeline_waves * GX_TL_KERNELS * 2);
        for (size_t i = 0; i < e->timeline_init.size(); i += 2) {
            e->timeline_init[i] = ~0ull;
            e->timeline_init[i + 1] = 0ull;
        }
        CK(cudaMemcpyAsync(e->d_timeline, e->timeline_init.data(), e->timeline_init.size() * 8,
                           cudaMemcpyHostToDevice, e->stream), "timeline reset");
    }

    R.grid = grid;
    R.threads = threads;
    R.max_waves = max_waves;
    return GEGS_OK;
}

// The transport of a run; with launch_only (persistent form) it returns once
// the graph is queued on the engine's stream, and run_finish completes it.
static gegs_status run_impl(gegs_engine *e, uint64_t hist_begin, uint64_t hist_end, const gegs_run_opts *opts,
                            bool launch_only)
{
    RunSetup R;
    gegs_status st = prepare_run(e, hist_begin, hist_end, opts, R);
    if (st != GEGS_OK) return st;
    const gegs_run_opts &o = R.o;
    const int grid = R.grid, threads = R.threads;
    const uint32_t max_waves = R.max_waves;
    for (int k = 0; k < 16; k++) { e->last.stage_ms[k] = 0.0; e->last.stage_launches[k] = 0; }
    if (o.mode == GEGS_MODE_PERSISTENT) {
        st = build_graph(e, grid, threads);
        if (st != GEGS_OK) return st;
        CK(cudaEventRecord(e->ev0, e->stream), "event");
        k_plan<<<1, 1, 0, e->stream>>>(e->ctx, e->d_sched);
        CK(cudaGraphLaunch(e->gexec[e->slot], e->stream), "graph launch");
        CK(cudaEventRecord(e->ev1, e->stream), "event");
    } else if (o.mode == GEGS_MODE_TIMED) {
        // Same kernels as the persistent graph, launched wave by wave with an
        // event pair around each launch to attribute device time per kernel.
        std::vector<cudaEvent_t> evs(32);
        for (auto &ev : evs) CK(cudaEventCreate(&ev), "event");
        CK(cudaEventRecord(e->ev0, e->stream), "event");
        SchedState hsr;
        float acc[16] = {0};
        unsigned long long nl[16] = {0};
        for (uint32_t w = 0; w < max_waves; w++) {
            CK(cudaEventRecord(evs[30], e->stream), "event");
            k_plan<<<1, 1, 0, e->stream>>>(e->ctx, e->d_sched);
            CK(cudaEventRecord(evs[31], e->stream), "event");
            CK(cudaMemcpyAsync(&hsr, e->d_sched, sizeof hsr, cudaMemcpyDeviceToHost, e->stream), "sched D2H");
            CK(cudaStreamSynchronize(e->stream), "timed sync");
            float t = 0.0f;
            cudaEventElapsedTime(&t, evs[30], evs[31]);
            acc[11] += t; nl[11]++;
            if (!hsr.pending) break;
            DevCtx C = e->ctx;
            C.overlap = 0u;             // one kernel at a time
            cudaStream_t s = e->stream;
            // codes 12 / 13: photon / electron consumers of the jaws, 14 / 15: of the MLC
            int slot[15] = {10, 12, 14, ST_PHOTON, ST_COMPTON, ST_PHOTO, ST_RAYLEIGH, ST_PAIR, 13, 15, ST_ELECTRON,
                            ST_MOLLER, ST_BREMS, ST_BHABHA, ST_ANNIH};
            for (int k = 0; k < 15; k++) {
                CK(cudaEventRecord(evs[2 * k], s), "event");
                switch (slot[k]) {
                case 10: k_source<<<grid, threads, 0, s>>>(C, e->d_sched); break;
                case 12: k_photon_jaws<<<grid, threads, C.stage_tables ? photon_smem_bytes(C.nmed) : 0, s>>>(C); break;
                case 13:
                    k_electron_jaws<<<grid, threads, 0, s>>>(C);
                    k_electron_jaws_near<<<grid, threads, 0, s>>>(C);
                    break;
                case 14: k_photon_mlc<<<grid, threads, C.stage_tables ? photon_smem_bytes(C.nmed) : 0, s>>>(C); break;
                case 15:
                    k_electron_mlc<<<grid, threads, 0, s>>>(C);
                    k_electron_mlc_near<<<grid, threads, 0, s>>>(C);
                    break;
                case ST_PHOTON: k_photon<<<grid, threads, C.stage_tables ? photon_smem_bytes(C.nmed) : 0, s>>>(C); break;
                case ST_COMPTON: k_interact<ST_COMPTON><<<grid, threads, 0, s>>>(C); break;
                case ST_PHOTO: k_interact<ST_PHOTO><<<grid, threads, 0, s>>>(C); break;
                case ST_RAYLEIGH: k_interact<ST_RAYLEIGH><<<grid, threads, 0, s>>>(C); break;
                case ST_PAIR: k_interact<ST_PAIR><<<grid, threads, 0, s>>>(C); break;
                case ST_ELECTRON: k_electron<<<grid, threads, 0, s>>>(C); break;
                case ST_MOLLER: k_interact<ST_MOLLER><<<grid, threads, 0, s>>>(C); break;
                case ST_BREMS: k_interact<ST_BREMS><<<grid, threads, 0, s>>>(C); break;
                case ST_BHABHA: k_interact<ST_BHABHA><<<grid, threads, 0, s>>>(C); break;
                default: k_interact<ST_ANNIH><<<grid, threads, 0, s>>>(C); break;
                }
                CK(cudaEventRecord(evs[2 * k + 1], s), "event");
            }
            CK(cudaStreamSynchronize(s), "timed sync");
            for (int k = 0; k < 15; k++) {
                float tk = 0.0f;
                cudaEventElapsedTime(&tk, evs[2 * k], evs[2 * k + 1]);
                acc[slot[k]] += tk;
                nl[slot[k]]++;
            }
        }
        CK(cudaEventRecord(e->ev1, e->stream), "event");
        for (auto &ev : evs) cudaEventDestroy(ev);
        for (int k = 0; k < 16; k++) { e->last.stage_ms[k] = acc[k]; e->last.stage_launches[k] = nl[k]; }
    } else {
        // Plain form: host-driven, one kernel per event type, synchronise and
        // read the queue counters back after every launch (CUDA_EGS.cu:226-365).
        CK(cudaEventRecord(e->ev0, e->stream), "event");
        uint32_t counts[GX_NQ];
        SchedState hsr;
        for (uint32_t w = 0; w < max_waves; w++) {
            k_plan<<<1, 1, 0, e->stream>>>(e->ctx, e->d_sched);
            CK(cudaMemcpyAsync(&hsr, e->d_sched, sizeof hsr, cudaMemcpyDeviceToHost, e->stream), "sched D2H");
            CK(cudaStreamSynchronize(e->stream), "plain sync");
            if (!hsr.pending) break;
            k_source<<<grid, threads, 0, e->stream>>>(e->ctx, e->d_sched);
            const int order[GX_NSTAGE] = {ST_PHOTON, ST_COMPTON, ST_PHOTO, ST_RAYLEIGH, ST_PAIR,
                                          ST_ELECTRON, ST_MOLLER, ST_BREMS, ST_BHABHA, ST_ANNIH};
            for (int k = 0; k < GX_NSTAGE; k++) {
                switch (order[k]) {
                case ST_PHOTON: k_plain<ST_PHOTON><<<grid, threads, 0, e->stream>>>(e->ctx); break;
                case ST_COMPTON: k_plain<ST_COMPTON><<<grid, threads, 0, e->stream>>>(e->ctx); break;
                case ST_PHOTO: k_plain<ST_PHOTO><<<grid, threads, 0, e->stream>>>(e->ctx); break;
                case ST_RAYLEIGH: k_plain<ST_RAYLEIGH><<<grid, threads, 0, e->stream>>>(e->ctx); break;
                case ST_PAIR: k_plain<ST_PAIR><<<grid, threads, 0, e->stream>>>(e->ctx); break;
                case ST_ELECTRON: k_plain<ST_ELECTRON><<<grid, threads, 0, e->stream>>>(e->ctx); break;
                case ST_MOLLER: k_plain<ST_MOLLER><<<grid, threads, 0, e->stream>>>(e->ctx); break;
                case ST_BREMS: k_plain<ST_BREMS><<<grid, threads, 0, e->stream>>>(e->ctx); break;
                case ST_BHABHA: k_plain<ST_BHABHA><<<grid, threads, 0, e->stream>>>(e->ctx); break;
                default: k_plain<ST_ANNIH><<<grid, threads, 0, e->stream>>>(e->ctx); break;
                }
                CK(cudaGetLastError(), "plain launch");
                CK(cudaMemcpyAsync(counts, e->d_qmeta, sizeof counts, cudaMemcpyDeviceToHost, e->stream), "counts D2H");
                CK(cudaStreamSynchronize(e->stream), "plain sync");
            }
        }
        CK(cudaEventRecord(e->ev1, e->stream), "event");
    }
    CK(cudaGetLastError(), "launch");
    if (launch_only && o.mode == GEGS_MODE_PERSISTENT) {
        e->in_flight = true;
        return GEGS_OK;
    }
    return run_finish(e);
}

// Fill the engine's run statistics from the device counters of a finished run
// (stats slots: processed per stage, photon and electron steps, then the steps
// in the jaws and the MLC per type) and turn the error bits into a status.
// Stage times and launch counts are left as the run set them.
static gegs_status finish_stats(gegs_engine *e, uint32_t errbits, const unsigned long long stats[16], uint32_t waves,
                                float ms)
{
    gegs_run_stats &R = e->last;
    for (int q = 0; q < GX_NSTAGE; q++) R.processed[q] = stats[q];
    R.photon_steps = stats[GX_NSTAGE];
    R.electron_steps = stats[GX_NSTAGE + 1];
    R.photon_steps_class[0] = stats[GX_NSTAGE + 2];
    R.photon_steps_class[1] = stats[GX_NSTAGE + 3];
    R.photon_steps_class[2] = R.photon_steps - stats[GX_NSTAGE + 2] - stats[GX_NSTAGE + 3];
    R.electron_steps_class[0] = stats[GX_NSTAGE + 4];
    R.electron_steps_class[1] = stats[GX_NSTAGE + 5];
    R.electron_steps_class[2] = R.electron_steps - stats[GX_NSTAGE + 4] - stats[GX_NSTAGE + 5];
    R.waves = waves;
    R.error_bits = errbits;
    R.device_ms = ms;
    if (errbits & GX_ERR_QUEUE_FULL) { e->err = "event queue overflow"; return GEGS_ERR_QUEUE_FULL; }
    if (errbits & GX_ERR_MODULE) { e->err = "particle in an unsupported module"; return GEGS_ERR_MODULE; }
    if (errbits & GX_ERR_SOURCE) { e->err = "history outside every field range"; return GEGS_ERR_SOURCE; }
    if (errbits & GX_ERR_STEP_BUDGET) { e->err = "wave budget exhausted"; return GEGS_ERR_STEP_BUDGET; }
    return GEGS_OK;
}

static gegs_status run_finish(gegs_engine *e)
{
    e->in_flight = false;
    CK(cudaStreamSynchronize(e->stream), "run sync");
    e->group.reset();
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e->ev0, e->ev1);
    uint32_t errbits = 0;
    unsigned long long stats[16];
    SchedState hsr;
    CK(cudaMemcpy(&errbits, e->d_err, sizeof errbits, cudaMemcpyDeviceToHost), "err D2H");
    CK(cudaMemcpy(stats, e->d_stats, sizeof stats, cudaMemcpyDeviceToHost), "stats D2H");
    CK(cudaMemcpy(&hsr, e->d_sched, sizeof hsr, cudaMemcpyDeviceToHost), "sched D2H");
    CK(cudaMemcpy(e->last.queue_peak, e->d_qmeta + 3 * GX_NQ, sizeof(uint32_t) * GX_NQ, cudaMemcpyDeviceToHost),
       "queue peaks D2H");
    for (int q = 0; q < GX_NQ; q++) e->last.queue_cap[q] = e->qcap[q];
    return finish_stats(e, errbits, stats, hsr.waves, ms);
}

extern "C" gegs_status gegs_run(gegs_engine *e, uint64_t hist_begin, uint64_t hist_end, const gegs_run_opts *opts)
{
    return run_impl(e, hist_begin, hist_end, opts, false);
}

extern "C" gegs_status gegs_launch(gegs_engine *e, uint64_t hist_begin, uint64_t hist_end, const gegs_run_opts *opts)
{
    gegs_run_opts o = {};
    if (opts) o = *opts;
    o.mode = GEGS_MODE_PERSISTENT;
    return run_impl(e, hist_begin, hist_end, &o, true);
}

extern "C" gegs_status gegs_wait(gegs_engine *e)
{
    if (!e) return GEGS_ERR_ARG;
    if (!e->in_flight) { e->err = "gegs_wait: no launched run"; return GEGS_ERR_ARG; }
    CK(cudaSetDevice(e->device), "cudaSetDevice");
    return run_finish(e);
}

extern "C" gegs_status gegs_set_field(gegs_engine *e, int32_t index, const gegs_field *F)
{
    if (!e || !F || !e->have_scene || index < 0 || index >= e->nfields) return GEGS_ERR_ARG;
    if (e->in_flight) { e->err = "a launched run has not been waited for (gegs_wait)"; return GEGS_ERR_ARG; }
    if (F->nrepeat < 0 || F->nrepeat > 255 || F->hist_end < F->hist_begin) {
        e->err = "gegs_set_field: bad history range or recycling count";
        return GEGS_ERR_ARG;
    }
    CK(cudaSetDevice(e->device), "cudaSetDevice");
    e->host_fields[(size_t)index] = *F;
    std::vector<float4> lines = jaw_edge_lines(e->host_fields.data(), e->nfields);
    // the device arrays keep their addresses: graphs built before stay valid
    CK(cudaMemcpyAsync(e->d_fields + index, F, sizeof(gegs_field), cudaMemcpyHostToDevice, e->stream), "field H2D");
    CK(cudaMemcpyAsync(e->d_jaw_lines, lines.data(), lines.size() * sizeof(float4), cudaMemcpyHostToDevice, e->stream),
       "jaw lines H2D");
    CK(cudaStreamSynchronize(e->stream), "field sync");
    return GEGS_OK;
}

extern "C" gegs_status gegs_set_stream(gegs_engine *e, void *cuda_stream)
{
    if (!e) return GEGS_ERR_ARG;
    if (e->in_flight) { e->err = "a launched run has not been waited for (gegs_wait)"; return GEGS_ERR_ARG; }
    CK(cudaSetDevice(e->device), "cudaSetDevice");
    CK(cudaStreamSynchronize(e->stream), "stream sync");      // work queued on the previous stream first
    e->stream = cuda_stream ? (cudaStream_t)cuda_stream : e->own_stream;
    return GEGS_OK;
}

extern "C" gegs_status gegs_launch_group(gegs_engine *const *engines, int32_t n, const uint64_t *hist_begin,
                                         const uint64_t *hist_end, const gegs_run_opts *opts)
{
    if (!engines || n < 1 || !hist_begin || !hist_end) return GEGS_ERR_ARG;
    for (int i = 0; i < n; i++) {
        if (!engines[i]) return GEGS_ERR_ARG;
        if (engines[i]->device != engines[0]->device) {
            engines[i]->err = "gegs_launch_group: the engines are on different devices";
            return GEGS_ERR_ARG;
        }
        for (int j = 0; j < i; j++)
            if (engines[j] == engines[i]) { engines[i]->err = "gegs_launch_group: an engine appears twice"; return GEGS_ERR_ARG; }
    }
    std::vector<RunSetup> R(n);
    for (int i = 0; i < n; i++) {
        gegs_run_opts o = {};
        if (opts) o = opts[i];
        o.mode = GEGS_MODE_PERSISTENT;
        gegs_status st = prepare_run(engines[i], hist_begin[i], hist_end[i], &o, R[i]);
        if (st != GEGS_OK) return st;
    }
    gegs_engine *e = engines[0];          // errors are reported on the first engine
    // the same engines in the same state as the last group launch reuse its graph
    std::vector<GroupKey> key(n);
    for (int i = 0; i < n; i++) key[i] = GroupKey{engines[i]->uid, engines[i]->ctx_gen, R[i].grid, R[i].threads};
    std::shared_ptr<GroupRun> grp = e->group_cache;
    bool reuse = grp && grp->key == key;
    for (int i = 1; reuse && i < n; i++) reuse = engines[i]->group_cache == grp;
    if (!reuse) {
        cudaGraph_t g;
        CK(cudaGraphCreate(&g, 0), "graph create");
        for (int i = 0; i < n; i++) {
            gegs_status st = add_wave_loop(engines[i], g, R[i].grid, R[i].threads, true);
            if (st != GEGS_OK) { cudaGraphDestroy(g); if (engines[i] != e) e->err = engines[i]->err; return st; }
        }
        grp = std::make_shared<GroupRun>();
        cudaError_t ce = cudaGraphInstantiate(&grp->exec, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) { e->err = std::string("group graph instantiate: ") + cudaGetErrorString(ce); return GEGS_ERR_CUDA; }
        grp->key = key;
        for (int i = 0; i < n; i++) engines[i]->group_cache = grp;
    }
    // the group runs on the first engine's stream once every engine's set-up is done
    cudaStream_t s = e->stream;
    for (int i = 1; i < n; i++) {
        CK(cudaEventRecord(engines[i]->ev_fork, engines[i]->stream), "event");
        CK(cudaStreamWaitEvent(s, engines[i]->ev_fork, 0), "stream wait");
    }
    for (int i = 0; i < n; i++) CK(cudaEventRecord(engines[i]->ev0, s), "event");
    CK(cudaGraphLaunch(grp->exec, s), "group graph launch");
    for (int i = 0; i < n; i++) {
        CK(cudaEventRecord(engines[i]->ev1, s), "event");
        if (i > 0) CK(cudaStreamWaitEvent(engines[i]->stream, engines[i]->ev1, 0), "stream wait");
        for (int k = 0; k < 16; k++) { engines[i]->last.stage_ms[k] = 0.0; engines[i]->last.stage_launches[k] = 0; }
        engines[i]->group = grp;
        engines[i]->in_flight = true;
    }
    return GEGS_OK;
}

extern "C" gegs_status gegs_get_tally(gegs_engine *e, int64_t *out, uint64_t nvox)
{
    if (!e || !out || nvox != e->nvox || !e->d_tally) return GEGS_ERR_ARG;
    CK(cudaMemcpyAsync(out, e->d_tally, nvox * 8, cudaMemcpyDeviceToHost, e->stream), "tally D2H");
    CK(cudaStreamSynchronize(e->stream), "tally sync");
    return GEGS_OK;
}

extern "C" gegs_status gegs_set_tally(gegs_engine *e, const int64_t *in, uint64_t nvox)
{
    if (!e || !in || nvox != e->nvox || !e->d_tally) return GEGS_ERR_ARG;
    if (e->in_flight) { e->err = "a launched run has not been waited for (gegs_wait)"; return GEGS_ERR_ARG; }
    CK(cudaMemcpyAsync(e->d_tally, in, nvox * 8, cudaMemcpyHostToDevice, e->stream), "tally H2D");
    CK(cudaStreamSynchronize(e->stream), "tally sync");
    return GEGS_OK;
}

extern "C" gegs_status gegs_probe_geometry(gegs_engine *e, uint32_t n, const gegs_probe_state *in, const float *t_in,
                                           uint32_t *far_region, float *far_t, gegs_probe_state *far_out, float *near_t)
{
    if (!e || !e->have_scene || !in || !t_in || !far_region || !far_t || !far_out || !near_t) return GEGS_ERR_ARG;
    if (e->in_flight) { e->err = "a launched run has not been waited for (gegs_wait)"; return GEGS_ERR_ARG; }
    if (n == 0) return GEGS_OK;
    CK(cudaSetDevice(e->device), "cudaSetDevice");
    const size_t ns = (size_t)n * sizeof(gegs_probe_state), nf = (size_t)n * 4;
    char *d = nullptr;
    CK(cudaMallocAsync(&d, 2 * ns + 4 * nf, e->stream), "probe buffers");
    gegs_probe_state *d_in = (gegs_probe_state *)d, *d_out = (gegs_probe_state *)(d + ns);
    float *d_t = (float *)(d + 2 * ns), *d_ft = d_t + n, *d_near = d_t + 2 * (size_t)n;
    uint32_t *d_reg = (uint32_t *)(d_t + 3 * (size_t)n);
    CK(cudaMemcpyAsync(d_in, in, ns, cudaMemcpyHostToDevice, e->stream), "probe H2D");
    CK(cudaMemcpyAsync(d_t, t_in, nf, cudaMemcpyHostToDevice, e->stream), "probe H2D");
    k_probe_geometry<<<(n + 127) / 128, 128, 0, e->stream>>>(e->ctx, n, d_in, d_t, d_reg, d_ft, d_out, d_near);
    CK(cudaGetLastError(), "probe kernel");
    CK(cudaMemcpyAsync(far_region, d_reg, nf, cudaMemcpyDeviceToHost, e->stream), "probe D2H");
    CK(cudaMemcpyAsync(far_t, d_ft, nf, cudaMemcpyDeviceToHost, e->stream), "probe D2H");
    CK(cudaMemcpyAsync(far_out, d_out, ns, cudaMemcpyDeviceToHost, e->stream), "probe D2H");
    CK(cudaMemcpyAsync(near_t, d_near, nf, cudaMemcpyDeviceToHost, e->stream), "probe D2H");
    cudaFreeAsync(d, e->stream);
    CK(cudaStreamSynchronize(e->stream), "probe sync");
    return GEGS_OK;
}

extern "C" gegs_status gegs_get_dose(gegs_engine *e, const float *voxel_mass, double dose_unit, double *out, uint64_t nvox)
{
    if (!e || !out || !voxel_mass || nvox != e->nvox || !e->d_tally) return GEGS_ERR_ARG;
    float *d_mass = nullptr;
    double *d_out = nullptr;
    CK(cudaMallocAsync(&d_mass, nvox * 4, e->stream), "mass");
    CK(cudaMallocAsync(&d_out, nvox * 8, e->stream), "dose");
    CK(cudaMemcpyAsync(d_mass, voxel_mass, nvox * 4, cudaMemcpyHostToDevice, e->stream), "mass H2D");
    k_dose<<<e->nsm * 4, 256, 0, e->stream>>>(e->d_tally, d_mass, dose_unit, d_out, nvox);
    CK(cudaGetLastError(), "dose kernel");
    CK(cudaMemcpyAsync(out, d_out, nvox * 8, cudaMemcpyDeviceToHost, e->stream), "dose D2H");
    cudaFreeAsync(d_mass, e->stream);
    cudaFreeAsync(d_out, e->stream);
    CK(cudaStreamSynchronize(e->stream), "dose sync");
    return GEGS_OK;
}

// ---- batch statistics (CUDA_EGS.cu:817-876, on the device) ------------------
extern "C" gegs_status gegs_stat_begin(gegs_engine *e)
{
    if (!e || !e->d_tally) return GEGS_ERR_ARG;
    if (e->in_flight) { e->err = "a launched run has not been waited for (gegs_wait)"; return GEGS_ERR_ARG; }
    CK(cudaSetDevice(e->device), "cudaSetDevice");
    if (e->stat_nvox != e->nvox) {
        CK(realloc_dev(&e->d_stat_s1, (size_t)e->nvox), "batch statistics");
        CK(realloc_dev(&e->d_stat_s2, (size_t)e->nvox), "batch statistics");
        CK(realloc_dev(&e->d_stat_snap, (size_t)e->nvox), "batch statistics");
        e->stat_nvox = e->nvox;
    }
    CK(cudaMemsetAsync(e->d_stat_s1, 0, e->nvox * sizeof(double), e->stream), "stat reset");
    CK(cudaMemsetAsync(e->d_stat_s2, 0, e->nvox * sizeof(double), e->stream), "stat reset");
    CK(cudaMemcpyAsync(e->d_stat_snap, e->d_tally, e->nvox * 8, cudaMemcpyDeviceToDevice, e->stream), "stat snapshot");
    CK(cudaStreamSynchronize(e->stream), "stat sync");
    e->stat_batches = 0;
    return GEGS_OK;
}

extern "C" gegs_status gegs_stat_fold(gegs_engine *e)
{
    if (!e || !e->d_stat_s1 || e->stat_nvox != e->nvox) { if (e) e->err = "gegs_stat_fold: no gegs_stat_begin"; return GEGS_ERR_ARG; }
    if (e->in_flight) { e->err = "a launched run has not been waited for (gegs_wait)"; return GEGS_ERR_ARG; }
    CK(cudaSetDevice(e->device), "cudaSetDevice");
    k_stat_fold<<<e->nsm * 8, 256, 0, e->stream>>>(e->d_tally, e->d_stat_snap, e->d_stat_s1, e->d_stat_s2, e->nvox);
    CK(cudaGetLastError(), "stat fold");
    CK(cudaStreamSynchronize(e->stream), "stat sync");
    e->stat_batches++;
    return GEGS_OK;
}

extern "C" gegs_status gegs_stat_get(gegs_engine *e, double *mean, double *rel_se, uint64_t nvox, uint32_t *nbatch)
{
    if (!e || !mean || !rel_se || !nbatch || nvox != e->nvox || !e->d_stat_s1 || e->stat_nvox != e->nvox)
        return GEGS_ERR_ARG;
    if (e->stat_batches < 2) { e->err = "gegs_stat_get: at least two folded batches are needed"; return GEGS_ERR_ARG; }
    CK(cudaSetDevice(e->device), "cudaSetDevice");
    double *d_mean = nullptr, *d_rel = nullptr;
    CK(cudaMallocAsync(&d_mean, nvox * 8, e->stream), "stat output");
    CK(cudaMallocAsync(&d_rel, nvox * 8, e->stream), "stat output");
    k_stat_final<<<e->nsm * 8, 256, 0, e->stream>>>(e->d_stat_s1, e->d_stat_s2, (double)e->stat_batches, d_mean, d_rel,
                                                   nvox);
    CK(cudaGetLastError(), "stat final");
    CK(cudaMemcpyAsync(mean, d_mean, nvox * 8, cudaMemcpyDeviceToHost, e->stream), "stat D2H");
    CK(cudaMemcpyAsync(rel_se, d_rel, nvox * 8, cudaMemcpyDeviceToHost, e->stream), "stat D2H");
    cudaFreeAsync(d_mean, e->stream);
    cudaFreeAsync(d_rel, e->stream);
    CK(cudaStreamSynchronize(e->stream), "stat sync");
    *nbatch = e->stat_batches;
    return GEGS_OK;
}

extern "C" gegs_status gegs_set_timeline(gegs_engine *e, uint32_t max_waves)
{
    if (!e) return GEGS_ERR_ARG;
    if (e->in_flight) { e->err = "a launched run has not been waited for (gegs_wait)"; return GEGS_ERR_ARG; }
    CK(cudaSetDevice(e->device), "cudaSetDevice");
    cudaFree(e->d_timeline);
    e->d_timeline = nullptr;
    e->timeline_waves = 0;
    if (max_waves) {
        CK(cudaMalloc(&e->d_timeline, (size_t)max_waves * GX_TL_KERNELS * 2 * sizeof(unsigned long long)), "timeline");
        e->timeline_waves = max_waves;
    }
    e->ctx.timeline = e->d_timeline;
    e->ctx.timeline_waves = e->timeline_waves;
    e->ctx_gen++;
    return GEGS_OK;
}

extern "C" gegs_status gegs_get_timeline(gegs_engine *e, uint64_t *out, uint32_t max_waves)
{
    if (!e || !out || !e->d_timeline) return GEGS_ERR_ARG;
    uint32_t m = max_waves < e->timeline_waves ? max_waves : e->timeline_waves;
    CK(cudaMemcpy(out, e->d_timeline, (size_t)m * GX_TL_KERNELS * 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost),
       "timeline D2H");
    return GEGS_OK;
}

extern "C" gegs_status gegs_set_trace(gegs_engine *e, uint32_t capacity)
{
    if (!e) return GEGS_ERR_ARG;
    CK(cudaSetDevice(e->device), "cudaSetDevice");
    cudaFree(e->d_trace);
    e->d_trace = nullptr;
    if (!e->d_trace_n) CK(cudaMalloc(&e->d_trace_n, sizeof(uint32_t)), "trace counter");
    CK(cudaMemset(e->d_trace_n, 0, sizeof(uint32_t)), "trace counter reset");
    if (capacity) CK(cudaMalloc(&e->d_trace, (size_t)capacity * sizeof(TraceRec)), "trace buffer");
    e->trace_cap = capacity;
    e->ctx.trace = e->d_trace;
    e->ctx.trace_n = e->d_trace_n;
    e->ctx.trace_cap = capacity;
    e->ctx_gen++;
    return GEGS_OK;
}

extern "C" gegs_status gegs_get_trace(gegs_engine *e, void *out, uint32_t capacity, uint32_t *n)
{
    if (!e || !n || !e->d_trace_n) return GEGS_ERR_ARG;
    uint32_t cnt = 0;
    CK(cudaMemcpy(&cnt, e->d_trace_n, sizeof cnt, cudaMemcpyDeviceToHost), "trace count");
    *n = cnt;
    uint32_t m = cnt < capacity ? cnt : capacity;
    if (m > e->trace_cap) m = e->trace_cap;
    if (m && out) CK(cudaMemcpy(out, e->d_trace, (size_t)m * sizeof(TraceRec), cudaMemcpyDeviceToHost), "trace D2H");
    CK(cudaMemset(e->d_trace_n, 0, sizeof(uint32_t)), "trace counter reset");
    return GEGS_OK;
}

extern "C" gegs_status gegs_get_stats(gegs_engine *e, gegs_run_stats *out)
{
    if (!e || !out) return GEGS_ERR_ARG;
    *out = e->last;
    return GEGS_OK;
}

extern "C" gegs_status gegs_tally_device_ptr(gegs_engine *e, void **out)
{
    if (!e || !out || !e->d_tally) return GEGS_ERR_ARG;
    *out = e->d_tally;
    return GEGS_OK;
}

// ---------------------------------------------------------------------------
// gegs_run_noalloc: the wave loop with every piece of scratch memory (queue
// counters, scheduler state, error word, counters, the 14 event queues and the
// electron continuation state) carved from one fixed device array, so that a
// run allocates nothing.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t noalloc_align(size_t x) { return (x + 255u) & ~(size_t)255u; }

// Upper bound of the carve-out at GEGS_NOALLOC_MAX_BATCH: every queue holds
// its capacity factor times the batch plus 4096 spare slots, each electron
// continuation queue as many step-state records.
constexpr size_t kNoallocBytes =
    noalloc_align(sizeof(uint32_t) * 3 * GX_NQ) + noalloc_align(sizeof(SchedState)) +
    noalloc_align(sizeof(uint32_t)) + noalloc_align(sizeof(unsigned long long) * 16) +
    (cap_factor_sum() * GEGS_NOALLOC_MAX_BATCH + (size_t)GX_NQ * 4096u) * sizeof(Part) + (size_t)GX_NQ * 256u +
    (estate_factor_sum() * GEGS_NOALLOC_MAX_BATCH + GX_NESTATE * 4096u) * sizeof(EStatePk) + GX_NESTATE * 256u;

constexpr int kNoallocMaxDevices = 64;

}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

static std::mutex g_noalloc_mu;
static unsigned char *g_noalloc_ptr[kNoallocMaxDevices] = {};

// Device address of g_noalloc_scratch on `device` (the current device); looked
// up once per device. Host code must not use the symbol itself as a pointer.
static cudaError_t noalloc_scratch(int device, unsigned char **out)
{
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
        void *p = nullptr;
        cudaError_t c = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (c != cudaSuccess) return c;
        g_noalloc_ptr[device] = (unsigned char *)p;
    }
    *out = g_noalloc_ptr[device];
    return cudaSuccess;
}

extern "C" gegs_status gegs_run_noalloc(gegs_engine *e, uint64_t hist_begin, uint64_t hist_end, uint32_t batch)
{
    if (!e) return GEGS_ERR_ARG;
    if (!e->have_scene || hist_end < hist_begin) { e->err = "gegs_run_noalloc: no scene, or hist_end < hist_begin"; return GEGS_ERR_ARG; }
    // a launched run still queued on the engine's stream owns the events and the run statistics
    if (e->in_flight) { e->err = "a launched run has not been waited for (gegs_wait)"; return GEGS_ERR_ARG; }
    if (batch == 0) batch = GEGS_NOALLOC_MAX_BATCH;
    if (batch > GEGS_NOALLOC_MAX_BATCH) {
        char buf[160];
        snprintf(buf, sizeof buf, "gegs_run_noalloc: batch %u exceeds the fixed scratch limit of %u particles "
                 "(GEGS_NOALLOC_MAX_BATCH)", batch, GEGS_NOALLOC_MAX_BATCH);
        e->err = buf;
        return GEGS_ERR_ARG;
    }
    if (e->device < 0 || e->device >= kNoallocMaxDevices) { e->err = "gegs_run_noalloc: device index out of range"; return GEGS_ERR_ARG; }
    CK(cudaSetDevice(e->device), "cudaSetDevice");
    unsigned char *base = nullptr;
    CK(noalloc_scratch(e->device, &base), "gegs_run_noalloc: cudaGetSymbolAddress of the scratch array");

    // carve the array
    size_t off = 0;
    auto take = [&](size_t bytes) { unsigned char *p = base + off; off += noalloc_align(bytes); return p; };
    uint32_t *qmeta = (uint32_t *)take(sizeof(uint32_t) * 3 * GX_NQ);
    SchedState *sched = (SchedState *)take(sizeof(SchedState));
    uint32_t *err = (uint32_t *)take(sizeof(uint32_t));
    unsigned long long *stats = (unsigned long long *)take(sizeof(unsigned long long) * 16);
    const size_t zero_bytes = off;   // counters, scheduler, error word and stats start at zero
    DevCtx c = e->ctx;
    for (int q = 0; q < GX_NQ; q++) {
        uint32_t cap = (uint32_t)(kCapFactor[q] * (float)batch) + 4096u;
        c.q.cap[q] = cap;
        c.q.buf[q] = (Part *)take((size_t)cap * sizeof(Part));
    }
    for (int k = 0; k < GX_NESTATE; k++)
        c.q.estate[k] = (EStatePk *)take((size_t)c.q.cap[GX_Q_ECONT + k] * sizeof(EStatePk));
    if (off > kNoallocBytes) { e->err = "gegs_run_noalloc: scratch layout exceeds the array"; return GEGS_ERR_ARG; }
    c.q.count = qmeta;
    c.q.head = qmeta + GX_NQ;
    c.q.done = qmeta + 2 * GX_NQ;
    c.q.peak = nullptr;
    c.err = err;
    c.stats = stats;
    c.wave = &sched->waves;
    c.budget_shift = &sched->budget_shift;
    c.photon_done = &sched->photon_done;
    c.electron_done = &sched->electron_done;
    c.overlap = 0u;                 // one kernel at a time
    c.pipelined = 0u;
    c.timeline = nullptr;
    c.timeline_waves = 0;
    c.trace = nullptr;
    c.trace_n = nullptr;
    c.trace_cap = 0;
    c.stage_tables = 0u;
    c.photon_budget = 16u;
    c.electron_budget = 8u;

    SchedState hs = {};
    hs.next = hist_begin;
    hs.end = hist_end;
    hs.batch = batch;
    hs.max_waves = 200000u;
    hs.refill_below = batch / 50u > 0u ? batch / 50u : 1u;
    hs.pending = 1u;                // k_plan_gated plans only while the run is pending
    cudaStream_t s = e->stream;
    CK(cudaMemsetAsync(base, 0, zero_bytes, s), "gegs_run_noalloc: scratch reset");
    CK(cudaMemcpyAsync(sched, &hs, sizeof hs, cudaMemcpyHostToDevice, s), "gegs_run_noalloc: scheduler H2D");

    const int threads = 256, grid = e->nsm * 4;
    CK(cudaEventRecord(e->ev0, s), "event");
    SchedState hsr = {};
    for (uint32_t w = 0; w < hs.max_waves;) {
        // a few waves between host checks; once a plan has ended the run, the
        // gated planner injects nothing and counts no wave, and the kernels of
        // the remaining waves find empty queues
        for (int k = 0; k < 8 && w < hs.max_waves; k++, w++) {
            k_plan_gated<<<1, 1, 0, s>>>(c, sched);
            k_source<<<grid, threads, 0, s>>>(c, sched);
            k_photon_jaws<<<grid, threads, 0, s>>>(c);
            k_photon_mlc<<<grid, threads, 0, s>>>(c);
            k_photon<<<grid, threads, 0, s>>>(c);
            k_interact<ST_COMPTON><<<grid, threads, 0, s>>>(c);
            k_interact<ST_PHOTO><<<grid, threads, 0, s>>>(c);
            k_interact<ST_RAYLEIGH><<<grid, threads, 0, s>>>(c);
            k_interact<ST_PAIR><<<grid, threads, 0, s>>>(c);
            k_electron_jaws<<<grid, threads, 0, s>>>(c);
            k_electron_jaws_near<<<grid, threads, 0, s>>>(c);
            k_electron_mlc<<<grid, threads, 0, s>>>(c);
            k_electron_mlc_near<<<grid, threads, 0, s>>>(c);
            k_electron<<<grid, threads, 0, s>>>(c);
            k_interact<ST_MOLLER><<<grid, threads, 0, s>>>(c);
            k_interact<ST_BREMS><<<grid, threads, 0, s>>>(c);
            k_interact<ST_BHABHA><<<grid, threads, 0, s>>>(c);
            k_interact<ST_ANNIH><<<grid, threads, 0, s>>>(c);
        }
        CK(cudaGetLastError(), "gegs_run_noalloc: launch");
        CK(cudaMemcpyAsync(&hsr, sched, sizeof hsr, cudaMemcpyDeviceToHost, s), "gegs_run_noalloc: scheduler D2H");
        CK(cudaStreamSynchronize(s), "gegs_run_noalloc: sync");
        if (!hsr.pending) break;
    }
    CK(cudaEventRecord(e->ev1, s), "event");
    uint32_t errbits = 0;
    unsigned long long st[16];
    CK(cudaMemcpyAsync(&errbits, err, sizeof errbits, cudaMemcpyDeviceToHost, s), "gegs_run_noalloc: err D2H");
    CK(cudaMemcpyAsync(st, stats, sizeof st, cudaMemcpyDeviceToHost, s), "gegs_run_noalloc: stats D2H");
    CK(cudaStreamSynchronize(s), "gegs_run_noalloc: sync");
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e->ev0, e->ev1);
    e->last = gegs_run_stats{};
    gegs_status fs = finish_stats(e, errbits, st, hsr.waves, ms);
    if (fs != GEGS_OK) return fs;
    if (hsr.pending) { e->err = "wave budget exhausted"; return GEGS_ERR_STEP_BUDGET; }
    return GEGS_OK;
}

// ---------------------------------------------------------------------------
// beamlet weights and the gradient replay
// ---------------------------------------------------------------------------
extern "C" gegs_status gegs_set_beamlet_weights(gegs_engine *e, const float *w, uint32_t n)
{
    if (!e || !e->have_scene) return GEGS_ERR_ARG;
    if (n != e->nbeamlets || (n && !w)) {
        e->err = "gegs_set_beamlet_weights: the count must equal nfields * bl_nx * bl_ny of the scene";
        return GEGS_ERR_ARG;
    }
    CK(cudaSetDevice(e->device), "cudaSetDevice");
    if (n) CK(cudaMemcpyAsync(e->d_blw, w, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, e->stream), "weights H2D");
    CK(cudaStreamSynchronize(e->stream), "weights sync");
    if (e->ctx.bl_weight != e->d_blw) { e->ctx.bl_weight = n ? e->d_blw : nullptr; e->ctx_gen++; }
    return GEGS_OK;
}

extern "C" gegs_status gegs_backward(gegs_engine *e, uint64_t hist_begin, uint64_t hist_end, const double *voxel_grad,
                                     double *beamlet_grad, uint32_t n, const gegs_run_opts *opts)
{
    if (!e || !e->have_scene || !voxel_grad || !beamlet_grad) return GEGS_ERR_ARG;
    if (n != e->nbeamlets || n == 0) {
        e->err = "gegs_backward: the scene has no beamlet grid, or n differs from its beamlet count";
        return GEGS_ERR_ARG;
    }
    CK(cudaSetDevice(e->device), "cudaSetDevice");
    bool fresh = false;
    if (!e->d_gvm) { CK(cudaMalloc(&e->d_gvm, e->nvox * sizeof(double)), "voxel gradient"); fresh = true; }
    CK(cudaMemcpyAsync(e->d_gvm, voxel_grad, e->nvox * sizeof(double), cudaMemcpyHostToDevice, e->stream), "gvm H2D");
    CK(cudaMemsetAsync(e->d_grad, 0, (size_t)n * GX_GRAD_COPIES * sizeof(double), e->stream), "grad reset");
    // replay the histories with unit fluence weights, scoring into the gradient
    DevCtx saved = e->ctx;
    e->ctx.bl_weight = nullptr;
    e->ctx.gvm = e->d_gvm;
    e->ctx.grad = e->d_grad;
    if (fresh) e->ctx_gen++;
    gegs_run_opts o = {};
    if (opts) o = *opts;
    o.mode = GEGS_MODE_PERSISTENT;
    e->slot = 1;
    gegs_status st = gegs_run(e, hist_begin, hist_end, &o);
    e->slot = 0;
    DevCtx after = e->ctx;
    e->ctx = saved;
    e->ctx.q = after.q;                          // queue buffers may have been re-sized by the run
    e->ctx.photon_budget = after.photon_budget;
    e->ctx.electron_budget = after.electron_budget;
    if (fresh) e->ctx_gen++;
    if (st != GEGS_OK) return st;
    std::vector<double> g((size_t)n * GX_GRAD_COPIES);
    CK(cudaMemcpy(g.data(), e->d_grad, g.size() * sizeof(double), cudaMemcpyDeviceToHost), "grad D2H");
    for (uint32_t b = 0; b < n; b++) {
        double acc = 0.0;
        for (int k = 0; k < GX_GRAD_COPIES; k++) acc += g[(size_t)k * n + b];
        beamlet_grad[b] = acc;
    }
    return GEGS_OK;
}
