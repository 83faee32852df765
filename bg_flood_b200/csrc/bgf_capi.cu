// C-ABI of the flow-step library (include/bg_flood_b200.h): handle life cycle,
// BUQ-layout uploads/downloads, boundary segments, the single-step entry point
// that stands in for FlowGPU, and the device-resident time loop.
#include <cuda_runtime.h>
#include <float.h>
#include <math.h>
#include <stddef.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <unordered_map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/bg_flood_b200.h"
#include "bgf_amr.cuh"
#include "bgf_internal.h"

using namespace bgf;
namespace ex = bgf::exact;
namespace fa = bgf::fast;

static thread_local std::string g_last_error;

void bgf::set_last_error(const std::string& msg) { g_last_error = msg; }

#define BGF_CUDA(call)                                                                 \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess) {                                                       \
            g_last_error = std::string(#call) + ": " + cudaGetErrorString(e_);         \
            return BGF_ECUDA;                                                          \
        }                                                                              \
    } while (0)

struct HostSeg {
    int type;
    std::vector<double> t, wl;
    std::vector<int> blk[4];
};

// Per-step control block of a handle: both time slots, both dt-minimum slots and the
// device error word, laid out alike in device memory and in a page-locked host
// mirror, so that a flow step moves its inputs with one copy in and its results
// with one copy out.
struct StepCtl {
    TimeState t[2];
    unsigned long long dtmin[2];
    int err;
    int pad[3];
};
static_assert(sizeof(StepCtl) <= 256, "the host mirror is one 256-byte page-locked slot");

// Host side of a device ring of gauge samples (GaugeRingDev): the gauges' cells and
// scenarios, the ring, and how many samples the host has drained.
struct GaugeRing {
    int n = 0, cap = 0;
    int* d_cell = nullptr;
    int* d_scen = nullptr;
    void* d_vals = nullptr;
    double* d_time = nullptr;
    unsigned long long* d_count = nullptr;
    unsigned long long read = 0;  // samples drained so far
    int64_t lost = 0;             // samples overwritten before they were drained
};

struct bgf_handle {
    bgf_param P;
    int nblkmem = 0, nblk = 0, dbl = 0, dev = 0, fast = 0;
    int split = 0;           // split precision: FP32 deviations from per-block datums
    int iodbl = 0;           // field pointers at the boundary are double* (doubleprecision or split)
    std::vector<double> datum, zbd;  // split: datum per block slot, bed as given (double)
    void* d_datum = nullptr;
    size_t esz = 4;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    // host copies of the tables
    std::vector<int> active, level, nbr;  // nbr as [8][nblkmem]
    std::vector<double> bxo, byo;         // block origins (values of the state precision)
    std::vector<HostSeg> segs;
    std::vector<double> rain_t, rain_r;
    std::vector<RiverDev> rivers;          // rivers with a non-zero discharge area
    std::vector<double> riv_t, riv_q;     // their discharge series, one after the other
    RiverDev* d_rivers = nullptr;
    RainMapDev rmap = {};                 // gridded rain (val: device frames), or none
    bool has_rmap = false;
    double *d_riv_t = nullptr, *d_riv_q = nullptr;
    // device buffers
    int *d_active = nullptr, *d_level = nullptr, *d_nbr = nullptr, *d_bndseg = nullptr, *d_err = nullptr;
    void *d_zb = nullptr, *d_dzbdx = nullptr, *d_dzbdy = nullptr, *d_cf = nullptr;
    uint8_t* d_rainmask = nullptr;
    float* d_qmean = nullptr;
    SegDev* d_segs = nullptr;
    double *d_seg_t = nullptr, *d_seg_wl = nullptr, *d_rain_t = nullptr, *d_rain_r = nullptr;
    void *d_h[2] = {nullptr, nullptr}, *d_u[2] = {nullptr, nullptr}, *d_v[2] = {nullptr, nullptr};
    void *d_dh = nullptr, *d_dhu = nullptr, *d_dhv = nullptr;
    StepCtl* d_ctl = nullptr;  // d_time, d_dtmin and d_err point into it
    TimeState* d_time = nullptr;
    unsigned long long* d_dtmin = nullptr;
    double* d_scratch = nullptr;
    StepCtl* h_ctl = nullptr;  // pinned mirror of d_ctl (single flow steps)
    std::vector<adapt::TargetMapDev> tmaps;  // Targetlevel maps (device node values)
    uint8_t* d_cflags = nullptr;             // coarsen flags of the Targetlevel criterion
    TimeState* h_time = nullptr;  // pinned
    // pinned scalars: [0] dt-minimum seed (H2D), [1] device error word (D2H)
    unsigned long long* h_misc = nullptr;
    // the per-block device arrays of bgf_create live in one allocation
    void* d_slab = nullptr;
    int cur = 0, parity = 0;
    bool has_blocks = false, has_bed = false, has_state = false, has_cf = false, has_rainmask = false;
    int nseg_dev = 0, rain_n_dev = 0;
    int64_t launches = 0;
    // graph of two consecutive steps (parities p, p^1)
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    bool graph_valid = false;
    // graph of one bgf_flow_step per parity: time-slot upload, the step, result download
    cudaGraphExec_t step_graph[2] = {nullptr, nullptr};
    int step_graph_launches[2] = {0, 0};
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double last_run_ms = 0.0;
    int64_t last_run_launches = 0;
    // per-kernel timing of bgf_flow_step (CUDA events on the handle's stream)
    int profiling = 0;
    cudaEvent_t pev[3] = {nullptr, nullptr, nullptr};
    double flux_ms = 0.0, update_ms = 0.0;
    int64_t profiled_steps = 0;
    // pinned staging buffer for host <-> device copies of BUQ fields
    void* pinned = nullptr;
    size_t pinned_bytes = 0;
    // page-locked staging of table uploads (pool rebuilds): while tstage_on, uploads
    // go through it and are queued without a wait per copy
    // Two areas used in turn by consecutive rebuilds: a rebuild queued behind a run in
    // flight (bgf_pool_prepare) must not overwrite the bytes of the previous rebuild's
    // copies, which may still wait in the stream ahead of that run.
    unsigned char* tstage[2] = {nullptr, nullptr};
    size_t tstage_bytes[2] = {0, 0};
    size_t tstage_used = 0;
    int tstage_sel = 0;
    bool tstage_on = false;
    cudaEvent_t tstage_ev[2] = {nullptr, nullptr};  // recorded after each area's copies
    // device tile scratch for the layout kernels (pinned caller arrays)
    void* d_tiles = nullptr;
    size_t tiles_bytes = 0;
    // multi-level meshes: stage tiles with halos, pre-prolongation gradients, face
    // arrays, wet/dry prolongation decisions and the active-list rank of each block
    bool amr = false;
    int gen = 2;  // single-level stage kernels: 1 one cell per thread, 2 two cells per thread
    int minlev = 0, maxlev = 0;
    int steps_launches = 2;  // kernel launches per step
    int grid = 0;            // CTAs of the fused kernels (0: one per block)
    int ntab = 0;            // table entries uploaded (highest active block id + 1)
    size_t seg_cap = 0, ser_cap = 0;  // capacities of the segment buffers
    void* d_W[2][4] = {{nullptr, nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr, nullptr}};
    void* d_G0[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    void* d_F[8] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    uint8_t* d_pflag = nullptr;
    int* d_rank = nullptr;
    // multi-level meshes split their active blocks: the chain runs on blocks with a
    // side facing another level, the single-level kernels on the rest ("pure")
    int* d_active_chain = nullptr;
    int* d_active_pure = nullptr;
    uint8_t* d_nolead = nullptr;  // zeros: the chain's kernels do not write the time slot
    int nchain = 0, npure = 0;
    // refinement pass: bathymetry grid, block origins, flags, children
    float* d_dem = nullptr;
    int dem_nx = 0, dem_ny = 0;
    double dem_xo = 0, dem_yo = 0, dem_dx = 0;
    double *d_bxo = nullptr, *d_byo = nullptr;
    uint8_t* d_flags = nullptr;
    int* d_child = nullptr;
    int* d_quads = nullptr;  // coarsened quads of an adaptation pass, 4 ids each
    // device table work of bgf_adapt (bgf_adapt_dev.cu): 1 when the mesh allows it
    int adapt_mode = 1;
    int regular_nbx = 0;          // > 0: single-level mesh that is a full regular grid of blocks
    int regular_nby = 0;
    unsigned regular_magic = 0;   // multiply-high divisor of block ids by regular_nbx, or 0
    void* d_adapt = nullptr;      // scratch, carved into adapt::DevAdaptScratch
    int* d_agrids = nullptr;      // per-level block index grids
    long long agrids_cap = 0;
    // gauges: the device ring, and the drained samples on the host ([sample][gauge]
    // times and [sample][gauge][4] values h, zs, u, v; gauge_nhost gauges per sample)
    GaugeRing gauges;
    std::vector<double> gauge_t, gauge_v;
    int gauge_nhost = 0;
    int64_t gauge_lost = 0;
};

// ---------------------------------------------------------------- helpers

template <class T> static DevModel<T> dev_model(bgf_handle* h)
{
    DevModel<T> m;
    m.nblk = h->nblk;
    m.nblkmem = h->nblkmem;
    m.active = h->d_active;
    m.level = h->d_level;
    m.nbr = h->d_nbr;
    m.zb = (const T*)h->d_zb;
    m.dzbdx = (const T*)h->d_dzbdx;
    m.dzbdy = (const T*)h->d_dzbdy;
    m.cf = h->has_cf ? (const T*)h->d_cf : nullptr;
    m.rainmask = h->has_rainmask ? h->d_rainmask : nullptr;
    m.bndseg = h->d_bndseg;
    m.qmean = h->d_qmean;
    m.segs = h->d_segs;
    m.seg_t = h->d_seg_t;
    m.seg_wl = h->d_seg_wl;
    m.rain_t = h->d_rain_t;
    m.rain_r = h->d_rain_r;
    m.rmap = h->rmap;
    m.rivers = h->d_rivers;
    m.riv_t = h->d_riv_t;
    m.riv_q = h->d_riv_q;
    m.bxo = h->d_bxo;
    m.byo = h->d_byo;
    for (int k = 0; k < 2; k++) {
        m.h[k] = (T*)h->d_h[k];
        m.u[k] = (T*)h->d_u[k];
        m.v[k] = (T*)h->d_v[k];
    }
    m.dh = (T*)h->d_dh;
    m.dhu = (T*)h->d_dhu;
    m.dhv = (T*)h->d_dhv;
    m.time = h->d_time;
    m.dtmin = h->d_dtmin;
    m.err = h->d_err;
    m.scen = nullptr;
    m.sparams = nullptr;
    m.lead = nullptr;
    m.hmax = nullptr;
    m.checklev = 0;
    m.datum = h->split ? (const T*)h->d_datum : nullptr;
    m.gen = h->gen;
    m.regular_nbx = h->amr ? 0 : h->regular_nbx;
    m.regular_nby = h->regular_nby;
    m.regular_magic = h->regular_magic;
    return m;
}

template <class T> static AmrDev<T> amr_dev(bgf_handle* h)
{
    AmrDev<T> a;
    for (int s = 0; s < 2; s++)
        for (int k = 0; k < 4; k++) a.W[s][k] = (T*)h->d_W[s][k];
    for (int k = 0; k < 6; k++) a.G0[k] = (T*)h->d_G0[k];
    for (int k = 0; k < 8; k++) a.F[k] = (T*)h->d_F[k];
    a.zb = (T*)h->d_zb;
    a.dzbdx = (T*)h->d_dzbdx;
    a.dzbdy = (T*)h->d_dzbdy;
    a.pflag = h->d_pflag;
    a.rank = h->d_rank;
    a.wetdryfix = h->P.wetdryfix ? 1 : 0;
    return a;
}

// Whether a series' times are non-decreasing (a NaN makes it unsorted); such series
// are searched by bisection on the device.
static bool series_sorted(const std::vector<double>& t)
{
    for (size_t k = 1; k < t.size(); k++)
        if (!(t[k - 1] <= t[k])) return false;
    return true;
}

template <class T> static StepParams<T> step_params(const bgf_handle* h)
{
    const bgf_param& P = h->P;
    StepParams<T> p;
    p.g = (T)P.g;
    p.eps = (T)P.eps;
    p.CFL = (T)P.CFL;
    p.theta = (T)P.theta;
    p.delta0 = (T)P.delta;
    p.delta0_d = P.delta;
    p.epsi = std::nextafter((T)1.0, (T)2.0) - (T)1.0;
    p.epsface = (T)P.eps + p.epsi;
    // Coriolis factor of updateEVCPU (src/Advection.cu:187) for a Cartesian grid
    p.fc = (T)((double)std::sin((T)(P.lat * 3.14159265 / 180.0)) * 3.14159265 / (double)(T)21600.0);
    p.eps_d = P.eps;
    p.dtparam = P.dt;
    p.bndfiltertime = P.bndfiltertime;
    p.bndrelaxtime = P.bndrelaxtime;
    p.bndtaper = P.bndtaper;
    p.inittime = P.inittime;
    p.zsinit = P.zsinit;
    p.zsoffset = std::isnan(P.zsoffset) ? 0.0 : P.zsoffset;
    p.dtmin = P.dtmin;
    p.cf = (T)P.cf;
    p.frictionmodel = P.frictionmodel;
    p.forcemass = P.ForceMassConserve;
    p.has_cf = h->has_cf ? 1 : 0;
    p.has_rain = (h->rain_n_dev > 0 || h->has_rmap) ? 1 : 0;
    p.rain_map = h->has_rmap ? 1 : 0;
    p.nseg = h->nseg_dev;
    p.rain_n = h->rain_n_dev;
    p.rain_off = 0;
    p.rain_sorted = series_sorted(h->rain_t) ? 1 : 0;
    p.xo_d = std::isnan(P.xo) ? 0.0 : P.xo;
    p.yo_d = std::isnan(P.yo) ? 0.0 : P.yo;
    p.nriver = (int)h->rivers.size();
    p.riv_first = 0;
    return p;
}

// Makes the handle's device current.  A launch error that other code of this host
// thread left pending (a host program whose own launches go unchecked -- the
// reference's FlowGPU leaves "invalid configuration argument" pending after a step)
// is taken off first, so that the check after each of this library's launches
// reports this library's errors only.  A sticky error (a fault that ended the
// context) is not cleared by this and fails the call all the same.
static int set_device(bgf_handle* h)
{
    (void)cudaGetLastError();
    BGF_CUDA(cudaSetDevice(h->dev));
    return BGF_OK;
}

template <class T> static T epsi_of() { return std::nextafter((T)1.0, (T)2.0) - (T)1.0; }

static unsigned long long dt_init_bits(int dbl)
{
    if (dbl) {
        double v = 1.0 / epsi_of<double>();
        unsigned long long b;
        memcpy(&b, &v, 8);
        return b;
    }
    float v = 1.0f / epsi_of<float>();
    unsigned int b;
    memcpy(&b, &v, 4);
    return (unsigned long long)b;
}

static void free_graphs(bgf_handle* h)
{
    for (int k = 0; k < 2; k++) {
        if (h->graph[k]) {
            cudaGraphExecDestroy(h->graph[k]);
            h->graph[k] = nullptr;
        }
        if (h->step_graph[k]) {
            cudaGraphExecDestroy(h->step_graph[k]);
            h->step_graph[k] = nullptr;
        }
    }
    h->graph_valid = false;
}

// Reads a BUQ field of the caller's precision into a T vector.
template <class T> static void buq_to(const void* src, int dbl, size_t n, std::vector<T>& out)
{
    out.resize(n);
    if (dbl) for (size_t k = 0; k < n; k++) out[k] = (T)((const double*)src)[k];
    else for (size_t k = 0; k < n; k++) out[k] = (T)((const float*)src)[k];
}

// Pinned staging area of at least `bytes` (grown on demand, kept for the handle).
// Page-locked staging buffers are kept in a process-wide cache by power-of-two size
// class: handles come and go per scenario when serving, and cudaMallocHost /
// cudaFreeHost cost milliseconds each and synchronise the device; under load a
// cudaFreeHost was measured holding every CUDA call of the process for up to two
// seconds.  The cache holds at most 8 GB (only what has been used is kept).
static std::mutex g_stage_mu;
static std::vector<std::pair<size_t, void*>> g_stage_free;  // (bytes, buffer)
static size_t g_stage_cached = 0;

static void stage_release(void* p, size_t bytes)
{
    if (!p) return;
    std::lock_guard<std::mutex> lk(g_stage_mu);
    if (g_stage_cached + bytes > ((size_t)8 << 30)) {
        cudaFreeHost(p);
        return;
    }
    g_stage_free.push_back({bytes, p});
    g_stage_cached += bytes;
}

static void* stage_acquire(size_t bytes, size_t* got)
{
    size_t cls = 1 << 16;
    while (cls < bytes) cls <<= 1;
    {
        std::lock_guard<std::mutex> lk(g_stage_mu);
        for (size_t k = 0; k < g_stage_free.size(); k++)
            if (g_stage_free[k].first == cls) {
                void* p = g_stage_free[k].second;
                g_stage_free.erase(g_stage_free.begin() + k);
                g_stage_cached -= cls;
                *got = cls;
                return p;
            }
    }
    void* p = nullptr;
    if (cudaMallocHost(&p, cls) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    *got = cls;
    return p;
}

static void* staging(bgf_handle* h, size_t bytes)
{
    if (h->pinned_bytes < bytes) {
        stage_release(h->pinned, h->pinned_bytes);
        h->pinned = nullptr;
        h->pinned_bytes = 0;
        size_t got = 0;
        h->pinned = stage_acquire(bytes, &got);
        if (!h->pinned) return nullptr;
        h->pinned_bytes = got;
    }
    return h->pinned;
}

// Device buffers owned by a handle come from the stream-ordered allocator on the
// handle's stream (released to the device's memory pool without a device-wide
// synchronisation); an allocation is complete before it returns, so any stream may
// use it.
// Debug aid: with BGF_DEBUG_FILL set in the environment, every device array of a
// handle starts as all-ones bytes (a NaN in both precisions) instead of whatever the
// memory pool held, so that a read of a cell no kernel wrote shows up in the results.
static bool debug_fill()
{
    static const bool on = getenv("BGF_DEBUG_FILL") != nullptr;
    return on;
}

static cudaError_t dalloc(bgf_handle* h, void** p, size_t bytes)
{
    cudaError_t e = cudaMallocAsync(p, bytes, h->stream);
    if (e == cudaSuccess && debug_fill()) e = cudaMemsetAsync(*p, 0xff, bytes, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    return e;
}

static void dfree(bgf_handle* h, void* p)
{
    if (p) cudaFreeAsync(p, h->stream);
}

// Host <-> device copies and fills of a handle's arrays, issued on the handle's
// stream and complete when they return.  Handle streams are created non-blocking,
// so the synchronous cudaMemcpy / cudaMemset (legacy default stream) would not be
// ordered with the handle's kernels: a bed upload could still be landing, or a
// fill of the bed gradients could run after the kernels that compute them.
static cudaError_t copy_on(cudaStream_t st, void* dst, const void* src, size_t bytes, cudaMemcpyKind kind)
{
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, kind, st);
    return e == cudaSuccess ? cudaStreamSynchronize(st) : e;
}

// Host -> device upload of a table.  Normally an asynchronous copy from the
// caller's (pageable) array, which the driver stages before it returns.  While the
// handle's table staging is on (a pool rebuild), the bytes are first copied into the
// handle's page-locked staging area and the copy is queued without any wait: the
// area is not reused before the stream has passed the copies (staging is reset only
// on an idle stream, and a full area is replaced only after a synchronisation).
static cudaError_t upload(bgf_handle* h, void* dst, const void* src, size_t bytes)
{
    if (bytes == 0) return cudaSuccess;
    if (!h->tstage_on) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, h->stream);
    const int a = h->tstage_sel;
    size_t off = (h->tstage_used + 255) & ~(size_t)255;
    if (off + bytes > h->tstage_bytes[a]) {
        // a larger area: wait for every copy queued so far, then replace it
        cudaError_t e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) return e;
        stage_release(h->tstage[a], h->tstage_bytes[a]);
        size_t got = 0;
        h->tstage[a] = (unsigned char*)stage_acquire(std::max(std::max(2 * h->tstage_bytes[a], bytes), (size_t)4 << 20), &got);
        h->tstage_bytes[a] = h->tstage[a] ? got : 0;
        off = 0;
        if (!h->tstage[a]) return cudaErrorMemoryAllocation;
    }
    memcpy(h->tstage[a] + off, src, bytes);
    h->tstage_used = off + bytes;
    return cudaMemcpyAsync(dst, h->tstage[a] + off, bytes, cudaMemcpyHostToDevice, h->stream);
}

// Allocation of a table buffer during a rebuild.  While table staging is on, the
// buffer is stream-ordered without a wait: it is used only by copies and kernels
// queued later on the handle's stream, and the buffer it replaces is freed in the
// same stream order (a rebuild queued behind a run must not wait for that run).
static cudaError_t dalloc_table(bgf_handle* h, void** p, size_t bytes)
{
    if (!h->tstage_on) return dalloc(h, p, bytes);
    cudaError_t e = cudaMallocAsync(p, bytes, h->stream);
    if (e == cudaSuccess && debug_fill()) e = cudaMemsetAsync(*p, 0xff, bytes, h->stream);
    return e;
}

// Starts a staged rebuild in the area the previous rebuild did not use, once the
// copies last queued from that area have run (its event; normally long done).
static void staging_begin(bgf_handle* h)
{
    h->tstage_sel ^= 1;
    if (h->tstage_ev[h->tstage_sel]) cudaEventSynchronize(h->tstage_ev[h->tstage_sel]);
    h->tstage_used = 0;
    h->tstage_on = true;
}

// Ends a staged rebuild: marks the point in the stream after its copies.
static void staging_end(bgf_handle* h)
{
    h->tstage_on = false;
    cudaEvent_t& ev = h->tstage_ev[h->tstage_sel];
    if (!ev && cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
        ev = nullptr;
        cudaGetLastError();
        cudaStreamSynchronize(h->stream);  // no event: wait here instead
        return;
    }
    cudaEventRecord(ev, h->stream);
}

// copy_on for host -> device table uploads: queued without a wait while staging is on.
static cudaError_t upload_on(bgf_handle* h, void* dst, const void* src, size_t bytes)
{
    return h->tstage_on ? upload(h, dst, src, bytes) : copy_on(h->stream, dst, src, bytes, cudaMemcpyHostToDevice);
}

static cudaError_t fill_on(cudaStream_t st, void* p, int value, size_t bytes)
{
    cudaError_t e = cudaMemsetAsync(p, value, bytes, st);
    return e == cudaSuccess ? cudaStreamSynchronize(st) : e;
}

// ---------------------------------------------------------------- gauge rings

static void gauge_free(bgf_handle* h, GaugeRing& g)
{
    for (void* q : {(void*)g.d_cell, (void*)g.d_scen, g.d_vals, (void*)g.d_time, (void*)g.d_count}) dfree(h, q);
    g = GaugeRing();
}

// A ring of cap samples for the given cells (block slot * 256 + j * 16 + i) and, for
// pools, their scenarios; allocated on h's stream, counter at zero.
static int gauge_alloc(bgf_handle* h, GaugeRing& g, const std::vector<int>& cells, const std::vector<int>& scen,
                       int cap)
{
    gauge_free(h, g);
    const int n = (int)cells.size();
    if (n == 0) return BGF_OK;
    bool ok = dalloc(h, (void**)&g.d_cell, sizeof(int) * n) == cudaSuccess &&
              dalloc(h, &g.d_vals, (size_t)cap * n * 4 * h->esz) == cudaSuccess &&
              dalloc(h, (void**)&g.d_time, (size_t)cap * n * sizeof(double)) == cudaSuccess &&
              dalloc(h, (void**)&g.d_count, sizeof(unsigned long long)) == cudaSuccess;
    if (ok && !scen.empty()) ok = dalloc(h, (void**)&g.d_scen, sizeof(int) * n) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        gauge_free(h, g);
        g_last_error = "cudaMalloc failed (gauge ring)";
        return BGF_ENOMEM;
    }
    g.n = n;
    g.cap = cap;
    BGF_CUDA(copy_on(h->stream, g.d_cell, cells.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    if (!scen.empty()) BGF_CUDA(copy_on(h->stream, g.d_scen, scen.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    BGF_CUDA(fill_on(h->stream, g.d_count, 0, sizeof(unsigned long long)));
    return BGF_OK;
}

template <class T> static GaugeRingDev<T> gauge_dev(const GaugeRing& g)
{
    return GaugeRingDev<T>{g.d_cell, g.d_scen, g.n, g.cap, (T*)g.d_vals, g.d_time, g.d_count};
}

// Copies the samples written since the last drain (ordered after the work queued on
// h's stream) and hands each (sample row, gauge, time, values) to sink.  Samples
// overwritten before this drain are counted in g.lost.
template <class T, class Sink> static int gauge_drain_t(bgf_handle* h, GaugeRing& g, Sink sink)
{
    if (g.n == 0) return BGF_OK;
    unsigned long long count = 0;
    BGF_CUDA(copy_on(h->stream, &count, g.d_count, sizeof(count), cudaMemcpyDeviceToHost));
    if (count <= g.read) return BGF_OK;
    if (count - g.read > (unsigned long long)g.cap) {
        g.lost += (int64_t)(count - g.read - g.cap);
        g.read = count - g.cap;
    }
    const size_t rows = (size_t)(count - g.read);
    std::vector<T> v(rows * g.n * 4);
    std::vector<double> t(rows * g.n);
    size_t done = 0;
    while (done < rows) {
        // contiguous run of ring rows from row (read + done) % cap
        const size_t r0 = (size_t)((g.read + done) % g.cap);
        const size_t nr = std::min(rows - done, (size_t)g.cap - r0);
        BGF_CUDA(cudaMemcpyAsync(v.data() + done * g.n * 4, (const T*)g.d_vals + r0 * g.n * 4, nr * g.n * 4 * sizeof(T),
                                 cudaMemcpyDeviceToHost, h->stream));
        BGF_CUDA(cudaMemcpyAsync(t.data() + done * g.n, g.d_time + r0 * g.n, nr * g.n * sizeof(double),
                                 cudaMemcpyDeviceToHost, h->stream));
        done += nr;
    }
    BGF_CUDA(cudaStreamSynchronize(h->stream));
    for (size_t r = 0; r < rows; r++)
        for (int q = 0; q < g.n; q++) {
            const T* x = v.data() + (r * g.n + q) * 4;
            const double vals[4] = {(double)x[0], (double)x[1], (double)x[2], (double)x[3]};
            sink(r, q, t[r * g.n + q], vals);
        }
    g.read = count;
    return BGF_OK;
}

// Drains a handle's own ring into its host buffer.
static int gauge_drain_handle(bgf_handle* h)
{
    if (h->gauges.n == 0) return BGF_OK;
    const int n = h->gauges.n;
    auto sink = [&](size_t, int, double t, const double* v) {
        if (std::isnan(t)) return;  // a replayed step after the loop ended
        h->gauge_t.push_back(t);
        h->gauge_v.insert(h->gauge_v.end(), v, v + 4);
    };
    const int64_t lost0 = h->gauges.lost;
    const int rc = h->dbl ? gauge_drain_t<double>(h, h->gauges, sink) : gauge_drain_t<float>(h, h->gauges, sink);
    h->gauge_lost += h->gauges.lost - lost0;
    h->gauge_nhost = n;
    return rc;
}

// Page-locked host slots of 256 bytes for the per-step scalars of a handle (dt seed,
// error word, two time states), handed out from 64 KB slabs that live until exit:
// cudaMallocHost per handle would cost about a millisecond each time.
static std::mutex g_pinned_mu;
static std::vector<void*> g_pinned_free;

static void* pinned_slot_get()
{
    std::lock_guard<std::mutex> lk(g_pinned_mu);
    if (g_pinned_free.empty()) {
        char* slab = nullptr;
        if (cudaMallocHost((void**)&slab, 65536) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        for (int k = 255; k >= 0; k--) g_pinned_free.push_back(slab + 256 * k);
    }
    void* p = g_pinned_free.back();
    g_pinned_free.pop_back();
    memset(p, 0, 256);
    return p;
}

static void pinned_slot_put(void* p)
{
    std::lock_guard<std::mutex> lk(g_pinned_mu);
    g_pinned_free.push_back(p);
}

// Device tile scratch of at least `bytes` (grown on demand, kept for the handle).
static void* tile_scratch(bgf_handle* h, size_t bytes)
{
    if (h->tiles_bytes < bytes) {
        dfree(h, h->d_tiles);
        h->d_tiles = nullptr;
        h->tiles_bytes = 0;
        if (dalloc(h, &h->d_tiles, bytes) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        h->tiles_bytes = bytes;
    }
    return h->d_tiles;
}

// True when p is page-locked host memory (cudaMallocHost / cudaHostRegister):
// such arrays can be copied by DMA as they are.
static bool host_pinned(const void* p)
{
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// ---------------------------------------------------------------- C ABI
// (C linkage comes from the declarations in include/bg_flood_b200.h)


void bgf_param_default(bgf_param* p)
{
    memset(p, 0, sizeof(*p));
    p->g = 9.81;
    p->eps = 0.0001;
    p->dt = 0.0;
    p->CFL = 0.5;
    p->theta = 1.3;
    p->cf = 0.0001;
    p->dx = NAN;
    p->delta = NAN;
    p->xo = 0.0;
    p->yo = 0.0;
    p->lat = 0.0;
    p->zsinit = NAN;
    p->zsoffset = 0.0;
    p->bndtaper = 0.0;
    p->bndrelaxtime = 3600.0;
    p->bndfiltertime = 60.0;
    p->inittime = 0.0;
    p->dtmin = 0.0005;
    p->dtinit = -1;
    p->mask = 9999.0;
    p->engine = 1;
    p->frictionmodel = 0;
    p->ForceMassConserve = 0;
    p->wetdryfix = 1;
    p->conserveElevation = 0;
    p->doubleprecision = 0;
    p->minlevel = 0;
    p->maxlevel = 0;
    p->initlevel = 0;
    p->aoibnd = 0;
    p->rainbnd = 0;
    p->GPUDEVICE = 0;
    p->fastmath = 0;
    p->splitprecision = 0;
}

const char* bgf_strerror(int s)
{
    switch (s) {
        case BGF_OK: return "ok";
        case BGF_EINVAL: return "invalid argument or unsupported configuration";
        case BGF_ECUDA: return "CUDA runtime error";
        case BGF_ENOMEM: return "device allocation failed";
        case BGF_EDT_UNDERFLOW: return "time step fell below dtmin (model crash)";
        case BGF_ENAN: return "non-finite value in the state";
        case BGF_ESTATE: return "call out of order";
        case BGF_EBUDGET: return "request exceeds the memory budget";
        case BGF_ETIMEOUT: return "bounded wait gave up";
        case BGF_ENOKERNEL: return "CUDA kernels unavailable on this device";
    }
    return "unknown status";
}

const char* bgf_last_error(void) { return g_last_error.c_str(); }

int bgf_device_supported(int dev)
{
    // two attribute queries (cudaGetDeviceProperties takes milliseconds)
    int major = 0, minor = 0;
    if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return major == 10 && minor == 0;
}

int bgf_create(const bgf_param* p, int nblkmem, void* stream, bgf_handle** out)
{
    if (!p || !out || nblkmem <= 0) return BGF_EINVAL;
    if (p->engine != 1 && p->engine != 2) return BGF_EINVAL;
    if (p->conserveElevation) return BGF_EINVAL;
    if (!(p->delta > 0.0)) return BGF_EINVAL;
    *out = nullptr;
    bgf_handle* h = new bgf_handle();
    h->P = *p;
    h->nblkmem = nblkmem;
    h->dbl = p->doubleprecision ? 1 : 0;
    h->esz = h->dbl ? 8 : 4;
    h->split = (p->splitprecision && !h->dbl) ? 1 : 0;
    h->iodbl = (h->dbl || h->split) ? 1 : 0;
    h->dev = p->GPUDEVICE;
    int rc;
    if ((rc = set_device(h)) != BGF_OK) { delete h; return rc; }
    if (!bgf_device_supported(h->dev)) {
        g_last_error = "device is not sm_100 (the library is built for sm_100a)";
        delete h;
        return BGF_ENOKERNEL;
    }
    h->fast = p->fastmath ? 1 : 0;
    // kernel attributes (dynamic shared memory) are set once per device, precision
    // and arithmetic variant
    static std::mutex cfg_mu;
    static bool configured[64][2][2] = {};
    cudaError_t e = cudaSuccess;
    {
        std::lock_guard<std::mutex> lk(cfg_mu);
        bool& done = configured[h->dev & 63][h->dbl][h->fast];
        if (!done) {
            e = h->dbl ? (h->fast ? fa::configure_kernels<double>() : ex::configure_kernels<double>())
                       : (h->fast ? fa::configure_kernels<float>() : ex::configure_kernels<float>());
            if (e == cudaSuccess)
                e = h->dbl ? (h->fast ? fa::configure_amr_kernels<double>() : ex::configure_amr_kernels<double>())
                           : (h->fast ? fa::configure_amr_kernels<float>() : ex::configure_amr_kernels<float>());
            done = e == cudaSuccess;
        }
    }
    if (e != cudaSuccess) {
        g_last_error = std::string("configure kernels: ") + cudaGetErrorString(e);
        delete h;
        return BGF_ENOKERNEL;
    }
    if (stream) h->stream = (cudaStream_t)stream;
    else {
        if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) { delete h; return BGF_ECUDA; }
        h->own_stream = true;
    }
    size_t nb = (size_t)nblkmem;
    size_t es = h->esz;
    struct A { void** p; size_t bytes; } allocs[] = {
        {(void**)&h->d_active, nb * sizeof(int)},        {(void**)&h->d_level, nb * sizeof(int)},
        {(void**)&h->d_nbr, 8 * nb * sizeof(int)},       {(void**)&h->d_bndseg, 4 * nb * sizeof(int)},
        {(void**)&h->d_ctl, sizeof(StepCtl)},            {&h->d_zb, nb * 324 * es},
        {&h->d_dzbdx, nb * 324 * es},                    {&h->d_dzbdy, nb * 324 * es},
        {&h->d_cf, nb * 256 * es},                       {(void**)&h->d_rainmask, nb * 256},
        {(void**)&h->d_qmean, nb * 64 * sizeof(float)},  {&h->d_h[0], nb * 256 * es},
        {&h->d_h[1], nb * 256 * es},                     {&h->d_u[0], nb * 256 * es},
        {&h->d_u[1], nb * 256 * es},                     {&h->d_v[0], nb * 256 * es},
        {&h->d_v[1], nb * 256 * es},                     {&h->d_dh, nb * 256 * es},
        {&h->d_dhu, nb * 256 * es},                      {&h->d_dhv, nb * 256 * es},
        {(void**)&h->d_scratch, 8 * sizeof(double)},
        {(void**)&h->d_bxo, nb * sizeof(double)},        {(void**)&h->d_byo, nb * sizeof(double)},
        {(void**)&h->d_flags, nb},                       {(void**)&h->d_child, 3 * nb * sizeof(int)},
        {(void**)&h->d_cflags, nb},                      {(void**)&h->d_quads, nb * sizeof(int)},
        {&h->d_datum, nb * es},
    };
    // one device allocation carved into 256-byte aligned pieces: handles are created
    // and destroyed per scenario when serving, and each cudaMalloc / cudaFree costs
    size_t total = 0;
    for (auto& a : allocs) total += (a.bytes + 255) & ~(size_t)255;
    // stream-ordered allocation from the device's memory pool, which keeps all freed
    // memory for reuse until the process exits instead of returning it to the driver
    // at synchronisation points: a release unmaps device memory, which waits for the
    // running kernels and held every CUDA call of a serving process (other threads
    // creating and destroying scenario handles) for tens of milliseconds to a second
    static std::mutex pool_mu;
    static bool pool_set[64] = {};
    {
        std::lock_guard<std::mutex> lk(pool_mu);
        if (!pool_set[h->dev & 63]) {
            cudaMemPool_t mp;
            if (cudaDeviceGetDefaultMemPool(&mp, h->dev) == cudaSuccess) {
                uint64_t keep = ~(uint64_t)0;
                cudaMemPoolSetAttribute(mp, cudaMemPoolAttrReleaseThreshold, &keep);
            }
            cudaGetLastError();
            pool_set[h->dev & 63] = true;
        }
    }
    if (cudaMallocAsync(&h->d_slab, total, h->stream) != cudaSuccess) {
        cudaGetLastError();
        g_last_error = "cudaMalloc failed";
        bgf_destroy(h);
        return BGF_ENOMEM;
    }
    if (debug_fill()) cudaMemsetAsync(h->d_slab, 0xff, total, h->stream);
    {
        char* q = (char*)h->d_slab;
        for (auto& a : allocs) {
            *a.p = q;
            q += (a.bytes + 255) & ~(size_t)255;
        }
        h->d_time = h->d_ctl->t;
        h->d_dtmin = h->d_ctl->dtmin;
        h->d_err = &h->d_ctl->err;
    }
    cudaMemsetAsync(h->d_bndseg, 0xff, 4 * nb * sizeof(int), h->stream);
    cudaMemsetAsync(h->d_qmean, 0, nb * 64 * sizeof(float), h->stream);
    cudaMemsetAsync(h->d_err, 0, sizeof(int), h->stream);
    cudaMemsetAsync(h->d_dh, 0, nb * 256 * es, h->stream);
    cudaMemsetAsync(h->d_dhu, 0, nb * 256 * es, h->stream);
    cudaMemsetAsync(h->d_dhv, 0, nb * 256 * es, h->stream);
    cudaMemsetAsync(h->d_datum, 0, nb * es, h->stream);
    h->h_misc = (unsigned long long*)pinned_slot_get();
    if (!h->h_misc) {
        bgf_destroy(h);
        return BGF_ENOMEM;
    }
    h->h_time = (TimeState*)(h->h_misc + 2);  // two time states after the two scalars
    h->h_ctl = (StepCtl*)pinned_slot_get();
    if (!h->h_ctl) {
        bgf_destroy(h);
        return BGF_ENOMEM;
    }
    cudaEventCreate(&h->ev0);
    cudaEventCreate(&h->ev1);
    for (int k = 0; k < 3; k++) cudaEventCreate(&h->pev[k]);
    // the slab and its initial values are in place before any other stream uses them
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) {
        g_last_error = "bgf_create: stream synchronisation failed";
        bgf_destroy(h);
        return BGF_ECUDA;
    }
    *out = h;
    return BGF_OK;
}

static void free_amr(bgf_handle* h)
{
    for (auto& st : h->d_W)
        for (void*& p : st) { dfree(h, p); p = nullptr; }
    for (void*& p : h->d_G0) { dfree(h, p); p = nullptr; }
    for (void*& p : h->d_F) { dfree(h, p); p = nullptr; }
    dfree(h, h->d_pflag);
    dfree(h, h->d_rank);
    dfree(h, h->d_active_chain);
    dfree(h, h->d_active_pure);
    dfree(h, h->d_nolead);
    h->d_pflag = nullptr;
    h->d_rank = nullptr;
    h->d_active_chain = h->d_active_pure = nullptr;
    h->d_nolead = nullptr;
}

int bgf_destroy(bgf_handle* h)
{
    if (!h) return BGF_EINVAL;
    cudaSetDevice(h->dev);
    if (h->stream) cudaStreamSynchronize(h->stream);
    free_graphs(h);
    // the per-block arrays of bgf_create are pieces of d_slab (back to the memory pool in
    // stream order); the rest are own allocations
    void* ptrs[] = {h->d_slab, h->d_segs, h->d_seg_t, h->d_seg_wl, h->d_rain_t, h->d_rain_r, h->d_dem,
                    h->d_rivers, h->d_riv_t, h->d_riv_q, (void*)h->rmap.val, h->d_tiles, h->d_adapt,
                    (void*)h->d_agrids};
    if (h->stream) {
        for (void* p : ptrs) dfree(h, p);
        for (auto& g : h->tmaps) dfree(h, (void*)g.val);
    }
    h->tmaps.clear();
    if (h->stream) gauge_free(h, h->gauges);
    h->d_slab = nullptr;
    free_amr(h);
    if (h->h_misc) pinned_slot_put(h->h_misc);
    if (h->h_ctl) pinned_slot_put(h->h_ctl);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    for (int k = 0; k < 3; k++)
        if (h->pev[k]) cudaEventDestroy(h->pev[k]);
    stage_release(h->pinned, h->pinned_bytes);
    for (int k = 0; k < 2; k++) {
        stage_release(h->tstage[k], h->tstage_bytes[k]);
        if (h->tstage_ev[k]) cudaEventDestroy(h->tstage_ev[k]);
    }
    if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return BGF_OK;
}

static int rebuild_segments(bgf_handle* h);

// Buffers of the multi-level path, allocated the first time a mesh with more than
// one level is set.
static int alloc_amr(bgf_handle* h)
{
    if (h->d_rank) return BGF_OK;
    const size_t nb = (size_t)h->nblkmem, es = h->esz;
    bool ok = true;
    for (auto& st : h->d_W)
        for (void*& p : st) ok = ok && dalloc(h, &p, nb * 324 * es) == cudaSuccess;
    for (void*& p : h->d_G0) ok = ok && dalloc(h, &p, nb * 324 * es) == cudaSuccess;
    for (void*& p : h->d_F) ok = ok && dalloc(h, &p, nb * NFX * es) == cudaSuccess;
    ok = ok && dalloc(h, (void**)&h->d_pflag, nb * 64) == cudaSuccess;
    ok = ok && dalloc(h, (void**)&h->d_rank, nb * sizeof(int)) == cudaSuccess;
    ok = ok && dalloc(h, (void**)&h->d_active_chain, nb * sizeof(int)) == cudaSuccess;
    ok = ok && dalloc(h, (void**)&h->d_active_pure, nb * sizeof(int)) == cudaSuccess;
    ok = ok && dalloc(h, (void**)&h->d_nolead, nb) == cudaSuccess;
    if (!ok) {
        free_amr(h);
        g_last_error = "cudaMalloc failed (multi-level buffers)";
        return BGF_ENOMEM;
    }
    BGF_CUDA(cudaMemsetAsync(h->d_pflag, 0, nb * 64, h->stream));
    BGF_CUDA(cudaMemsetAsync(h->d_nolead, 0, nb, h->stream));
    return BGF_OK;
}

// Uploads the host tables (active, level, neighbours, origins), classifies the
// mesh as single- or multi-level and prepares the multi-level buffers.
static int upload_tables(bgf_handle* h)
{
    const int nb = h->nblkmem;
    int rc = set_device(h);
    if (rc) return rc;
    // only the slots up to the highest active id are uploaded (pools hand out low ids first)
    int nt = 0;
    for (int ibl = 0; ibl < h->nblk; ibl++) nt = std::max(nt, h->active[ibl] + 1);
    h->ntab = nt;
    // gauge cells name block slots of the previous mesh
    if (h->gauges.n) gauge_free(h, h->gauges);
    BGF_CUDA(upload(h, h->d_active, h->active.data(), sizeof(int) * h->nblk));
    BGF_CUDA(upload(h, h->d_level, h->level.data(), sizeof(int) * nt));
    for (int k = 0; k < 8; k++) BGF_CUDA(upload(h, h->d_nbr + (size_t)k * nb, h->nbr.data() + (size_t)k * nb, sizeof(int) * nt));
    BGF_CUDA(upload(h, h->d_bxo, h->bxo.data(), sizeof(double) * nt));
    BGF_CUDA(upload(h, h->d_byo, h->byo.data(), sizeof(double) * nt));
    // a mesh is multi-level when some active block has a neighbour on another level
    h->amr = false;
    h->minlev = h->maxlev = h->level[h->active[0]];
    for (int ibl = 0; ibl < h->nblk; ibl++) {
        int ib = h->active[ibl];
        h->minlev = std::min(h->minlev, h->level[ib]);
        h->maxlev = std::max(h->maxlev, h->level[ib]);
        for (int k = 0; k < 8; k++) h->amr = h->amr || h->level[h->nbr[(size_t)k * nb + ib]] != h->level[ib];
    }
    if (h->amr && h->split) {
        g_last_error = "split precision supports single-level meshes only";
        return BGF_EINVAL;
    }
    // a full regular grid of blocks in row-major ids: the two-cell kernels derive the
    // ids the tables hold instead of loading them
    h->regular_nbx = 0;
    h->regular_nby = 0;
    h->regular_magic = 0;
    if (!h->amr) {
        int nbx = 0;
        for (int k = 0; k < h->nblk && !nbx; k++)
            if (h->active[k] != k) break;
            else if (h->nbr[(size_t)2 * nb + k] == k) nbx = k + 1;
        bool ok = nbx > 0 && h->nblk % nbx == 0;
        const int nby = ok ? h->nblk / nbx : 0;
        for (int k = 0; ok && k < h->nblk; k++) {
            const int bx = k % nbx, by = k / nbx;
            const int want[4] = {bx > 0 ? k - 1 : k, bx < nbx - 1 ? k + 1 : k, by > 0 ? k - nbx : k,
                                 by < nby - 1 ? k + nbx : k};
            ok = h->active[k] == k;
            for (int q = 0; ok && q < 8; q++) ok = h->nbr[(size_t)q * nb + k] == want[q >> 1];
        }
        if (ok) {
            h->regular_nbx = nbx;
            h->regular_nby = nby;
            // block row by = ib / nbx as the high word of ib * ceil(2^32 / nbx), kept only if
            // it equals the quotient for every block id of this mesh
            h->regular_magic = 0;
            if (nbx > 1) {
                const unsigned mg = (unsigned)((((unsigned long long)1 << 32) + nbx - 1) / nbx);
                bool exact = true;
                for (int k = 0; exact && k < h->nblk; k++)
                    exact = (int)(((unsigned long long)(unsigned)k * mg) >> 32) == k / nbx;
                if (exact) h->regular_magic = mg;
            }
        }
    }
    if (h->amr) {
        rc = alloc_amr(h);
        if (rc) return rc;
        std::vector<int> rank(nt, 0);
        for (int ibl = 0; ibl < h->nblk; ibl++) rank[h->active[ibl]] = ibl;
        BGF_CUDA(upload(h, h->d_rank, rank.data(), sizeof(int) * nt));
        // chain: blocks with a side facing another level; pure: the rest, in active order
        std::vector<int> chain, pure;
        for (int ibl = 0; ibl < h->nblk; ibl++) {
            const int ib = h->active[ibl];
            bool cross = false;
            for (int k = 0; k < 8; k++) cross = cross || h->level[h->nbr[(size_t)k * nb + ib]] != h->level[ib];
            (cross ? chain : pure).push_back(ib);
        }
        h->nchain = (int)chain.size();
        h->npure = (int)pure.size();
        if (h->nchain) BGF_CUDA(upload(h, h->d_active_chain, chain.data(), sizeof(int) * h->nchain));
        if (h->npure) BGF_CUDA(upload(h, h->d_active_pure, pure.data(), sizeof(int) * h->npure));
    }
    // (staged uploads need no wait: their bytes are in the staging area already)
    if (!h->tstage_on) BGF_CUDA(cudaStreamSynchronize(h->stream));
    h->has_blocks = true;
    free_graphs(h);
    return BGF_OK;
}

int bgf_set_blocks(bgf_handle* h, const bgf_blockp* b)
{
    if (!h || !b || b->nblk <= 0 || b->nblk > h->nblkmem || !b->active || !b->level) return BGF_EINVAL;
    const int* tabs[8] = {b->LeftBot, b->LeftTop, b->RightBot, b->RightTop, b->BotLeft, b->BotRight, b->TopLeft, b->TopRight};
    for (int k = 0; k < 8; k++)
        if (!tabs[k]) return BGF_EINVAL;
    int nb = h->nblkmem;
    for (int ibl = 0; ibl < b->nblk; ibl++) {
        int ib = b->active[ibl];
        if (ib < 0 || ib >= nb) return BGF_EINVAL;
        for (int k = 0; k < 8; k++) {
            int q = tabs[k][ib];
            if (q < 0 || q >= nb) return BGF_EINVAL;
        }
    }
    h->nblk = b->nblk;
    h->active.assign(b->active, b->active + b->nblk);
    h->level.assign(b->level, b->level + nb);
    h->nbr.assign((size_t)8 * nb, 0);
    for (int k = 0; k < 8; k++)
        for (int ib = 0; ib < nb; ib++) h->nbr[(size_t)k * nb + ib] = tabs[k][ib];
    h->bxo.assign(nb, 0.0);
    h->byo.assign(nb, 0.0);
    if (b->xo && b->yo)
        for (int ib = 0; ib < nb; ib++) {
            h->bxo[ib] = h->iodbl ? ((const double*)b->xo)[ib] : (double)((const float*)b->xo)[ib];
            h->byo[ib] = h->iodbl ? ((const double*)b->yo)[ib] : (double)((const float*)b->yo)[ib];
        }
    int rc = upload_tables(h);
    if (rc) return rc;
    return rebuild_segments(h);
}

template <class T>
static int set_bed_t(bgf_handle* h, const void* zb, const void* dzbdx, const void* dzbdy, const void* cf,
                     const int* activeCell)
{
    size_t nb = h->nblkmem;
    std::vector<T> z;
    buq_to<T>(zb, h->iodbl, nb * 324, z);
    if (h->split) {
        // datum per block: the mean depth below zero of its interior, in whole metres
        h->zbd.assign((const double*)zb, (const double*)zb + nb * 324);
        h->datum.assign(nb, 0.0);
        std::vector<T> dt(nb, (T)0);
        for (int ibl = 0; ibl < h->nblk; ibl++) {
            const size_t ib = h->active[ibl];
            double sum = 0.0;
            for (int j = 0; j < 16; j++)
                for (int i = 0; i < 16; i++) sum += h->zbd[ib * 324 + (i + 1) + (j + 1) * 18];
            h->datum[ib] = std::max(0.0, std::round(-sum / 256.0));
            dt[ib] = (T)h->datum[ib];
        }
        BGF_CUDA(copy_on(h->stream, h->d_datum, dt.data(), nb * sizeof(T), cudaMemcpyHostToDevice));
    }
    BGF_CUDA(copy_on(h->stream, h->d_zb, z.data(), nb * 324 * sizeof(T), cudaMemcpyHostToDevice));
    if (dzbdx && dzbdy) {
        // the caller's bed halo and gradients are taken as they are
        std::vector<T> gx, gy;
        buq_to<T>(dzbdx, h->iodbl, nb * 324, gx);
        buq_to<T>(dzbdy, h->iodbl, nb * 324, gy);
        BGF_CUDA(copy_on(h->stream, h->d_dzbdx, gx.data(), nb * 324 * sizeof(T), cudaMemcpyHostToDevice));
        BGF_CUDA(copy_on(h->stream, h->d_dzbdy, gy.data(), nb * 324 * sizeof(T), cudaMemcpyHostToDevice));
    } else {
        // bed halo and bed gradients from the interior, as the reference prepares
        // them at initialisation (src/InitialConditions.cu:140-144)
        BGF_CUDA(fill_on(h->stream, h->d_dzbdx, 0, nb * 324 * sizeof(T)));
        BGF_CUDA(fill_on(h->stream, h->d_dzbdy, 0, nb * 324 * sizeof(T)));
        DevModel<T> m = dev_model<T>(h);
        StepParams<T> p = step_params<T>(h);
        int n = h->fast ? fa::launch_bed_init<T>(m, p, (T*)h->d_zb, (T*)h->d_dzbdx, (T*)h->d_dzbdy, h->stream)
                        : ex::launch_bed_init<T>(m, p, (T*)h->d_zb, (T*)h->d_dzbdx, (T*)h->d_dzbdy, h->stream);
        h->launches += n;
        BGF_CUDA(cudaGetLastError());
        BGF_CUDA(cudaStreamSynchronize(h->stream));
    }
    h->has_cf = cf != nullptr;
    if (cf) {
        std::vector<T> c(nb * 256);
        for (size_t ib = 0; ib < nb; ib++)
            for (int j = 0; j < 16; j++)
                for (int i = 0; i < 16; i++) {
                    size_t s = ib * 324 + (i + 1) + (j + 1) * 18;
                    c[ib * 256 + j * 16 + i] = h->iodbl ? (T)((const double*)cf)[s] : (T)((const float*)cf)[s];
                }
        BGF_CUDA(copy_on(h->stream, h->d_cf, c.data(), nb * 256 * sizeof(T), cudaMemcpyHostToDevice));
    }
    h->has_rainmask = activeCell != nullptr;
    if (activeCell) {
        std::vector<uint8_t> r(nb * 256);
        for (size_t ib = 0; ib < nb; ib++)
            for (int j = 0; j < 16; j++)
                for (int i = 0; i < 16; i++) r[ib * 256 + j * 16 + i] = (uint8_t)(activeCell[ib * 324 + (i + 1) + (j + 1) * 18] != 0);
        BGF_CUDA(copy_on(h->stream, h->d_rainmask, r.data(), nb * 256, cudaMemcpyHostToDevice));
    }
    h->has_bed = true;
    free_graphs(h);
    return BGF_OK;
}

int bgf_set_bed(bgf_handle* h, const void* zb, const void* dzbdx, const void* dzbdy, const void* cf,
                const int* activeCell)
{
    if (!h || !zb) return BGF_EINVAL;
    if (!h->has_blocks) return BGF_ESTATE;
    int rc = set_device(h);
    if (rc) return rc;
    return h->dbl ? set_bed_t<double>(h, zb, dzbdx, dzbdy, cf, activeCell)
                  : set_bed_t<float>(h, zb, dzbdx, dzbdy, cf, activeCell);
}

// Per-block side -> segment table.  A block belongs to one segment; each of its
// domain-edge sides is handled by that segment, in the segment order of
// FlowbndFlux (src/Boundary.cu:108-195).
static int rebuild_segments(bgf_handle* h)
{
    int nb = h->nblkmem;
    const int nt = h->ntab > 0 ? h->ntab : nb;
    std::vector<int> side(4 * (size_t)nt, -1);
    std::vector<SegDev> sd;
    std::vector<double> st, swl;
    for (size_t k = 0; k < h->segs.size(); k++) {
        const HostSeg& s = h->segs[k];
        SegDev d;
        d.type = s.type;
        d.n = (int)s.t.size();
        d.off = (int)st.size();
        d.sorted = series_sorted(s.t) ? 1 : 0;
        sd.push_back(d);
        st.insert(st.end(), s.t.begin(), s.t.end());
        swl.insert(swl.end(), s.wl.begin(), s.wl.end());
        for (int sidx = 0; sidx < 4; sidx++)
            for (int ib : s.blk[sidx]) {
                if (ib < 0 || ib >= nb) return BGF_EINVAL;
                if (ib < nt) side[(size_t)ib * 4 + sidx] = (int)k;
            }
    }
    int rc = set_device(h);
    if (rc) return rc;
    if (!h->tstage_on) BGF_CUDA(cudaStreamSynchronize(h->stream));
    // segment buffers only grow (pools rebuild them on every admission)
    size_t ns = std::max<size_t>(1, sd.size()), nser = std::max<size_t>(1, st.size());
    if (ns > h->seg_cap || !h->d_segs) {
        dfree(h, h->d_segs);
        h->seg_cap = std::max(ns, 2 * h->seg_cap);
        BGF_CUDA(dalloc_table(h, (void**)&h->d_segs, h->seg_cap * sizeof(SegDev)));
    }
    if (nser > h->ser_cap || !h->d_seg_t) {
        dfree(h, h->d_seg_t);
        dfree(h, h->d_seg_wl);
        h->ser_cap = std::max(nser, 2 * h->ser_cap);
        BGF_CUDA(dalloc_table(h, (void**)&h->d_seg_t, h->ser_cap * sizeof(double)));
        BGF_CUDA(dalloc_table(h, (void**)&h->d_seg_wl, h->ser_cap * sizeof(double)));
    }
    if (!sd.empty()) BGF_CUDA(upload_on(h, h->d_segs, sd.data(), sd.size() * sizeof(SegDev)));
    if (!st.empty()) {
        BGF_CUDA(upload_on(h, h->d_seg_t, st.data(), st.size() * sizeof(double)));
        BGF_CUDA(upload_on(h, h->d_seg_wl, swl.data(), swl.size() * sizeof(double)));
    }
    BGF_CUDA(upload_on(h, h->d_bndseg, side.data(), side.size() * sizeof(int)));
    h->nseg_dev = (int)sd.size();
    free_graphs(h);
    return BGF_OK;
}

int bgf_add_bnd_segment(bgf_handle* h, int type, int n, const double* t, const double* wl, const int nblk_side[4],
                        const int* const blk_side[4])
{
    if (!h || type < 0 || type > 3 || n < 0 || (n > 0 && (!t || !wl)) || n == 1) return BGF_EINVAL;
    HostSeg s;
    s.type = type;
    for (int k = 0; k < n; k++) {
        s.t.push_back(t[k]);
        s.wl.push_back(wl[k]);
    }
    for (int sd = 0; sd < 4; sd++) {
        int c = nblk_side ? nblk_side[sd] : 0;
        if (c < 0) return BGF_EINVAL;
        for (int k = 0; k < c; k++) s.blk[sd].push_back(blk_side[sd][k]);
    }
    h->segs.push_back(s);
    return rebuild_segments(h);
}

int bgf_set_rain_series(bgf_handle* h, int n, const double* t, const double* r)
{
    if (!h || n < 0 || n == 1 || (n > 0 && (!t || !r))) return BGF_EINVAL;
    int rc = set_device(h);
    if (rc) return rc;
    BGF_CUDA(cudaStreamSynchronize(h->stream));
    dfree(h, h->d_rain_t);
    dfree(h, h->d_rain_r);
    h->d_rain_t = h->d_rain_r = nullptr;
    h->rain_n_dev = n;
    h->rain_t.assign(t, t + n);
    h->rain_r.assign(r, r + n);
    dfree(h, (void*)h->rmap.val);  // a uniform series replaces a gridded one
    h->rmap = RainMapDev{};
    h->has_rmap = false;
    if (n > 0) {
        BGF_CUDA(dalloc(h, (void**)&h->d_rain_t, n * sizeof(double)));
        BGF_CUDA(dalloc(h, (void**)&h->d_rain_r, n * sizeof(double)));
        BGF_CUDA(copy_on(h->stream, h->d_rain_t, t, n * sizeof(double), cudaMemcpyHostToDevice));
        BGF_CUDA(copy_on(h->stream, h->d_rain_r, r, n * sizeof(double), cudaMemcpyHostToDevice));
    }
    free_graphs(h);
    return BGF_OK;
}

int bgf_set_rain_map(bgf_handle* h, int nx, int ny, double xo, double yo, double dx, double dy, int nt, double to,
                     double dt, const float* frames)
{
    if (!h || nx < 2 || ny < 2 || nt < 2 || !(dx > 0.0) || !(dy > 0.0) || !(dt > 0.0) || !frames) return BGF_EINVAL;
    int rc = set_device(h);
    if (rc) return rc;
    BGF_CUDA(cudaStreamSynchronize(h->stream));
    dfree(h, (void*)h->rmap.val);
    h->rmap = RainMapDev{};
    h->has_rmap = false;
    // a gridded series replaces a uniform one
    dfree(h, h->d_rain_t);
    dfree(h, h->d_rain_r);
    h->d_rain_t = h->d_rain_r = nullptr;
    h->rain_n_dev = 0;
    h->rain_t.clear();
    h->rain_r.clear();
    const size_t n = (size_t)nx * ny * nt;
    float* d = nullptr;
    BGF_CUDA(dalloc(h, (void**)&d, n * sizeof(float)));
    BGF_CUDA(copy_on(h->stream, d, frames, n * sizeof(float), cudaMemcpyHostToDevice));
    RainMapDev& r = h->rmap;
    r.val = d;
    r.nx = nx;
    r.ny = ny;
    r.nt = nt;
    r.xo = xo;
    r.yo = yo;
    r.dx = dx;
    r.dy = dy;
    r.xmax = xo + (nx - 1) * dx;
    r.ymax = yo + (ny - 1) * dy;
    r.to = to;
    r.dt = dt;
    h->has_rmap = true;
    free_graphs(h);
    return BGF_OK;
}

// Rivers: InitRivers (src/InitialConditions.cu:336-420) for the discharge area,
// with the handle's current blocks; the series go to the device with the others.
int bgf_add_river(bgf_handle* h, double xstart, double xend, double ystart, double yend, int n, const double* t,
                  const double* q, double* area)
{
    if (!h || n < 2 || !t || !q) return BGF_EINVAL;
    if (!h->has_blocks) return BGF_ESTATE;
    if ((int)h->rivers.size() >= BGF_MAX_RIVERS) return BGF_EINVAL;
    for (int k = 1; k < n; k++)
        if (!(t[k] > t[k - 1])) return BGF_EINVAL;
    int rc = set_device(h);
    if (rc) return rc;
    const bgf_param& P = h->P;
    const double xo = std::isnan(P.xo) ? 0.0 : P.xo, yo = std::isnan(P.yo) ? 0.0 : P.yo;
    double a = 0.0;
    for (int ibl = 0; ibl < h->nblk; ibl++) {
        const int ib = h->active[ibl];
        const int lev = h->level[ib];
        const double levdx = lev < 0 ? P.dx * (1 << -lev) : P.dx / (1 << lev);
        const double levdelta = lev < 0 ? P.delta * (1 << -lev) : P.delta / (1 << lev);
        for (int j = 0; j < 16; j++)
            for (int i = 0; i < 16; i++) {
                const double xi = xo + h->bxo[ib] + i * levdx, yi = yo + h->byo[ib] + j * levdx;
                const double xl = xi - 0.5 * levdx, yb = yi - 0.5 * levdx, xr = xi + 0.5 * levdx, yt = yi + 0.5 * levdx;
                if (xstart <= xr && xend >= xl && ystart <= yt && yend >= yb) a = a + levdelta * levdelta;
            }
    }
    if (area) *area = a;
    if (a == 0.0) return BGF_OK;  // outside the model: the reference drops such a river
    BGF_CUDA(cudaStreamSynchronize(h->stream));
    RiverDev r;
    r.xs = xstart;
    r.xe = xend;
    r.ys = ystart;
    r.ye = yend;
    r.area = a;
    r.off = (int)h->riv_t.size();
    r.n = n;
    h->rivers.push_back(r);
    h->riv_t.insert(h->riv_t.end(), t, t + n);
    h->riv_q.insert(h->riv_q.end(), q, q + n);
    for (void** d : {(void**)&h->d_rivers, (void**)&h->d_riv_t, (void**)&h->d_riv_q})
        if (*d) { dfree(h, *d); *d = nullptr; }
    BGF_CUDA(dalloc(h, (void**)&h->d_rivers, h->rivers.size() * sizeof(RiverDev)));
    BGF_CUDA(dalloc(h, (void**)&h->d_riv_t, h->riv_t.size() * sizeof(double)));
    BGF_CUDA(dalloc(h, (void**)&h->d_riv_q, h->riv_q.size() * sizeof(double)));
    BGF_CUDA(copy_on(h->stream, h->d_rivers, h->rivers.data(), h->rivers.size() * sizeof(RiverDev), cudaMemcpyHostToDevice));
    BGF_CUDA(copy_on(h->stream, h->d_riv_t, h->riv_t.data(), h->riv_t.size() * sizeof(double), cudaMemcpyHostToDevice));
    BGF_CUDA(copy_on(h->stream, h->d_riv_q, h->riv_q.data(), h->riv_q.size() * sizeof(double), cudaMemcpyHostToDevice));
    free_graphs(h);
    return BGF_OK;
}

// Runs fn(b0, b1) over the block range [0, n) in contiguous pieces on up to 8 host
// threads when the range is large enough to pay for starting them.
template <class F> static void parallel_blocks(size_t n, F fn)
{
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const unsigned nt = std::min<unsigned>(8, hw);
    if (n < 1024 || nt <= 1) {
        fn((size_t)0, n);
        return;
    }
    std::vector<std::thread> th;
    const size_t chunk = (n + nt - 1) / nt;
    for (unsigned t = 0; t < nt; t++) {
        const size_t b0 = t * chunk, b1 = std::min(n, b0 + chunk);
        if (b0 >= b1) break;
        th.emplace_back(fn, b0, b1);
    }
    for (auto& x : th) x.join();
}

// Interior cells of BUQ tiles (324 per block, source type S) to compact blocks
// (256 per block, type T), blocks [b0, b1).
template <class T, class S> static void tiles_to_compact(const S* src, T* dst, size_t b0, size_t b1)
{
    for (size_t ib = b0; ib < b1; ib++)
        for (int j = 0; j < 16; j++) {
            const S* r = src + ib * 324 + (size_t)(j + 1) * 18 + 1;
            T* w = dst + ib * 256 + (size_t)j * 16;
            for (int i = 0; i < 16; i++) w[i] = (T)r[i];
        }
}

template <class T> static int set_state_t(bgf_handle* h, const bgf_evolving* ev)
{
    size_t nb = h->nblkmem;
    T* a = (T*)staging(h, 3 * nb * 256 * sizeof(T));
    if (!a) return BGF_ENOMEM;
    void* dst[3] = {h->d_h[h->cur], h->d_u[h->cur], h->d_v[h->cur]};
    const void* src[3] = {ev->h, ev->u, ev->v};
    const bool split = h->split != 0, iodbl = h->iodbl != 0;
    if (!split && host_pinned(src[0]) && host_pinned(src[1]) && host_pinned(src[2])) {
        // pinned caller arrays: whole tiles by DMA, interiors picked out on the device
        T* tiles = (T*)tile_scratch(h, 3 * nb * 324 * sizeof(T));
        if (!tiles) return BGF_ENOMEM;
        for (int f = 0; f < 3; f++)
            BGF_CUDA(cudaMemcpyAsync(tiles + f * nb * 324, src[f], nb * 324 * sizeof(T), cudaMemcpyHostToDevice,
                                     h->stream));
        layout::launch_tiles_to_compact<T>(tiles, (T*)dst[0], (T*)dst[1], (T*)dst[2], nb, h->stream);
        BGF_CUDA(cudaGetLastError());
        BGF_CUDA(cudaStreamSynchronize(h->stream));
        h->has_state = true;
        return BGF_OK;
    }
    // one pass over the blocks converts the three fields
    parallel_blocks(nb, [=](size_t b0, size_t b1) {
        for (int f = 0; f < 3; f++) {
            T* o = a + f * nb * 256;
            if (split && f == 0) {
                // deviation from the datum, chosen so that the model surface
                // zb (as stored) + datum + deviation is the given zb + h
                const double* hs = (const double*)src[0];
                for (size_t ib = b0; ib < b1; ib++) {
                    const double D = h->datum[ib];
                    for (int j = 0; j < 16; j++)
                        for (int i = 0; i < 16; i++) {
                            const size_t s = ib * 324 + (i + 1) + (j + 1) * 18;
                            const double hv = hs[s];
                            const double zf = (double)(T)h->zbd[s];
                            const double dev = hv > 0.0 ? (h->zbd[s] + hv) - zf - D : -D;
                            o[ib * 256 + j * 16 + i] = (T)std::max(dev, -D);
                        }
                }
            } else if (iodbl) {
                tiles_to_compact<T, double>((const double*)src[f], o, b0, b1);
            } else {
                tiles_to_compact<T, float>((const float*)src[f], o, b0, b1);
            }
        }
    });
    for (int f = 0; f < 3; f++)
        BGF_CUDA(cudaMemcpyAsync(dst[f], a + f * nb * 256, nb * 256 * sizeof(T), cudaMemcpyHostToDevice, h->stream));
    BGF_CUDA(cudaStreamSynchronize(h->stream));
    h->has_state = true;
    return BGF_OK;
}

int bgf_set_state(bgf_handle* h, const bgf_evolving* ev)
{
    if (!h || !ev || !ev->h || !ev->u || !ev->v) return BGF_EINVAL;
    int rc = set_device(h);
    if (rc) return rc;
    BGF_CUDA(cudaStreamSynchronize(h->stream));
    if (h->split && h->datum.empty()) return BGF_ESTATE;  // split mode: bed (and datums) first
    return h->dbl ? set_state_t<double>(h, ev) : set_state_t<float>(h, ev);
}

// Compact blocks (type T) back into BUQ tiles (type O): the interior cells of the
// active blocks hold the state (zs = zb + h in T; in double from the datum in split
// mode), every other entry of the nblkmem tiles is set to 0.
template <class T, class O> static void compact_to_tiles(const bgf_handle* h, const T* hh, const T* uu, const T* vv,
                                                         const T* zb, bgf_evolving* ev)
{
    O* outs[4] = {(O*)ev->zs, (O*)ev->h, (O*)ev->u, (O*)ev->v};
    std::vector<uint8_t> isact(h->nblkmem, 0);
    for (int ibl = 0; ibl < h->nblk; ibl++) isact[h->active[ibl]] = 1;
    const uint8_t* act = isact.data();
    const bool split = h->split != 0;
    parallel_blocks((size_t)h->nblkmem, [=](size_t b0, size_t b1) {
        for (size_t ib = b0; ib < b1; ib++) {
            if (!act[ib]) {
                for (O* o : outs)
                    if (o) memset(o + ib * 324, 0, 324 * sizeof(O));
                continue;
            }
            const double D = split ? h->datum[ib] : 0.0;
            for (O* o : outs)
                if (o) {
                    memset(o + ib * 324, 0, 18 * sizeof(O));
                    memset(o + ib * 324 + 17 * 18, 0, 18 * sizeof(O));
                }
            for (int j = 0; j < 16; j++) {
                const size_t d0 = ib * 324 + (size_t)(j + 1) * 18, s0 = ib * 256 + (size_t)j * 16;
                for (O* o : outs)
                    if (o) o[d0] = o[d0 + 17] = (O)0;
                for (int i = 0; i < 16; i++) {
                    const size_t d = d0 + 1 + i, s = s0 + i;
                    if (split) {
                        // full depth and surface in double from the datum and the deviation
                        if (outs[1]) outs[1][d] = (O)(D + (double)hh[s]);
                        if (outs[0]) outs[0][d] = (O)((double)zb[d] + D + (double)hh[s]);
                    } else {
                        if (outs[1]) outs[1][d] = (O)hh[s];
                        if (outs[0]) outs[0][d] = (O)(T)(zb[d] + hh[s]);
                    }
                    if (outs[2]) outs[2][d] = (O)uu[s];
                    if (outs[3]) outs[3][d] = (O)vv[s];
                }
            }
        }
    });
}

template <class T> static int get_state_t(bgf_handle* h, bgf_evolving* ev)
{
    size_t nb = h->nblkmem;
    if (!h->split && host_pinned(ev->zs) && host_pinned(ev->h) && host_pinned(ev->u) && host_pinned(ev->v)) {
        // pinned caller arrays: tiles composed on the device, then copied by DMA
        T* tiles = (T*)tile_scratch(h, 4 * nb * 324 * sizeof(T));
        if (!tiles) return BGF_ENOMEM;
        BGF_CUDA(cudaMemsetAsync(tiles, 0, 4 * nb * 324 * sizeof(T), h->stream));
        layout::launch_compact_to_tiles<T>(h->d_active, h->nblk, (const T*)h->d_h[h->cur], (const T*)h->d_u[h->cur],
                                           (const T*)h->d_v[h->cur], (const T*)h->d_zb, tiles, nb, h->stream);
        BGF_CUDA(cudaGetLastError());
        void* outs[4] = {ev->zs, ev->h, ev->u, ev->v};
        for (int f = 0; f < 4; f++)
            BGF_CUDA(cudaMemcpyAsync(outs[f], tiles + f * nb * 324, nb * 324 * sizeof(T), cudaMemcpyDeviceToHost,
                                     h->stream));
        BGF_CUDA(cudaStreamSynchronize(h->stream));
        return BGF_OK;
    }
    T* a = (T*)staging(h, (3 * nb * 256 + nb * 324) * sizeof(T));
    if (!a) return BGF_ENOMEM;
    T *hh = a, *uu = a + nb * 256, *vv = a + 2 * nb * 256, *zb = a + 3 * nb * 256;
    BGF_CUDA(cudaMemcpyAsync(hh, h->d_h[h->cur], nb * 256 * sizeof(T), cudaMemcpyDeviceToHost, h->stream));
    BGF_CUDA(cudaMemcpyAsync(uu, h->d_u[h->cur], nb * 256 * sizeof(T), cudaMemcpyDeviceToHost, h->stream));
    BGF_CUDA(cudaMemcpyAsync(vv, h->d_v[h->cur], nb * 256 * sizeof(T), cudaMemcpyDeviceToHost, h->stream));
    BGF_CUDA(cudaMemcpyAsync(zb, h->d_zb, nb * 324 * sizeof(T), cudaMemcpyDeviceToHost, h->stream));
    BGF_CUDA(cudaStreamSynchronize(h->stream));
    if (h->split || h->dbl) compact_to_tiles<T, double>(h, hh, uu, vv, zb, ev);
    else compact_to_tiles<T, float>(h, hh, uu, vv, zb, ev);
    return BGF_OK;
}

int bgf_get_state(bgf_handle* h, bgf_evolving* ev)
{
    if (!h || !ev) return BGF_EINVAL;
    if (!h->has_state) return BGF_ESTATE;
    int rc = set_device(h);
    if (rc) return rc;
    BGF_CUDA(cudaStreamSynchronize(h->stream));
    return h->dbl ? get_state_t<double>(h, ev) : get_state_t<float>(h, ev);
}

static int check_ready(bgf_handle* h)
{
    if (!h) return BGF_EINVAL;
    if (!h->has_blocks || !h->has_bed || !h->has_state) return BGF_ESTATE;
    return set_device(h);
}

static int check_err_word(bgf_handle* h)
{
    int err = 0;
    BGF_CUDA(copy_on(h->stream, &err, h->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) {
        g_last_error = "mesh has cross-level neighbours, which this build does not support yet";
        return BGF_EINVAL;
    }
    return BGF_OK;
}

template <class T> static int init_dt_t(bgf_handle* h, bgf_loop* loop)
{
    unsigned long long init = dt_init_bits(h->dbl);
    BGF_CUDA(cudaMemcpyAsync(h->d_dtmin, &init, sizeof(init), cudaMemcpyHostToDevice, h->stream));
    DevModel<T> m = dev_model<T>(h);
    StepParams<T> p = step_params<T>(h);
    if (h->fast) fa::launch_initdt<T>(m, p, h->cur, h->d_dtmin, h->stream);
    else ex::launch_initdt<T>(m, p, h->cur, h->d_dtmin, h->stream);
    h->launches++;
    BGF_CUDA(cudaGetLastError());
    unsigned long long bits = 0;
    BGF_CUDA(cudaMemcpyAsync(&bits, h->d_dtmin, sizeof(bits), cudaMemcpyDeviceToHost, h->stream));
    BGF_CUDA(cudaStreamSynchronize(h->stream));
    T dt;
    if (sizeof(T) == 8) memcpy(&dt, &bits, 8);
    else { unsigned int b = (unsigned int)bits; memcpy(&dt, &b, 4); }
    // initdt (src/Mainloop.cu:515-554) on a local copy of the loop
    int maxlevel = h->P.maxlevel;
    double dtmaxloc = h->P.dtinit > 0 ? h->P.dtinit / 1.5
                                      : (maxlevel < 0 ? h->P.delta * (double)(1 << (-maxlevel)) : h->P.delta / (double)(1 << maxlevel)) /
                                            (sqrt(h->P.g * 10.0));
    T one_over_epsi = (T)1.0 / epsi_of<T>();
    if (one_over_epsi < dt) dt = one_over_epsi;  // reduction starts at 1/epsi (timestepreductionCPU)
    if ((double)dt > (1.5 * dtmaxloc)) dt = (T)(1.5 * dtmaxloc);
    if (ceil((loop->nextoutputtime - loop->totaltime) / (double)dt) > 0.0)
        dt = (T)((loop->nextoutputtime - loop->totaltime) / ceil((loop->nextoutputtime - loop->totaltime) / (double)dt));
    loop->dtmax = (double)dt;
    return BGF_OK;
}

int bgf_init_dt(bgf_handle* h, bgf_loop* loop)
{
    int rc = check_ready(h);
    if (rc) return rc;
    if (!loop) return BGF_EINVAL;
    return h->dbl ? init_dt_t<double>(h, loop) : init_dt_t<float>(h, loop);
}

// A multi-level mesh's two block sets: the multi-level chain over the blocks with a
// side facing another level, and the fused single-level kernels over the rest.
// Without pools only one kernel may write the time slot: the single-level
// corrector's first block when it has blocks, else the chain's.
template <class T> static DevModel<T> chain_model(const bgf_handle* h, DevModel<T> m, bool pool)
{
    m.active = h->d_active_chain;
    m.nblk = h->nchain;
    if (!pool && h->npure) m.lead = h->d_nolead;
    return m;
}
template <class T> static DevModel<T> pure_model(const bgf_handle* h, DevModel<T> m)
{
    m.active = h->d_active_pure;
    m.nblk = h->npure;
    return m;
}

// One stage of a multi-level step over model m (a handle's or a pool's): predictor
// (stage 0) = single-level flux kernel on the pure blocks and the chain's predictor;
// corrector = the chain's corrector and the single-level update kernel.
template <class T>
static int enqueue_amr_stage(bgf_handle* h, const DevModel<T>& m, const StepParams<T>& p, int parity, int stage,
                             bool pool)
{
    int n = 0;
    const DevModel<T> mc = chain_model<T>(h, m, pool), mp = pure_model<T>(h, m);
    if (stage == 0 && h->npure) {
        if (h->fast) fa::launch_flux<T>(mp, p, h->P.engine, parity, h->stream, 0);
        else ex::launch_flux<T>(mp, p, h->P.engine, parity, h->stream, 0);
        n++;
    }
    n += h->fast ? fa::launch_amr_stage<T>(mc, amr_dev<T>(h), p, h->P.engine, parity, stage, h->minlev, h->maxlev,
                                          h->stream)
                 : ex::launch_amr_stage<T>(mc, amr_dev<T>(h), p, h->P.engine, parity, stage, h->minlev, h->maxlev,
                                          h->stream);
    if (stage == 1 && h->npure) {
        if (h->fast) fa::launch_update<T>(mp, p, h->P.engine, parity, h->stream, 0);
        else ex::launch_update<T>(mp, p, h->P.engine, parity, h->stream, 0);
        n++;
    }
    return n;
}

// First and second half of a step: the fused predictor / corrector kernels, or
// the predictor / corrector stages of a multi-level mesh.  Return the number of
// kernels launched.
template <class T> static int enqueue_flux(bgf_handle* h, int parity)
{
    if (h->amr) return enqueue_amr_stage<T>(h, dev_model<T>(h), step_params<T>(h), parity, 0, false);
    if (h->fast) fa::launch_flux<T>(dev_model<T>(h), step_params<T>(h), h->P.engine, parity, h->stream, h->grid);
    else ex::launch_flux<T>(dev_model<T>(h), step_params<T>(h), h->P.engine, parity, h->stream, h->grid);
    return 1;
}

template <class T> static int enqueue_update(bgf_handle* h, int parity)
{
    if (h->amr) return enqueue_amr_stage<T>(h, dev_model<T>(h), step_params<T>(h), parity, 1, false);
    if (h->fast) fa::launch_update<T>(dev_model<T>(h), step_params<T>(h), h->P.engine, parity, h->stream, h->grid);
    else ex::launch_update<T>(dev_model<T>(h), step_params<T>(h), h->P.engine, parity, h->stream, h->grid);
    return 1;
}

// The gauge samples of a step, after its corrector.
template <class T> static int enqueue_gauges(bgf_handle* h, int parity)
{
    if (h->gauges.n == 0) return 0;
    launch_gauges<T>(dev_model<T>(h), gauge_dev<T>(h->gauges), parity, h->stream);
    return 1;
}

template <class T> static int enqueue_step(bgf_handle* h, int parity)
{
    int n = enqueue_flux<T>(h, parity);
    n += enqueue_update<T>(h, parity);
    return n + enqueue_gauges<T>(h, parity);
}

// The host side of write_time_slot: fills the pinned time slot and dt seed.
static TimeState make_time_state(const bgf_handle* h, const bgf_loop* loop, double endtime, double outputtimestep,
                                 long long maxsteps)
{
    TimeState ts;
    memset(&ts, 0, sizeof(ts));
    ts.totaltime = loop->totaltime;
    ts.dt = loop->dt;
    ts.dtmax = loop->dtmax;
    ts.nextoutputtime = loop->nextoutputtime;
    ts.endtime = endtime;
    ts.outputtimestep = outputtimestep;
    ts.nstep = 0;
    ts.maxsteps = maxsteps;
    ts.cur = h->cur;
    ts.done = 0;
    ts.status = 0;
    return ts;
}

static void set_time_slot_host(bgf_handle* h, const bgf_loop* loop, double endtime, double outputtimestep,
                               long long maxsteps)
{
    h->h_time[0] = make_time_state(h, loop, endtime, outputtimestep, maxsteps);
    h->h_misc[0] = dt_init_bits(h->dbl);
}

// Writes the loop state into the device time slot of the current parity and seeds
// the dt minimum.  Both copies read pinned slots that are not written again before
// the caller's next stream synchronisation, so no synchronisation is needed here.
static int write_time_slot(bgf_handle* h, const bgf_loop* loop, double endtime, double outputtimestep, long long maxsteps)
{
    set_time_slot_host(h, loop, endtime, outputtimestep, maxsteps);
    BGF_CUDA(cudaMemcpyAsync(h->d_time + h->parity, &h->h_time[0], sizeof(TimeState), cudaMemcpyHostToDevice, h->stream));
    BGF_CUDA(cudaMemcpyAsync(h->d_dtmin + h->parity, &h->h_misc[0], sizeof(unsigned long long), cudaMemcpyHostToDevice,
                             h->stream));
    return BGF_OK;
}

// After a step's result reached the pinned slots: error word, loop update, parity.
static int finish_step(bgf_handle* h, bgf_loop* loop, int err, const TimeState& nt)
{
    if (err) {
        g_last_error = "mesh has cross-level neighbours, which this build does not support yet";
        return BGF_EINVAL;
    }
    loop->dt = nt.dt;
    loop->dtmax = nt.dtmax;
    h->cur = nt.cur;
    h->parity ^= 1;
    if (nt.status == BGF_ENAN) {
        g_last_error = "non-finite value in the state";
        return BGF_ENAN;
    }
    return BGF_OK;
}

// One flow step for parity p as a graph: one copy of the control block's time and
// dt slots in (slot p carries the step's loop state; the other slots are overwritten
// by the step itself), the step's kernels, and one copy out from time slot p ^ 1 to
// the error word.  One launch per bgf_flow_step.
static int build_step_graph(bgf_handle* h, int p)
{
    cudaGraph_t g;
    BGF_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    cudaMemcpyAsync(h->d_ctl, h->h_ctl, offsetof(StepCtl, err), cudaMemcpyHostToDevice, h->stream);
    h->step_graph_launches[p] = h->dbl ? enqueue_step<double>(h, p) : enqueue_step<float>(h, p);
    const size_t off = offsetof(StepCtl, t) + (size_t)(p ^ 1) * sizeof(TimeState);
    cudaMemcpyAsync((char*)h->h_ctl + off, (const char*)h->d_ctl + off, offsetof(StepCtl, err) + sizeof(int) - off,
                    cudaMemcpyDeviceToHost, h->stream);
    cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    if (e != cudaSuccess) {
        g_last_error = std::string("graph capture: ") + cudaGetErrorString(e);
        return BGF_ECUDA;
    }
    e = cudaGraphInstantiate(&h->step_graph[p], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        h->step_graph[p] = nullptr;
        g_last_error = std::string("graph instantiate: ") + cudaGetErrorString(e);
        return BGF_ECUDA;
    }
    return BGF_OK;
}

int bgf_flow_step(bgf_handle* h, bgf_loop* loop)
{
    int rc = check_ready(h);
    if (rc) return rc;
    if (!loop) return BGF_EINVAL;
    if (!h->profiling) {
        const int p = h->parity;
        if (!h->step_graph[p] && (rc = build_step_graph(h, p))) return rc;
        // the host block the graph copies from and to (not in use: the previous call
        // synchronised); both dt slots are armed, slot p ^ 1 is re-armed by the step too
        StepCtl* c = h->h_ctl;
        c->t[p] = make_time_state(h, loop, INFINITY, 0.0, 1);
        c->t[p ^ 1] = c->t[p];
        c->dtmin[0] = c->dtmin[1] = dt_init_bits(h->dbl);
        BGF_CUDA(cudaGraphLaunch(h->step_graph[p], h->stream));
        h->launches += h->step_graph_launches[p];
        BGF_CUDA(cudaStreamSynchronize(h->stream));
        return finish_step(h, loop, c->err, c->t[p ^ 1]);
    }
    rc = write_time_slot(h, loop, INFINITY, 0.0, 1);
    if (rc) return rc;
    int n = 0;
    if (h->profiling) {
        BGF_CUDA(cudaEventRecord(h->pev[0], h->stream));
        if (h->dbl) {
            n += enqueue_flux<double>(h, h->parity);
            BGF_CUDA(cudaEventRecord(h->pev[1], h->stream));
            n += enqueue_update<double>(h, h->parity);
        } else {
            n += enqueue_flux<float>(h, h->parity);
            BGF_CUDA(cudaEventRecord(h->pev[1], h->stream));
            n += enqueue_update<float>(h, h->parity);
        }
        BGF_CUDA(cudaEventRecord(h->pev[2], h->stream));
        n += h->dbl ? enqueue_gauges<double>(h, h->parity) : enqueue_gauges<float>(h, h->parity);
    } else if (h->dbl) {
        n = enqueue_step<double>(h, h->parity);
    } else {
        n = enqueue_step<float>(h, h->parity);
    }
    h->launches += n;
    BGF_CUDA(cudaGetLastError());
    // the step's time state and the device error word, read back with one synchronisation
    BGF_CUDA(cudaMemcpyAsync(&h->h_time[1], h->d_time + (h->parity ^ 1), sizeof(TimeState), cudaMemcpyDeviceToHost,
                             h->stream));
    BGF_CUDA(cudaMemcpyAsync(&h->h_misc[1], h->d_err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    BGF_CUDA(cudaStreamSynchronize(h->stream));
    if (h->profiling) {
        float a = 0.f, b = 0.f;
        cudaEventElapsedTime(&a, h->pev[0], h->pev[1]);
        cudaEventElapsedTime(&b, h->pev[1], h->pev[2]);
        h->flux_ms += a;
        h->update_ms += b;
        h->profiled_steps++;
    }
    return finish_step(h, loop, *(const int*)&h->h_misc[1], h->h_time[1]);
}

static int build_graphs(bgf_handle* h)
{
    for (int k = 0; k < 2; k++)  // the run graphs only; the single-step graphs stay valid
        if (h->graph[k]) {
            cudaGraphExecDestroy(h->graph[k]);
            h->graph[k] = nullptr;
        }
    for (int p0 = 0; p0 < 2; p0++) {
        cudaGraph_t g;
        BGF_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        int n = 0;
        for (int k = 0; k < 2; k++) n += h->dbl ? enqueue_step<double>(h, p0 ^ k) : enqueue_step<float>(h, p0 ^ k);
        h->steps_launches = n / 2;
        cudaError_t e = cudaStreamEndCapture(h->stream, &g);
        if (e != cudaSuccess) {
            g_last_error = std::string("graph capture: ") + cudaGetErrorString(e);
            return BGF_ECUDA;
        }
        e = cudaGraphInstantiate(&h->graph[p0], g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            g_last_error = std::string("graph instantiate: ") + cudaGetErrorString(e);
            return BGF_ECUDA;
        }
    }
    h->graph_valid = true;
    return BGF_OK;
}

int bgf_run(bgf_handle* h, bgf_loop* loop, double endtime, double outputtimestep, int maxsteps, int* nsteps)
{
    int rc = check_ready(h);
    if (rc) return rc;
    if (!loop || maxsteps < 0) return BGF_EINVAL;
    if (nsteps) *nsteps = 0;
    if (!h->graph_valid) {
        rc = build_graphs(h);
        if (rc) return rc;
    }
    rc = write_time_slot(h, loop, endtime, outputtimestep, maxsteps);
    if (rc) return rc;
    const int p0 = h->parity;
    double gpu_ms = 0.0;
    int64_t launched = 0;
    TimeState ts = h->h_time[0];
    double dtguess = loop->dtmax > 0 ? loop->dtmax : 1.0;
    while (true) {
        double remaining = (endtime - ts.totaltime) / (dtguess > 0 ? dtguess : 1.0);
        long long left = (long long)maxsteps - ts.nstep;
        long long want = (long long)std::min<double>(remaining * 1.02 + 2.0, (double)left);
        int batch = (int)std::max<long long>(1, std::min<long long>((want + 1) / 2, 512));
        BGF_CUDA(cudaEventRecord(h->ev0, h->stream));
        for (int b = 0; b < batch; b++) BGF_CUDA(cudaGraphLaunch(h->graph[p0], h->stream));
        BGF_CUDA(cudaEventRecord(h->ev1, h->stream));
        launched += 2LL * h->steps_launches * batch;
        // after whole graphs the latest time state is in slot p0
        BGF_CUDA(cudaMemcpyAsync(&h->h_time[1], h->d_time + p0, sizeof(TimeState), cudaMemcpyDeviceToHost, h->stream));
        BGF_CUDA(cudaStreamSynchronize(h->stream));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, h->ev0, h->ev1);
        gpu_ms += ms;
        ts = h->h_time[1];
        // at most 1024 steps per batch: the 4096-sample gauge ring cannot overflow
        if ((rc = gauge_drain_handle(h))) return rc;
        if (ts.dt > 0) dtguess = ts.dt;
        if (ts.done || ts.totaltime >= endtime || ts.nstep >= maxsteps) break;
    }
    h->launches += launched;
    h->last_run_ms = gpu_ms;
    h->last_run_launches = launched;
    rc = check_err_word(h);
    if (rc) return rc;
    loop->totaltime = ts.totaltime;
    loop->dt = ts.dt;
    loop->dtmax = ts.dtmax;
    loop->nextoutputtime = ts.nextoutputtime;
    h->cur = ts.cur;
    // parity stays p0: every graph replay advances it by two
    if (nsteps) *nsteps = (int)ts.nstep;
    if (ts.status == BGF_EDT_UNDERFLOW || ts.status == BGF_ENAN) return ts.status;
    return BGF_OK;
}

int bgf_volume(bgf_handle* h, double* volume)
{
    int rc = check_ready(h);
    if (rc) return rc;
    if (!volume) return BGF_EINVAL;
    BGF_CUDA(cudaMemsetAsync(h->d_scratch, 0, sizeof(double), h->stream));
    if (h->dbl) ex::launch_volume<double>(dev_model<double>(h), (double)h->P.delta, h->cur, h->d_scratch, h->stream);
    else ex::launch_volume<float>(dev_model<float>(h), (float)h->P.delta, h->cur, h->d_scratch, h->stream);
    h->launches++;
    BGF_CUDA(cudaGetLastError());
    BGF_CUDA(cudaMemcpyAsync(volume, h->d_scratch, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    BGF_CUDA(cudaStreamSynchronize(h->stream));
    return BGF_OK;
}

int64_t bgf_kernel_launches(bgf_handle* h) { return h ? h->launches : -1; }

int bgf_set_profiling(bgf_handle* h, int on)
{
    if (!h) return BGF_EINVAL;
    h->profiling = on ? 1 : 0;
    h->flux_ms = h->update_ms = 0.0;
    h->profiled_steps = 0;
    return BGF_OK;
}

int bgf_kernel_timing(bgf_handle* h, double* flux_ms, double* update_ms, int64_t* steps)
{
    if (!h) return BGF_EINVAL;
    if (flux_ms) *flux_ms = h->flux_ms;
    if (update_ms) *update_ms = h->update_ms;
    if (steps) *steps = h->profiled_steps;
    return BGF_OK;
}

int bgf_run_timing(bgf_handle* h, double* gpu_ms, int64_t* launches)
{
    if (!h) return BGF_EINVAL;
    if (gpu_ms) *gpu_ms = h->last_run_ms;
    if (launches) *launches = h->last_run_launches;
    return BGF_OK;
}

// ---------------------------------------------------------------- refinement pass

int bgf_set_bathy(bgf_handle* h, int nx, int ny, double xo, double yo, double dx, const float* val)
{
    if (!h || nx < 2 || ny < 2 || !(dx > 0.0) || !val) return BGF_EINVAL;
    int rc = set_device(h);
    if (rc) return rc;
    dfree(h, h->d_dem);
    h->d_dem = nullptr;
    BGF_CUDA(dalloc(h, (void**)&h->d_dem, sizeof(float) * (size_t)nx * ny));
    BGF_CUDA(copy_on(h->stream, h->d_dem, val, sizeof(float) * (size_t)nx * ny, cudaMemcpyHostToDevice));
    h->dem_nx = nx;
    h->dem_ny = ny;
    h->dem_xo = xo;
    h->dem_yo = yo;
    h->dem_dx = dx;
    return BGF_OK;
}

int bgf_add_target_level_map(bgf_handle* h, int nx, int ny, double xo, double yo, double dx, const int* levels)
{
    if (!h || nx < 2 || ny < 2 || !(dx > 0.0) || !levels) return BGF_EINVAL;
    int rc = set_device(h);
    if (rc) return rc;
    const size_t n = (size_t)nx * ny;
    std::vector<float> v(n);
    for (size_t k = 0; k < n; k++) v[k] = (float)levels[k];
    adapt::TargetMapDev g{};
    BGF_CUDA(dalloc(h, (void**)&g.val, sizeof(float) * n));
    BGF_CUDA(copy_on(h->stream, (void*)g.val, v.data(), sizeof(float) * n, cudaMemcpyHostToDevice));
    g.nx = nx;
    g.ny = ny;
    g.xo = xo;
    g.yo = yo;
    g.dx = dx;
    g.dy = dx;
    g.xmax = xo + (nx - 1) * dx;
    g.ymax = yo + (ny - 1) * dx;
    h->tmaps.push_back(g);
    return BGF_OK;
}

int bgf_clear_target_level_maps(bgf_handle* h)
{
    if (!h) return BGF_EINVAL;
    int rc = set_device(h);
    if (rc) return rc;
    for (auto& g : h->tmaps) dfree(h, (void*)g.val);
    h->tmaps.clear();
    return BGF_OK;
}

int bgf_get_blocks(bgf_handle* h, int* nblk, int* active, int* level, int* nbr8, double* xo, double* yo)
{
    if (!h || !nblk) return BGF_EINVAL;
    if (!h->has_blocks) return BGF_ESTATE;
    const int nb = h->nblkmem;
    *nblk = h->nblk;
    if (active) memcpy(active, h->active.data(), sizeof(int) * h->nblk);
    if (level) memcpy(level, h->level.data(), sizeof(int) * nb);
    if (nbr8)
        for (int ib = 0; ib < nb; ib++)
            for (int k = 0; k < 8; k++) nbr8[8 * ib + k] = h->nbr[(size_t)k * nb + ib];
    if (xo) memcpy(xo, h->bxo.data(), sizeof(double) * nb);
    if (yo) memcpy(yo, h->byo.data(), sizeof(double) * nb);
    return BGF_OK;
}

template <class T> static adapt::AdaptDev<T> adapt_dev(bgf_handle* h)
{
    adapt::AdaptDev<T> a;
    for (int k = 0; k < 4; k++) a.W[k] = (T*)h->d_W[0][k];
    a.zs = (T*)h->d_dh;  // the flow step's scratch is free between steps
    a.dem = h->d_dem;
    a.dnx = h->dem_nx;
    a.dny = h->dem_ny;
    a.dxo = h->dem_xo;
    a.dyo = h->dem_yo;
    a.ddx = h->dem_dx;
    a.dxmax = h->dem_xo + (h->dem_nx - 1) * h->dem_dx;
    a.dymax = h->dem_yo + (h->dem_ny - 1) * h->dem_dx;
    a.child = h->d_child;
    a.flags = h->d_flags;
    return a;
}

// refinesanitycheck on the handle's tables (bgf_adapt_sanity); coarsening flags
// survive only with allow_coarsen.
static int sanity(bgf_handle* h, const bgf_adapt_param* ap, std::vector<uint8_t>& refine,
                  std::vector<uint8_t>& coarsen)
{
    const int nb = h->nblkmem;
    std::vector<int> nbr8((size_t)8 * nb);
    for (int ib = 0; ib < nb; ib++)
        for (int k = 0; k < 8; k++) nbr8[8 * ib + k] = h->nbr[(size_t)k * nb + ib];
    return bgf_adapt_sanity(h->nblk, h->active.data(), h->level.data(), nbr8.data(), nb, h->P.minlevel, h->P.maxlevel,
                            h->bxo.data(), h->byo.data(), h->P.dx, ap->allow_coarsen ? 1 : 0, refine.data(),
                            coarsen.data());
}

// AdaptCriteria (src/AdaptCriteria.cu:20-130) on the device, then the host sanity
// pass.  refine/coarsen are indexed by block id (nblkmem bytes each).
template <class T> static int adapt_flags_t(bgf_handle* h, const bgf_adapt_param* ap, std::vector<uint8_t>& refine,
                                            std::vector<uint8_t>& coarsen)
{
    const int nb = h->nblkmem;
    DevModel<T> m = dev_model<T>(h);
    if (ap->criterion == BGF_ADAPT_TARGETLEVEL) {
        // AdaptCriteria runs targetlevelcriteria once per map (the last map decides)
        if (h->tmaps.empty()) {
            g_last_error = "the Targetlevel criterion needs at least one target-level map";
            return BGF_EINVAL;
        }
        for (const auto& g : h->tmaps) {
            adapt::launch_target_level<T>(m, g, std::isnan(h->P.xo) ? 0.0 : h->P.xo, std::isnan(h->P.yo) ? 0.0 : h->P.yo,
                                          h->P.dx, h->d_flags, h->d_cflags, h->stream);
            h->launches++;
        }
        BGF_CUDA(cudaGetLastError());
        refine.assign(nb, 0);
        coarsen.assign(nb, 0);
        BGF_CUDA(cudaMemcpyAsync(refine.data(), h->d_flags, nb, cudaMemcpyDeviceToHost, h->stream));
        BGF_CUDA(cudaMemcpyAsync(coarsen.data(), h->d_cflags, nb, cudaMemcpyDeviceToHost, h->stream));
        BGF_CUDA(cudaStreamSynchronize(h->stream));
        std::vector<uint8_t> mask(nb, 0);
        for (int ibl = 0; ibl < h->nblk; ibl++) mask[h->active[ibl]] = 1;
        for (int ib = 0; ib < nb; ib++) {
            refine[ib] = mask[ib] ? refine[ib] : 0;
            coarsen[ib] = mask[ib] ? coarsen[ib] : 0;
        }
        return sanity(h, ap, refine, coarsen);
    }
    if (ap->criterion == BGF_ADAPT_HGRAD) {
        adapt::launch_hgrad<T>(m, (const T*)h->d_dh, h->cur, h->P.eps, ap->arg1, ap->arg2, h->P.dx, h->d_flags,
                               h->d_cflags, h->stream);
        h->launches++;
        BGF_CUDA(cudaGetLastError());
        refine.assign(nb, 0);
        coarsen.assign(nb, 0);
        BGF_CUDA(cudaMemcpyAsync(refine.data(), h->d_flags, nb, cudaMemcpyDeviceToHost, h->stream));
        BGF_CUDA(cudaMemcpyAsync(coarsen.data(), h->d_cflags, nb, cudaMemcpyDeviceToHost, h->stream));
        BGF_CUDA(cudaStreamSynchronize(h->stream));
        std::vector<uint8_t> mask(nb, 0);
        for (int ibl = 0; ibl < h->nblk; ibl++) mask[h->active[ibl]] = 1;
        for (int ib = 0; ib < nb; ib++) {
            refine[ib] = mask[ib] ? refine[ib] : 0;
            coarsen[ib] = mask[ib] ? coarsen[ib] : 0;
        }
        return sanity(h, ap, refine, coarsen);
    }
    const T* z = nullptr;
    int stride324 = 0;
    switch (ap->var) {
    case BGF_VAR_H: z = (const T*)h->d_h[h->cur]; break;
    case BGF_VAR_ZS: z = (const T*)h->d_dh; break;
    case BGF_VAR_U: z = (const T*)h->d_u[h->cur]; break;
    case BGF_VAR_V: z = (const T*)h->d_v[h->cur]; break;
    case BGF_VAR_ZB: z = (const T*)h->d_zb; stride324 = 1; break;
    default: return BGF_EINVAL;
    }
    adapt::launch_criteria<T>(m, z, stride324, ap->criterion, (T)ap->arg1, (T)ap->arg2, h->d_flags, h->stream);
    h->launches++;
    BGF_CUDA(cudaGetLastError());
    refine.assign(nb, 0);
    coarsen.assign(nb, 0);
    BGF_CUDA(cudaMemcpyAsync(refine.data(), h->d_flags, nb, cudaMemcpyDeviceToHost, h->stream));
    BGF_CUDA(cudaStreamSynchronize(h->stream));
    std::vector<uint8_t> mask(nb, 0);
    for (int ibl = 0; ibl < h->nblk; ibl++) mask[h->active[ibl]] = 1;
    for (int ib = 0; ib < nb; ib++) {
        refine[ib] = mask[ib] ? refine[ib] : 0;
        coarsen[ib] = mask[ib] ? !refine[ib] : 0;  // Thresholdcriteria: coarsen = !refine
    }
    return sanity(h, ap, refine, coarsen);
}

static int check_adapt_param(const bgf_adapt_param* ap)
{
    if (!ap) return BGF_EINVAL;
    if (ap->allow_coarsen != 0 && ap->allow_coarsen != 1) return BGF_EINVAL;
    if (ap->criterion == BGF_ADAPT_TARGETLEVEL) return BGF_OK;  // var, arg1 and arg2 are not used
    if (ap->criterion == BGF_ADAPT_HGRAD) return ap->arg1 >= 0.0 && ap->arg2 >= 0.0 ? BGF_OK : BGF_EINVAL;
    if (ap->criterion != BGF_ADAPT_THRESHOLD && ap->criterion != BGF_ADAPT_INRANGE) return BGF_EINVAL;
    if (ap->var < BGF_VAR_H || ap->var > BGF_VAR_ZB) return BGF_EINVAL;
    return BGF_OK;
}

template <class T> static void zs_from_state(bgf_handle* h)
{
    adapt::launch_zs<T>(dev_model<T>(h), (T*)h->d_dh, h->cur, h->stream);
    h->launches++;
}

int bgf_adapt_flags(bgf_handle* h, const bgf_adapt_param* ap, uint8_t* refine, uint8_t* coarsen)
{
    int rc = check_ready(h);
    if (rc) return rc;
    if ((rc = check_adapt_param(ap))) return rc;
    std::vector<uint8_t> r, c;
    if (h->dbl) {
        zs_from_state<double>(h);
        rc = adapt_flags_t<double>(h, ap, r, c);
    } else {
        zs_from_state<float>(h);
        rc = adapt_flags_t<float>(h, ap, r, c);
    }
    if (rc) return rc;
    for (int ibl = 0; ibl < h->nblk; ibl++) {
        if (refine) refine[ibl] = r[h->active[ibl]];
        if (coarsen) coarsen[ibl] = c[h->active[ibl]];
    }
    return BGF_OK;
}

// Adaptation (src/Adaptation.cu:17-121): repeats {criteria, sanity pass, refine,
// bed re-interpolation, wet/dry fix-up} until the block count stops changing or
// maxiteration passes ran, then prepares the bed halo and gradients of the new
// mesh and carries the boundary segments over to the children of refined blocks.
template <class T>
static int adapt_dev_t(bgf_handle* h, const bgf_adapt_param* ap, const adapt::GridSpec& gs, int* niter,
                       bool& changed_any);

// gs: the level grids when the table work runs on the device (adapt_dev_t), else
// NULL for the host tables.
template <class T> static int adapt_t(bgf_handle* h, const bgf_adapt_param* ap, int* niter, const adapt::GridSpec* gs)
{
    const int nb = h->nblkmem;
    int rc = alloc_amr(h);  // stage tiles double as the old-mesh halo tiles
    if (rc) return rc;
    const int maxit = ap->maxiteration > 0 ? ap->maxiteration : 20;
    int it = 0;
    bool changed_any = false;
    if (gs) {
        if ((rc = adapt_dev_t<T>(h, ap, *gs, &it, changed_any))) return rc;
    } else {
    zs_from_state<T>(h);
    while (it < maxit) {
        it++;
        std::vector<uint8_t> refine, coarsen;
        if ((rc = adapt_flags_t<T>(h, ap, refine, coarsen))) return rc;
        std::vector<int> act(nb, -1), lev = h->level, nbr8((size_t)8 * nb), child((size_t)3 * nb, -1),
            sib((size_t)3 * nb, -1);
        std::copy(h->active.begin(), h->active.end(), act.begin());
        for (int ib = 0; ib < nb; ib++)
            for (int k = 0; k < 8; k++) nbr8[8 * ib + k] = h->nbr[(size_t)k * nb + ib];
        std::vector<double> xo = h->bxo, yo = h->byo;
        int n = h->nblk;
        rc = bgf_adapt_tables(&n, act.data(), lev.data(), nbr8.data(), xo.data(), yo.data(), nb, h->P.dx, h->dbl,
                              refine.data(), ap->allow_coarsen ? coarsen.data() : nullptr, child.data(), sib.data());
        if (rc) {
            if (rc == BGF_ENOMEM) g_last_error = "refinement needs more block slots than nblkmem";
            return rc;
        }
        bool refined = false;
        std::vector<int> quads;
        for (int ibl = 0; ibl < h->nblk; ibl++) {
            const int ib = h->active[ibl];
            refined = refined || child[3 * ib] >= 0;
            if (sib[3 * ib] >= 0) {
                quads.push_back(ib);
                for (int q = 0; q < 3; q++) quads.push_back(sib[3 * ib + q]);
            }
        }
        const int nquads = (int)quads.size() / 4;
        const bool changed = refined || nquads > 0;
        adapt::AdaptDev<T> a = adapt_dev<T>(h);
        DevModel<T> m = dev_model<T>(h);
        if (changed) {
            // children and merged quads from the old mesh (old tables still on the device)
            if (refined)
                BGF_CUDA(cudaMemcpyAsync(h->d_child, child.data(), sizeof(int) * 3 * nb, cudaMemcpyHostToDevice,
                                         h->stream));
            if (nquads)
                BGF_CUDA(cudaMemcpyAsync(h->d_quads, quads.data(), sizeof(int) * quads.size(), cudaMemcpyHostToDevice,
                                         h->stream));
            h->launches += adapt::launch_children<T>(m, a, h->cur, h->has_cf ? (T*)h->d_cf : nullptr,
                                                     h->has_rainmask ? h->d_rainmask : nullptr, h->d_quads, nquads,
                                                     refined, h->stream);
            BGF_CUDA(cudaGetLastError());
            // segments: the children on a listed side inherit it; a merged quad's
            // blocks give way to the parent, listed once
            std::vector<int> parent_of(nb, -1);
            for (int k = 0; k < nquads; k++)
                for (int q = 0; q < 4; q++) parent_of[quads[4 * k + q]] = quads[4 * k];
            const int kids_side[4][2] = {{0, 2}, {1, 3}, {2, 3}, {0, 1}};  // left, right, top, bot: child slots
            for (HostSeg& sg : h->segs)
                for (int sidx = 0; sidx < 4; sidx++) {
                    std::vector<int> out;
                    for (int ib : sg.blk[sidx]) {
                        if (ib >= 0 && ib < nb && child[3 * ib] >= 0) {
                            const int kids[4] = {ib, child[3 * ib], child[3 * ib + 1], child[3 * ib + 2]};
                            out.push_back(kids[kids_side[sidx][0]]);
                            out.push_back(kids[kids_side[sidx][1]]);
                        } else if (ib >= 0 && ib < nb && parent_of[ib] >= 0) {
                            const int p = parent_of[ib];
                            if (std::find(out.begin(), out.end(), p) == out.end()) out.push_back(p);
                        } else {
                            out.push_back(ib);
                        }
                    }
                    sg.blk[sidx] = out;
                }
            changed_any = true;
        }
        h->nblk = n;
        h->active.assign(act.begin(), act.begin() + n);
        h->level = lev;
        for (int ib = 0; ib < nb; ib++)
            for (int k = 0; k < 8; k++) h->nbr[(size_t)k * nb + ib] = nbr8[8 * ib + k];
        h->bxo = xo;
        h->byo = yo;
        if ((rc = upload_tables(h))) return rc;
        m = dev_model<T>(h);
        adapt::launch_bed<T>(m, a, step_params<T>(h), h->cur, (T*)h->d_zb, std::isnan(h->P.xo) ? 0.0 : h->P.xo,
                             std::isnan(h->P.yo) ? 0.0 : h->P.yo, h->d_bxo, h->d_byo, h->P.mask,
                             h->has_rainmask ? h->d_rainmask : nullptr, h->stream);
        h->launches++;
        BGF_CUDA(cudaGetLastError());
        if (!changed) break;
    }
    }
    // bed halo and gradients of the new mesh
    BGF_CUDA(cudaMemsetAsync(h->d_dzbdx, 0, (size_t)nb * 324 * sizeof(T), h->stream));
    BGF_CUDA(cudaMemsetAsync(h->d_dzbdy, 0, (size_t)nb * 324 * sizeof(T), h->stream));
    DevModel<T> m = dev_model<T>(h);
    int nl = h->fast ? fa::launch_bed_init<T>(m, step_params<T>(h), (T*)h->d_zb, (T*)h->d_dzbdx, (T*)h->d_dzbdy, h->stream)
                     : ex::launch_bed_init<T>(m, step_params<T>(h), (T*)h->d_zb, (T*)h->d_dzbdx, (T*)h->d_dzbdy, h->stream);
    h->launches += nl;
    BGF_CUDA(cudaGetLastError());
    BGF_CUDA(cudaStreamSynchronize(h->stream));
    if (changed_any && (rc = rebuild_segments(h))) return rc;
    free_graphs(h);
    if (niter) *niter = it;
    return BGF_OK;
}

// ---------------------------------------------------------------- adaptation tables on the device

// The level grids of the device table rebuild: levels 0..maxlevel of the domain's
// level-0 block extent.  False when the mesh or its size leaves the device path
// out (a level below 0, more than 16 levels, grids above 64 M entries).
static bool adapt_grid_spec(const bgf_handle* h, int maxlevel, adapt::GridSpec& gs)
{
    if (h->P.minlevel < 0 || maxlevel < 0 || maxlevel > 15) return false;
    const int nb = h->nblkmem;
    (void)nb;
    int nbx0 = 0, nby0 = 0;
    for (int ibl = 0; ibl < h->nblk; ibl++) {
        const int ib = h->active[ibl];
        const int l = h->level[ib];
        if (l < 0 || l > maxlevel) return false;
        const double dxl = h->P.dx / (double)(1 << l);
        const int bx = (int)floor((h->bxo[ib] / dxl - 0.5) / 16.0 + 0.5);
        const int by = (int)floor((h->byo[ib] / dxl - 0.5) / 16.0 + 0.5);
        if (bx < 0 || by < 0) return false;
        nbx0 = std::max(nbx0, (bx >> l) + 1);
        nby0 = std::max(nby0, (by >> l) + 1);
    }
    gs.nlev = maxlevel + 1;
    long long tot = 0;
    for (int l = 0; l < 16; l++) {
        gs.off[l] = 0;
        gs.w[l] = gs.h[l] = 0;
        if (l >= gs.nlev) continue;
        gs.off[l] = (int)tot;
        gs.w[l] = nbx0 << l;
        gs.h[l] = nby0 << l;
        tot += (long long)gs.w[l] * gs.h[l];
        if (tot > (64ll << 20)) return false;
    }
    gs.total = tot;
    return true;
}

// Scratch of the device table work, carved from one allocation sized for nblkmem.
static int adapt_scratch(bgf_handle* h, const adapt::GridSpec& gs, adapt::DevAdaptScratch& S, int*& d_err)
{
    const size_t nb = (size_t)h->nblkmem;
    struct Piece {
        void** p;
        size_t bytes;
    };
    const size_t ntile = nb / 1024 + 2;
    Piece pieces[] = {
        {(void**)&S.pos, nb * 4},     {(void**)&S.parent, nb},     {(void**)&S.gone, nb},
        {(void**)&S.fr, nb * 4},      {(void**)&S.fq, nb * 4},     {(void**)&S.fk, nb * 4},
        {(void**)&S.ff, nb * 4},      {(void**)&S.sr, nb * 4},     {(void**)&S.sq, nb * 4},
        {(void**)&S.sk, nb * 4},      {(void**)&S.sf, nb * 4},     {(void**)&S.tiles, ntile * 4},
        {(void**)&S.counts, 64},      {(void**)&S.avail, nb * 4},  {(void**)&S.nact, nb * 4},
        {(void**)&S.nlev, nb * 4},    {(void**)&S.nxo, nb * 8},    {(void**)&S.nyo, nb * 8},
        {(void**)&S.reflist, nb * 16}, {(void**)&S.bx, nb * 4},    {(void**)&S.by, nb * 4},
        {(void**)&S.nnbr, nb * 32},   {(void**)&d_err, 64},
    };
    size_t total = 0;
    for (auto& q : pieces) total += (q.bytes + 255) & ~(size_t)255;
    if (!h->d_adapt) {
        BGF_CUDA(dalloc(h, &h->d_adapt, total));
    }
    unsigned char* base = (unsigned char*)h->d_adapt;
    for (auto& q : pieces) {
        *q.p = base;
        base += (q.bytes + 255) & ~(size_t)255;
    }
    if (gs.total > h->agrids_cap) {
        if (h->d_agrids) dfree(h, (void*)h->d_agrids);
        h->d_agrids = nullptr;
        h->agrids_cap = 0;
        BGF_CUDA(dalloc(h, (void**)&h->d_agrids, sizeof(int) * (size_t)gs.total));
        h->agrids_cap = gs.total;
    }
    S.grids = h->d_agrids;
    return BGF_OK;
}

// The criterion on the device into d_flags (refine) and, for the criteria that
// have one, d_cflags (coarsen).  Returns in fill whether coarsen is !refine.
template <class T> static int launch_flag_criteria(bgf_handle* h, const bgf_adapt_param* ap, int& fill)
{
    DevModel<T> m = dev_model<T>(h);
    fill = 0;
    if (ap->criterion == BGF_ADAPT_TARGETLEVEL) {
        if (h->tmaps.empty()) {
            g_last_error = "the Targetlevel criterion needs at least one target-level map";
            return BGF_EINVAL;
        }
        for (const auto& g : h->tmaps) {
            adapt::launch_target_level<T>(m, g, std::isnan(h->P.xo) ? 0.0 : h->P.xo, std::isnan(h->P.yo) ? 0.0 : h->P.yo,
                                          h->P.dx, h->d_flags, h->d_cflags, h->stream);
            h->launches++;
        }
    } else if (ap->criterion == BGF_ADAPT_HGRAD) {
        adapt::launch_hgrad<T>(m, (const T*)h->d_dh, h->cur, h->P.eps, ap->arg1, ap->arg2, h->P.dx, h->d_flags,
                               h->d_cflags, h->stream);
        h->launches++;
    } else {
        const T* z = nullptr;
        int stride324 = 0;
        switch (ap->var) {
        case BGF_VAR_H: z = (const T*)h->d_h[h->cur]; break;
        case BGF_VAR_ZS: z = (const T*)h->d_dh; break;
        case BGF_VAR_U: z = (const T*)h->d_u[h->cur]; break;
        case BGF_VAR_V: z = (const T*)h->d_v[h->cur]; break;
        case BGF_VAR_ZB: z = (const T*)h->d_zb; stride324 = 1; break;
        default: return BGF_EINVAL;
        }
        adapt::launch_criteria<T>(m, z, stride324, ap->criterion, (T)ap->arg1, (T)ap->arg2, h->d_flags, h->stream);
        h->launches++;
        fill = 1;
    }
    BGF_CUDA(cudaGetLastError());
    return BGF_OK;
}

// Boundary segments after a pass: the children on a listed side inherit it; a
// merged quad's blocks give way to the parent, listed once.  kids(ib, out[3]) and
// parent(ib) describe the pass.
template <class Kids, class Parent> static void segments_after_pass(bgf_handle* h, Kids kids, Parent parent)
{
    const int nb = h->nblkmem;
    const int kids_side[4][2] = {{0, 2}, {1, 3}, {2, 3}, {0, 1}};  // left, right, top, bot: child slots
    for (HostSeg& sg : h->segs)
        for (int sidx = 0; sidx < 4; sidx++) {
            std::vector<int> out;
            for (int ib : sg.blk[sidx]) {
                int k3[3];
                if (ib >= 0 && ib < nb && kids(ib, k3)) {
                    const int q4[4] = {ib, k3[0], k3[1], k3[2]};
                    out.push_back(q4[kids_side[sidx][0]]);
                    out.push_back(q4[kids_side[sidx][1]]);
                } else if (ib >= 0 && ib < nb && parent(ib) >= 0) {
                    const int p = parent(ib);
                    if (std::find(out.begin(), out.end(), p) == out.end()) out.push_back(p);
                } else {
                    out.push_back(ib);
                }
            }
            sg.blk[sidx] = out;
        }
}

// adapt_t with the sanity pass and the tables on the device (same results); the
// host mirrors of the tables are refreshed once at the end.
template <class T>
static int adapt_dev_t(bgf_handle* h, const bgf_adapt_param* ap, const adapt::GridSpec& gs, int* niter,
                       bool& changed_any)
{
    const int nb = h->nblkmem;
    int rc = alloc_amr(h);  // stage tiles double as the old-mesh halo tiles
    if (rc) return rc;
    adapt::DevAdaptScratch S;
    int* d_err = nullptr;
    if ((rc = adapt_scratch(h, gs, S, d_err))) return rc;
    BGF_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), h->stream));
    zs_from_state<T>(h);
    const int maxit = ap->maxiteration > 0 ? ap->maxiteration : 20;
    const int allow = ap->allow_coarsen ? 1 : 0;
    int it = 0;
    changed_any = false;
    while (it < maxit) {
        it++;
        int fill = 0;
        if ((rc = launch_flag_criteria<T>(h, ap, fill))) return rc;
        const adapt::DevTables t{h->d_active, h->nblk, nb, h->d_level, h->d_nbr, h->d_bxo, h->d_byo};
        h->launches += adapt::dev_sanity(t, S, h->d_flags, h->d_cflags, h->P.minlevel, h->P.maxlevel, allow, fill,
                                         h->P.dx, h->stream);
        h->launches += adapt::dev_tables_count(t, S, h->d_flags, h->d_cflags, h->stream);
        BGF_CUDA(cudaGetLastError());
        int cnt[5];
        BGF_CUDA(cudaMemcpyAsync(cnt, S.counts, sizeof(int) * 4, cudaMemcpyDeviceToHost, h->stream));
        BGF_CUDA(cudaMemcpyAsync(cnt + 4, d_err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
        BGF_CUDA(cudaStreamSynchronize(h->stream));
        const int nref = cnt[0], nq = cnt[1], nkeep = cnt[2], nfree = cnt[3];
        if (cnt[4]) {
            g_last_error = "device adaptation: a block lies outside the level grids";
            return BGF_EINVAL;
        }
        if (3 * nref > nfree) {
            g_last_error = "refinement needs more block slots than nblkmem";
            return BGF_ENOMEM;
        }
        const bool changed = nref > 0 || nq > 0;
        adapt::AdaptDev<T> a = adapt_dev<T>(h);
        DevModel<T> m = dev_model<T>(h);
        if (changed) {
            const int nnew = nkeep + 3 * nref;
            h->launches += adapt::dev_tables_build(t, S, h->d_flags, h->d_cflags, h->P.dx, h->dbl, nkeep, nnew,
                                                   h->d_child, h->d_quads, gs, d_err, h->stream);
            // children and merged quads from the old mesh (old tables still in place)
            h->launches += adapt::launch_children<T>(m, a, h->cur, h->has_cf ? (T*)h->d_cf : nullptr,
                                                     h->has_rainmask ? h->d_rainmask : nullptr, h->d_quads, nq,
                                                     nref > 0, h->stream);
            BGF_CUDA(cudaGetLastError());
            if (!h->segs.empty()) {
                std::vector<int> rl((size_t)4 * nref), ql((size_t)4 * nq);
                if (nref)
                    BGF_CUDA(cudaMemcpyAsync(rl.data(), S.reflist, sizeof(int) * rl.size(), cudaMemcpyDeviceToHost,
                                             h->stream));
                if (nq)
                    BGF_CUDA(cudaMemcpyAsync(ql.data(), h->d_quads, sizeof(int) * ql.size(), cudaMemcpyDeviceToHost,
                                             h->stream));
                BGF_CUDA(cudaStreamSynchronize(h->stream));
                std::unordered_map<int, int> kid_at, parent_of;
                for (int k = 0; k < nref; k++) kid_at[rl[4 * k]] = k;
                for (int k = 0; k < nq; k++)
                    for (int q = 0; q < 4; q++) parent_of[ql[4 * k + q]] = ql[4 * k];
                segments_after_pass(
                    h,
                    [&](int ib, int* out) {
                        auto f = kid_at.find(ib);
                        if (f == kid_at.end()) return false;
                        for (int q = 0; q < 3; q++) out[q] = rl[4 * f->second + 1 + q];
                        return true;
                    },
                    [&](int ib) {
                        auto f = parent_of.find(ib);
                        return f == parent_of.end() ? -1 : f->second;
                    });
            }
            // the new tables replace the old ones
            BGF_CUDA(cudaMemcpyAsync(h->d_active, S.nact, sizeof(int) * nnew, cudaMemcpyDeviceToDevice, h->stream));
            BGF_CUDA(cudaMemcpyAsync(h->d_level, S.nlev, sizeof(int) * nb, cudaMemcpyDeviceToDevice, h->stream));
            BGF_CUDA(cudaMemcpyAsync(h->d_nbr, S.nnbr, sizeof(int) * 8 * (size_t)nb, cudaMemcpyDeviceToDevice, h->stream));
            BGF_CUDA(cudaMemcpyAsync(h->d_bxo, S.nxo, sizeof(double) * nb, cudaMemcpyDeviceToDevice, h->stream));
            BGF_CUDA(cudaMemcpyAsync(h->d_byo, S.nyo, sizeof(double) * nb, cudaMemcpyDeviceToDevice, h->stream));
            h->nblk = nnew;
            changed_any = true;
            m = dev_model<T>(h);
        }
        adapt::launch_bed<T>(m, a, step_params<T>(h), h->cur, (T*)h->d_zb, std::isnan(h->P.xo) ? 0.0 : h->P.xo,
                             std::isnan(h->P.yo) ? 0.0 : h->P.yo, h->d_bxo, h->d_byo, h->P.mask,
                             h->has_rainmask ? h->d_rainmask : nullptr, h->stream);
        h->launches++;
        BGF_CUDA(cudaGetLastError());
        if (!changed) break;
    }
    // host mirrors of the final tables
    int err = 0;
    h->active.assign(h->nblk, 0);
    std::vector<int> nbrT((size_t)8 * nb);
    BGF_CUDA(cudaMemcpyAsync(h->active.data(), h->d_active, sizeof(int) * h->nblk, cudaMemcpyDeviceToHost, h->stream));
    BGF_CUDA(cudaMemcpyAsync(h->level.data(), h->d_level, sizeof(int) * nb, cudaMemcpyDeviceToHost, h->stream));
    BGF_CUDA(cudaMemcpyAsync(h->nbr.data(), h->d_nbr, sizeof(int) * 8 * (size_t)nb, cudaMemcpyDeviceToHost, h->stream));
    BGF_CUDA(cudaMemcpyAsync(h->bxo.data(), h->d_bxo, sizeof(double) * nb, cudaMemcpyDeviceToHost, h->stream));
    BGF_CUDA(cudaMemcpyAsync(h->byo.data(), h->d_byo, sizeof(double) * nb, cudaMemcpyDeviceToHost, h->stream));
    BGF_CUDA(cudaMemcpyAsync(&err, d_err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    BGF_CUDA(cudaStreamSynchronize(h->stream));
    if (err) {
        g_last_error = "device adaptation: a block lies outside the level grids";
        return BGF_EINVAL;
    }
    if ((rc = upload_tables(h))) return rc;
    if (niter) *niter = it;
    return BGF_OK;
}

int bgf_set_adapt_mode(bgf_handle* h, int mode)
{
    if (!h || (mode != 0 && mode != 1)) return BGF_EINVAL;
    h->adapt_mode = mode;
    return BGF_OK;
}

int bgf_adapt(bgf_handle* h, const bgf_adapt_param* ap, int* nblk, int* niter)
{
    int rc = check_ready(h);
    if (rc) return rc;
    if ((rc = check_adapt_param(ap))) return rc;
    if (!h->d_dem) {
        g_last_error = "bgf_adapt needs the bathymetry grid (bgf_set_bathy)";
        return BGF_ESTATE;
    }
    if (h->split) {
        g_last_error = "bgf_adapt does not support split precision";
        return BGF_EINVAL;
    }
    adapt::GridSpec gs;
    const bool on_device = h->adapt_mode && adapt_grid_spec(h, std::max(h->P.maxlevel, h->maxlev), gs);
    rc = h->dbl ? adapt_t<double>(h, ap, niter, on_device ? &gs : nullptr)
                : adapt_t<float>(h, ap, niter, on_device ? &gs : nullptr);
    if (nblk) *nblk = h->nblk;
    return rc;
}

int bgf_get_bed(bgf_handle* h, void* zb)
{
    if (!h || !zb) return BGF_EINVAL;
    if (!h->has_bed) return BGF_ESTATE;
    int rc = set_device(h);
    if (rc) return rc;
    BGF_CUDA(cudaStreamSynchronize(h->stream));
    BGF_CUDA(copy_on(h->stream, zb, h->d_zb, (size_t)h->nblkmem * 324 * h->esz, cudaMemcpyDeviceToHost));
    return BGF_OK;
}

int bgf_set_grid(bgf_handle* h, int grid)
{
    if (!h || grid < 0) return BGF_EINVAL;
    h->grid = grid;
    free_graphs(h);
    return BGF_OK;
}

int bgf_set_gauges(bgf_handle* h, int n, const int* block, const int* i, const int* j)
{
    if (!h || n < 0 || (n > 0 && (!block || !i || !j))) return BGF_EINVAL;
    if (!h->has_blocks) return BGF_ESTATE;
    int rc = set_device(h);
    if (rc) return rc;
    std::vector<int> cells(n);
    std::vector<uint8_t> isact(h->nblkmem, 0);
    for (int ibl = 0; ibl < h->nblk; ibl++) isact[h->active[ibl]] = 1;
    for (int k = 0; k < n; k++) {
        if (block[k] < 0 || block[k] >= h->nblkmem || !isact[block[k]] || i[k] < 0 || i[k] >= 16 || j[k] < 0 ||
            j[k] >= 16) {
            g_last_error = "gauge outside the active blocks";
            return BGF_EINVAL;
        }
        cells[k] = block[k] * 256 + j[k] * 16 + i[k];
    }
    BGF_CUDA(cudaStreamSynchronize(h->stream));
    if ((rc = gauge_drain_handle(h))) return rc;
    if ((rc = gauge_alloc(h, h->gauges, cells, {}, 4096))) return rc;
    h->gauge_t.clear();
    h->gauge_v.clear();
    h->gauge_nhost = n;
    free_graphs(h);
    return BGF_OK;
}

int bgf_read_gauges(bgf_handle* h, int max_samples, double* times, double* values, int* nsamples, int64_t* lost)
{
    if (!h || max_samples < 0 || !nsamples) return BGF_EINVAL;
    int rc = set_device(h);
    if (rc) return rc;
    if ((rc = gauge_drain_handle(h))) return rc;
    const int n = h->gauge_nhost;
    const size_t have = n > 0 ? h->gauge_t.size() / n : 0;
    const size_t take = std::min(have, (size_t)max_samples);
    if (take && (!times || !values)) return BGF_EINVAL;
    if (take) {
        std::copy(h->gauge_t.begin(), h->gauge_t.begin() + take * n, times);
        std::copy(h->gauge_v.begin(), h->gauge_v.begin() + take * n * 4, values);
        h->gauge_t.erase(h->gauge_t.begin(), h->gauge_t.begin() + take * n);
        h->gauge_v.erase(h->gauge_v.begin(), h->gauge_v.begin() + take * n * 4);
    }
    *nsamples = (int)take;
    if (lost) *lost = h->gauge_lost;
    return BGF_OK;
}

int bgf_set_kernel_layout(bgf_handle* h, int cells_per_thread)
{
    if (!h || cells_per_thread < 1 || cells_per_thread > 3) return BGF_EINVAL;
    h->gen = cells_per_thread;
    free_graphs(h);
    return BGF_OK;
}

// ---------------------------------------------------------------- launch-shape autotuner

// Launch shapes tried by the autotuner: one CTA per block (0), then persistent grids
// of 2, 3, 4, 5, 6 and 8 CTAs per SM (only those smaller than the block count).
static std::vector<int> tune_candidates(int dev, int nblk)
{
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    std::vector<int> c = {0};
    for (int k : {2, 3, 4, 5, 6, 8})
        if (k * sms < nblk) c.push_back(k * sms);
    return c;
}

// Device bytes to save and restore around tuning runs: (pointer, bytes) pairs.
struct TuneSave {
    std::vector<std::pair<void*, size_t>> areas;
    void* d_copy = nullptr;
    size_t total = 0;
};

static int tune_save(bgf_handle* h, TuneSave& t)
{
    for (auto& a : t.areas) t.total += a.second;
    if (dalloc(h, &t.d_copy, std::max<size_t>(t.total, 1)) != cudaSuccess) return BGF_ENOMEM;
    size_t off = 0;
    for (auto& a : t.areas) {
        BGF_CUDA(cudaMemcpyAsync((char*)t.d_copy + off, a.first, a.second, cudaMemcpyDeviceToDevice, h->stream));
        off += a.second;
    }
    BGF_CUDA(cudaStreamSynchronize(h->stream));
    return BGF_OK;
}

static int tune_restore(bgf_handle* h, TuneSave& t)
{
    size_t off = 0;
    for (auto& a : t.areas) {
        BGF_CUDA(cudaMemcpyAsync(a.first, (char*)t.d_copy + off, a.second, cudaMemcpyDeviceToDevice, h->stream));
        off += a.second;
    }
    BGF_CUDA(cudaStreamSynchronize(h->stream));
    dfree(h, t.d_copy);
    t.d_copy = nullptr;
    return BGF_OK;
}

// Times `steps` steps (after two untimed ones) of the handle's step graphs with the
// current launch shape, from the time slot written by the caller.
static int tune_time_handle(bgf_handle* h, int steps, double* ms)
{
    int rc = build_graphs(h);
    if (rc) return rc;
    const int p0 = h->parity;
    BGF_CUDA(cudaGraphLaunch(h->graph[p0], h->stream));
    BGF_CUDA(cudaEventRecord(h->ev0, h->stream));
    for (int k = 0; k < (steps + 1) / 2; k++) BGF_CUDA(cudaGraphLaunch(h->graph[p0], h->stream));
    BGF_CUDA(cudaEventRecord(h->ev1, h->stream));
    BGF_CUDA(cudaStreamSynchronize(h->stream));
    float t = 0.f;
    BGF_CUDA(cudaEventElapsedTime(&t, h->ev0, h->ev1));
    *ms = t / (2 * ((steps + 1) / 2));
    return BGF_OK;
}

int bgf_autotune(bgf_handle* h, const bgf_loop* loop, int steps, int* grid, double* ms_per_step)
{
    int rc = check_ready(h);
    if (rc) return rc;
    if (!loop || steps <= 0) return BGF_EINVAL;
    if (h->amr) {
        // the multi-level chain launches one CTA per block; nothing to choose
        if (grid) *grid = 0;
        if (ms_per_step) *ms_per_step = 0.0;
        return BGF_OK;
    }
    BGF_CUDA(cudaStreamSynchronize(h->stream));
    const size_t nb = h->nblkmem, es = h->esz;
    TuneSave save;
    for (int b = 0; b < 2; b++)
        for (void* a : {h->d_h[b], h->d_u[b], h->d_v[b]}) save.areas.push_back({a, nb * 256 * es});
    save.areas.push_back({h->d_qmean, nb * 64 * sizeof(float)});
    save.areas.push_back({h->d_time, 2 * sizeof(TimeState)});
    if ((rc = tune_save(h, save))) return rc;
    const int cur0 = h->cur, par0 = h->parity, grid0 = h->grid;
    int best = grid0;
    double best_ms = INFINITY;
    for (int g : tune_candidates(h->dev, h->nblk)) {
        h->grid = g;
        h->cur = cur0;
        h->parity = par0;
        if ((rc = write_time_slot(h, loop, INFINITY, 0.0, (long long)1 << 60))) break;
        double ms = 0.0;
        if ((rc = tune_time_handle(h, steps, &ms))) break;
        if (ms < best_ms) {
            best_ms = ms;
            best = g;
        }
    }
    h->cur = cur0;
    h->parity = par0;
    int rc2 = tune_restore(h, save);
    if (rc) {
        h->grid = grid0;
        free_graphs(h);
        return rc;
    }
    if (rc2) return rc2;
    h->grid = best;
    free_graphs(h);
    if (grid) *grid = best;
    if (ms_per_step) *ms_per_step = best_ms;
    return BGF_OK;
}

// ---------------------------------------------------------------- batched pools

#include "bgf_pool.inc"
