// Allocation-free flow step: the same two kernels as bgf_flow_step, with all
// their scratch memory in one file-scope device array instead of handle-owned
// allocations.
//
// Who needs it: host programs that must not change their device-memory
// footprint once they are running.  An operational flood-forecast service that
// reserves its GPU memory pool at start-up and treats any later cudaMalloc as a
// fault, or a host model that already owns every device array (as BG_Flood's
// own Model<T> does) and steps it from code where a cudaMalloc / cudaFree -- which
// can synchronise the whole device -- is not allowed, cannot create a handle.
// They pass device pointers to their own state and tables and get one step.
//
// The scratch array is sized for at most BGF_NOALLOC_MAX_BLOCKS blocks in double
// precision; every GPU that loads the library holds it until the process exits.
// All calls share it and it keeps the contents of the last call, so calls whose
// GPU work overlaps (two streams, two host threads) race on it.  The absorbing-
// boundary running means live in it too and carry from call to call, as the
// reference's qmean carries from step to step (src/Boundary.cu:481-537); they are
// cleared at the first set-up on a device and when the caller asks (reset_means).
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <mutex>
#include <string>

#include "../../include/bg_flood_b200.h"
#include "bgf_flow.cuh"
#include "bgf_internal.h"

using namespace bgf;

namespace {

constexpr size_t kMaxBlocks = BGF_NOALLOC_MAX_BLOCKS;
// layout (bytes, every part 256-aligned): dh, dhu, dhv (double-sized), qmean,
// two time slots, two dt slots, error word, the four-entry segment table
constexpr size_t kAdv = kMaxBlocks * 256 * sizeof(double);
constexpr size_t kQmean = kMaxBlocks * 64 * sizeof(float);
constexpr size_t kOffDh = 0, kOffDhu = kAdv, kOffDhv = 2 * kAdv, kOffQmean = 3 * kAdv;
constexpr size_t kOffTime = kOffQmean + kQmean;
constexpr size_t kOffDt = kOffTime + 256;
constexpr size_t kOffErr = kOffDt + 256;
constexpr size_t kOffSegs = kOffErr + 256;
constexpr size_t kBytes = kOffSegs + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kBytes];

// Device address of g_noalloc_scratch per device, found once per device.
constexpr int kMaxDevices = 64;
unsigned char* g_scratch_ptr[kMaxDevices] = {nullptr};
std::mutex g_setup_mutex;

// The set-up copies run on the caller's stream and complete before the step is
// queued behind them (a non-blocking caller stream is not ordered with the legacy
// default stream of cudaMemcpy).
int scratch_for_device(int dev, cudaStream_t st, unsigned char** out)
{
    if (dev < 0 || dev >= kMaxDevices) return BGF_EINVAL;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            bgf::set_last_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            return BGF_ECUDA;
        }
        // segment table: entry k is a boundary of type k without a water-level series
        SegDev segs[4];
        for (int k = 0; k < 4; k++) segs[k] = SegDev{k, 0, 0, 0};
        e = cudaMemcpyAsync((unsigned char*)p + kOffSegs, segs, sizeof(segs), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            bgf::set_last_error(std::string("scratch set-up: ") + cudaGetErrorString(e));
            return BGF_ECUDA;
        }
        // the running means start from zero, as the reference's segment sides do
        e = cudaMemsetAsync((unsigned char*)p + kOffQmean, 0, kQmean, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            bgf::set_last_error(std::string("scratch set-up: ") + cudaGetErrorString(e));
            return BGF_ECUDA;
        }
        g_scratch_ptr[dev] = (unsigned char*)p;
    }
    *out = g_scratch_ptr[dev];
    return BGF_OK;
}

template <class T>
int step_noalloc(const bgf_param* P, const bgf_noalloc_args* a, bgf_loop* loop, cudaStream_t st, unsigned char* sc)
{
    cudaError_t e = P->fastmath ? fast::configure_kernels<T>() : exact::configure_kernels<T>();
    if (e != cudaSuccess) {
        bgf::set_last_error(std::string("configure kernels: ") + cudaGetErrorString(e));
        return BGF_ENOKERNEL;
    }
    DevModel<T> m;
    memset(&m, 0, sizeof(m));
    m.nblk = a->nblk;
    m.nblkmem = a->nblkmem;
    m.active = a->active;
    m.level = a->level;
    m.nbr = a->nbr;
    m.zb = (const T*)a->zb;
    m.dzbdx = (const T*)a->dzbdx;
    m.dzbdy = (const T*)a->dzbdy;
    m.cf = nullptr;
    m.rainmask = nullptr;
    m.bndseg = a->bndtype;
    m.qmean = (float*)(sc + kOffQmean);
    m.segs = (const SegDev*)(sc + kOffSegs);
    m.h[0] = (T*)a->h_in;
    m.u[0] = (T*)a->u_in;
    m.v[0] = (T*)a->v_in;
    m.h[1] = (T*)a->h_out;
    m.u[1] = (T*)a->u_out;
    m.v[1] = (T*)a->v_out;
    m.dh = (T*)(sc + kOffDh);
    m.dhu = (T*)(sc + kOffDhu);
    m.dhv = (T*)(sc + kOffDhv);
    m.time = (TimeState*)(sc + kOffTime);
    m.dtmin = (unsigned long long*)(sc + kOffDt);
    m.err = (int*)(sc + kOffErr);
    m.scen = nullptr;
    m.sparams = nullptr;
    m.lead = nullptr;
    m.hmax = nullptr;
    m.checklev = 1;
    m.datum = nullptr;
    m.rmap = RainMapDev{};
    m.rivers = nullptr;
    m.riv_t = nullptr;
    m.riv_q = nullptr;
    m.bxo = nullptr;
    m.byo = nullptr;

    StepParams<T> p;
    p.g = (T)P->g;
    p.eps = (T)P->eps;
    p.CFL = (T)P->CFL;
    p.theta = (T)P->theta;
    p.delta0 = (T)P->delta;
    p.delta0_d = P->delta;
    p.epsi = std::nextafter((T)1.0, (T)2.0) - (T)1.0;
    p.epsface = (T)P->eps + p.epsi;
    p.fc = (T)((double)std::sin((T)(P->lat * 3.14159265 / 180.0)) * 3.14159265 / (double)(T)21600.0);
    p.eps_d = P->eps;
    p.dtparam = P->dt;
    p.bndfiltertime = P->bndfiltertime;
    p.bndrelaxtime = P->bndrelaxtime;
    p.bndtaper = P->bndtaper;
    p.inittime = P->inittime;
    p.zsinit = P->zsinit;
    p.zsoffset = std::isnan(P->zsoffset) ? 0.0 : P->zsoffset;
    p.dtmin = P->dtmin;
    p.cf = (T)P->cf;
    p.frictionmodel = P->frictionmodel;
    p.forcemass = P->ForceMassConserve;
    p.has_cf = 0;
    p.has_rain = 0;
    p.nseg = 4;
    p.rain_n = 0;
    p.rain_off = 0;
    p.rain_sorted = 0;
    p.xo_d = 0.0;
    p.yo_d = 0.0;
    p.nriver = 0;
    p.rain_map = 0;
    p.riv_first = 0;

    // per-call state: time slot 0 from the caller's loop, the dt minimum and the error
    // word; the absorbing-boundary running means persist unless the caller resets them
    TimeState ts;
    memset(&ts, 0, sizeof(ts));
    ts.totaltime = loop->totaltime;
    ts.dt = loop->dt;
    ts.dtmax = loop->dtmax;
    ts.nextoutputtime = loop->nextoutputtime;
    ts.endtime = INFINITY;
    ts.maxsteps = 1;
    T inv = (T)1.0 / p.epsi;
    unsigned long long bits = 0;
    memcpy(&bits, &inv, sizeof(T));
    if ((e = cudaMemcpyAsync(m.time, &ts, sizeof(ts), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(m.dtmin, &bits, sizeof(bits), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemsetAsync(m.err, 0, sizeof(int), st)) != cudaSuccess ||
        (a->reset_means &&
         (e = cudaMemsetAsync(m.qmean, 0, (size_t)a->nblkmem * 64 * sizeof(float), st)) != cudaSuccess)) {
        bgf::set_last_error(std::string("scratch reset: ") + cudaGetErrorString(e));
        return BGF_ECUDA;
    }
    if (P->fastmath) {
        fast::launch_flux<T>(m, p, P->engine, 0, st, 0);
        fast::launch_update<T>(m, p, P->engine, 0, st, 0);
    } else {
        exact::launch_flux<T>(m, p, P->engine, 0, st, 0);
        exact::launch_update<T>(m, p, P->engine, 0, st, 0);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) {
        bgf::set_last_error(std::string("launch: ") + cudaGetErrorString(e));
        return BGF_ECUDA;
    }
    TimeState nt;
    int err = 0;
    if ((e = cudaMemcpyAsync(&nt, m.time + 1, sizeof(nt), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&err, m.err, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess) {
        bgf::set_last_error(std::string("readback: ") + cudaGetErrorString(e));
        return BGF_ECUDA;
    }
    if (err) {
        bgf::set_last_error("mesh has cross-level neighbours, which this entry point does not support");
        return BGF_EINVAL;
    }
    loop->dt = nt.dt;
    loop->dtmax = nt.dtmax;
    if (nt.status == BGF_ENAN) {
        bgf::set_last_error("non-finite value in the state");
        return BGF_ENAN;
    }
    return BGF_OK;
}

}  // namespace

int bgf_flow_step_noalloc(const bgf_param* p, const bgf_noalloc_args* a, bgf_loop* loop, void* stream)
{
    if (!p || !a || !loop) return BGF_EINVAL;
    if (a->nblk <= 0 || a->nblkmem <= 0 || a->nblk > a->nblkmem) return BGF_EINVAL;
    if ((size_t)a->nblkmem > kMaxBlocks) {
        bgf::set_last_error("nblkmem exceeds BGF_NOALLOC_MAX_BLOCKS");
        return BGF_EINVAL;
    }
    if (p->engine != 1 && p->engine != 2) return BGF_EINVAL;
    if (!a->active || !a->level || !a->nbr || !a->zb || !a->bndtype || !a->h_in || !a->u_in || !a->v_in ||
        !a->h_out || !a->u_out || !a->v_out)
        return BGF_EINVAL;
    if (p->engine == 1 && (!a->dzbdx || !a->dzbdy)) return BGF_EINVAL;
    // the kernels copy each block's bed tile into shared memory in 16-byte pieces
    if (((uintptr_t)a->zb & 15) != 0) {
        bgf::set_last_error("zb must be 16-byte aligned (as cudaMalloc returns it)");
        return BGF_EINVAL;
    }
    if (p->frictionmodel != 0 && p->frictionmodel != -1 && p->frictionmodel != 1) return BGF_EINVAL;
    if (p->splitprecision || p->conserveElevation) {
        bgf::set_last_error("the allocation-free step takes neither split precision nor conserveElevation");
        return BGF_EINVAL;
    }
    int caller_dev = 0;
    (void)cudaGetLastError();  // a launch error other code left pending is not this call's
    if (cudaGetDevice(&caller_dev) != cudaSuccess) return BGF_ECUDA;
    if (cudaSetDevice(p->GPUDEVICE) != cudaSuccess) return BGF_ECUDA;
    unsigned char* sc = nullptr;
    cudaStream_t st = (cudaStream_t)stream;
    int rc = scratch_for_device(p->GPUDEVICE, st, &sc);
    if (!rc) {
        rc = p->doubleprecision ? step_noalloc<double>(p, a, loop, st, sc) : step_noalloc<float>(p, a, loop, st, sc);
    }
    cudaSetDevice(caller_dev);
    return rc;
}
