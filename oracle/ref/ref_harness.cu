// Test harness over the UNMODIFIED reference BG_Flood sources (compiled in
// place by oracle/ref/Makefile).  It is test infrastructure: tests/ and the
// CPU-baseline leg of bench.py load oracle/_ref/libbgf_ref.so to run the
// reference's own FlowCPU (src/FlowCPU.cu:15) -- and, on a GPU box, its
// FlowGPU (src/FlowGPU.cu:14) -- on in-memory setups, exactly the way the
// reference's own tests drive it (src/Testing.cu:418-629: Param built in
// memory, a flat bathymetry, checkparamsanity, InitMesh, InitialConditions,
// then the evolving fields overwritten before the time loop).
//
// The harness exposes a small extern "C" surface (ref_*) with plain pointers.
#include "General.h"
#include "Param.h"
#include "Arrays.h"
#include "Forcing.h"
#include "ReadInput.h"
#include "Mesh.h"
#include "InitialConditions.h"
#include "FlowCPU.h"
#include "FlowGPU.h"
#include "Setup_GPU.h"
#include "Mainloop.h"
#include "Adaptation.h"
#include "AdaptCriteria.h"
#include "Updateforcing.h"
#include "Gradients.h"
#include "Halo.h"
#include "ReadForcing.h"

#include <memory>
#include <vector>
#include <sstream>

namespace {

struct RefBase {
    virtual ~RefBase() {}
    virtual int step(int nsteps, double* dts) = 0;
    virtual int get(const char* name, double* out) = 0;
    virtual int get_blocks(int* level, double* xo, double* yo, int* nbr8) = 0;
    virtual int adapt() = 0;
    virtual int set(const char* name, const double* buq) = 0;
    virtual int reinit(double nextout) = 0;
    virtual int get_active(int* out) = 0;
    virtual int adaptation() = 0;
    virtual int flags(unsigned char* refine, unsigned char* coarsen) = 0;
    virtual int set_bathy(int nx, int ny, double xo, double yo, double dx, const double* val) = 0;
    virtual int setup_loaded() = 0;
    virtual double loop_nextoutputtime() = 0;
    virtual int get_active_cell(int* out) = 0;
    virtual double loop_dtmax() = 0;
    Param P;
    Forcing<float> F;
    double totaltime = 0.0, nextoutputtime = 0.0, dtmax = 0.0;
    int gpu = -1;
};

template <class T> struct RefModel : RefBase {
    Model<T> M;
    Model<T> Mg;
    Loop<T> L;
    Loop<T> Lg;

    int setup(const char* paramtext, int nx, int ny, double dx, double xo, double yo,
              const double* zb, const double* h, const double* u, const double* v,
              const double* cf, double nextout)
    {
        // Parameters through the reference's own key parser (src/ReadInput.cu:162).
        std::istringstream ss(paramtext ? paramtext : "");
        std::string line;
        int engine_override = -1;
        while (std::getline(ss, line)) {
            if (line.empty()) continue;
            // The reference parser maps every "engine" value other than 1 to engine 5
            // (src/ReadInput.cu:193-213), so engine 2 (Kurganov) can only be chosen in
            // code, as src/Testing.cu does; "harness_engine = N" does that here.
            if (line.rfind("harness_engine", 0) == 0) {
                engine_override = std::stoi(line.substr(line.find('=') + 1));
                continue;
            }
            P = readparamstr(line, P);
            F = readparamstr(line, F);
        }
        if (engine_override > 0) P.engine = engine_override;
        P.dx = dx;
        P.xo = xo;
        P.yo = yo;
        P.xmax = xo + nx * dx;
        P.ymax = yo + ny * dx;
        gpu = P.GPUDEVICE;

        // Flat 3x3 bathymetry covering the domain, as src/Testing.cu:490-513.
        StaticForcingP<float> bathy;
        F.Bathy.push_back(bathy);
        F.Bathy[0].xo = xo - dx;
        F.Bathy[0].yo = yo - dx;
        F.Bathy[0].nx = 3;
        F.Bathy[0].ny = 3;
        F.Bathy[0].dx = (nx * dx + 2 * dx) / 2.0;
        F.Bathy[0].dy = F.Bathy[0].dx;
        F.Bathy[0].xmax = F.Bathy[0].xo + 2 * F.Bathy[0].dx;
        F.Bathy[0].ymax = F.Bathy[0].yo + 2 * F.Bathy[0].dx;
        AllocateCPU(3, 3, F.Bathy[0].val);
        for (int k = 0; k < 9; k++) F.Bathy[0].val[k] = 0.0f;

        checkparamsanity(P, F);
        InitMesh(P, F, M);
        InitialConditions(P, F, M);

        // Overwrite the fields on interior cells (row-major global cell grid).
        int nbx = nx / 16;
        for (int ibl = 0; ibl < P.nblk; ibl++) {
            int ib = M.blocks.active[ibl];
            int bx = (int)llround(M.blocks.xo[ib] / (16.0 * dx));
            int by = (int)llround(M.blocks.yo[ib] / (16.0 * dx));
            (void)nbx;
            for (int iy = 0; iy < 16; iy++)
                for (int ix = 0; ix < 16; ix++) {
                    int n = memloc(P, ix, iy, ib);
                    size_t g = (size_t)(by * 16 + iy) * nx + (bx * 16 + ix);
                    M.zb[n] = T(zb[g]);
                    M.evolv.h[n] = T(h[g]);
                    M.evolv.u[n] = T(u[g]);
                    M.evolv.v[n] = T(v[g]);
                    M.evolv.zs[n] = M.zb[n] + M.evolv.h[n];
                    if (cf) M.cf[n] = T(cf[g]);
                }
        }
        // Bed halo and gradients, as src/Testing.cu:583-588.
        fillHaloC(P, M.blocks, M.zb);
        gradientC(P, M.blocks, M.zb, M.grad.dzbdx, M.grad.dzbdy);
        gradientHalo(P, M.blocks, M.zb, M.grad.dzbdx, M.grad.dzbdy);
        refine_linear(P, M.blocks, M.zb, M.grad.dzbdx, M.grad.dzbdy);
        gradientHalo(P, M.blocks, M.zb, M.grad.dzbdx, M.grad.dzbdy);

        L.hugenegval = std::numeric_limits<T>::min();
        L.hugeposval = std::numeric_limits<T>::max();
        L.epsilon = std::numeric_limits<T>::epsilon();
        L.totaltime = 0.0;
        L.nextoutputtime = nextout;
        L.dtmax = initdt(P, L, M);
        if (gpu >= 0) {
            SetupGPU(P, M, F, Mg);
            Lg.hugenegval = L.hugenegval;
            Lg.hugeposval = L.hugeposval;
            Lg.epsilon = L.epsilon;
            Lg.totaltime = L.totaltime;
            Lg.nextoutputtime = L.nextoutputtime;
            Lg.dtmax = L.dtmax;
            // SetupGPU copies the model state; the bed halo/gradients computed above are
            // copied again explicitly so the GPU starts from the same arrays.
            CopytoGPU(P.nblkmem, P.blksize, M.zb, Mg.zb);
            CopytoGPU(P.nblkmem, P.blksize, M.grad.dzbdx, Mg.grad.dzbdx);
            CopytoGPU(P.nblkmem, P.blksize, M.grad.dzbdy, Mg.grad.dzbdy);
        }
        return 0;
    }

    // The reference's own start-up after Readparamfile, readforcing and
    // checkparamsanity (src/BG_Flood.cu:132-152): InitMesh, InitialConditions,
    // InitialAdaptation, then the loop as InitLoop (src/Mainloop.cu:207-240) and
    // the first mapoutput (src/Mainloop.cu:323-340) leave it.  CPU only.
    int setup_loaded() override
    {
        gpu = -1;
        InitMesh(P, F, M);
        InitialConditions(P, F, M);
        InitialAdaptation(P, F, M);
        L.hugeposval = std::numeric_limits<T>::max();
        L.hugenegval = T(-1.0) * L.hugeposval;
        L.epsilon = std::numeric_limits<T>::epsilon();
        L.totaltime = P.totaltime;
        L.nextoutputtime = M.OutputT.empty() ? P.endtime : M.OutputT[0];
        L.dtmax = initdt(P, L, M);
        if (M.OutputT.size() > 1) L.nextoutputtime = std::min(M.OutputT[1], P.endtime);
        return 0;
    }

    // activeCell (rain mask) tiles in active-block order, 18x18 per block.
    int get_active_cell(int* out) override
    {
        for (int ibl = 0; ibl < P.nblk; ibl++) {
            int ib = M.blocks.active[ibl];
            for (int k = 0; k < P.blksize; k++) out[(size_t)ibl * P.blksize + k] = M.blocks.activeCell[(size_t)ib * P.blksize + k];
        }
        return P.nblk;
    }

    double loop_nextoutputtime() override { return gpu >= 0 ? Lg.nextoutputtime : L.nextoutputtime; }
    double loop_dtmax() override { return gpu >= 0 ? Lg.dtmax : L.dtmax; }

    int step(int nsteps, double* dts) override
    {
        for (int s = 0; s < nsteps; s++) {
            if (gpu >= 0) {
                updateforcing(P, Lg, F);
                FlowGPU(P, Lg, F, Mg);
                Lg.totaltime = Lg.totaltime + Lg.dt;
                if (dts) dts[s] = Lg.dt;
            } else {
                updateforcing(P, L, F);
                FlowCPU(P, L, F, M);
                L.totaltime = L.totaltime + L.dt;
                if (dts) dts[s] = L.dt;
            }
        }
        return 0;
    }

    T* field(const char* name, bool devicecopy)
    {
        Model<T>& X = M;
        std::string s(name);
        T* p = nullptr;
        if (s == "zs") p = X.evolv.zs;
        else if (s == "h") p = X.evolv.h;
        else if (s == "u") p = X.evolv.u;
        else if (s == "v") p = X.evolv.v;
        else if (s == "zb") p = X.zb;
        else if (s == "dzbdx") p = X.grad.dzbdx;
        else if (s == "dzbdy") p = X.grad.dzbdy;
        else if (s == "cf") p = X.cf;
        if (p && devicecopy && gpu >= 0) {
            T* pg = nullptr;
            if (s == "zs") pg = Mg.evolv.zs;
            else if (s == "h") pg = Mg.evolv.h;
            else if (s == "u") pg = Mg.evolv.u;
            else if (s == "v") pg = Mg.evolv.v;
            else if (s == "zb") pg = Mg.zb;
            else if (s == "dzbdx") pg = Mg.grad.dzbdx;
            else if (s == "dzbdy") pg = Mg.grad.dzbdy;
            else if (s == "cf") pg = Mg.cf;
            if (pg) cudaMemcpy(p, pg, sizeof(T) * (size_t)P.nblkmem * P.blksize, cudaMemcpyDeviceToHost);
        }
        return p;
    }

    // Full 18x18 tiles of every allocated block, in block-index order.
    int get(const char* name, double* out) override
    {
        T* p = field(name, true);
        if (!p) return -1;
        size_t n = (size_t)P.nblk * P.blksize;
        for (int ibl = 0; ibl < P.nblk; ibl++) {
            int ib = M.blocks.active[ibl];
            for (int k = 0; k < P.blksize; k++)
                out[(size_t)ibl * P.blksize + k] = double(p[(size_t)ib * P.blksize + k]);
        }
        (void)n;
        return 0;
    }

    int get_blocks(int* level, double* xo, double* yo, int* nbr8) override
    {
        for (int ibl = 0; ibl < P.nblk; ibl++) {
            int ib = M.blocks.active[ibl];
            if (level) level[ibl] = M.blocks.level[ib];
            if (xo) xo[ibl] = double(M.blocks.xo[ib]);
            if (yo) yo[ibl] = double(M.blocks.yo[ib]);
            if (nbr8) {
                int* q = nbr8 + 8 * ibl;
                q[0] = M.blocks.LeftBot[ib];  q[1] = M.blocks.LeftTop[ib];
                q[2] = M.blocks.RightBot[ib]; q[3] = M.blocks.RightTop[ib];
                q[4] = M.blocks.BotLeft[ib];  q[5] = M.blocks.BotRight[ib];
                q[6] = M.blocks.TopLeft[ib];  q[7] = M.blocks.TopRight[ib];
            }
        }
        return P.nblk;
    }

    // The reference's own initial mesh adaptation (InitialAdaptation,
    // src/Adaptation.cu:133-146: Adaptation then InitialConditions, which also
    // rebuilds the boundary block lists) on the current state, with the criterion
    // given by the "Adaptation" key.
    int adapt() override
    {
        CopyArrayBUQ(P, M.blocks, M.evolv, M.evolv_o);
        InitialAdaptation(P, F, M);
        return P.nblk;
    }

    // Whole 18x18 tiles in active-block order (the layout of get()).
    int set(const char* name, const double* buq) override
    {
        T* p = field(name, false);
        if (!p) return -1;
        for (int ibl = 0; ibl < P.nblk; ibl++) {
            int ib = M.blocks.active[ibl];
            for (int k = 0; k < P.blksize; k++) p[(size_t)ib * P.blksize + k] = T(buq[(size_t)ibl * P.blksize + k]);
        }
        return 0;
    }

    // After fields were set on an adapted mesh: bed halo and gradients as
    // src/Testing.cu:583-588 does, zs = zb + h, state copy, fresh loop and initdt.
    int reinit(double nextout) override
    {
        fillHaloC(P, M.blocks, M.zb);
        gradientC(P, M.blocks, M.zb, M.grad.dzbdx, M.grad.dzbdy);
        gradientHalo(P, M.blocks, M.zb, M.grad.dzbdx, M.grad.dzbdy);
        refine_linear(P, M.blocks, M.zb, M.grad.dzbdx, M.grad.dzbdy);
        gradientHalo(P, M.blocks, M.zb, M.grad.dzbdx, M.grad.dzbdy);
        for (int ibl = 0; ibl < P.nblk; ibl++) {
            int ib = M.blocks.active[ibl];
            for (int iy = 0; iy < 16; iy++)
                for (int ix = 0; ix < 16; ix++) {
                    int n = memloc(P, ix, iy, ib);
                    M.evolv.zs[n] = M.zb[n] + M.evolv.h[n];
                }
        }
        CopyArrayBUQ(P, M.blocks, M.evolv, M.evolv_o);
        L.totaltime = 0.0;
        L.dt = 0.0;
        L.nextoutputtime = nextout;
        L.dtmax = initdt(P, L, M);
        return 0;
    }

    int get_active(int* out) override
    {
        for (int ibl = 0; ibl < P.nblk; ibl++) out[ibl] = M.blocks.active[ibl];
        return P.nblk;
    }

    // The reference's Adaptation() alone (src/Adaptation.cu:17-121), as a time loop
    // would call it between steps: criteria, sanity pass, refinement, bed
    // re-interpolation from the bathymetry forcing, wet/dry fix-up, state copy.
    int adaptation() override
    {
        CopyArrayBUQ(P, M.blocks, M.evolv, M.evolv_o);
        Adaptation(P, F, M);
        return P.nblk;
    }

    // Refine / coarsen flags of one pass of AdaptCriteria + refinesanitycheck, read
    // off one iteration of Adaptation (refinesanitycheck is not exported by the
    // reference build): a block was flagged for refinement when its level rose, for
    // coarsening when it left the active list or its level fell.  Written per block
    // of the active list before the pass; the model is adapted by one iteration.
    int flags(unsigned char* refine, unsigned char* coarsen) override
    {
        const int n0 = P.nblk;
        std::vector<int> act(M.blocks.active, M.blocks.active + n0), lev(n0);
        for (int k = 0; k < n0; k++) lev[k] = M.blocks.level[act[k]];
        const int saved = P.adaptmaxiteration;
        P.adaptmaxiteration = 1;
        CopyArrayBUQ(P, M.blocks, M.evolv, M.evolv_o);
        Adaptation(P, F, M);
        P.adaptmaxiteration = saved;
        std::vector<char> still(P.nblkmem, 0);
        for (int ibl = 0; ibl < P.nblk; ibl++) still[M.blocks.active[ibl]] = 1;
        for (int k = 0; k < n0; k++) {
            const int ib = act[k];
            refine[k] = still[ib] && M.blocks.level[ib] > lev[k];
            coarsen[k] = !still[ib] || M.blocks.level[ib] < lev[k];
        }
        return n0;
    }

    // Replaces the bathymetry forcing (Forcing.Bathy[0], a regular grid of nx*ny
    // nodes from (xo, yo) with spacing dx) used when Adaptation re-interpolates zb.
    int set_bathy(int nx, int ny, double xo, double yo, double dx, const double* val) override
    {
        StaticForcingP<float>& b = F.Bathy[0];
        b.nx = nx;
        b.ny = ny;
        b.xo = xo;
        b.yo = yo;
        b.dx = dx;
        b.dy = dx;
        b.xmax = xo + (nx - 1) * dx;
        b.ymax = yo + (ny - 1) * dx;
        AllocateCPU(nx, ny, b.val);
        for (int k = 0; k < nx * ny; k++) b.val[k] = (float)val[k];
        return 0;
    }
};

}  // namespace

extern "C" {

// Creates an in-memory reference model on a uniform nx*ny cell grid (multiples of 16),
// overwriting bed and state with the given row-major cell arrays.
void* ref_create(const char* paramtext, int use_double, int nx, int ny, double dx, double xo,
                 double yo, const double* zb, const double* h, const double* u, const double* v,
                 const double* cf, double nextoutputtime)
{
    if (use_double) {
        auto* m = new RefModel<double>();
        m->setup(paramtext, nx, ny, dx, xo, yo, zb, h, u, v, cf, nextoutputtime);
        return m;
    }
    auto* m = new RefModel<float>();
    m->setup(paramtext, nx, ny, dx, xo, yo, zb, h, u, v, cf, nextoutputtime);
    return m;
}

// Adds a boundary segment on one side BEFORE ref_create is not possible through this
// surface; segments are instead declared in paramtext with the reference's own keys
// ("left = 2,file" needs a file), so uniform series are injected here after creation.
int ref_set_segment_series(void* hdl, int iseg, int n, const double* t, const double* wl)
{
    RefBase* m = (RefBase*)hdl;
    if (iseg < 0 || iseg >= (int)m->F.bndseg.size()) return -1;
    bndsegment& s = m->F.bndseg[iseg];
    s.data.clear();
    for (int k = 0; k < n; k++) {
        Windin w;
        w.time = t[k];
        w.wspeed = wl[k];
        s.data.push_back(w);
    }
    s.on = true;
    s.uniform = true;
    return 0;
}

int ref_adaptation(void* hdl) { return ((RefBase*)hdl)->adaptation(); }
int ref_flags(void* hdl, unsigned char* refine, unsigned char* coarsen) { return ((RefBase*)hdl)->flags(refine, coarsen); }
int ref_set_bathy(void* hdl, int nx, int ny, double xo, double yo, double dx, const double* val)
{
    return ((RefBase*)hdl)->set_bathy(nx, ny, xo, yo, dx, val);
}

// Appends a target-level map (an entry of the reference's Forcing.targetadapt, which
// readforcing fills from the files of "Adaptation = Targetlevel,<file>,..."): nx*ny
// integer nodes from (xo, yo) with spacing dx in x and y.
int ref_add_target_map(void* hdl, int nx, int ny, double xo, double yo, double dx, const int* val)
{
    StaticForcingP<int> m;
    m.nx = nx;
    m.ny = ny;
    m.xo = xo;
    m.yo = yo;
    m.dx = dx;
    m.dy = dx;
    m.xmax = xo + (nx - 1) * dx;
    m.ymax = yo + (ny - 1) * dx;
    m.val = (int*)malloc(sizeof(int) * (size_t)nx * ny);
    if (!m.val) return 1;
    for (int k = 0; k < nx * ny; k++) m.val[k] = val[k];
    ((RefBase*)hdl)->F.targetadapt.push_back(m);
    return 0;
}
int ref_nblkmem(void* hdl) { return ((RefBase*)hdl)->P.nblkmem; }

int ref_set_rain_series(void* hdl, int n, const double* t, const double* r)
{
    RefBase* m = (RefBase*)hdl;
    m->F.Rain.inputfile = "uniform_rain_series";
    m->F.Rain.uniform = true;
    m->F.Rain.unidata.clear();
    for (int k = 0; k < n; k++) {
        Windin w;
        w.time = t[k];
        w.wspeed = r[k];
        m->F.Rain.unidata.push_back(w);
    }
    return 0;
}

// A model set up by the reference's own start-up from a BG_param.txt file (paths
// in it relative to the working directory), on the CPU.  The reference leaves the
// y spacing (dy) of an .asc bathymetry at 0, which its bilinear interp2BUQ
// divides by; with fix_asc_dy the harness sets dy = dx after reading, as the
// reference's .md reader does.
void* ref_create_from_file(const char* paramfile, int fix_asc_dy)
{
    Param P;
    Forcing<float> F;
    Readparamfile(P, F, std::string(paramfile));
    P.GPUDEVICE = -1;
    readforcing(P, F);
    if (fix_asc_dy)
        for (auto& b : F.Bathy)
            if (b.dy == 0.0) b.dy = b.dx;
    checkparamsanity(P, F);
    RefBase* m;
    if (P.doubleprecision) m = new RefModel<double>();
    else m = new RefModel<float>();
    m->P = P;
    m->F = F;
    m->setup_loaded();
    return m;
}

// readbathyASCHead / readbathyASCzb (src/ReadForcing.cu:2067-2220) as they are.
int ref_read_asc_head(const char* path, int* nx, int* ny, double* dx, double* xo, double* yo, double* grdalpha)
{
    readbathyASCHead(std::string(path), *nx, *ny, *dx, *xo, *yo, *grdalpha);
    return 0;
}
int ref_read_asc(const char* path, int nx, int ny, float* val)
{
    readbathyASCzb<float>(std::string(path), nx, ny, val);
    return 0;
}

// Scalars of the set-up model: xo, yo, xmax, ymax, dx, delta, nx, ny, nblk, nblkmem,
// doubleprecision, zsinit, zsoffset, endtime, totaltime, loop nextoutputtime,
// loop dtmax, CFL, engine, mask, initlevel, minlevel, maxlevel, rain samples, segments.
int ref_param(void* hdl, double* out)
{
    RefBase* m = (RefBase*)hdl;
    const Param& P = m->P;
    double v[] = {P.xo, P.yo, P.xmax, P.ymax, P.dx, P.delta, (double)P.nx, (double)P.ny, (double)P.nblk,
                  (double)P.nblkmem, (double)P.doubleprecision, P.zsinit, P.zsoffset, P.endtime, P.totaltime,
                  m->loop_nextoutputtime(), m->loop_dtmax(), P.CFL, (double)P.engine, P.mask, (double)P.initlevel,
                  (double)P.minlevel, (double)P.maxlevel, (double)m->F.Rain.unidata.size(), (double)m->F.bndseg.size()};
    const int n = (int)(sizeof(v) / sizeof(v[0]));
    for (int k = 0; k < n; k++) out[k] = v[k];
    return n;
}

// Uniform rain series (time, mm/h) as the reference read it.
int ref_rain(void* hdl, double* t, double* r)
{
    RefBase* m = (RefBase*)hdl;
    const auto& d = m->F.Rain.unidata;
    for (size_t k = 0; k < d.size(); k++) {
        t[k] = d[k].time;
        r[k] = d[k].wspeed;
    }
    return (int)d.size();
}

// Segment iseg: type, number of samples; times and levels of a uniform series.
int ref_segment(void* hdl, int iseg, int* type, double* t, double* wl)
{
    RefBase* m = (RefBase*)hdl;
    if (iseg < 0 || iseg >= (int)m->F.bndseg.size()) return -1;
    const bndsegment& s = m->F.bndseg[iseg];
    *type = s.type;
    for (size_t k = 0; k < s.data.size(); k++) {
        if (t) t[k] = s.data[k].time;
        if (wl) wl[k] = s.data[k].wspeed;
    }
    return (int)s.data.size();
}

int ref_get_active_cell(void* hdl, int* out) { return ((RefBase*)hdl)->get_active_cell(out); }

// Gridded rain of two frames (before at time `to`, after at to + dt) installed as
// the reference holds a netCDF rain map after its first read (DynForcingP with
// instep = 1, so Forcingthisstep interpolates without reading a file while the
// time stays below to + dt).  Its CPU time interpolation counts from time 0
// (InterpstepCPU, src/GridManip.cu:602-621), so `to` must be 0.
int ref_set_rain_map(void* hdl, int nx, int ny, double xo, double yo, double dx, double dy, double to, double dt,
                     const float* before, const float* after)
{
    RefBase* m = (RefBase*)hdl;
    DynForcingP<float>& R = m->F.Rain;
    R.inputfile = "rain_map";
    R.uniform = false;
    R.nx = nx;
    R.ny = ny;
    R.xo = xo;
    R.yo = yo;
    R.dx = dx;
    R.dy = dy;
    R.xmax = xo + (nx - 1) * dx;
    R.ymax = yo + (ny - 1) * dy;
    R.nt = 2;
    R.to = to;
    R.dt = dt;
    R.tmax = to + dt;
    R.instep = 1;
    const size_t n = (size_t)nx * ny;
    R.before = (float*)malloc(n * sizeof(float));
    R.after = (float*)malloc(n * sizeof(float));
    R.val = (float*)malloc(n * sizeof(float));
    R.now = R.val;
    for (size_t k = 0; k < n; k++) {
        R.before[k] = before[k];
        R.after[k] = after[k];
        R.val[k] = before[k];
    }
    return 0;
}

int ref_step(void* hdl, int nsteps, double* dts) { return ((RefBase*)hdl)->step(nsteps, dts); }
int ref_adapt(void* hdl) { return ((RefBase*)hdl)->adapt(); }
int ref_set(void* hdl, const char* name, const double* buq) { return ((RefBase*)hdl)->set(name, buq); }
int ref_reinit(void* hdl, double nextout) { return ((RefBase*)hdl)->reinit(nextout); }
int ref_get_active(void* hdl, int* out) { return ((RefBase*)hdl)->get_active(out); }
int ref_nblk(void* hdl) { return ((RefBase*)hdl)->P.nblk; }
int ref_nseg(void* hdl) { return (int)((RefBase*)hdl)->F.bndseg.size(); }
int ref_get(void* hdl, const char* name, double* out) { return ((RefBase*)hdl)->get(name, out); }
int ref_get_blocks(void* hdl, int* level, double* xo, double* yo, int* nbr8)
{
    return ((RefBase*)hdl)->get_blocks(level, xo, yo, nbr8);
}
void ref_destroy(void* hdl) { delete (RefBase*)hdl; }

}
