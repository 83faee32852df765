// Fused flow-step kernels for sm_100a.
//
// One step of the reference (FlowGPU, src/FlowGPU.cu:14-315) is two launches:
//
//   flux_kernel   (predictor): per 16x16 block, assemble the state tile with a
//                 two-cell ring from the neighbour tables (fillHalo + the
//                 stencils of gradientHalo), limited gradients, wet-slope reset,
//                 X/Y face fluxes, boundary-segment fluxes, the per-cell dtmax and
//                 the block's share of the global CFL minimum, then the flux
//                 divergence (updateEV).  Writes dh, dhu, dhv only.
//
//   update_kernel (corrector): turns the global minimum into dt with the
//                 reference clamps (CalctimestepGPU), rebuilds the half-step state
//                 h* = Advance(h, dh, dt/2) on the fly for its tile and ring (the
//                 predictor advance is pointwise, so the ring values equal what a
//                 halo exchange of h* would deliver), repeats gradients / fluxes /
//                 boundaries on h*, and applies the full-step advance, friction and
//                 rain, writing the next state into the other ping-pong buffer.
//
// Per cell-update HBM traffic is h,u,v,zb read + dh,dhu,dhv written (predictor)
// and h,u,v,dh,dhu,dhv,zb read + h,u,v written (corrector): 68 B in FP32 with a
// uniform friction coefficient, the algorithmic minimum of the two-stage scheme.
#pragma once
#include <stdint.h>

#include "bgf_numerics.cuh"
#include "bgf_split.cuh"

namespace bgf {

constexpr int BW = 16;      // block width in cells
constexpr int TW = 20;      // tile width: 16 interior + 2 rings each side
constexpr int NTHREADS = 256;

// Device time-loop state (reference Loop<T> members, src/Arrays.h:359-404), kept in
// two slots that alternate with the step parity.
struct TimeState {
    double totaltime;
    double dt;          // dt of the last step taken (the "previous dt" of the next one)
    double dtmax;       // clamp reference for the next dt (XLoop.dtmax)
    double nextoutputtime;
    double endtime;
    double outputtimestep;
    long long nstep;
    long long maxsteps;
    int cur;            // state buffer holding the current state
    int done;           // 1: the loop condition failed; further steps are no-ops
    int status;         // 0 ok, BGF_EDT_UNDERFLOW, BGF_ENAN
    int pad;
};

struct SegDev {
    int type;  // 0 wall, 1 Neumann, 2 Dirichlet, 3 absorbing
    int n;     // series length (0: no series, zsbnd from zsinit)
    int off;   // offset in the series arrays
    int sorted;  // 1: the series times are non-decreasing (the sample is found by bisection)
};

template <class T> struct StepParams {
    T g, eps, CFL, theta, delta0, epsi, epsface, fc;
    double eps_d, dtparam, bndfiltertime, bndrelaxtime, bndtaper, inittime, zsinit, zsoffset, dtmin;
    double delta0_d;  // level-0 spacing in double (refine_linear left/top offsets)
    double xo_d, yo_d;  // domain origin (river boxes)
    T cf;        // uniform friction coefficient
    int frictionmodel, forcemass, has_cf, has_rain, nseg, rain_n, rain_off;
    int nriver, riv_first;  // rivers of this scenario: entries riv_first .. riv_first + nriver - 1
    int rain_map;           // 1: the rain rate is a gridded series (m.rmap), else the uniform series
    int rain_sorted;        // 1: the uniform rain series' times are non-decreasing
};

// A gridded rain series (the reference's DynForcingP<float> Rain read from a
// file): nt frames of nx*ny nodes from (xo, yo) with spacings dx, dy, frame k at
// time to + k*dt; frames row-major with row 0 at yo.
struct RainMapDev {
    const float* val;
    int nx, ny, nt;
    double xo, yo, dx, dy, xmax, ymax, to, dt;
};

// A river (the reference's River / RiverInfo): discharge box, discharge area (sum
// of the cell areas the box overlaps, InitRivers) and its discharge series at
// riv_t / riv_q [off, off + n).
struct RiverDev {
    double xs, xe, ys, ye, area;
    int off, n;
};

template <class T> struct DevModel {
    int nblk, nblkmem;
    const int* active;
    const int* level;
    const int* nbr;  // [8][nblkmem]: LB, LT, RB, RT, BL, BR, TL, TR
    const T* zb;     // 324 per block (halo filled)
    const T* dzbdx;  // 324 per block (engine 1)
    const T* dzbdy;
    const T* cf;     // 256 per block (optional)
    const uint8_t* rainmask;  // 256 per block (optional)
    const int* bndseg;        // 4 per block: segment index per side or -1
    float* qmean;             // 64 per block
    const SegDev* segs;
    const double* seg_t;
    const double* seg_wl;
    const double* rain_t;
    const double* rain_r;
    RainMapDev rmap;
    const RiverDev* rivers;
    const double* riv_t;
    const double* riv_q;
    const double* bxo;  // block origins relative to the domain origin (values of the state precision)
    const double* byo;
    T* h[2];
    T* u[2];
    T* v[2];
    T* dh;
    T* dhu;
    T* dhv;
    TimeState* time;       // [nscen][2]
    unsigned long long* dtmin;  // [nscen][2] bit patterns of the running minimum (dt > 0: integer order)
    int* err;              // device error word (0 ok)
    // batched pools (all null for a single scenario)
    const int* scen;                  // per block slot: scenario index
    const StepParams<T>* sparams;     // per scenario
    const uint8_t* lead;              // per block slot: 1 for the first block of its scenario
    T* hmax;                          // per cell (256 per block): running maximum depth, or null
    const T* datum;                   // per block slot: datum depth of split mode, or null
    int checklev;                     // fused kernels: verify that neighbours share the block's level
    int gen;                          // thread layout of the single-level stage kernels: 1 one cell per
                                      // thread, otherwise two cells per thread (read by the launchers)
    int regular_nbx;                  // > 0: the mesh is a full regular grid of regular_nbx blocks per
                                      // row in row-major ids (active[w] == w, neighbours at +-1 and
                                      // +-regular_nbx, a domain edge its own block); the two-cell
                                      // kernels then derive ids instead of loading them
    int regular_nby;                  // rows of that grid (nblk / regular_nbx)
    unsigned regular_magic;           // > 0: ib / regular_nbx == umulhi(ib, regular_magic) for every
                                      // block id (checked on the host), else a division
};

// Device ring of gauge samples (bgf_gauge.cu): row k % cap holds, for each of the n
// gauges, the time of sample k and h, zs, u, v at the gauge cell.
template <class T> struct GaugeRingDev {
    const int* cell;   // per gauge: block slot * 256 + j * 16 + i
    const int* scen;   // per gauge: scenario index (pools), or null
    int n, cap;
    T* vals;           // [cap][n][4]
    double* time;      // [cap][n]
    unsigned long long* count;  // samples written
};

// Positive floating-point values order like their bit patterns.
__device__ __forceinline__ unsigned long long dt_bits(float v) { return (unsigned long long)__float_as_uint(v); }
__device__ __forceinline__ unsigned long long dt_bits(double v) { return (unsigned long long)__double_as_longlong(v); }
template <class T> __device__ __forceinline__ T dt_from_bits(unsigned long long b);
template <> __device__ __forceinline__ float dt_from_bits<float>(unsigned long long b) { return __uint_as_float((unsigned int)b); }
template <> __device__ __forceinline__ double dt_from_bits<double>(unsigned long long b) { return __longlong_as_double((long long)b); }

// Global BUQ tile index (memloc within a block).
__device__ __forceinline__ int hi18(int x, int y) { return (y + 1) * 18 + (x + 1); }

// Shared-memory layouts.  A warp covers two rows of 16 cells (tx, ty), so a row
// pair is free of bank conflicts when the two rows start 16 words apart modulo 32
// words; interior rows are therefore stored with stride 16 (or in even/odd halves
// for the 20-wide tile) and edge columns apart.
constexpr int TODD = 336;   // first odd row of the 20x20 tile (16 modulo 32 words)
constexpr int TSIZE = 656;  // words of one 20x20 tile variable
__device__ __forceinline__ int ti(int x, int y)  // 20x20 tile, x, y = -2..17
{
    const int Y = y + 2;
    return ((Y & 1) ? TODD : 0) + (Y >> 1) * 32 + (x + 2);
}
__device__ __forceinline__ int si(int x, int y)  // 18x18 tile, x, y = -1..16
{
    return (x >= 0 && x < BW) ? (y + 1) * 16 + x : (x < 0 ? 288 : 306) + (y + 1);
}
__device__ __forceinline__ int gxi(int x, int y)  // x-gradients, x = -1..16, y = 0..15
{
    return (x >= 0 && x < BW) ? y * 16 + x : (x < 0 ? 256 : 272) + y;
}
__device__ __forceinline__ int gyi(int x, int y) { return (y + 1) * 16 + x; }  // y-gradients, y = -1..16
__device__ __forceinline__ int fxi(int x, int y) { return x < BW ? y * 16 + x : 256 + y; }  // X faces x = 0..16
__device__ __forceinline__ int fyi(int x, int y) { return y * 16 + x; }                     // Y faces y = 0..16

// Source cell of tile position (x, y) for a single-level neighbourhood: the
// interior cell whose value fillHalo copies into ring 1 (src/Halo.cu:2083-2286)
// and whose value gradientHalo uses as the outer stencil point for ring 2
// (src/Gradients.cu:2713-3290).  At a domain edge (neighbour == self) both rings
// take the block's own edge cell.  Returns false for cross-level sides.
// checklev: also verify that the neighbour is on the block's level (callers that
// cannot know the mesh is single-level); the handle path knows it and skips the
// dependent level loads.
__device__ __forceinline__ bool tile_source(const int* nbr, int nblkmem, const int* level, int ib, int x, int y,
                                            int& sb, int& sx, int& sy, bool checklev = true)
{
    sb = ib;
    sx = x;
    sy = y;
    if (x < 0) {
        int nb = nbr[0 * nblkmem + ib];
        if (nb == ib) { sx = 0; return nbr[1 * nblkmem + ib] == ib; }
        if (checklev && level[nb] != level[ib]) return false;
        sb = nb; sx = BW + x;
    } else if (x >= BW) {
        int nb = nbr[2 * nblkmem + ib];
        if (nb == ib) { sx = BW - 1; return nbr[3 * nblkmem + ib] == ib; }
        if (checklev && level[nb] != level[ib]) return false;
        sb = nb; sx = x - BW;
    } else if (y < 0) {
        int nb = nbr[4 * nblkmem + ib];
        if (nb == ib) { sy = 0; return nbr[5 * nblkmem + ib] == ib; }
        if (checklev && level[nb] != level[ib]) return false;
        sb = nb; sy = BW + y;
    } else if (y >= BW) {
        int nb = nbr[6 * nblkmem + ib];
        if (nb == ib) { sy = BW - 1; return nbr[7 * nblkmem + ib] == ib; }
        if (checklev && level[nb] != level[ib]) return false;
        sb = nb; sy = y - BW;
    }
    return true;
}

// Ring position k in [0,128): side = k/32 (left, right, bot, top), ring = (k/16)&1, t = k&15.
__device__ __forceinline__ void ring_pos(int k, int& x, int& y)
{
    int side = k >> 5, ring = (k >> 4) & 1, t = k & 15;
    if (side == 0) { x = -1 - ring; y = t; }
    else if (side == 1) { x = BW + ring; y = t; }
    else if (side == 2) { x = t; y = -1 - ring; }
    else { x = t; y = BW + ring; }
}

// Variables of the state tile / gradient arrays
enum { VH = 0, VZS = 1, VU = 2, VV = 3 };

template <class T> struct Smem {
    T t[4][TSIZE];             // h, zs, u, v on the 20x20 tile (layout ti)
    T zb[18 * 18];             // layout si
    T gx[4][18 * 16];          // x-gradients at x=-1..16, rows 0..15
    T gy[4][16 * 18];          // y-gradients at y=-1..16, cols 0..15
    T dzbx[18 * 16], dzby[16 * 18];
    T Fhu[17 * 16], Fqux[17 * 16], Su[17 * 16], Fqvx[17 * 16];
    T Fhv[16 * 17], Fqvy[16 * 17], Sv[16 * 17], Fquy[16 * 17];
    // state n on the 18x18 tile (corrector: evolv for the boundary and the advance)
    T h0[18 * 18], u0[18 * 18], v0[18 * 18];
    T red[NTHREADS / 32];
};

// Correctly rounded quotient x / d for a divisor shared by a whole block, from the
// precomputed r = RN(1/d): one product and two Newton-Raphson correction steps with
// exact residuals (Markstein, "Computation of elementary functions on the IBM
// RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990; the last step is
// Markstein's correctly-rounding theorem).  Tiny numerators, whose residual could
// underflow, take the IEEE division.
template <class T> __device__ __forceinline__ T div_by(T x, T d, T r);
#if BGF_FAST
// fast-math build: one product with the rounded reciprocal (within about an ulp)
template <> __device__ __forceinline__ float div_by<float>(float x, float d, float r) { return x * r; }
template <> __device__ __forceinline__ double div_by<double>(double x, double d, double r) { return x * r; }
#else
template <> __device__ __forceinline__ float div_by<float>(float x, float d, float r)
{
    if (fabsf(x) < 0x1p-90f) return x / d;
    float q = x * r;
    float e = fmaf(-q, d, x);
    q = fmaf(e, r, q);
    e = fmaf(-q, d, x);
    return fmaf(e, r, q);
}
template <> __device__ __forceinline__ double div_by<double>(double x, double d, double r)
{
    if (fabs(x) < 0x1p-960) return x / d;
    double q = x * r;
    double e = fma(-q, d, x);
    q = fma(e, r, q);
    e = fma(-q, d, x);
    return fma(e, r, q);
}
#endif

// Source-term substitution at coarse/fine faces (src/Kurganov.cu:602-616,
// src/Reimann.cu:350-365): on a side whose neighbour is coarser, the depth and bed
// of the coarse neighbour's cell next to the face replace those of the halo cell.
// Sides 0..3 = left, right, bottom, top; entry t along the side.
template <class T> struct SubFaces {
    T h[4][BW];
    T z[4][BW];
    int on[4];
};

// One X (isx) or Y face of the tile, written to the face arrays of s.
template <class T, int ENGINE, bool SUB = false, bool SPLIT = false>
__device__ __forceinline__ Face<T> tile_face(Smem<T>& s, const StepParams<T>& p, T delta, bool isx, int x, int y,
                                             const SubFaces<T>* sub = nullptr, T D = (T)0)
{
    FaceIn<T, ENGINE> f;
    int ci = ti(x, y), cn = isx ? ti(x - 1, y) : ti(x, y - 1);
    f.hi = s.t[VH][ci]; f.hn = s.t[VH][cn];
    f.zsi = s.t[VZS][ci]; f.zsn = s.t[VZS][cn];
    if (isx) {
        int gi = gxi(x, y), gn = gxi(x - 1, y);
        f.uni = s.t[VU][ci]; f.unn = s.t[VU][cn]; f.uti = s.t[VV][ci]; f.utn = s.t[VV][cn];
        f.dhi = s.gx[VH][gi]; f.dhn = s.gx[VH][gn]; f.dzsi = s.gx[VZS][gi]; f.dzsn = s.gx[VZS][gn];
        f.duni = s.gx[VU][gi]; f.dunn = s.gx[VU][gn]; f.duti = s.gx[VV][gi]; f.dutn = s.gx[VV][gn];
    } else {
        int gi = gyi(x, y), gn = gi - 16;
        f.uni = s.t[VV][ci]; f.unn = s.t[VV][cn]; f.uti = s.t[VU][ci]; f.utn = s.t[VU][cn];
        f.dhi = s.gy[VH][gi]; f.dhn = s.gy[VH][gn]; f.dzsi = s.gy[VZS][gi]; f.dzsn = s.gy[VZS][gn];
        f.duni = s.gy[VV][gi]; f.dunn = s.gy[VV][gn]; f.duti = s.gy[VU][gi]; f.dutn = s.gy[VU][gn];
    }
    f.hsi = f.hi;
    f.hsn = f.hn;
    if (ENGINE == 1) {
        f.zbi = s.zb[si(x, y)];
        f.zbn = isx ? s.zb[si(x - 1, y)] : s.zb[si(x, y - 1)];
        f.zsrci = f.zbi;
        f.zsrcn = f.zbn;
    } else {
        f.zsrci = f.zsi - f.hi;
        f.zsrcn = f.zsn - f.hn;
    }
    if (SUB) {
        if (isx) {
            if (x == BW && sub->on[1]) { f.hsi = sub->h[1][y]; f.zsrci = sub->z[1][y]; }
            if (x == 0 && sub->on[0]) { f.hsn = sub->h[0][y]; f.zsrcn = sub->z[0][y]; }
        } else {
            if (y == BW && sub->on[3]) { f.hsi = sub->h[3][x]; f.zsrci = sub->z[3][x]; }
            if (y == 0 && sub->on[2]) { f.hsn = sub->h[2][x]; f.zsrcn = sub->z[2][x]; }
        }
    }
    Face<T> r;
    if (SPLIT) r = face_flux_split<T, ENGINE>(f, D, p.g, p.CFL, p.epsi, p.epsface, delta);
    else r = face_flux<T, ENGINE>(f, p.g, p.CFL, p.epsi, p.epsface, delta);
    if (isx) {
        int fi = fxi(x, y);
        s.Fhu[fi] = r.Fh; s.Fqux[fi] = r.Fq; s.Su[fi] = r.S; s.Fqvx[fi] = r.Ft;
    } else {
        int fi = fyi(x, y);
        s.Fhv[fi] = r.Fh; s.Fqvy[fi] = r.Fq; s.Sv[fi] = r.S; s.Fquy[fi] = r.Ft;
    }
    return r;
}

// Gradients, wet-slope reset and face fluxes on an assembled tile (s.h/u/v/zs/zb).
// Restates gradientCPU (src/Gradients.cu:971-1054) on a single-level tile, then
// the engine's X and Y sweeps.  Returns this thread's cell dtmax (the value the
// reference leaves in dtmax[i] after both sweeps).
template <class T, int ENGINE, bool SUB = false, bool SPLIT = false>
__device__ __forceinline__ T tile_fluxes(Smem<T>& s, const StepParams<T>& p, T delta, int tid,
                                         const SubFaces<T>* sub = nullptr, T D = (T)0)
{
    const T theta = p.theta;
    const T rdelta = (T)1.0 / delta;
    const int tx = tid & 15, ty = tid >> 4;
    {
        // interior cell of this thread: x- and y-gradients of h, zs, u, v
        const int c = ti(tx, ty), gi = gxi(tx, ty), gj = gyi(tx, ty);
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const T* a = s.t[k];
            s.gx[k][gi] = div_by(minmod2(theta, a[c - 1], a[c], a[c + 1]), delta, rdelta);
            s.gy[k][gj] = div_by(minmod2(theta, a[ti(tx, ty - 1)], a[c], a[ti(tx, ty + 1)]), delta, rdelta);
        }
        // one ring gradient per thread: ring cell r = tid/4 (64 cells), variable tid%4;
        // x-gradients on the left/right ring columns, y-gradients on the bottom/top rows
        const int r = tid >> 2, k = tid & 3, side = r >> 4, q = r & 15;
        const T* a = s.t[k];
        int cm, cr, cp;
        T* out;
        if (side == 0) { cm = ti(-2, q); cr = ti(-1, q); cp = ti(0, q); out = &s.gx[k][gxi(-1, q)]; }
        else if (side == 1) { cm = ti(BW - 1, q); cr = ti(BW, q); cp = ti(BW + 1, q); out = &s.gx[k][gxi(BW, q)]; }
        else if (side == 2) { cm = ti(q, -2); cr = ti(q, -1); cp = ti(q, 0); out = &s.gy[k][gyi(q, -1)]; }
        else { cm = ti(q, BW - 1); cr = ti(q, BW); cp = ti(q, BW + 1); out = &s.gy[k][gyi(q, BW)]; }
        *out = div_by(minmod2(theta, a[cm], a[cr], a[cp]), delta, rdelta);
        if (ENGINE == 1) {
            // Wet-slope reset, in the same phase: each thread resets the zs gradients of its
            // own interior cell (WetsloperesetCPU; its y test compares both reconstructions
            // with zs[yminus]); the lane holding a ring cell's zs gradient reads that cell's
            // h gradient, written by the previous lane of the same warp (halo variants).
            const T* zs = s.t[VZS];
            const T* hh = s.t[VH];
            {
                const int c = ti(tx, ty), gi = gxi(tx, ty), gj = gyi(tx, ty);
                const T hc = SPLIT ? D + hh[c] : hh[c];
                const T zsm = zs[ti(tx, ty - 1)];
                s.gx[VZS][gi] = wetslope(delta, zs[c], hc, zs[c - 1], zs[c + 1], s.gx[VZS][gi], s.gx[VH][gi], s.dzbx[gi]);
                s.gy[VZS][gj] = wetslope(delta, zs[c], hc, zsm, zsm, s.gy[VZS][gj], s.gy[VH][gj], s.dzby[gj]);
            }
            __syncwarp();
            if (k == VZS) {
                const T hc = SPLIT ? D + hh[cr] : hh[cr];
                if (side < 2) {
                    const int g = side == 0 ? gxi(-1, q) : gxi(BW, q);
                    s.gx[VZS][g] = wetslope(delta, zs[cr], hc, zs[cr - 1], zs[cr + 1], s.gx[VZS][g], s.gx[VH][g], s.dzbx[g]);
                } else {
                    const int g = side == 2 ? gyi(q, -1) : gyi(q, BW);
                    s.gy[VZS][g] = wetslope(delta, zs[cr], hc, zs[cm], zs[cp], s.gy[VZS][g], s.gy[VH][g], s.dzby[g]);
                }
            }
        }
    }
    __syncthreads();
    // Thread (tx,ty) owns the left (X) and bottom (Y) faces of its cell; threads
    // 0..15 also take X face x=16 and threads 32..47 Y face y=16 (the faces the
    // reference computes in the right / top halo column).
    Face<T> fx = tile_face<T, ENGINE, SUB, SPLIT>(s, p, delta, true, tx, ty, sub, D);
    T celldt = fx.dt;  // dtmax after the X sweep (hugeposval exceeds any finite dt)
    Face<T> fy = tile_face<T, ENGINE, SUB, SPLIT>(s, p, delta, false, tx, ty, sub, D);
    celldt = fy.wet ? (fy.dt < celldt ? fy.dt : celldt) : fy.dt;
    // the extra X faces on warp 0 and the extra Y faces on warp 1: each warp runs one
    // more face pass, instead of warp 0 running two half-empty ones
    if (tid < 16) tile_face<T, ENGINE, SUB, SPLIT>(s, p, delta, true, BW, tid, sub, D);
    else if (tid >= 32 && tid < 48) tile_face<T, ENGINE, SUB, SPLIT>(s, p, delta, false, tid - 32, BW, sub, D);
    return celldt;
}

}  // namespace bgf
