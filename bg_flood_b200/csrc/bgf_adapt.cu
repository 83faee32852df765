// Device side of the refinement pass (the reference's Adapt, src/Adaptation.cu:
// 435-532, with AdaptCriteria, src/AdaptCriteria.cu:20-238):
//
//   adapt_criteria_kernel   Threshold / Inrange criterion per block (any cell)
//   adapt_hgrad_kernel      depth-or-slope criterion with coarsening (extension)
//   adapt_halo_kernel       halos of the old mesh as the reference's adaptation
//                           fills them: h and zs like the flow step, u and v with
//                           the flux-type rules (fillHaloF)
//   adapt_halo_late_kernel  the u/v halo cells that read a coarser neighbour's own
//                           halo (left/bottom sides, last cell of the upper half)
//   adapt_corner_kernel     the four corner cells (fillCorners)
//   adapt_children_kernel   bilinear interpolation of h, zs, u, v from the parent
//                           tile (with halo and corners) into its four children;
//                           per-cell friction and rain mask by covering cell
//   adapt_coarsen_kernel    quads merged into their parent (mean of four cells)
//   adapt_bed_kernel        bed re-interpolated from the bathymetry grid for every
//                           block (interp2BUQ), domain-edge cells copied from the
//                           next row (setedges), then the wet/dry fix-up of h, zs
//
// Compiled once, without FMA contraction: the pass reproduces the reference's
// arithmetic whatever variant the flow kernels use.
#include <cuda_runtime.h>

#include "bgf_amr.cuh"
#include "bgf_internal.h"

namespace bgf {
namespace adapt {


// ---------------------------------------------------------------- criteria

template <class T>
__global__ void __launch_bounds__(256) adapt_criteria_kernel(DevModel<T> m, const T* z, int stride324, int kind, T a1,
                                                             T a2, uint8_t* flags)
{
    const int ib = m.active[blockIdx.x];
    const int tid = threadIdx.x, x = tid & 15, y = tid >> 4;
    const T v = stride324 ? z[(size_t)ib * 324 + hi18(x, y)] : z[(size_t)ib * 256 + tid];
    // Thresholdcriteria: z > threshold; inrangecriteria: zmin <= z <= zmax
    const bool hit = kind == 1 ? v > a1 : (v >= a1 && v <= a2);
    const int any = __syncthreads_or(hit ? 1 : 0);
    if (tid == 0) flags[ib] = any ? 1 : 0;
}

// Depth-or-slope criterion (extension): refine when some cell has h > hthr or a
// wet-surface slope above gthr, coarsening candidate when every cell has h <=
// hthr/2 and slope <= gthr/2.  The slope comes from wet cells of the block only:
// central difference over two wet neighbours, one-sided towards a single wet one,
// 0 with none; squares are compared, in T, without contraction.
template <class T>
__global__ void __launch_bounds__(256) adapt_hgrad_kernel(DevModel<T> m, const T* zs, int cur, T eps, T hthr, T gthr,
                                                          double dx0, uint8_t* refine, uint8_t* coarsen)
{
    __shared__ T sh[256], sz[256];
    const int ib = m.active[blockIdx.x];
    const int tid = threadIdx.x, x = tid & 15, y = tid >> 4;
    const size_t g = (size_t)ib * 256 + tid;
    const T hv = m.h[cur][g];
    sh[tid] = hv;
    sz[tid] = zs[g];
    __syncthreads();
    const T dxl = (T)calcres<double>(dx0, m.level[ib]);
    auto wet = [&](int k) { return sh[k] > eps; };
    auto slope = [&](int km, bool okm, int kp, bool okp) -> T {
        if (okm && okp) return (sz[kp] - sz[km]) / ((T)2 * dxl);
        if (okp) return (sz[kp] - sz[tid]) / dxl;
        if (okm) return (sz[tid] - sz[km]) / dxl;
        return (T)0;
    };
    T g2 = (T)0;
    if (wet(tid)) {
        const T gx = slope(tid - 1, x > 0 && wet(tid - 1), tid + 1, x < 15 && wet(tid + 1));
        const T gy = slope(tid - 16, y > 0 && wet(tid - 16), tid + 16, y < 15 && wet(tid + 16));
        g2 = gx * gx + gy * gy;  // this file is compiled without contraction
    }
    const T hh = hthr * (T)0.5, gh = gthr * (T)0.5;
    const int up = __syncthreads_or(hv > hthr || g2 > gthr * gthr ? 1 : 0);
    const int keep = __syncthreads_or(hv > hh || g2 > gh * gh ? 1 : 0);
    if (tid == 0) {
        refine[ib] = up ? 1 : 0;
        coarsen[ib] = keep ? 0 : 1;
    }
}

// targetlevelcriteria (src/AdaptCriteria.cu:179-232): at every cell of a block the
// map's level, interp2BUQ's bilinear value (src/GridManip.cu:456-495, in double from
// the clamped cell position) rounded in T; the block refines when some cell's level
// is above its own and keeps its level (no coarsening) when some cell's level equals
// it.  Every map rewrites the flags of all blocks, so the last map decides.
template <class T>
__global__ void __launch_bounds__(256) target_level_kernel(DevModel<T> m, TargetMapDev g, T xo, T yo, double dx0,
                                                           uint8_t* refine, uint8_t* coarsen)
{
    const int ib = m.active[blockIdx.x];
    const int tid = threadIdx.x, ix = tid & 15, iy = tid >> 4;
    const int lev = m.level[ib];
    const T delta = (T)calcres<double>(dx0, lev);
    const T x = xo + (T)m.bxo[ib] + (T)ix * delta;
    const T y = yo + (T)m.byo[ib] + (T)iy * delta;
    const double xi = fmax(fmin((double)x, g.xmax), g.xo);
    const double yi = fmax(fmin((double)y, g.ymax), g.yo);
    const int cfi = min(max((int)floor((xi - g.xo) / g.dx), 0), g.nx - 2), cfip = cfi + 1;
    const int cfj = min(max((int)floor((yi - g.yo) / g.dy), 0), g.ny - 2), cfjp = cfj + 1;
    const double x1 = g.xo + g.dx * cfi, x2 = g.xo + g.dx * cfip;
    const double y1 = g.yo + g.dy * cfj, y2 = g.yo + g.dy * cfjp;
    const double q11 = g.val[cfi + cfj * g.nx], q12 = g.val[cfi + cfjp * g.nx];
    const double q21 = g.val[cfip + cfj * g.nx], q22 = g.val[cfip + cfjp * g.nx];
    const double x2x1 = x2 - x1, y2y1 = y2 - y1, x2x = x2 - xi, y2y = y2 - yi, yy1 = yi - y1, xx1 = xi - x1;
    const T v = (T)(1.0 / (x2x1 * y2y1) * (q11 * x2x * y2y + q21 * xx1 * y2y + q12 * x2x * yy1 + q22 * xx1 * yy1));
    const int target = (int)round(v);
    const int up = __syncthreads_or(target > lev ? 1 : 0);
    const int same = __syncthreads_or(target == lev ? 1 : 0);
    if (tid == 0) {
        refine[ib] = up ? 1 : 0;
        coarsen[ib] = up || same ? 0 : 1;
    }
}

template <class T> __global__ void __launch_bounds__(256) adapt_zs_kernel(DevModel<T> m, T* zs, int cur)
{
    const int ib = m.active[blockIdx.x];
    const int tid = threadIdx.x;
    zs[(size_t)ib * 256 + tid] = m.zb[(size_t)ib * 324 + hi18(tid & 15, tid >> 4)] + m.h[cur][(size_t)ib * 256 + tid];
}

// ---------------------------------------------------------------- old-mesh halos

// fillLeftFlux / fillRightFlux / fillBotFlux / fillTopFlux with prolongation
// (src/Halo.cu:2678-2810, 3022-3160, 4256-4390, 4602-4740), as the reference's
// adaptation fills u and v: a finer neighbour gives the mean of its two edge
// cells next to the face, a coarser one its edge cell (left/bottom sides round the
// position up, right/top sides down).  Returns false for the one cell that reads
// the coarser neighbour's halo (handled by adapt_halo_late_kernel).
template <class T>
__device__ bool flux_halo(const int* nbr, int nbm, const int* lv, int ib, int s, int j, const Acc256<T>& z, T& out)
{
    const int nb1 = nbr[(2 * s) * nbm + ib], nb2 = nbr[(2 * s + 1) * nbm + ib];
    int x, y, x2, y2;
    auto own = [&]() {
        own_xy(s, 0, j, x, y);
        out = z(ib, x, y);
    };
    auto mean2 = [&](int nb, int jj) {
        nb_xy(s, 0, jj, x, y);
        nb_xy(s, 0, jj + 1, x2, y2);
        out = (T)0.5 * (z(nb, x, y) + z(nb, x2, y2));
    };
    if (nb1 == ib) {
        if (j < BW / 2 || nb2 == ib) own();
        else mean2(nb2, (j - BW / 2) * 2);
    } else if (lv[ib] == lv[nb1]) {
        nb_xy(s, 0, j, x, y);
        out = z(nb1, x, y);
    } else if (lv[nb1] > lv[ib]) {
        if (j < BW / 2) mean2(nb1, 2 * j);
        else if (nb2 == ib) own();
        else mean2(nb2, (j - BW / 2) * 2);
    } else {
        const bool low = nbr[(2 * (s ^ 1)) * nbm + nb1] == ib;
        const int half = (s == 0 || s == 2) ? (j + 1) >> 1 : j >> 1;
        const int jj = low ? half : half + BW / 2;
        if (jj >= BW) return false;
        nb_xy(s, 0, jj, x, y);
        out = z(nb1, x, y);
    }
    return true;
}

template <class T>
__global__ void __launch_bounds__(256) adapt_halo_kernel(DevModel<T> m, AdaptDev<T> a, int cur)
{
    const int ib = m.active[blockIdx.x];
    const int tid = threadIdx.x, nbm = m.nblkmem;
    const size_t base = (size_t)ib * 324;
    const T* src[4] = {m.h[cur], a.zs, m.u[cur], m.v[cur]};
    {
        const size_t g = (size_t)ib * 256 + tid;
        const int c = hi18(tid & 15, tid >> 4);
#pragma unroll
        for (int f = 0; f < 4; f++) a.W[f][base + c] = src[f][g];
    }
    if (tid < 64) {
        const int s = tid >> 4, j = tid & 15;
        int hx, hy;
        halo_xy(s, j, hx, hy);
        const int hc = hi18(hx, hy);
        const CellRule<T> r = halo_rule<T>(m.nbr, nbm, m.level, ib, s, j);
        a.W[0][base + hc] = rule_eval(r, Acc256<T>{src[0]});
        a.W[1][base + hc] = rule_eval(r, Acc256<T>{src[1]});
#pragma unroll
        for (int f = 2; f < 4; f++) {
            T v;
            if (flux_halo<T>(m.nbr, nbm, m.level, ib, s, j, Acc256<T>{src[f]}, v)) a.W[f][base + hc] = v;
        }
    }
}

// The coarser neighbour's halo cell read by the last cell of the upper half of a
// left or bottom side (the reference fills blocks in active order, so that cell
// already holds the neighbour's filled halo value).
template <class T> __global__ void __launch_bounds__(32) adapt_halo_late_kernel(DevModel<T> m, AdaptDev<T> a)
{
    if (threadIdx.x >= 4) return;
    const int ib = m.active[blockIdx.x];
    const int side = (threadIdx.x & 1) ? 2 : 0, f = 2 + (threadIdx.x >> 1);
    const int nbm = m.nblkmem;
    const int nb1 = m.nbr[(2 * side) * nbm + ib];
    if (!(m.level[nb1] < m.level[ib])) return;
    if (m.nbr[(2 * (side ^ 1)) * nbm + nb1] == ib) return;  // lower half: the cell lies inside the neighbour
    int x, y, hx, hy;
    nb_xy(side, 0, BW, x, y);
    halo_xy(side, BW - 1, hx, hy);
    a.W[f][(size_t)ib * 324 + hi18(hx, hy)] = a.W[f][(size_t)nb1 * 324 + hi18(x, y)];
}

// fillCorners (src/Halo.cu:5277-5408) for one variable: bottom-left, top-left,
// top-right, bottom-right, each from the diagonal block found through a side
// neighbour; when that block is coarser the reference's top-right rule tests the
// top-left diagonal and keeps the previous corner's value otherwise, and its
// bottom-right rule reads the top-left diagonal block -- both reproduced.
template <class T> __device__ void corners(const DevModel<T>& m, T* W, int ib)
{
    const int nbm = m.nblkmem;
    const int* lv = m.level;
    auto Z = [&](int b, int x, int y) -> T { return W[(size_t)b * 324 + hi18(x, y)]; };
    auto N = [&](int k, int b) { return m.nbr[k * nbm + b]; };
    const int LB = 0, LT = 1, RB = 2, BL = 4, BR = 5, TL = 6, TR = 7;
    const int l = lv[ib];
    T zz = (T)0;
    // bottom left
    {
        const int c = N(LT, N(BL, ib));
        if (c == N(BL, ib)) zz = (T)0.5 * (Z(ib, -1, 0) + Z(ib, 0, -1));
        else if (lv[c] == l) zz = Z(c, BW - 1, BW - 1);
        else if (lv[c] > l) zz = (T)0.25 * (Z(c, BW - 1, BW - 1) + Z(c, BW - 1, BW - 2) + Z(c, BW - 2, BW - 1) + Z(c, BW - 2, BW - 2));
        else zz = (T)0.5 * Z(c, BW - 1, BW - 1) + (T)0.25 * (Z(ib, -1, 0) + Z(ib, 0, -1));
        W[(size_t)ib * 324 + hi18(-1, -1)] = zz;
    }
    const int ctl = N(LB, N(TL, ib));
    // top left
    {
        if (ctl == N(TL, ib)) zz = (T)0.5 * (Z(ib, -1, BW - 1) + Z(ib, 0, BW));
        else if (lv[ctl] == l) zz = Z(ctl, BW - 1, 0);
        else if (lv[ctl] > l) zz = (T)0.25 * (Z(ctl, BW - 1, 0) + Z(ctl, BW - 1, 1) + Z(ctl, BW - 2, 0) + Z(ctl, BW - 2, 1));
        else zz = (T)0.5 * Z(ctl, BW - 1, 0) + (T)0.25 * (Z(ib, -1, BW - 1) + Z(ib, 0, BW));
        W[(size_t)ib * 324 + hi18(-1, BW)] = zz;
    }
    // top right
    {
        const int c = N(RB, N(TR, ib));
        if (c == N(TR, ib)) zz = (T)0.5 * (Z(ib, BW, BW - 1) + Z(ib, BW - 1, BW));
        else if (lv[c] == l) zz = Z(c, 0, 0);
        else if (lv[c] > l) zz = (T)0.25 * (Z(c, 0, 0) + Z(c, 0, 1) + Z(c, 1, 0) + Z(c, 1, 1));
        else if (lv[ctl] < l) zz = (T)0.5 * Z(ctl, 0, 0) + (T)0.25 * (Z(ib, BW, BW - 1) + Z(ib, BW - 1, BW));
        W[(size_t)ib * 324 + hi18(BW, BW)] = zz;
    }
    // bottom right
    {
        const int c = N(RB, N(BR, ib));
        if (c == N(BR, ib)) zz = (T)0.5 * (Z(ib, BW - 1, -1) + Z(ib, BW, 0));
        else if (lv[c] == l) zz = Z(c, 0, BW - 1);
        else if (lv[c] > l) zz = (T)0.25 * (Z(c, 0, BW - 1) + Z(c, 0, BW - 2) + Z(c, 1, BW - 1) + Z(c, 1, BW - 2));
        else zz = (T)0.5 * Z(ctl, 0, BW - 1) + (T)0.25 * (Z(ib, BW - 1, -1) + Z(ib, BW, 0));
        W[(size_t)ib * 324 + hi18(BW, -1)] = zz;
    }
}

template <class T> __global__ void __launch_bounds__(4) adapt_corner_kernel(DevModel<T> m, AdaptDev<T> a)
{
    corners<T>(m, a.W[threadIdx.x], m.active[blockIdx.x]);
}

// ---------------------------------------------------------------- children

// refine, step 1 (src/Adaptation.cu:1030-1094): child kk of a refined block takes
// at cell (ix, iy) the bilinear interpolation of the parent tile at
// (ix/2 - 1/4 + kx, iy/2 - 1/4 + ky), kx, ky in {0, 8}; the parent's id is the
// bottom-left child.
template <class T>
__global__ void __launch_bounds__(256) adapt_children_kernel(DevModel<T> m, AdaptDev<T> a, int cur, T* cf,
                                                             uint8_t* rainmask)
{
    __shared__ T tile[4][324];
    __shared__ T cfp[256];
    __shared__ uint8_t rmp[256];
    const int ib = m.active[blockIdx.x];
    const int* ch = a.child + (size_t)ib * 3;
    if (ch[0] < 0) return;
    const int tid = threadIdx.x;
    for (int k = tid; k < 324; k += 256)
#pragma unroll
        for (int f = 0; f < 4; f++) tile[f][k] = a.W[f][(size_t)ib * 324 + k];
    if (cf) cfp[tid] = cf[(size_t)ib * 256 + tid];
    if (rainmask) rmp[tid] = rainmask[(size_t)ib * 256 + tid];
    __syncthreads();
    const int ix = tid & 15, iy = tid >> 4;
    const int kids[4] = {ib, ch[0], ch[1], ch[2]};
    const T lx = (T)ix * (T)0.5 - (T)0.25, ly = (T)iy * (T)0.5 - (T)0.25;
    const int flx = (int)floor(lx), clx = (int)ceil(lx), fly = (int)floor(ly), cly = (int)ceil(ly);
    T* dst[4] = {m.h[cur], a.zs, m.u[cur], m.v[cur]};
#pragma unroll
    for (int kk = 0; kk < 4; kk++) {
        const int kx = (kk & 1) * (BW / 2), ky = (kk >> 1) * (BW / 2);
        const int fx = flx + kx, cx = clx + kx, fy = fly + ky, cy = cly + ky;
        const T rx = lx + (T)kx, ry = ly + (T)ky;
        const int ii = hi18(fx, fy), ir = hi18(cx, fy), it = hi18(fx, cy), itr = hi18(cx, cy);
        const size_t o = (size_t)kids[kk] * 256 + tid;
#pragma unroll
        for (int f = 0; f < 4; f++) {
            const T* z = tile[f];
            // BilinearInterpolation(q11, q12, q21, q22, x1, x2, y1, y2, x, y), src/Util_CPU.cu:129-144
            const T x1 = (T)fx, x2 = (T)cx, y1 = (T)fy, y2 = (T)cy;
            const T x2x1 = x2 - x1, y2y1 = y2 - y1, x2x = x2 - rx, y2y = y2 - ry, yy1 = ry - y1, xx1 = rx - x1;
            dst[f][o] = (T)1.0 / (x2x1 * y2y1) *
                        (z[ii] * x2x * y2y + z[ir] * xx1 * y2y + z[it] * x2x * yy1 + z[itr] * xx1 * yy1);
        }
        // per-cell inputs without a map to re-interpolate from: the covering parent cell
        const int pc = (ky + (iy >> 1)) * 16 + kx + (ix >> 1);
        if (cf) cf[o] = cfp[pc];
        if (rainmask) rainmask[o] = rmp[pc];
    }
    // boundary running means of the new blocks start at zero
    if (tid < 64) {
#pragma unroll
        for (int kk = 1; kk < 4; kk++) m.qmean[(size_t)kids[kk] * 64 + tid] = 0.f;
    }
}

// ---------------------------------------------------------------- coarsening

// coarsen, step 1 (src/Adaptation.cu:690-770): the parent (the quad's lower-left
// block, which keeps its id) takes at cell (ix, iy) the mean of the four cells of
// the quadrant's block it covers, T(0.25) * (((c00 + c10) + c01) + c11), for h, zs,
// u and v, read from the old mesh's tiles; per-cell friction is averaged the same
// way and the rain mask is set when any covered cell has it (the bed pass
// recomputes it from the new bed).  quads[4k..4k+3] = parent, right, top, top-right.
template <class T>
__global__ void __launch_bounds__(256) adapt_coarsen_kernel(DevModel<T> m, AdaptDev<T> a, const int* quads, int cur,
                                                            T* cf, uint8_t* rainmask)
{
    __shared__ T cfq[4][256];
    __shared__ uint8_t rmq[4][256];
    const int* q = quads + 4 * (size_t)blockIdx.x;
    const int ib = q[0];
    const int tid = threadIdx.x, ix = tid & 15, iy = tid >> 4;
    if (cf || rainmask) {
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if (cf) cfq[k][tid] = cf[(size_t)q[k] * 256 + tid];
            if (rainmask) rmq[k][tid] = rainmask[(size_t)q[k] * 256 + tid];
        }
    }
    __syncthreads();
    const int kq = (ix >= 8 ? 1 : 0) + (iy >= 8 ? 2 : 0);
    const int src = q[kq];
    const int cx = 2 * (ix & 7), cy = 2 * (iy & 7);
    const size_t sb = (size_t)src * 324;
    const int ii = hi18(cx, cy), ir = hi18(cx + 1, cy), it = hi18(cx, cy + 1), itr = hi18(cx + 1, cy + 1);
    T* dst[4] = {m.h[cur], a.zs, m.u[cur], m.v[cur]};
    const size_t o = (size_t)ib * 256 + tid;
#pragma unroll
    for (int f = 0; f < 4; f++) {
        const T* W = a.W[f] + sb;
        dst[f][o] = (T)0.25 * (((W[ii] + W[ir]) + W[it]) + W[itr]);
    }
    const int c00 = cy * 16 + cx;
    if (cf) {
        const T* c = cfq[kq];
        cf[o] = (T)0.25 * (((c[c00] + c[c00 + 1]) + c[c00 + 16]) + c[c00 + 17]);
    }
    if (rainmask) {
        const uint8_t* r = rmq[kq];
        rainmask[o] = (r[c00] | r[c00 + 1] | r[c00 + 16] | r[c00 + 17]) ? 1 : 0;
    }
    // boundary running means of the merged block start at zero
    if (tid < 64) m.qmean[(size_t)ib * 64 + tid] = 0.f;
}

// ---------------------------------------------------------------- bed

// interp2BUQ (src/GridManip.cu:456-575): bilinear between grid nodes when the
// block spacing is not coarser than the grid, else the mean of the grid nodes
// inside the cell.
template <class T> __device__ T dem_value(const AdaptDev<T>& a, T x, T y, T dx)
{
    if (dx <= (T)a.ddx) {
        const double xi = fmax(fmin((double)x, a.dxmax), a.dxo);
        const double yi = fmax(fmin((double)y, a.dymax), a.dyo);
        const int cfi = min(max((int)floor((xi - a.dxo) / a.ddx), 0), a.dnx - 2), cfip = cfi + 1;
        const int cfj = min(max((int)floor((yi - a.dyo) / a.ddx), 0), a.dny - 2), cfjp = cfj + 1;
        const double x1 = a.dxo + a.ddx * cfi, x2 = a.dxo + a.ddx * cfip;
        const double y1 = a.dyo + a.ddx * cfj, y2 = a.dyo + a.ddx * cfjp;
        const double q11 = a.dem[cfi + cfj * a.dnx], q12 = a.dem[cfi + cfjp * a.dnx];
        const double q21 = a.dem[cfip + cfj * a.dnx], q22 = a.dem[cfip + cfjp * a.dnx];
        const double x2x1 = x2 - x1, y2y1 = y2 - y1, x2x = x2 - xi, y2y = y2 - yi, yy1 = yi - y1, xx1 = xi - x1;
        return (T)(1.0 / (x2x1 * y2y1) * (q11 * x2x * y2y + q21 * xx1 * y2y + q12 * x2x * yy1 + q22 * xx1 * yy1));
    }
    const double xmin = x - dx * 0.5, xmax = x + dx * 0.5, ymin = y - dx * 0.5, ymax = y + dx * 0.5;
    const int imin = max((int)floor((xmin - a.dxo) / a.ddx), 0), imax = min((int)floor((xmax - a.dxo) / a.ddx), a.dnx - 1);
    const int jmin = max((int)floor((ymin - a.dyo) / a.ddx), 0), jmax = min((int)floor((ymax - a.dyo) / a.ddx), a.dny - 1);
    const int ni = max(imax - imin + 1, 1), nj = max(jmax - jmin + 1, 1);
    T z = (T)0.0;
    for (int i = 0; i < ni; i++)
        for (int j = 0; j < nj; j++) z = z + (T)a.dem[min(imin + i, a.dnx - 1) + min(jmin + j, a.dny - 1) * a.dnx];
    return z / (T)(ni * nj);
}

template <class T>
__global__ void __launch_bounds__(256) adapt_bed_kernel(DevModel<T> m, AdaptDev<T> a, StepParams<T> p, int cur, T* zb,
                                                        double xo0, double yo0, const double* bxo, const double* byo,
                                                        double mask, uint8_t* rainmask)
{
    __shared__ T z[324];
    const int ib = m.active[blockIdx.x];
    const int tid = threadIdx.x, ix = tid & 15, iy = tid >> 4;
    const int nbm = m.nblkmem;
    const double blkdx = calcres<double>(p.delta0_d, m.level[ib]);
    const T x = (T)(xo0 + bxo[ib] + ix * blkdx), y = (T)(yo0 + byo[ib] + iy * blkdx);
    z[hi18(ix, iy)] = dem_value<T>(a, x, y, (T)blkdx);
    __syncthreads();
    // setedges (src/GridManip.cu:222-330): left, right, top, bottom, one after the
    // other; the left/right test looks at the first neighbour only, as the reference does
    auto N = [&](int k) { return m.nbr[k * nbm + ib]; };
    if (tid < 16) {
        const int j = tid;
        if (N(0) == ib && j >= 0 && j < (N(1) == ib ? BW : BW / 2)) z[hi18(0, j)] = z[hi18(1, j)];
    }
    __syncthreads();
    if (tid < 16) {
        const int j = tid;
        if (N(2) == ib && j < (N(3) == ib ? BW : BW / 2)) z[hi18(BW - 1, j)] = z[hi18(BW - 2, j)];
    }
    __syncthreads();
    if (tid < 16) {
        const int i = tid;
        if (N(6) == ib || N(7) == ib) {
            const int i0 = N(6) == ib ? 0 : BW / 2, i1 = N(7) == ib ? BW : BW / 2;
            if (i >= i0 && i < i1) z[hi18(i, BW - 1)] = z[hi18(i, BW - 2)];
        }
    }
    __syncthreads();
    if (tid < 16) {
        const int i = tid;
        if (N(4) == ib || N(5) == ib) {
            const int i0 = N(4) == ib ? 0 : BW / 2, i1 = N(5) == ib ? BW : BW / 2;
            if (i >= i0 && i < i1) z[hi18(i, 0)] = z[hi18(i, 1)];
        }
    }
    __syncthreads();
    const T zbv = z[hi18(ix, iy)];
    zb[(size_t)ib * 324 + hi18(ix, iy)] = zbv;
    // zb cannot be conserved through refinement: wet cells keep their surface,
    // dry cells take the bed as surface (src/Adaptation.cu:500-525)
    const size_t g = (size_t)ib * 256 + tid;
    T hv = m.h[cur][g];
    if ((double)hv > p.eps_d) {
        const T d = a.zs[g] - zbv;
        m.h[cur][g] = (T)p.eps_d < d ? d : (T)p.eps_d;
    } else {
        a.zs[g] = zbv;
    }
    if (rainmask) rainmask[g] = (double)zbv < mask ? 1 : 0;
}

// ---------------------------------------------------------------- launchers

template <class T> void launch_criteria(const DevModel<T>& m, const T* z, int stride324, int kind, T a1, T a2,
                                        uint8_t* flags, cudaStream_t st)
{
    adapt_criteria_kernel<T><<<m.nblk, 256, 0, st>>>(m, z, stride324, kind, a1, a2, flags);
}

template <class T>
void launch_target_level(const DevModel<T>& m, const TargetMapDev& g, double xo, double yo, double dx0,
                         uint8_t* refine, uint8_t* coarsen, cudaStream_t st)
{
    target_level_kernel<T><<<m.nblk, 256, 0, st>>>(m, g, (T)xo, (T)yo, dx0, refine, coarsen);
}

template <class T> void launch_zs(const DevModel<T>& m, T* zs, int cur, cudaStream_t st)
{
    adapt_zs_kernel<T><<<m.nblk, 256, 0, st>>>(m, zs, cur);
}

template <class T>
void launch_hgrad(const DevModel<T>& m, const T* zs, int cur, double eps, double hthr, double gthr, double dx0,
                  uint8_t* refine, uint8_t* coarsen, cudaStream_t st)
{
    adapt_hgrad_kernel<T><<<m.nblk, 256, 0, st>>>(m, zs, cur, (T)eps, (T)hthr, (T)gthr, dx0, refine, coarsen);
}

template <class T> int launch_children(const DevModel<T>& m, const AdaptDev<T>& a, int cur, T* cf, uint8_t* rainmask,
                                       const int* quads, int nquads, bool refine, cudaStream_t st)
{
    adapt_halo_kernel<T><<<m.nblk, 256, 0, st>>>(m, a, cur);
    adapt_halo_late_kernel<T><<<m.nblk, 32, 0, st>>>(m, a);
    adapt_corner_kernel<T><<<m.nblk, 4, 0, st>>>(m, a);
    int n = 3;
    if (refine) {
        adapt_children_kernel<T><<<m.nblk, 256, 0, st>>>(m, a, cur, cf, rainmask);
        n++;
    }
    if (nquads > 0) {
        adapt_coarsen_kernel<T><<<nquads, 256, 0, st>>>(m, a, quads, cur, cf, rainmask);
        n++;
    }
    return n;
}

template <class T> void launch_bed(const DevModel<T>& m, const AdaptDev<T>& a, const StepParams<T>& p, int cur, T* zb,
                                   double xo0, double yo0, const double* bxo, const double* byo, double mask,
                                   uint8_t* rainmask, cudaStream_t st)
{
    adapt_bed_kernel<T><<<m.nblk, 256, 0, st>>>(m, a, p, cur, zb, xo0, yo0, bxo, byo, mask, rainmask);
}

#define BGF_ADAPT_INST(T)                                                                                          \
    template void launch_criteria<T>(const DevModel<T>&, const T*, int, int, T, T, uint8_t*, cudaStream_t);       \
    template void launch_zs<T>(const DevModel<T>&, T*, int, cudaStream_t);                                         \
    template void launch_target_level<T>(const DevModel<T>&, const TargetMapDev&, double, double, double, uint8_t*, \
                                         uint8_t*, cudaStream_t);                                                  \
    template int launch_children<T>(const DevModel<T>&, const AdaptDev<T>&, int, T*, uint8_t*, const int*, int, bool, \
                                    cudaStream_t);                                                                 \
    template void launch_hgrad<T>(const DevModel<T>&, const T*, int, double, double, double, double, uint8_t*,      \
                                  uint8_t*, cudaStream_t);                                                         \
    template void launch_bed<T>(const DevModel<T>&, const AdaptDev<T>&, const StepParams<T>&, int, T*, double,      \
                                double, const double*, const double*, double, uint8_t*, cudaStream_t);
BGF_ADAPT_INST(float)
BGF_ADAPT_INST(double)

}  // namespace adapt
}  // namespace bgf
