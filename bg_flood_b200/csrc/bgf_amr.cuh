// Multi-level (quadtree) meshes: device buffers and the per-cell rules of the
// halo exchange across refinement levels.
//
// A mesh whose blocks sit on more than one level cannot assemble a block's
// stencil tile from the neighbours' interiors alone: the reference fills the
// halo of every block (restriction from finer, barycentric interpolation from
// coarser neighbours), computes gradients, rebuilds the halos next to coarser
// blocks by linear reconstruction, applies the wet/dry corrections, and only then
// evaluates fluxes, whose coarse-side faces are finally replaced by the mean of
// the two fine faces.  Each of those phases reads what the previous one wrote in
// *other* blocks, so the multi-level step is a short chain of per-block kernels
// (bgf_amr.cu) over stage arrays that keep the 18x18 BUQ tiles with their halos.
#pragma once
#include <stdint.h>

#include "bgf_flow.cuh"

namespace bgf {

template <class T> struct AmrDev {
    T* W[2][4];        // stage state on 18x18 tiles: h, zs, u, v (stage 0 state n, stage 1 half step)
    T* G0[6];          // dhdx, dhdy, dudx, dudy, dvdx, dvdy on 18x18 tiles (interior, before prolongation)
    T* F[8];           // Fhu, Fqux, Su, Fqvx (17x16 per block), Fhv, Fqvy, Sv, Fquy (16x17 per block)
    T* zb;             // bed on 18x18 tiles; the wet/dry prolongation edits its halo
    T* dzbdx;
    T* dzbdy;
    uint8_t* pflag;    // 64 per block: halo cell takes its parent's depth and bed (wet/dry prolongation)
    const int* rank;   // position of each block in the active list (the reference's loop order)
    int wetdryfix;
};

constexpr int NFX = 17 * 16;  // X faces per block (x = 0..16, rows 0..15)

// Cell coordinates along side s (0 left, 1 right, 2 bottom, 3 top) of a block.
// nb_xy: the cell at depth k from the edge that faces us, tangential position j,
// in a neighbour across side s.  own_xy: depth k from our own edge on side s.
__device__ __forceinline__ void nb_xy(int s, int k, int j, int& x, int& y)
{
    if (s == 0) { x = BW - 1 - k; y = j; }
    else if (s == 1) { x = k; y = j; }
    else if (s == 2) { x = j; y = BW - 1 - k; }
    else { x = j; y = k; }
}
__device__ __forceinline__ void own_xy(int s, int k, int j, int& x, int& y)
{
    if (s == 0) { x = k; y = j; }
    else if (s == 1) { x = BW - 1 - k; y = j; }
    else if (s == 2) { x = j; y = k; }
    else { x = j; y = BW - 1 - k; }
}
__device__ __forceinline__ void halo_xy(int s, int j, int& x, int& y)
{
    if (s == 0) { x = -1; y = j; }
    else if (s == 1) { x = BW; y = j; }
    else if (s == 2) { x = j; y = -1; }
    else { x = j; y = BW; }
}
// Neighbour-table entries (LB, LT, RB, RT, BL, BR, TL, TR = 0..7): the first and
// second neighbour across side s are 2s and 2s+1; a neighbour's first entry on the
// side facing back is 2(s^1).  The corner neighbours used at the ends of a coarse
// side: BR of LB, BL of RB, LT of BL, LB of TL (low end) and TR of LT, TL of RT,
// RT of BR, RB of TR (high end).
__device__ __forceinline__ int corner_low(int s) { return (0x0145 >> (4 * s)) & 0xF; }
__device__ __forceinline__ int corner_high(int s) { return (0x2367 >> (4 * s)) & 0xF; }

template <class T> struct Acc324 {
    const T* a;
    __device__ __forceinline__ T operator()(int b, int x, int y) const { return a[(size_t)b * 324 + (y + 1) * 18 + (x + 1)]; }
};
template <class T> struct Acc256 {
    const T* a;
    __device__ __forceinline__ T operator()(int b, int x, int y) const { return a[(size_t)b * 256 + y * 16 + x]; }
};

// How one halo cell (or one outer stencil value) is formed from block cells.
template <class T> struct CellRule {
    int kind;  // 0 copy, 1 mean of four, 2 three-point weights, 3 bilinear in one coarse 2x2 cell patch
    int b[4], x[4], y[4];
    T w1, w2, w3;  // kind 2 weights; kind 3: w1, w2 = interpolation point
};

template <class T> __device__ __forceinline__ void rule_cell(CellRule<T>& r, int k, int b, int x, int y)
{
    r.b[k] = b;
    r.x[k] = x;
    r.y[k] = y;
}

// fillLeft / fillRight / fillBot / fillTop (src/Halo.cu:2083-2286, 2818-3020,
// 3685-3900, 4394-4600): halo cell j of side s of block ib.  A domain edge
// (neighbour == self) copies the block's own edge cell; a same-level neighbour is
// copied; a finer one is restricted (mean of its 2x2 cells next to the face); a
// coarser one is interpolated with the barycentric weights 1/3, 1/6, 1/2 and the
// reference's special weights at the two ends of the side.
template <class T> __device__ CellRule<T> halo_rule(const int* nbr, int nbm, const int* lv, int ib, int s, int j)
{
    CellRule<T> r;
    r.w1 = r.w2 = r.w3 = (T)0;
    const int nb1 = nbr[(2 * s) * nbm + ib], nb2 = nbr[(2 * s + 1) * nbm + ib];
    int x, y;
    auto copy_own = [&]() {
        r.kind = 0;
        own_xy(s, 0, j, x, y);
        rule_cell(r, 0, ib, x, y);
    };
    auto mean4 = [&](int nb, int jj) {
        r.kind = 1;
        for (int k = 0; k < 4; k++) {
            nb_xy(s, k & 1, jj + (k >> 1), x, y);
            rule_cell(r, k, nb, x, y);
        }
    };
    if (nb1 == ib) {
        if (j < BW / 2 || nb2 == ib) copy_own();
        else mean4(nb2, (j - BW / 2) * 2);
    } else if (lv[nb1] == lv[ib]) {
        r.kind = 0;
        nb_xy(s, 0, j, x, y);
        rule_cell(r, 0, nb1, x, y);
    } else if (lv[nb1] > lv[ib]) {
        if (j < BW / 2) mean4(nb1, 2 * j);
        else if (nb2 == ib) copy_own();
        else mean4(nb2, (j - BW / 2) * 2);
    } else {
        const int cj = (j + 1) >> 1;  // ceil(j / 2)
        const bool low = nbr[(2 * (s ^ 1)) * nbm + nb1] == ib;
        const int jj = low ? cj : cj + BW / 2;
        T w1 = (T)(1.0 / 3.0);
        T w2 = cj * 2 > j ? (T)(1.0 / 6.0) : (T)(0.5);
        T w3 = cj * 2 > j ? (T)(0.5) : (T)(1.0 / 6.0);
        int bir = nb1, jr = jj, bit = nb1, jt = jj - 1;
        if (low) {
            if (j == 0) {
                const int c = nbr[corner_low(s) * nbm + nb1];
                if (c == nb1) {
                    // the left side evaluates this weight in T, the other sides in double
                    w3 = s == 0 ? (T)0.5 * ((T)1.0 - w1) : (T)(0.5 * (1.0 - (double)w1));
                    w2 = w3;
                    bit = bir;
                    jt = jr;
                } else if (lv[c] < lv[nb1]) {
                    w1 = (T)(4.0 / 10.0); w2 = (T)(5.0 / 10.0); w3 = (T)(1.0 / 10.0);
                    bit = c; jt = BW - 1;
                } else if (lv[c] == lv[nb1]) {
                    bit = c; jt = BW - 1;
                } else {
                    w1 = (T)(1.0 / 4.0); w2 = (T)(1.0 / 2.0); w3 = (T)(1.0 / 4.0);
                    bit = c; jt = BW - 1;
                }
            }
        } else if (j == BW - 1) {
            const int c = nbr[corner_high(s) * nbm + nb2];
            if (c == nb2) {
                w3 = (T)(0.5 * (1.0 - (double)w1));
                w2 = w3;
                bir = bit;
                jr = jt;
            } else if (lv[c] < lv[nb2]) {
                w1 = (T)(4.0 / 10.0); w2 = (T)(1.0 / 10.0); w3 = (T)(5.0 / 10.0);
                bir = c; jr = 0;
            } else if (lv[c] == lv[nb2]) {
                bir = c; jr = 0;
            } else {
                w1 = (T)(1.0 / 4.0); w2 = (T)(1.0 / 2.0); w3 = (T)(1.0 / 4.0);
                bir = c; jr = 0;
            }
        }
        r.kind = 2;
        own_xy(s, 0, j, x, y);
        rule_cell(r, 0, ib, x, y);
        nb_xy(s, 0, jr, x, y);
        rule_cell(r, 1, bir, x, y);
        nb_xy(s, 0, jt, x, y);
        rule_cell(r, 2, bit, x, y);
        r.w1 = w1; r.w2 = w2; r.w3 = w3;
    }
    return r;
}

// BilinearInterpolation (src/Util_CPU.cu:129-144) on the unit square.
template <class T> __device__ __forceinline__ T bilinear01(T q11, T q12, T q21, T q22, T x, T y)
{
    const T x1 = (T)0.0, x2 = (T)1.0, y1 = (T)0.0, y2 = (T)1.0;
    T x2x1 = x2 - x1, y2y1 = y2 - y1, x2x = x2 - x, y2y = y2 - y, yy1 = y - y1, xx1 = x - x1;
    return (T)1.0 / (x2x1 * y2y1) * (q11 * x2x * y2y + q21 * xx1 * y2y + q12 * x2x * yy1 + q22 * xx1 * yy1);
}

// Outer stencil value of the halo gradients and the halo wet-slope reset
// (gradientHalo{Left,Right,Bot,Top}, src/Gradients.cu:2713-3290;
// WetsloperesetHalo*CPU, src/Gradients.cu:1399-2580): the value one cell beyond
// halo cell t of side s.  Restrictions of a finer neighbour average the cells at
// depth 2 and 3 (left/bottom sides list depth 2 first, right/top depth 3 first);
// a coarser neighbour is interpolated bilinearly inside its 2x2 patch, which may
// reach into that neighbour's own halo.
template <class T> __device__ CellRule<T> outer_rule(const int* nbr, int nbm, const int* lv, int ib, int s, int t)
{
    CellRule<T> r;
    r.w1 = r.w2 = r.w3 = (T)0;
    const int nb1 = nbr[(2 * s) * nbm + ib], nb2 = nbr[(2 * s + 1) * nbm + ib];
    int x, y;
    auto copy_own = [&]() {
        r.kind = 0;
        own_xy(s, 0, t, x, y);
        rule_cell(r, 0, ib, x, y);
    };
    const int d0 = (s == 0 || s == 2) ? 2 : 3, d1 = 5 - d0;
    auto mean4 = [&](int nb, int jj) {
        r.kind = 1;
        for (int k = 0; k < 4; k++) {
            nb_xy(s, (k & 1) ? d1 : d0, jj + (k >> 1), x, y);
            rule_cell(r, k, nb, x, y);
        }
    };
    if (nb1 == ib) {
        if (t < BW / 2 || nb2 == ib) copy_own();
        else mean4(nb2, (t - BW / 2) * 2);
    } else if (lv[ib] == lv[nb1]) {
        r.kind = 0;
        nb_xy(s, 1, t, x, y);
        rule_cell(r, 0, nb1, x, y);
    } else if (lv[nb1] > lv[ib]) {
        if (t < BW / 2) mean4(nb1, 2 * t);
        else if (nb2 == ib) copy_own();
        else mean4(nb2, (t - BW / 2) * 2);
    } else {
        const int cj = (t + 1) >> 1;
        const int jj = nbr[(2 * (s ^ 1)) * nbm + nb1] == ib ? cj : cj + BW / 2;
        const T jr = cj * 2 > t ? (T)0.25 : (T)0.75;
        // ii = (depth 0, jj), ir = (depth 1, jj), it = (depth 0, jj-1), itr = (depth 1, jj-1)
        int xi, yi, xr, yr, xt, yt, xtr, ytr;
        nb_xy(s, 0, jj, xi, yi);
        nb_xy(s, 1, jj, xr, yr);
        nb_xy(s, 0, jj - 1, xt, yt);
        nb_xy(s, 1, jj - 1, xtr, ytr);
        r.kind = 3;
        // corner order q11, q12, q21, q22 and the interpolation point of each side
        if (s == 0) {
            rule_cell(r, 0, nb1, xtr, ytr); rule_cell(r, 1, nb1, xr, yr);
            rule_cell(r, 2, nb1, xt, yt); rule_cell(r, 3, nb1, xi, yi);
            r.w1 = (T)0.75; r.w2 = jr;
        } else if (s == 1) {
            rule_cell(r, 0, nb1, xt, yt); rule_cell(r, 1, nb1, xi, yi);
            rule_cell(r, 2, nb1, xtr, ytr); rule_cell(r, 3, nb1, xr, yr);
            r.w1 = (T)0.25; r.w2 = jr;
        } else if (s == 2) {
            rule_cell(r, 0, nb1, xtr, ytr); rule_cell(r, 1, nb1, xt, yt);
            rule_cell(r, 2, nb1, xr, yr); rule_cell(r, 3, nb1, xi, yi);
            r.w1 = jr; r.w2 = (T)0.75;
        } else {
            rule_cell(r, 0, nb1, xt, yt); rule_cell(r, 1, nb1, xtr, ytr);
            rule_cell(r, 2, nb1, xi, yi); rule_cell(r, 3, nb1, xr, yr);
            r.w1 = jr; r.w2 = (T)0.25;
        }
    }
    return r;
}

template <class T, class A> __device__ __forceinline__ T rule_eval(const CellRule<T>& r, const A& a)
{
    if (r.kind == 0) return a(r.b[0], r.x[0], r.y[0]);
    if (r.kind == 1)
        return (T)0.25 * (a(r.b[0], r.x[0], r.y[0]) + a(r.b[1], r.x[1], r.y[1]) + a(r.b[2], r.x[2], r.y[2]) +
                          a(r.b[3], r.x[3], r.y[3]));
    if (r.kind == 2)
        return r.w1 * a(r.b[0], r.x[0], r.y[0]) + r.w2 * a(r.b[1], r.x[1], r.y[1]) + r.w3 * a(r.b[2], r.x[2], r.y[2]);
    return bilinear01<T>(a(r.b[0], r.x[0], r.y[0]), a(r.b[1], r.x[1], r.y[1]), a(r.b[2], r.x[2], r.y[2]),
                         a(r.b[3], r.x[3], r.y[3]), r.w1, r.w2);
}

// Parent of a prolongated halo cell: the coarse neighbour's cell that contains it
// (refine_linear* and WetDryProlongation, src/Halo.cu:1044-1394,
// src/ConserveElevation.cu:80-203).  Returns false when side s of block ib does not
// face a coarser block.
__device__ __forceinline__ bool parent_cell(const int* nbr, int nbm, const int* lv, int ib, int s, int j, int& pb,
                                            int& px, int& py)
{
    const int nb1 = nbr[(2 * s) * nbm + ib];
    if (!(lv[nb1] < lv[ib])) return false;
    const int fj = j >> 1;
    const int jp = nbr[(2 * (s ^ 1)) * nbm + nb1] == ib ? fj : fj + BW / 2;
    pb = nb1;
    nb_xy(s, 0, jp, px, py);
    return true;
}

// Linear reconstruction of a halo cell inside its coarser parent
// (refine_linear_{Left,Right,Bot,Top}, src/Halo.cu:1044-1394): the parent value
// plus the parent's limited gradients times half the fine spacing, toward the
// halo cell.  Left and top evaluate the offset in double, right and bottom in T.
template <class T, class A>
__device__ __forceinline__ T refine_value(const A& z, const A& gx, const A& gy, int s, int j, int pb, int px, int py,
                                          int level, T delta0, double delta0_d)
{
    const T zi = z(pb, px, py), dx = gx(pb, px, py), dy = gy(pb, px, py);
    const T odd = (j & 1) ? (T)1.0 : (T)-1.0;  // fj * 2 < j - 0.01
    T faclr, facbt;
    if (s == 0) { faclr = (T)1.0; facbt = odd; }
    else if (s == 1) { faclr = (T)-1.0; facbt = odd; }
    else if (s == 2) { facbt = (T)1.0; faclr = odd; }
    else { facbt = (T)-1.0; faclr = odd; }
    if (s == 0 || s == 3) {
        const double ilevdx = (level < 0 ? delta0_d * (double)(1 << (-level)) : delta0_d / (double)(1 << level)) *
                              (double)(T)0.5;
        return (T)((double)zi + (double)(faclr * dx + facbt * dy) * ilevdx);
    }
    const T ilevdx = calcres<T>(delta0, level) * (T)0.5;
    return zi + (faclr * dx + facbt * dy) * ilevdx;
}

namespace adapt {

// Device view of the refinement pass (bgf_adapt.cu).
// A target-level map of the Targetlevel criterion: nx*ny nodes from (xo, yo) with
// spacings dx, dy (integer levels held as float, which represents them exactly).
struct TargetMapDev {
    const float* val;
    int nx, ny;
    double xo, yo, dx, dy, xmax, ymax;
};

template <class T> struct AdaptDev {
    T* W[4];            // h, zs, u, v on 18x18 tiles of the old mesh
    T* zs;              // zs of the state, 256 per block
    const float* dem;   // bathymetry grid, dnx * dny nodes
    int dnx, dny;
    double dxo, dyo, ddx, dxmax, dymax;
    const int* child;   // [nblkmem][3]: bottom-right, top-left, top-right children, or -1
    uint8_t* flags;     // one byte per block id
};

}  // namespace adapt
}  // namespace bgf
