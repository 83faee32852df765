// Host side of the refinement pass: the sanity pass over the refine flags and
// the new block tables (ids, levels, origins, neighbours, active list).
//
// The reference rewires the eight neighbour tables of every refined block and of
// its neighbours incrementally (refine, src/Adaptation.cu:1017-1792).  Here the
// tables are rebuilt from the geometry of the resulting quadtree instead: every
// active block has integer coordinates (bx, by) at its level, and each side's
// neighbours are found by looking up the same level, the parent level and the
// child level.  On a 2:1-balanced quadtree this yields the reference's tables:
// a same-level or coarser neighbour fills both entries of a side, two finer
// neighbours fill the low and high entries, and a side with no block is the block
// itself.  New block ids, the order of the active list and the block origins
// follow the reference exactly, since they are visible in its outputs.
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <unordered_map>
#include <vector>

#include "../../include/bg_flood_b200.h"

namespace {

inline double calcres_d(double dx, int level)
{
    return level < 0 ? dx * (double)(1 << (-level)) : dx / (double)(1 << level);
}

inline uint64_t key(int level, int bx, int by)
{
    return ((uint64_t)(uint32_t)(level + 64) << 48) ^ ((uint64_t)(uint32_t)(bx & 0xFFFFFF) << 24) ^
           (uint64_t)(uint32_t)(by & 0xFFFFFF);
}

// Integer position of a block at its level from its origin (the first cell
// centre, relative to the domain origin): xo = (16 bx + 1/2) dx_l.
inline int block_index(double o, double dxl) { return (int)floor((o / dxl - 0.5) / 16.0 + 0.5); }

}  // namespace

// refinesanitycheck (src/Adaptation.cu:157-296), checkneighbourrefine (:298-312).
// The reference cancels every coarsening flag (:173-175); with allow_coarsen the
// flags are kept and its coarsening rules apply, in its order.
extern "C" int bgf_adapt_sanity(int nblk, const int* active, const int* level, const int* nbr8, int nblkmem,
                                int minlevel, int maxlevel, const double* xo, const double* yo, double dx,
                                int allow_coarsen, uint8_t* refine, uint8_t* coarsen)
{
    if (nblk <= 0 || nblkmem < nblk || !active || !level || !nbr8 || !refine || !coarsen) return BGF_EINVAL;
    if (allow_coarsen && (!xo || !yo || !(dx > 0.0))) return BGF_EINVAL;
    for (int ibl = 0; ibl < nblk; ibl++) {
        const int ib = active[ibl];
        if (ib < 0 || ib >= nblkmem) return BGF_EINVAL;
        for (int k = 0; k < 8; k++)
            if (nbr8[8 * ib + k] < 0 || nbr8[8 * ib + k] >= nblkmem) return BGF_EINVAL;
        if (refine[ib] && level[ib] == maxlevel) refine[ib] = 0;
        if (coarsen[ib] && level[ib] == minlevel) coarsen[ib] = 0;
        if (!allow_coarsen || refine[ib]) coarsen[ib] = 0;
    }
    auto N = [&](int ib, int k) { return nbr8[8 * ib + k]; };
    enum { LB = 0, LT = 1, RB = 2, RT = 3, BL = 4, BR = 5, TL = 6, TR = 7 };
    if (allow_coarsen) {
        // no coarsening next to a refining block
        for (int ibl = 0; ibl < nblk; ibl++) {
            const int ib = active[ibl];
            if (refine[ib])
                for (int k = 0; k < 8; k++) coarsen[N(ib, k)] = 0;
        }
        // no coarsening next to a finer block (first neighbour of each side)
        for (int ibl = 0; ibl < nblk; ibl++) {
            const int ib = active[ibl];
            const int l = level[ib];
            if (coarsen[ib] && (l < level[N(ib, LB)] || l < level[N(ib, RB)] || l < level[N(ib, TL)] ||
                                l < level[N(ib, BL)]))
                coarsen[ib] = 0;
        }
    }
    // a refining block forces its coarser first neighbours (top-left, bottom-left,
    // left-bottom, right-bottom) to refine and keeps same-level ones from coarsening,
    // until nothing changes
    static const int side_first[4] = {TL, BL, LB, RB};
    bool changed = true;
    while (changed) {
        changed = false;
        for (int ibl = 0; ibl < nblk; ibl++) {
            const int ib = active[ibl];
            if (!refine[ib]) continue;
            for (int k : side_first) {
                const int nb = N(ib, k);
                if (!refine[nb] && level[nb] < level[ib]) {
                    refine[nb] = 1;
                    coarsen[nb] = 0;
                    changed = true;
                }
                if (level[nb] == level[ib]) coarsen[nb] = 0;
            }
        }
    }
    if (!allow_coarsen) return BGF_OK;
    // a block keeps its flag only as the lower-left block of a quad whose right, top
    // and top-right blocks are on its level and flagged; active order, in place
    for (int ibl = 0; ibl < nblk; ibl++) {
        const int ib = active[ibl];
        if (!coarsen[ib]) continue;
        const double dxl = calcres_d(dx, level[ib]);
        const int ix = (int)(xo[ib] / dxl / 16.0), iy = (int)(yo[ib] / dxl / 16.0);
        const int r = N(ib, RB), t = N(ib, TL), tr = N(N(ib, TR), RB);
        const int l = level[ib];
        const bool corner = ix % 2 == 0 && iy % 2 == 0 && r != ib && t != ib && tr != N(ib, TR);
        if (!(corner && level[r] == l && level[t] == l && level[tr] == l && coarsen[r] && coarsen[t] && coarsen[tr]))
            coarsen[ib] = 0;
    }
    return BGF_OK;
}

extern "C" int bgf_refine_sanity(int nblk, const int* active, const int* level, const int* nbr8, int nblkmem,
                                 int minlevel, int maxlevel, uint8_t* refine, uint8_t* coarsen)
{
    return bgf_adapt_sanity(nblk, active, level, nbr8, nblkmem, minlevel, maxlevel, nullptr, nullptr, 0.0, 0, refine,
                            coarsen);
}

// Coarsening and refinement of the flagged blocks on host tables (CalcAvailblk,
// coarsen, refine and Adaptationcleanup, src/Adaptation.cu:535-596, 677-1015,
// 1017-1876).  Arrays are indexed by block id and sized nblkmem; nbr8 is
// [nblkmem][8] (LB, LT, RB, RT, BL, BR, TL, TR).
//   coarsen: a flagged quad parent keeps its id at level - 1; its right, top and
//   top-right blocks (siblings[3*ib + 0..2]) leave the active list and join the
//   free ids only after this pass, as the reference appends them behind the free
//   list that the refinement draws from.
//   refine: a refined block keeps its id as the bottom-left child; the k-th refined
//   block of the active list takes the free ids 3k, 3k+1, 3k+2 (ascending) of the
//   ids inactive before the pass for its bottom-right, top-left and top-right
//   children, which are appended to the active list in that order.
//   children[3*ib + 0..2] receives those ids (or -1).
// Returns BGF_ENOMEM when nblkmem has too few free block slots.
extern "C" int bgf_adapt_tables(int* nblk_io, int* active, int* level, int* nbr8, double* xo, double* yo,
                                int nblkmem, double dx, int doubleprecision, const uint8_t* refine,
                                const uint8_t* coarsen, int* children, int* siblings)
{
    if (!nblk_io || !active || !level || !nbr8 || !xo || !yo || !refine || !children) return BGF_EINVAL;
    if (coarsen && !siblings) return BGF_EINVAL;
    const int nblk = *nblk_io;
    if (nblk <= 0 || nblk > nblkmem) return BGF_EINVAL;
    std::vector<char> isactive(nblkmem, 0);
    int nref = 0;
    for (int ibl = 0; ibl < nblk; ibl++) {
        const int ib = active[ibl];
        if (ib < 0 || ib >= nblkmem || isactive[ib]) return BGF_EINVAL;
        isactive[ib] = 1;
        if (refine[ib]) nref++;
    }
    std::vector<int> avail;
    for (int ib = 0; ib < nblkmem; ib++)
        if (!isactive[ib]) avail.push_back(ib);
    if ((int)avail.size() < 3 * nref) return BGF_ENOMEM;
    for (int ib = 0; ib < nblkmem; ib++) children[3 * ib] = children[3 * ib + 1] = children[3 * ib + 2] = -1;
    if (siblings)
        for (int ib = 0; ib < nblkmem; ib++) siblings[3 * ib] = siblings[3 * ib + 1] = siblings[3 * ib + 2] = -1;

    auto round_t = [&](double v) { return doubleprecision ? v : (double)(float)v; };
    // integer positions before the pass
    std::vector<int> bx(nblkmem, 0), by(nblkmem, 0);
    std::unordered_map<uint64_t, int> old;
    old.reserve((size_t)nblk * 2);
    for (int ibl = 0; ibl < nblk; ibl++) {
        const int ib = active[ibl];
        const double dxl = calcres_d(dx, level[ib]);
        bx[ib] = block_index(xo[ib], dxl);
        by[ib] = block_index(yo[ib], dxl);
        old[key(level[ib], bx[ib], by[ib])] = ib;
    }
    // coarsening: quads merge into their lower-left block
    std::vector<char> gone(nblkmem, 0);
    if (coarsen) {
        for (int ibl = 0; ibl < nblk; ibl++) {
            const int ib = active[ibl];
            if (!coarsen[ib]) continue;
            const int l = level[ib], x = bx[ib], y = by[ib];
            if (refine[ib] || gone[ib] || (x & 1) || (y & 1)) return BGF_EINVAL;
            int sib[3];
            for (int q = 1; q < 4; q++) {
                auto it = old.find(key(l, x + (q & 1), y + (q >> 1)));
                if (it == old.end()) return BGF_EINVAL;
                const int s = it->second;
                if (refine[s] || coarsen[s] || gone[s]) return BGF_EINVAL;
                sib[q - 1] = s;
            }
            for (int q = 0; q < 3; q++) {
                siblings[3 * ib + q] = sib[q];
                gone[sib[q]] = 1;
            }
            // the reference adds T(calcres(dx, level + 1)) to the T origin
            const double c = round_t(calcres_d(dx, l + 1));
            xo[ib] = round_t(xo[ib] + c);
            yo[ib] = round_t(yo[ib] + c);
            level[ib] = l - 1;
            bx[ib] = x >> 1;
            by[ib] = y >> 1;
        }
    }
    int n = 0;
    for (int ibl = 0; ibl < nblk; ibl++)
        if (!gone[active[ibl]]) active[n++] = active[ibl];
    const int nkeep = n;
    int k = 0;
    for (int ibl = 0; ibl < nkeep; ibl++) {
        const int ib = active[ibl];
        if (!refine[ib]) continue;
        const int ibr = avail[3 * k], ibtl = avail[3 * k + 1], ibtr = avail[3 * k + 2];
        k++;
        children[3 * ib] = ibr;
        children[3 * ib + 1] = ibtl;
        children[3 * ib + 2] = ibtr;
        // origins as the reference computes them (double, stored in T)
        const double delx = calcres_d(dx, level[ib] + 1);
        const double xoblk = xo[ib] - 0.5 * delx, yoblk = yo[ib] - 0.5 * delx;
        xo[ib] = round_t(xoblk);
        yo[ib] = round_t(yoblk);
        xo[ibr] = round_t(xoblk + 16 * delx);
        yo[ibr] = round_t(yoblk);
        xo[ibtl] = round_t(xoblk);
        yo[ibtl] = round_t(yoblk + 16 * delx);
        xo[ibtr] = round_t(xoblk + 16 * delx);
        yo[ibtr] = round_t(yoblk + 16 * delx);
        const int l = level[ib] + 1, x2 = 2 * bx[ib], y2 = 2 * by[ib];
        const int kids[4] = {ib, ibr, ibtl, ibtr};
        for (int q = 0; q < 4; q++) {
            level[kids[q]] = l;
            bx[kids[q]] = x2 + (q & 1);
            by[kids[q]] = y2 + (q >> 1);
        }
        active[n] = ibr;
        active[n + 1] = ibtl;
        active[n + 2] = ibtr;
        n += 3;
    }
    for (int ibl = n; ibl < nblk; ibl++) active[ibl] = -1;
    // neighbours from the geometry of the new quadtree
    std::unordered_map<uint64_t, int> at;
    at.reserve((size_t)n * 2);
    for (int ibl = 0; ibl < n; ibl++) {
        const int ib = active[ibl];
        at[key(level[ib], bx[ib], by[ib])] = ib;
    }
    auto find = [&](int l, int x, int y) -> int {
        if (x < 0 || y < 0) return -1;
        auto it = at.find(key(l, x, y));
        return it == at.end() ? -1 : it->second;
    };
    for (int ibl = 0; ibl < n; ibl++) {
        const int ib = active[ibl];
        const int l = level[ib], x = bx[ib], y = by[ib];
        int* q = nbr8 + 8 * ib;
        // side s: (dx, dy) to the neighbour cell; fine children of that cell facing us
        const int sdx[4] = {-1, 1, 0, 0}, sdy[4] = {0, 0, -1, 1};
        for (int s = 0; s < 4; s++) {
            const int nx = x + sdx[s], ny = y + sdy[s];
            int lo = find(l, nx, ny), hi = lo;
            if (lo < 0 && nx >= 0 && ny >= 0) {
                lo = hi = find(l - 1, nx >> 1, ny >> 1);
                if (lo < 0) {
                    int fx0, fy0, fx1, fy1;
                    if (s < 2) {  // left / right: the two children in the column facing us
                        fx0 = fx1 = 2 * nx + (s == 0 ? 1 : 0);
                        fy0 = 2 * ny;
                        fy1 = 2 * ny + 1;
                    } else {      // bottom / top: the two children in the row facing us
                        fy0 = fy1 = 2 * ny + (s == 2 ? 1 : 0);
                        fx0 = 2 * nx;
                        fx1 = 2 * nx + 1;
                    }
                    lo = find(l + 1, fx0, fy0);
                    hi = find(l + 1, fx1, fy1);
                    if (lo < 0 || hi < 0) lo = hi = -1;
                }
            }
            if (lo < 0) lo = hi = ib;
            q[2 * s] = lo;
            q[2 * s + 1] = hi;
        }
    }
    *nblk_io = n;
    return BGF_OK;
}

extern "C" int bgf_refine_tables(int* nblk_io, int* active, int* level, int* nbr8, double* xo, double* yo,
                                 int nblkmem, double dx, int doubleprecision, const uint8_t* refine, int* children)
{
    return bgf_adapt_tables(nblk_io, active, level, nbr8, xo, yo, nblkmem, dx, doubleprecision, refine, nullptr,
                            children, nullptr);
}
