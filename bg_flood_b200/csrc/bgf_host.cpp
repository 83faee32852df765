// Host-side preparation done once per mesh: the uniform BUQ mesh (block origins
// and neighbour tables) and the bed halo / bed gradients.  These run at set-up
// time in the reference too (src/Mesh.cu:257-433, src/InitialConditions.cu:140-144).
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <vector>

#include "../../include/bg_flood_b200.h"
#include "bgf_internal.h"

namespace bgf {

namespace {

inline int ml(int i, int j, int ib) { return (i + 1) + (j + 1) * 18 + ib * 324; }

template <class T> T calcres_h(T dx, int level) { return level < 0 ? dx * (T)(1 << (-level)) : dx / (T)(1 << level); }

template <class T> T minmod2_h(T theta, T s0, T s1, T s2)
{
    if (s0 < s1 && s1 < s2) {
        T d1 = theta * (s1 - s0);
        T d2 = (s2 - s0) / (T)2.0;
        T d3 = theta * (s2 - s1);
        if (d2 < d1) d1 = d2;
        return fmin(d1, d3);
    }
    if (s0 > s1 && s1 > s2) {
        T d1 = theta * (s1 - s0), d2 = (s2 - s0) / (T)2.0, d3 = theta * (s2 - s1);
        if (d2 > d1) d1 = d2;
        return fmax(d1, d3);
    }
    return (T)0.0;
}

}  // namespace

// gradientC + gradientHalo on the bed (src/Gradients.cu:921-957, 2713-3290) for
// single-level neighbourhoods; nbr8soa is [8][nblkmem] (LB, LT, RB, RT, BL, BR, TL, TR).
template <class T>
int host_bed_gradients(int nblk, const int* active, const int* level, const int* nbr, int nblkmem, double delta_d,
                       double theta_d, const T* zb, T* dzbdx, T* dzbdy)
{
    const T theta = (T)theta_d;
    for (int ibl = 0; ibl < nblk; ibl++) {
        int ib = active[ibl];
        T delta = calcres_h<T>((T)delta_d, level[ib]);
        for (int iy = 0; iy < 16; iy++)
            for (int ix = 0; ix < 16; ix++) {
                int i = ml(ix, iy, ib);
                dzbdx[i] = minmod2_h<T>(theta, zb[ml(ix - 1, iy, ib)], zb[i], zb[ml(ix + 1, iy, ib)]) / delta;
                dzbdy[i] = minmod2_h<T>(theta, zb[ml(ix, iy - 1, ib)], zb[i], zb[ml(ix, iy + 1, ib)]) / delta;
            }
    }
    for (int ibl = 0; ibl < nblk; ibl++) {
        int ib = active[ibl];
        T delta = calcres_h<T>((T)delta_d, level[ib]);
        int LB = nbr[0 * nblkmem + ib], LT = nbr[1 * nblkmem + ib], RB = nbr[2 * nblkmem + ib],
            RT = nbr[3 * nblkmem + ib], BL = nbr[4 * nblkmem + ib], BR = nbr[5 * nblkmem + ib],
            TL = nbr[6 * nblkmem + ib], TR = nbr[7 * nblkmem + ib];
        for (int t = 0; t < 16; t++) {
            T aleft, aright, abot, atop;
            if (LB == ib) { if (LT != ib) return BGF_EINVAL; aleft = zb[ml(0, t, ib)]; }
            else if (level[LB] == level[ib]) aleft = zb[ml(14, t, LB)];
            else return BGF_EINVAL;
            if (RB == ib) { if (RT != ib) return BGF_EINVAL; aright = zb[ml(15, t, ib)]; }
            else if (level[RB] == level[ib]) aright = zb[ml(1, t, RB)];
            else return BGF_EINVAL;
            if (BL == ib) { if (BR != ib) return BGF_EINVAL; abot = zb[ml(t, 0, ib)]; }
            else if (level[BL] == level[ib]) abot = zb[ml(t, 14, BL)];
            else return BGF_EINVAL;
            if (TL == ib) { if (TR != ib) return BGF_EINVAL; atop = zb[ml(t, 15, ib)]; }
            else if (level[TL] == level[ib]) atop = zb[ml(t, 1, TL)];
            else return BGF_EINVAL;
            int i;
            i = ml(-1, t, ib);
            dzbdx[i] = minmod2_h<T>(theta, aleft, zb[i], zb[ml(0, t, ib)]) / delta;
            i = ml(16, t, ib);
            dzbdx[i] = minmod2_h<T>(theta, zb[ml(15, t, ib)], zb[i], aright) / delta;
            i = ml(t, -1, ib);
            dzbdy[i] = minmod2_h<T>(theta, abot, zb[i], zb[ml(t, 0, ib)]) / delta;
            i = ml(t, 16, ib);
            dzbdy[i] = minmod2_h<T>(theta, zb[ml(t, 15, ib)], zb[i], atop) / delta;
        }
    }
    return BGF_OK;
}

template int host_bed_gradients<float>(int, const int*, const int*, const int*, int, double, double, const float*,
                                       float*, float*);
template int host_bed_gradients<double>(int, const int*, const int*, const int*, int, double, double, const double*,
                                        double*, double*);

}  // namespace bgf

extern "C" int bgf_mesh_uniform(int nbx, int nby, double levdx, const uint8_t* present, int* nblk, int* level,
                                int* nbr8, double* xo, double* yo)
{
    if (nbx <= 0 || nby <= 0 || !nblk || !level || !nbr8) return BGF_EINVAL;
    // InitBlockxoyo (src/Mesh.cu:257-347): row-major candidate blocks, masked ones skipped.
    std::vector<int> id((size_t)nbx * nby, -1);
    int n = 0;
    for (int by = 0; by < nby; by++)
        for (int bx = 0; bx < nbx; bx++) {
            size_t k = (size_t)by * nbx + bx;
            if (present && !present[k]) continue;
            id[k] = n;
            level[n] = 0;
            if (xo) xo[n] = bx * 16.0 * levdx + 0.5 * levdx;
            if (yo) yo[n] = by * 16.0 * levdx + 0.5 * levdx;
            n++;
        }
    // InitBlockneighbours (src/Mesh.cu:351-433): neighbours by position, self at edges.
    for (int by = 0; by < nby; by++)
        for (int bx = 0; bx < nbx; bx++) {
            int b = id[(size_t)by * nbx + bx];
            if (b < 0) continue;
            int L = bx > 0 ? id[(size_t)by * nbx + bx - 1] : -1;
            int R = bx < nbx - 1 ? id[(size_t)by * nbx + bx + 1] : -1;
            int B = by > 0 ? id[(size_t)(by - 1) * nbx + bx] : -1;
            int T = by < nby - 1 ? id[(size_t)(by + 1) * nbx + bx] : -1;
            if (L < 0) L = b;
            if (R < 0) R = b;
            if (B < 0) B = b;
            if (T < 0) T = b;
            int* q = nbr8 + 8 * b;
            q[0] = L; q[1] = L; q[2] = R; q[3] = R; q[4] = B; q[5] = B; q[6] = T; q[7] = T;
        }
    *nblk = n;
    return BGF_OK;
}
