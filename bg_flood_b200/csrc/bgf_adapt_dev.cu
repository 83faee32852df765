// The table work of the refinement pass on the device: the sanity pass over the
// refine / coarsen flags, the new block ids and active list, and the neighbour
// tables of the new quadtree.  Same rules and same results as the host version in
// bgf_adapt_host.cpp (refinesanitycheck, CalcAvailblk, coarsen, refine,
// Adaptationcleanup; src/Adaptation.cu:157-312, 535-596, 677-1876):
//
//  * sanity: clamps at min/max level; with coarsening allowed, no coarsening next to
//    a refining block or a finer first neighbour; the forced refinement of coarser
//    first neighbours (checkneighbourrefine) is a monotone fixpoint, iterated here
//    a fixed number of times (the chain of forced blocks steps one level coarser
//    each time, so levels + 1 rounds reach it); the reference's in-place quad rule
//    in active order becomes: the lower-left block keeps its flag when its three
//    siblings are flagged and all come after it in the active list.
//  * ids: the k-th refined block of the active list takes the free ids 3k..3k+2 of
//    the ids inactive before the pass (prefix sums over the ids), merged quads keep
//    their lower-left id, the active list keeps its order without the merged
//    siblings and appends the children (prefix sums over the active list).
//  * neighbours: every block of the new mesh is entered in a dense index grid of
//    its level (integer block coordinates from its origin); each side then finds a
//    same-level block, a coarser one or two finer ones, as the host rebuild does.
//
// Compiled without FMA contraction, so the origins are computed as on the host.
#include <cuda_runtime.h>

#include "bgf_internal.h"

namespace bgf {
namespace adapt {

namespace {

enum { LB = 0, LT = 1, RB = 2, RT = 3, BL = 4, BR = 5, TL = 6, TR = 7 };

__device__ __forceinline__ double calcres_dd(double dx, int level)
{
    return level < 0 ? dx * (double)(1 << (-level)) : dx / (double)(1 << level);
}
__device__ __forceinline__ int block_index_d(double o, double dxl) { return (int)floor((o / dxl - 0.5) / 16.0 + 0.5); }
__device__ __forceinline__ double round_t(double v, int dbl) { return dbl ? v : (double)(float)v; }

// ---------------------------------------------------------------- prefix sums
constexpr int SCAN_T = 256, SCAN_V = 4, SCAN_TILE = SCAN_T * SCAN_V;

__device__ __forceinline__ int block_excl_scan(int v, int* sh, int& total)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[w] = x;
    __syncthreads();
    if (w == 0) {
        int s = lane < SCAN_T / 32 ? sh[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < SCAN_T / 32) sh[lane] = s;
    }
    __syncthreads();
    const int before = (w > 0 ? sh[w - 1] : 0) + x - v;
    total = sh[SCAN_T / 32 - 1];
    __syncthreads();
    return before;
}

// tile-local exclusive sums and tile totals
__global__ void __launch_bounds__(SCAN_T) scan_tiles_kernel(const int* in, int* out, int n, int* tile_sum)
{
    __shared__ int sh[SCAN_T / 32];
    const int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_V;
    int v[SCAN_V], s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_V; k++) {
        v[k] = base + k < n ? in[base + k] : 0;
        s += v[k];
    }
    int total;
    int run = block_excl_scan(s, sh, total);
#pragma unroll
    for (int k = 0; k < SCAN_V; k++) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
    if (threadIdx.x == 0) tile_sum[blockIdx.x] = total;
}

// exclusive sums of the tile totals (one CTA, any number of tiles); total into *sum
__global__ void __launch_bounds__(SCAN_T) scan_sums_kernel(int* tile_sum, int ntiles, int* sum)
{
    __shared__ int sh[SCAN_T / 32];
    int carry = 0;
    for (int b = 0; b < ntiles; b += SCAN_T) {
        const int i = b + threadIdx.x;
        const int v = i < ntiles ? tile_sum[i] : 0;
        int total;
        const int before = block_excl_scan(v, sh, total);
        if (i < ntiles) tile_sum[i] = carry + before;
        carry += total;
    }
    if (threadIdx.x == 0) *sum = carry;
}

__global__ void __launch_bounds__(SCAN_T) scan_add_kernel(int* out, int n, const int* tile_sum)
{
    const int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_V;
    const int add = tile_sum[blockIdx.x];
#pragma unroll
    for (int k = 0; k < SCAN_V; k++)
        if (base + k < n) out[base + k] += add;
}

// ---------------------------------------------------------------- sanity pass
__global__ void pos_kernel(const int* active, int nblk, int* pos)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < nblk) pos[active[p]] = p;
}

__global__ void coarsen_not_refine_kernel(const int* active, int nblk, const uint8_t* refine, uint8_t* coarsen)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < nblk) coarsen[active[p]] = refine[active[p]] ? 0 : 1;
}

__global__ void clamp_kernel(const int* active, int nblk, const int* level, int minlevel, int maxlevel, int allow,
                             uint8_t* refine, uint8_t* coarsen)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nblk) return;
    const int ib = active[p];
    if (refine[ib] && level[ib] == maxlevel) refine[ib] = 0;
    if (coarsen[ib] && level[ib] == minlevel) coarsen[ib] = 0;
    if (!allow || refine[ib]) coarsen[ib] = 0;
}

__global__ void no_coarsen_near_refine_kernel(const int* active, int nblk, const int* nbr, int nbm,
                                              const uint8_t* refine, uint8_t* coarsen)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nblk) return;
    const int ib = active[p];
    if (!refine[ib]) return;
    for (int k = 0; k < 8; k++) coarsen[nbr[k * nbm + ib]] = 0;
}

__global__ void no_coarsen_near_finer_kernel(const int* active, int nblk, const int* nbr, int nbm, const int* level,
                                             uint8_t* coarsen)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nblk) return;
    const int ib = active[p];
    const int l = level[ib];
    if (coarsen[ib] && (l < level[nbr[LB * nbm + ib]] || l < level[nbr[RB * nbm + ib]] || l < level[nbr[TL * nbm + ib]] ||
                        l < level[nbr[BL * nbm + ib]]))
        coarsen[ib] = 0;
}

__global__ void cascade_kernel(const int* active, int nblk, const int* nbr, int nbm, const int* level, uint8_t* refine,
                               uint8_t* coarsen)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nblk) return;
    const int ib = active[p];
    if (!refine[ib]) return;
    const int sides[4] = {TL, BL, LB, RB};
    for (int k = 0; k < 4; k++) {
        const int nb = nbr[sides[k] * nbm + ib];
        if (level[nb] < level[ib] && !refine[nb]) {
            refine[nb] = 1;
            coarsen[nb] = 0;
        }
        if (level[nb] == level[ib]) coarsen[nb] = 0;
    }
}

// the quad rule on the flags in `cin`; result in `cout`
__global__ void quad_kernel(const int* active, int nblk, const int* nbr, int nbm, const int* level, const double* xo,
                            const double* yo, double dx, const int* pos, const uint8_t* cin, uint8_t* cout)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nblk) return;
    const int ib = active[p];
    uint8_t keep = 0;
    if (cin[ib]) {
        const int l = level[ib];
        const double dxl = calcres_dd(dx, l);
        const int ix = (int)(xo[ib] / dxl / 16.0), iy = (int)(yo[ib] / dxl / 16.0);
        const int r = nbr[RB * nbm + ib], t = nbr[TL * nbm + ib], trn = nbr[TR * nbm + ib];
        const int tr = nbr[RB * nbm + trn];
        const bool corner = ix % 2 == 0 && iy % 2 == 0 && r != ib && t != ib && tr != trn;
        keep = corner && level[r] == l && level[t] == l && level[tr] == l && cin[r] && cin[t] && cin[tr] &&
               pos[r] > p && pos[t] > p && pos[tr] > p;
    }
    cout[ib] = keep;
}

// ---------------------------------------------------------------- ids and tables
// per active position: refine, parent and keep flags; the siblings of a parent are gone
__global__ void mark_kernel(const int* active, int nblk, const int* nbr, int nbm, const uint8_t* refine,
                            const uint8_t* parent, int* fr, int* fq, uint8_t* gone)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nblk) return;
    const int ib = active[p];
    fr[p] = refine[ib] ? 1 : 0;
    fq[p] = parent[ib] ? 1 : 0;
    if (parent[ib]) {
        const int r = nbr[RB * nbm + ib], t = nbr[TL * nbm + ib], tr = nbr[TL * nbm + r];
        gone[r] = gone[t] = gone[tr] = 1;
    }
}

__global__ void keep_kernel(const int* active, int nblk, const uint8_t* gone, int* fk)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < nblk) fk[p] = gone[active[p]] ? 0 : 1;
}

__global__ void free_kernel(const int* pos, int nbm, int* ff)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nbm) ff[i] = pos[i] < 0 ? 1 : 0;
}

__global__ void avail_kernel(const int* pos, int nbm, const int* sf, int* avail)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nbm && pos[i] < 0) avail[sf[i]] = i;
}

// New active list, levels and origins; children (three per refined block, -1
// otherwise), merged quads (parent, right, top, top-right) and the refined blocks
// with their children in active order.
__global__ void build_kernel(const int* active, int nblk, const int* nbr, int nbm, const int* level, const double* xo,
                             const double* yo, double dx, int dbl, const uint8_t* refine, const uint8_t* parent,
                             const uint8_t* gone, const int* sr, const int* sq, const int* sk, int nkeep,
                             const int* avail, int* nact, int* nlev, double* nxo, double* nyo, int* child, int* quads,
                             int* reflist)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nblk) return;
    const int ib = active[p];
    if (gone[ib]) return;
    nact[sk[p]] = ib;
    const int l = level[ib];
    if (parent[ib]) {
        // coarsen: the reference adds T(calcres(dx, level + 1)) to the T origin
        const double c = round_t(calcres_dd(dx, l + 1), dbl);
        nxo[ib] = round_t(xo[ib] + c, dbl);
        nyo[ib] = round_t(yo[ib] + c, dbl);
        nlev[ib] = l - 1;
        const int r = nbr[RB * nbm + ib], t = nbr[TL * nbm + ib], tr = nbr[TL * nbm + r];
        int* q = quads + 4 * (size_t)sq[p];
        q[0] = ib; q[1] = r; q[2] = t; q[3] = tr;
    }
    if (refine[ib]) {
        const int k = sr[p];
        const int kids[4] = {ib, avail[3 * k], avail[3 * k + 1], avail[3 * k + 2]};
        const double delx = calcres_dd(dx, l + 1);
        const double xoblk = xo[ib] - 0.5 * delx, yoblk = yo[ib] - 0.5 * delx;
        for (int q = 0; q < 4; q++) {
            nxo[kids[q]] = round_t(xoblk + (q & 1 ? 16 * delx : 0.0), dbl);
            nyo[kids[q]] = round_t(yoblk + (q >> 1 ? 16 * delx : 0.0), dbl);
            nlev[kids[q]] = l + 1;
        }
        for (int q = 1; q < 4; q++) {
            child[3 * (size_t)ib + q - 1] = kids[q];
            nact[nkeep + 3 * k + q - 1] = kids[q];
        }
        int* rl = reflist + 4 * (size_t)k;
        rl[0] = ib; rl[1] = kids[1]; rl[2] = kids[2]; rl[3] = kids[3];
    }
}

struct GridsDev {
    int* g;            // all levels' grids
    int off[16];       // start of level l's grid
    int w[16], hgt[16];
    int nlev;
};

__global__ void coords_kernel(const int* nact, int n, const int* nlev, const double* nxo, const double* nyo, double dx,
                              GridsDev G, int* bx, int* by, int* err)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int ib = nact[p];
    const int l = nlev[ib];
    const double dxl = calcres_dd(dx, l);
    const int x = block_index_d(nxo[ib], dxl), y = block_index_d(nyo[ib], dxl);
    bx[ib] = x;
    by[ib] = y;
    if (l < 0 || l >= G.nlev || x < 0 || y < 0 || x >= G.w[l] || y >= G.hgt[l]) {
        atomicOr(err, 1);
        return;
    }
    G.g[G.off[l] + (size_t)y * G.w[l] + x] = ib;
}

__device__ __forceinline__ int grid_find(const GridsDev& G, int l, int x, int y)
{
    if (l < 0 || l >= G.nlev || x < 0 || y < 0 || x >= G.w[l] || y >= G.hgt[l]) return -1;
    return G.g[G.off[l] + (size_t)y * G.w[l] + x];
}

// neighbour tables of the new mesh (the host rebuild's rules)
__global__ void neighbours_kernel(const int* nact, int n, const int* nlev, const int* bx, const int* by, GridsDev G,
                                  int* nnbr, int nbm)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int ib = nact[p];
    const int l = nlev[ib], x = bx[ib], y = by[ib];
    const int sdx[4] = {-1, 1, 0, 0}, sdy[4] = {0, 0, -1, 1};
    for (int s = 0; s < 4; s++) {
        const int nx = x + sdx[s], ny = y + sdy[s];
        int lo = grid_find(G, l, nx, ny), hi = lo;
        if (lo < 0 && nx >= 0 && ny >= 0) {
            lo = hi = grid_find(G, l - 1, nx >> 1, ny >> 1);
            if (lo < 0) {
                int fx0, fy0, fx1, fy1;
                if (s < 2) {
                    fx0 = fx1 = 2 * nx + (s == 0 ? 1 : 0);
                    fy0 = 2 * ny;
                    fy1 = 2 * ny + 1;
                } else {
                    fy0 = fy1 = 2 * ny + (s == 2 ? 1 : 0);
                    fx0 = 2 * nx;
                    fx1 = 2 * nx + 1;
                }
                lo = grid_find(G, l + 1, fx0, fy0);
                hi = grid_find(G, l + 1, fx1, fy1);
                if (lo < 0 || hi < 0) lo = hi = -1;
            }
        }
        if (lo < 0) lo = hi = ib;
        nnbr[(size_t)(2 * s) * nbm + ib] = lo;
        nnbr[(size_t)(2 * s + 1) * nbm + ib] = hi;
    }
}

inline int cdiv(int a, int b) { return (a + b - 1) / b; }

}  // namespace

// ---------------------------------------------------------------- host driver

void scan_excl(const int* in, int* out, int n, int* tile_sum, int* total, cudaStream_t st)
{
    const int tiles = cdiv(n, SCAN_TILE);
    if (n > 0) scan_tiles_kernel<<<tiles, SCAN_T, 0, st>>>(in, out, n, tile_sum);
    scan_sums_kernel<<<1, SCAN_T, 0, st>>>(tile_sum, n > 0 ? tiles : 0, total);
    if (n > 0) scan_add_kernel<<<tiles, SCAN_T, 0, st>>>(out, n, tile_sum);
}

int dev_sanity(const DevTables& t, const DevAdaptScratch& s, uint8_t* refine, uint8_t* coarsen, int minlevel,
               int maxlevel, int allow, int fill_coarsen, double dx, cudaStream_t st)
{
    const int n = t.nblk, nb = t.nblkmem, B = 256, g = cdiv(n, B);
    cudaMemsetAsync(s.pos, 0xff, sizeof(int) * nb, st);
    pos_kernel<<<g, B, 0, st>>>(t.active, n, s.pos);
    if (fill_coarsen) coarsen_not_refine_kernel<<<g, B, 0, st>>>(t.active, n, refine, coarsen);
    clamp_kernel<<<g, B, 0, st>>>(t.active, n, t.level, minlevel, maxlevel, allow, refine, coarsen);
    int launches = 4;
    if (allow) {
        no_coarsen_near_refine_kernel<<<g, B, 0, st>>>(t.active, n, t.nbr, nb, refine, coarsen);
        no_coarsen_near_finer_kernel<<<g, B, 0, st>>>(t.active, n, t.nbr, nb, t.level, coarsen);
        launches += 2;
    }
    const int rounds = (maxlevel - minlevel) + 2;
    for (int r = 0; r < rounds; r++) cascade_kernel<<<g, B, 0, st>>>(t.active, n, t.nbr, nb, t.level, refine, coarsen);
    launches += rounds;
    if (allow) {
        quad_kernel<<<g, B, 0, st>>>(t.active, n, t.nbr, nb, t.level, t.xo, t.yo, dx, s.pos, coarsen, s.parent);
        cudaMemcpyAsync(coarsen, s.parent, nb, cudaMemcpyDeviceToDevice, st);
        launches++;
    }
    return launches;
}

int dev_tables_count(const DevTables& t, const DevAdaptScratch& s, const uint8_t* refine, const uint8_t* coarsen,
                     cudaStream_t st)
{
    const int n = t.nblk, nb = t.nblkmem, B = 256, g = cdiv(n, B);
    cudaMemsetAsync(s.gone, 0, nb, st);
    mark_kernel<<<g, B, 0, st>>>(t.active, n, t.nbr, nb, refine, coarsen, s.fr, s.fq, s.gone);
    keep_kernel<<<g, B, 0, st>>>(t.active, n, s.gone, s.fk);
    free_kernel<<<cdiv(nb, B), B, 0, st>>>(s.pos, nb, s.ff);
    scan_excl(s.fr, s.sr, n, s.tiles, s.counts + 0, st);
    scan_excl(s.fq, s.sq, n, s.tiles, s.counts + 1, st);
    scan_excl(s.fk, s.sk, n, s.tiles, s.counts + 2, st);
    scan_excl(s.ff, s.sf, nb, s.tiles, s.counts + 3, st);
    avail_kernel<<<cdiv(nb, B), B, 0, st>>>(s.pos, nb, s.sf, s.avail);
    return 4 + 4 * 3 + 1;
}

int dev_tables_build(const DevTables& t, const DevAdaptScratch& s, const uint8_t* refine, const uint8_t* coarsen,
                     double dx, int dbl, int nkeep, int nnew, int* child, int* quads, const GridSpec& gs, int* err,
                     cudaStream_t st)
{
    const int n = t.nblk, nb = t.nblkmem, B = 256;
    cudaMemcpyAsync(s.nlev, t.level, sizeof(int) * nb, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(s.nxo, t.xo, sizeof(double) * nb, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(s.nyo, t.yo, sizeof(double) * nb, cudaMemcpyDeviceToDevice, st);
    cudaMemsetAsync(child, 0xff, sizeof(int) * 3 * (size_t)nb, st);
    build_kernel<<<cdiv(n, B), B, 0, st>>>(t.active, n, t.nbr, nb, t.level, t.xo, t.yo, dx, dbl, refine, coarsen, s.gone,
                                           s.sr, s.sq, s.sk, nkeep, s.avail, s.nact, s.nlev, s.nxo, s.nyo, child, quads,
                                           s.reflist);
    GridsDev G;
    G.g = s.grids;
    G.nlev = gs.nlev;
    for (int l = 0; l < 16; l++) {
        G.off[l] = l < gs.nlev ? gs.off[l] : 0;
        G.w[l] = l < gs.nlev ? gs.w[l] : 0;
        G.hgt[l] = l < gs.nlev ? gs.h[l] : 0;
    }
    cudaMemsetAsync(s.grids, 0xff, sizeof(int) * (size_t)gs.total, st);
    coords_kernel<<<cdiv(nnew, B), B, 0, st>>>(s.nact, nnew, s.nlev, s.nxo, s.nyo, dx, G, s.bx, s.by, err);
    neighbours_kernel<<<cdiv(nnew, B), B, 0, st>>>(s.nact, nnew, s.nlev, s.bx, s.by, G, s.nnbr, nb);
    return 4;
}

}  // namespace adapt
}  // namespace bgf
