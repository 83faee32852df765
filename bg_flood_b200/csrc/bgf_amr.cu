// Multi-level flow step and the bed preparation (see bgf_amr.cuh for the design).
//
// One stage (predictor or corrector) of a step on a mesh with several refinement
// levels is this chain of launches over all active blocks:
//
//   amr_halo_kernel     halo of h, u, v from the neighbours' interiors (fillHalo),
//                       wet/dry restriction next to finer blocks, zs = zb + h, and
//                       the interior gradients of h, u, v of blocks that have a
//                       finer neighbour (what the neighbour's prolongation reads)
//   amr_refine_kernel   halos next to coarser blocks rebuilt by linear
//                       reconstruction in the coarse cell (refine_linear)
//   amr_wetdry_kernel   wet/dry prolongation decisions, one launch per level
//                       above the coarsest (the reference visits blocks in order,
//                       so a decision may see a coarser block's halo that the
//                       same pass already changed)
//   amr_apply_kernel    the decisions applied (depth and bed of the parent), zs
//                       recomputed on the prolongated halo
//   amr_flux2_kernel    tile with its outer stencil ring, gradients, wet-slope
//                       reset, faces with the coarse/fine source substitution,
//                       cell dtmax and the block minimum (predictor only);
//                       faces written to the stage face arrays
//   amr_update_kernel   faces next to finer blocks replaced by the mean of the two
//                       fine faces, boundary segments, flux divergence, advance
//                       (predictor: half step into the scratch arrays; corrector:
//                       full step, friction, rain, next state, time slot)
//
// The reference counterpart is FlowGPU/FlowCPU with its fillHalo, gradient,
// refine_linear, WetDryProlongation and HaloFlux calls (src/FlowCPU.cu:15-253).
#include <cuda_runtime.h>

#include "bgf_amr.cuh"
#include "bgf_internal.h"

#ifndef BGF_VARIANT
#define BGF_VARIANT exact
#endif

namespace bgf {
namespace BGF_VARIANT {

#include "bgf_stage.cuh"
#include "bgf_pair.cuh"
#include "bgf_flow2.cuh"

__device__ __forceinline__ bool has_coarser_side(const int* nbr, int nbm, const int* lv, int ib)
{
    const int l = lv[ib];
    return lv[nbr[0 * nbm + ib]] < l || lv[nbr[2 * nbm + ib]] < l || lv[nbr[4 * nbm + ib]] < l ||
           lv[nbr[6 * nbm + ib]] < l;
}

__device__ __forceinline__ bool has_finer_neighbour(const int* nbr, int nbm, const int* lv, int ib)
{
    const int l = lv[ib];
    bool f = false;
#pragma unroll
    for (int k = 0; k < 8; k++) f |= lv[nbr[k * nbm + ib]] > l;
    return f;
}

// wetdryrestriction (src/ConserveElevation.cu:676-726): a halo cell next to a finer
// neighbour whose four cells are partly wet takes the depth-weighted surface of the
// wet ones minus its own bed.  hv is the restricted depth from the halo fill.
template <class T, class HA>
__device__ __forceinline__ T wetdry_restrict(const HA& h, const Acc324<T>& zb, T eps, T zbw, int nb, int s, int j,
                                             T hv)
{
    const int jj = j < BW / 2 ? 2 * j : (j - BW / 2) * 2;
    int x0, y0;
    if (s == 0) { x0 = BW - 2; y0 = jj; }
    else if (s == 1) { x0 = 0; y0 = jj; }
    else if (s == 2) { x0 = jj; y0 = BW - 2; }
    else { x0 = jj; y0 = 0; }
    const T hii = h(nb, x0, y0), hir = h(nb, x0 + 1, y0), hit = h(nb, x0, y0 + 1), hitr = h(nb, x0 + 1, y0 + 1);
    const T iiwet = hii > eps ? (T)1.0 : (T)0.0;
    const T irwet = hir > eps ? (T)1.0 : (T)0.0;
    const T itwet = hit > eps ? (T)1.0 : (T)0.0;
    const T itrwet = hitr > eps ? (T)1.0 : (T)0.0;
    const T cwet = (iiwet + irwet + itwet + itrwet);
    T hwet = (iiwet * hii + irwet * hir + itwet * hit + itrwet * hitr);
    T zswet = (iiwet * hii) * (zb(nb, x0, y0) + hii) + (irwet * hir) * (zb(nb, x0 + 1, y0) + hir) +
              (itwet * hit) * (zb(nb, x0, y0 + 1) + hit) + (itrwet * hitr) * (zb(nb, x0 + 1, y0 + 1) + hitr);
    if (cwet > (T)0.0 && cwet < (T)4.0) {
        zswet = zswet / hwet;
        return ((T)0.0 < zswet - zbw) ? zswet - zbw : (T)0.0;
    }
    return hv;
}

// ---------------------------------------------------------------- stage state

// State of any cell as a stage reads it: state n in the predictor; in the corrector
// the half-step state h* = Advance(state n, predictor tendencies, dt / 2), rebuilt
// from the stored tendencies (the predictor advance is pointwise, so this is the
// value the reference's half-step state holds at that cell).  Blocks on one level
// among same-level neighbours run the single-level kernels, which store the same
// tendencies, so every block reads its neighbours the same way.
template <class T> struct StageState {
    const DevModel<T>& m;
    const StepParams<T>& p;
    int cur;
    bool half;
    T halfdt;
    double time;
    __device__ __forceinline__ void get(int b, int x, int y, T& ho, T& uo, T& vo) const
    {
        const size_t g = (size_t)b * 256 + y * 16 + x;
        const T hv = m.h[cur][g], uv = m.u[cur][g], vv = m.v[cur][g];
        if (!half) {
            ho = hv; uo = uv; vo = vv;
            return;
        }
        // the predictor's river source of the cell (AddRiverForcing after updateEV)
        const T dhs = add_rivers<T>(m, p, b, x, y, m.dh[g], time);
        advance<T>(halfdt, p.eps, p.eps_d, p.forcemass != 0, hv, uv, vv, dhs, m.dhu[g], m.dhv[g], ho, uo, vo);
    }
};
template <class T> struct StageComp {
    const StageState<T>& s;
    int f;
    __device__ __forceinline__ T operator()(int b, int x, int y) const
    {
        T a0, a1, a2;
        s.get(b, x, y, a0, a1, a2);
        return f == 0 ? a0 : f == 1 ? a1 : a2;
    }
};

// rule_eval of the three state components of a rule, each cell's state formed once;
// the arithmetic of each component is rule_eval's.
template <class T>
__device__ __forceinline__ void rule_eval_state(const CellRule<T>& r, const StageState<T>& S, T& ho, T& uo, T& vo)
{
    T c[4][3];
    const int nc = r.kind == 0 ? 1 : r.kind == 2 ? 3 : 4;
    for (int k = 0; k < nc; k++) S.get(r.b[k], r.x[k], r.y[k], c[k][0], c[k][1], c[k][2]);
    T out[3];
#pragma unroll
    for (int f = 0; f < 3; f++) {
        if (r.kind == 0) out[f] = c[0][f];
        else if (r.kind == 1) out[f] = (T)0.25 * (c[0][f] + c[1][f] + c[2][f] + c[3][f]);
        else if (r.kind == 2) out[f] = r.w1 * c[0][f] + r.w2 * c[1][f] + r.w3 * c[2][f];
        else out[f] = bilinear01<T>(c[0][f], c[1][f], c[2][f], c[3][f], r.w1, r.w2);
    }
    ho = out[0]; uo = out[1]; vo = out[2];
}

// ---------------------------------------------------------------- stage kernels

// Threads 0..255 copy the interior cells and threads 256..319 (two more warps) fill
// the 64 halo cells, so that the halo rules do not wait behind an interior copy.
constexpr int HALO_THREADS = NTHREADS + 64;

template <class T>
__global__ void __launch_bounds__(HALO_THREADS) amr_halo_kernel(DevModel<T> m, AmrDev<T> a, StepParams<T> p0,
                                                                 int parity, int stage)
{
    __shared__ T th[3][324];
    const int tid = threadIdx.x;
    const int ib = m.active[blockIdx.x];
    const int sc = scen_of(m, ib);
    const TimeState ts = m.time[2 * sc + parity];
    if (!step_live(ts)) return;
    const StepParams<T>& p = m.sparams ? m.sparams[sc] : p0;
    const int nbm = m.nblkmem;
    const T halfdt = stage == 0 ? (T)0 : step_dt<T>(ts, m.dtmin[2 * sc + parity]) * (T)0.5;
    const StageState<T> S{m, p, ts.cur, stage != 0, halfdt, ts.totaltime};
    T* const* W = a.W[stage];
    const size_t base = (size_t)ib * 324;
    const int x = tid & 15, y = (tid >> 4) & 15, c = hi18(x, y);
    if (tid < NTHREADS) {
        S.get(ib, x, y, th[0][c], th[1][c], th[2][c]);
        W[0][base + c] = th[0][c];
        W[2][base + c] = th[1][c];
        W[3][base + c] = th[2][c];
        W[1][base + c] = a.zb[base + c] + th[0][c];
    } else {
        const int s = (tid - NTHREADS) >> 4, j = tid & 15;
        const CellRule<T> r = halo_rule<T>(m.nbr, nbm, m.level, ib, s, j);
        T hv, uv, vv;
        rule_eval_state<T>(r, S, hv, uv, vv);
        int hx, hy;
        halo_xy(s, j, hx, hy);
        const int hc = hi18(hx, hy);
        const int nbh = m.nbr[(2 * s + (j >= BW / 2 ? 1 : 0)) * nbm + ib];
        if (a.wetdryfix && m.level[nbh] > m.level[ib])
            hv = wetdry_restrict<T>(StageComp<T>{S, 0}, Acc324<T>{a.zb}, p.eps, a.zb[base + hc], nbh, s, j, hv);
        th[0][hc] = hv;
        th[1][hc] = uv;
        th[2][hc] = vv;
        W[0][base + hc] = hv;
        W[2][base + hc] = uv;
        W[3][base + hc] = vv;
        W[1][base + hc] = a.zb[base + hc] + hv;
    }
    // gradientC (src/Gradients.cu:921-957) of h, u, v for the prolongation of the
    // finer neighbours' halos
    if (!has_finer_neighbour(m.nbr, nbm, m.level, ib)) return;
    __syncthreads();
    if (tid >= NTHREADS) return;
    const T delta = calcres<T>(p.delta0, m.level[ib]);
    const T rdelta = (T)1.0 / delta;
#pragma unroll
    for (int f = 0; f < 3; f++) {
        const T* t = th[f];
        a.G0[2 * f][base + c] = div_by(minmod2(p.theta, t[c - 1], t[c], t[c + 1]), delta, rdelta);
        a.G0[2 * f + 1][base + c] = div_by(minmod2(p.theta, t[c - 18], t[c], t[c + 18]), delta, rdelta);
    }
}

template <class T>
__global__ void __launch_bounds__(64) amr_refine_kernel(DevModel<T> m, AmrDev<T> a, StepParams<T> p0, int parity,
                                                        int stage)
{
    const int ib = m.active[blockIdx.x];
    const int sc = scen_of(m, ib);
    const TimeState ts = m.time[2 * sc + parity];
    if (!step_live(ts)) return;
    const StepParams<T>& p = m.sparams ? m.sparams[sc] : p0;
    const int s = threadIdx.x >> 4, j = threadIdx.x & 15;
    int pb, px, py;
    if (!parent_cell(m.nbr, m.nblkmem, m.level, ib, s, j, pb, px, py)) return;
    int hx, hy;
    halo_xy(s, j, hx, hy);
    const size_t o = (size_t)ib * 324 + hi18(hx, hy);
    T* const* W = a.W[stage];
#pragma unroll
    for (int f = 0; f < 3; f++) {
        const int wf = f == 0 ? 0 : f + 1;  // h, u, v in W order h, zs, u, v
        W[wf][o] = refine_value<T>(Acc324<T>{W[wf]}, Acc324<T>{a.G0[2 * f]}, Acc324<T>{a.G0[2 * f + 1]}, s, j, pb, px,
                                   py, m.level[ib], p.delta0, p.delta0_d);
    }
}

// WetDryProlongation (src/ConserveElevation.cu:80-203) for the blocks of one level:
// a halo cell next to a coarser block whose parent or any of the parent's four
// neighbours is dry takes the parent's depth and bed.  The reference visits the
// blocks in active-list order and changes halos as it goes, so the four neighbours
// of a parent that lie in the coarse block's own halo are read as already changed
// when that coarse block comes earlier in the list and its decision (made by the
// launch for its level, which runs first) says so.
template <class T>
__global__ void __launch_bounds__(64) amr_wetdry_kernel(DevModel<T> m, AmrDev<T> a, StepParams<T> p0, int parity,
                                                        int stage, int level)
{
    const int ib = m.active[blockIdx.x];
    const TimeState ts = m.time[2 * scen_of(m, ib) + parity];
    if (!step_live(ts)) return;
    if (m.level[ib] != level) return;
    const int nbm = m.nblkmem;
    const int s = threadIdx.x >> 4, j = threadIdx.x & 15;
    int pb, px, py;
    if (!parent_cell(m.nbr, nbm, m.level, ib, s, j, pb, px, py)) return;
    const T* H = a.W[stage][0];
    const T eps = (m.sparams ? m.sparams[scen_of(m, ib)] : p0).eps;
    const bool earlier = a.rank[pb] < a.rank[ib];
    auto hval = [&](int x, int y) -> T {
        const T v = H[(size_t)pb * 324 + hi18(x, y)];
        if (!earlier) return v;
        int hs, hj;
        if (x < 0) { hs = 0; hj = y; }
        else if (x >= BW) { hs = 1; hj = y; }
        else if (y < 0) { hs = 2; hj = x; }
        else if (y >= BW) { hs = 3; hj = x; }
        else return v;
        int qb, qx, qy;
        if (!parent_cell(m.nbr, nbm, m.level, pb, hs, hj, qb, qx, qy)) return v;
        if (!a.pflag[(size_t)pb * 64 + hs * 16 + hj]) return v;
        return H[(size_t)qb * 324 + hi18(qx, qy)];
    };
    const bool dry = !(hval(px, py) > eps && hval(px - 1, py) > eps && hval(px + 1, py) > eps &&
                       hval(px, py + 1) > eps && hval(px, py - 1) > eps);
    a.pflag[(size_t)ib * 64 + s * 16 + j] = dry ? 1 : 0;
}

// The prolongation decisions applied, then RecalculateZs (src/Halo.cu:72-107) on
// the halo cells next to coarser blocks.
template <class T>
__global__ void __launch_bounds__(64) amr_apply_kernel(DevModel<T> m, AmrDev<T> a, StepParams<T> p, int parity,
                                                       int stage)
{
    const int ib = m.active[blockIdx.x];
    const TimeState ts = m.time[2 * scen_of(m, ib) + parity];
    if (!step_live(ts)) return;
    const int s = threadIdx.x >> 4, j = threadIdx.x & 15;
    int pb, px, py;
    if (!parent_cell(m.nbr, m.nblkmem, m.level, ib, s, j, pb, px, py)) return;
    int hx, hy;
    halo_xy(s, j, hx, hy);
    const size_t o = (size_t)ib * 324 + hi18(hx, hy);
    const size_t po = (size_t)pb * 324 + hi18(px, py);
    T* H = a.W[stage][0];
    if (a.wetdryfix && a.pflag[(size_t)ib * 64 + s * 16 + j]) {
        H[o] = H[po];
        a.zb[o] = a.zb[po];
    }
    a.W[stage][1][o] = a.zb[o] + H[o];
}

// Resident CTAs per SM of the FP32 stage kernels (launch bounds): six, the shared-
// memory limit.  Since the tile and face loads were spread over the warps, six beat
// four or five in both builds (flux +3 % fast / +10 % bit-exact, update +6 % / +5 %)
// despite a few spilled registers; FP64 instantiations keep more registers.
template <class T> struct AmrOcc {
    static constexpr int update = sizeof(T) == 4 ? 6 : 3;
    static constexpr int flux = sizeof(T) == 4 ? 6 : 3;
};

// The multi-level flux kernel, in the two-cells-per-thread layout of the single-level kernels
// (bgf_flow2.cuh): 128 threads per block, thread (x, p) owning cells (x, 2p) and
// (x, 2p+1).  The tile comes from the stage tile W (interior and ring 1, whose
// halos the chain filled) and the outer ring rules (ring 2); gradients, wet-slope
// reset and faces are the single-level kernels' own, with the coarse/fine source
// substitution on the sides whose neighbour is coarser.  The faces go to the stage
// face arrays in the layout amr_update_kernel reads.  The same operations in the
// same order as the reference's FlowCPU: the exact build matches the oracle bit for bit.
template <class T, int ENGINE>
__global__ void __launch_bounds__(NT2, AmrOcc<T>::flux) amr_flux2_kernel(DevModel<T> m, AmrDev<T> a, StepParams<T> p0,
                                                                            int parity, int stage)
{
    using V = V2<T>;
    extern __shared__ __align__(16) unsigned char smem_raw2[];
    Smem2<T>& s = *reinterpret_cast<Smem2<T>*>(smem_raw2);
    __shared__ SubFaces<T> sub;
    const int tid = threadIdx.x;
    const int w4 = tid >> 5, lane = tid & 31;
    const int x = lane & 15;
    const int py = (w4 & 1) + 4 * (w4 >> 1) + 2 * (lane >> 4);
    const int y = 2 * py;
    const int ib = m.active[blockIdx.x];
    const int sc = scen_of(m, ib);
    const StepParams<T>& p = m.sparams ? m.sparams[sc] : p0;
    const int nbm = m.nblkmem;
    T* const* W = a.W[stage];
    const size_t base = (size_t)ib * 324;
    const T* zbt = m.zb + base;
    // every load that does not depend on the block's time slot is issued before it
    // arrives: the bed tile and gradients, the own pair and ring 1 from the stage
    // tile, the coarse/fine sources, and ring 2 inside a coarser neighbour's patch
    load_bed2<T>(s, zbt, tid);
    const BedGrad<T> bg = load_bedgrad<T, ENGINE>(m, ib, tid, x, y);
    V c[4];
#pragma unroll
    for (int v = 0; v < 4; v++) c[v] = V{W[v][base + hi18(x, y)], W[v][base + hi18(x, y + 1)]};
    CellRule<T> r{};  // ring 2 (threads 64..127)
    int o2 = 0;
    if (tid < 64) {
        // ring 1 (the block's halo, corners excluded) and the coarse/fine substitution
        const int sd = tid >> 4, t = tid & 15;
        int hx, hy;
        halo_xy(sd, t, hx, hy);
        const int c18 = hi18(hx, hy), o = p2t(hx, hy);
#pragma unroll
        for (int v = 0; v < 4; v++) s.t[v][o] = W[v][base + c18];
        int pb, px, pyy;
        const bool coarse = parent_cell(m.nbr, nbm, m.level, ib, sd, t, pb, px, pyy);
        if (t == 0) sub.on[sd] = coarse ? 1 : 0;
        if (coarse) {
            sub.h[sd][t] = W[0][(size_t)pb * 324 + hi18(px, pyy)];
            sub.z[sd][t] = a.zb[(size_t)pb * 324 + hi18(px, pyy)];
        }
    } else {
        // ring 2: the outer stencil values of the halo gradients
        const int k = tid - 64;
        const int sd = k >> 4, t = k & 15;
        r = outer_rule<T>(m.nbr, nbm, m.level, ib, sd, t);
        int rx, ry;
        halo_xy(sd, t, rx, ry);
        if (sd == 0) rx = -2;
        else if (sd == 1) rx = BW + 1;
        else if (sd == 2) ry = -2;
        else ry = BW + 1;
        o2 = p2t(rx, ry);
        if (r.kind == 3) {
            // inside a coarser neighbour's 2x2 patch, which may reach into its halo:
            // that neighbour has a finer neighbour, so it runs this chain and its
            // stage tile is filled
#pragma unroll
            for (int v = 0; v < 4; v++) s.t[v][o2] = rule_eval(r, Acc324<T>{W[v]});
        }
    }
    const TimeState ts = m.time[2 * sc + parity];
    if (!step_live(ts)) {
        bed_wait();  // (no bed copy outlives the block)
        return;
    }
    const T delta = calcres<T>(p.delta0, m.level[ib]);
    if (tid >= 64 && r.kind != 3) {
        // ring 2 at interior cells of this block or of a same-level or finer
        // neighbour, read as the stage reads any cell (the neighbour may run the
        // single-level kernels and have no stage tile): the state of the step
        const T halfdt = stage == 0 ? (T)0 : step_dt<T>(ts, m.dtmin[2 * sc + parity]) * (T)0.5;
        const StageState<T> S{m, p, ts.cur, stage != 0, halfdt, ts.totaltime};
        T cv[4][4];  // per rule cell: h, zs, u, v
        const int nc = r.kind == 0 ? 1 : 4;
        for (int q = 0; q < nc; q++) {
            S.get(r.b[q], r.x[q], r.y[q], cv[q][0], cv[q][2], cv[q][3]);
            cv[q][1] = a.zb[(size_t)r.b[q] * 324 + hi18(r.x[q], r.y[q])] + cv[q][0];
        }
#pragma unroll
        for (int v = 0; v < 4; v++)
            s.t[v][o2] = r.kind == 0 ? cv[0][v] : (T)0.25 * (cv[0][v] + cv[1][v] + cv[2][v] + cv[3][v]);
    }
    const int ct = p2t(x, y);
#pragma unroll
    for (int k = 0; k < 4; k++) st2<T>(s.t[k], ct, c[k]);
    bed_wait();
    __syncthreads();
    V xm[4], gxo[4], gyo[4];
    T ym[4];
    gradients2<T, ENGINE>(s, bg, p.theta, delta, tid, x, py, c, xm, ym, gxo, gyo);
    __syncthreads();
    V cdt = faces2<T, ENGINE, false, true>(s, p, delta, tid, x, py, c, xm, ym, gxo, gyo, (T)0, &sub);
    if (stage == 0) {
        cdt = finite_dt2<T>(c[VH], c[VU], c[VV], cdt);
        T v = cdt.b < cdt.a ? cdt.b : cdt.a;
        for (int o = 16; o > 0; o >>= 1) {
            const T q = __shfl_xor_sync(0xffffffffu, v, o);
            v = q < v ? q : v;
        }
        if (lane == 0) s.red[w4] = v;
    }
    __syncthreads();  // every face written (the right column and top row by warp 0)
    // faces to the stage face arrays: X faces at fxi(x, y) (x = 16 after the 256
    // interior faces), Y faces at fyi(x, y)
    const size_t fb = (size_t)ib * NFX;
    for (int k = tid; k < NFX; k += NT2) {
        const int ox = k < 256 ? p2fx(k & 15, k >> 4) : p2fx(BW, k - 256);
        const int oy = p2fy(k & 15, k >> 4);
#pragma unroll
        for (int v = 0; v < 4; v++) {
            a.F[v][fb + k] = s.fx[v][ox];
            a.F[4 + v][fb + k] = s.fy[v][oy];
        }
    }
    if (stage == 0 && tid == 0) {
        T b = s.red[0];
        for (int k = 1; k < NT2 / 32; k++) b = s.red[k] < b ? s.red[k] : b;
        atomicMin(&m.dtmin[2 * sc + parity], dt_bits(b));
    }
}

template <class T, int ENGINE>
__global__ void __launch_bounds__(NTHREADS, AmrOcc<T>::update) amr_update_kernel(DevModel<T> m, AmrDev<T> a, StepParams<T> p0, int parity,
                                                                 int stage)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem<T>& s = *reinterpret_cast<Smem<T>*>(smem_raw);
    const int tid = threadIdx.x;
    const int ib = m.active[blockIdx.x];
    const int sc = scen_of(m, ib);
    const bool lead = lead_of(m, ib, blockIdx.x);
    const TimeState ts = m.time[2 * sc + parity];
    if (!step_live(ts)) {
        if (stage == 1 && lead && tid == 0) {
            TimeState nt = ts;
            nt.done = 1;
            m.time[2 * sc + (parity ^ 1)] = nt;
        }
        return;
    }
    const StepParams<T>& p = m.sparams ? m.sparams[sc] : p0;
    const int nbm = m.nblkmem;
    const T delta = calcres<T>(p.delta0, m.level[ib]);
    const T dt = step_dt<T>(ts, m.dtmin[2 * sc + parity]);
    const double dtd = (double)dt;
    const size_t base = (size_t)ib * 324;
    const size_t fb = (size_t)ib * NFX;
    // one face entry and one tile entry per thread; the 16 face entries beyond 256 go
    // to threads 240..255 and the 68 tile entries beyond 256 to threads 128..195, so
    // that no warp loads three rounds while others load two
    static_assert(NTHREADS == 256 && NFX == 272, "entries beyond 256 on the upper threads");
    auto load_faces = [&](int k) {
        s.Fhu[k] = a.F[0][fb + k];
        s.Fqux[k] = a.F[1][fb + k];
        s.Su[k] = a.F[2][fb + k];
        s.Fqvx[k] = a.F[3][fb + k];
        s.Fhv[k] = a.F[4][fb + k];
        s.Fqvy[k] = a.F[5][fb + k];
        s.Sv[k] = a.F[6][fb + k];
        s.Fquy[k] = a.F[7][fb + k];
    };
    // state n on the 18x18 tile (boundary segments, full-step advance) and the bed
    auto load_tile = [&](int k) {
        const int q = si(k % 18 - 1, k / 18 - 1);
        s.zb[q] = a.zb[base + k];
        s.h0[q] = a.W[0][0][base + k];
        s.u0[q] = a.W[0][2][base + k];
        s.v0[q] = a.W[0][3][base + k];
    };
    load_faces(tid);
    load_tile(tid);
    if (tid >= 240) load_faces(tid + 16);
    if (tid >= 128 && tid < 196) load_tile(tid + 128);
    // uniform rain: the depth of the step is the same for every cell of the scenario;
    // one thread evaluates the series (AddrainforcingImplicitCPU) for the block
    __shared__ T rain_step;
    if (stage == 1 && p.has_rain && !p.rain_map && tid == 0) {
        const T r = (T)series_at(m.rain_t + p.rain_off, m.rain_r + p.rain_off, p.rain_n, ts.totaltime,
                                 p.rain_sorted != 0);
        rain_step = M<T>::fmax_(r / (T)1000.0 / (T)3600.0 * (T)dtd, (T)0.0);
    }
    __syncthreads();
    // HaloFluxCPULR / HaloFluxCPUBT (src/Halo.cu:1441-1540, 1766-1850): the faces of
    // a side with finer neighbours take the mean of the two fine faces
    if (tid < 64) {
        const int sd = tid >> 4, j = tid & 15;
        const int nbh = m.nbr[(2 * sd + (j >= BW / 2 ? 1 : 0)) * nbm + ib];
        if (m.level[nbh] > m.level[ib]) {
            const int jj = j < BW / 2 ? 2 * j : (j - BW / 2) * 2;
            const size_t nf = (size_t)nbh * NFX;
            int own, f0, f1, a0;
            if (sd == 0) { own = fxi(0, j); f0 = fxi(BW, jj); f1 = fxi(BW, jj + 1); a0 = 0; }
            else if (sd == 1) { own = fxi(BW, j); f0 = fxi(0, jj); f1 = fxi(0, jj + 1); a0 = 0; }
            else if (sd == 2) { own = fyi(j, 0); f0 = fyi(jj, BW); f1 = fyi(jj + 1, BW); a0 = 4; }
            else { own = fyi(j, BW); f0 = fyi(jj, 0); f1 = fyi(jj + 1, 0); a0 = 4; }
            T* dst[4];
            if (a0 == 0) { dst[0] = s.Fhu; dst[1] = s.Fqux; dst[2] = s.Su; dst[3] = s.Fqvx; }
            else { dst[0] = s.Fhv; dst[1] = s.Fqvy; dst[2] = s.Sv; dst[3] = s.Fquy; }
#pragma unroll
            for (int q = 0; q < 4; q++) dst[q][own] = (T)0.5 * (a.F[a0 + q][nf + f0] + a.F[a0 + q][nf + f1]);
        }
    }
    __syncthreads();
    if (block_has_segments<T>(m, ib)) {  // interior blocks skip the step and its barrier
        apply_boundaries<T>(s, m, p, ib, stage == 0 ? ts.totaltime + ts.dt * 0.5 : ts.totaltime + dtd, tid);
        __syncthreads();
    }
    const int x = tid & 15, y = tid >> 4;
    const int c18 = hi18(x, y), q18 = si(x, y);
    const T hs = a.W[stage][0][base + c18], us = a.W[stage][2][base + c18], vs = a.W[stage][3][base + c18];
    T dh, dhu, dhv;
    flux_divergence<T>(s, p, (T)1.0 / ((T)1.0 * delta), x, y, hs, us, vs, dh, dhu, dhv);
    const size_t g = (size_t)ib * 256 + tid;
    if (stage == 0) {
        // predictor: the tendencies (before the river source), from which the
        // corrector rebuilds the half-step state of any cell (StageState)
        m.dh[g] = dh;
        m.dhu[g] = dhu;
        m.dhv[g] = dhv;
        return;
    }
    dh = add_rivers<T>(m, p, ib, x, y, dh, ts.totaltime);
    const T hold = s.h0[q18], uold = s.u0[q18], vold = s.v0[q18];
    T ho, uo, vo;
    advance<T>(dt, p.eps, p.eps_d, p.forcemass != 0, hold, uold, vold, dh, dhu, dhv, ho, uo, vo);
    const T cfv = p.has_cf ? m.cf[g] : p.cf;
    bottom_friction<T>(p.frictionmodel, p.g, p.eps, dt, cfv, ho, uo, vo);
    if (p.has_rain) {
        // AddrainforcingImplicitCPU (src/Updateforcing.cu:530-580): the rain rate at the
        // start of the step, uniform or gridded
        T Rainhh;
        const T mask = m.rainmask ? (T)m.rainmask[g] : (T)1;
        if (p.rain_map) {
            const T xc = (T)p.xo_d + (T)m.bxo[ib] + (T)x * delta;
            const T yc = (T)p.yo_d + (T)m.byo[ib] + (T)y * delta;
            Rainhh = rain_map_at<T>(m.rmap, xc, yc, ts.totaltime);
            Rainhh = M<T>::fmax_(Rainhh / (T)1000.0 / (T)3600.0 * (T)dtd, (T)0.0) * mask;
        } else {
            Rainhh = rain_step * mask;
        }
        const T hi = ho;
        const T qvol = hi / (hi + Rainhh);
        ho = hi + Rainhh;
        if ((double)hi > p.eps_d) {
            uo = uo * qvol;
            vo = vo * qvol;
        }
    }
    const int nxt = ts.cur ^ 1;
    m.h[nxt][g] = ho;
    m.u[nxt][g] = uo;
    m.v[nxt][g] = vo;
    if (m.hmax) m.hmax[g] = ho > m.hmax[g] ? ho : m.hmax[g];
    if (lead && tid == 0) m.time[2 * sc + (parity ^ 1)] = next_time_state<T>(ts, p, dtd, nxt, m.dtmin + 2 * sc, parity);
}

// ---------------------------------------------------------------- bed preparation

// fillHaloC on the bed (src/Halo.cu:16-51): halo from the neighbours' interiors.
template <class T> __global__ void __launch_bounds__(64) bed_halo_kernel(DevModel<T> m, T* zb)
{
    const int ib = m.active[blockIdx.x];
    const int s = threadIdx.x >> 4, j = threadIdx.x & 15;
    const CellRule<T> r = halo_rule<T>(m.nbr, m.nblkmem, m.level, ib, s, j);
    int hx, hy;
    halo_xy(s, j, hx, hy);
    zb[(size_t)ib * 324 + hi18(hx, hy)] = rule_eval(r, Acc324<T>{zb});
}

// gradientC on the bed (src/Gradients.cu:921-957)
template <class T>
__global__ void __launch_bounds__(NTHREADS) bed_grad_kernel(DevModel<T> m, StepParams<T> p, const T* zb, T* gx, T* gy)
{
    const int ib = m.active[blockIdx.x];
    const int tid = threadIdx.x, x = tid & 15, y = tid >> 4;
    const size_t i = (size_t)ib * 324 + hi18(x, y);
    const T delta = calcres<T>(p.delta0, m.level[ib]);
    const T rdelta = (T)1.0 / delta;
    gx[i] = div_by(minmod2(p.theta, zb[i - 1], zb[i], zb[i + 1]), delta, rdelta);
    gy[i] = div_by(minmod2(p.theta, zb[i - 18], zb[i], zb[i + 18]), delta, rdelta);
}

// gradientHalo on the bed (src/Gradients.cu:2584-2605, 2713-3290)
template <class T>
__global__ void __launch_bounds__(64) bed_grad_halo_kernel(DevModel<T> m, StepParams<T> p, const T* zb, T* gx, T* gy)
{
    const int ib = m.active[blockIdx.x];
    const int s = threadIdx.x >> 4, t = threadIdx.x & 15;
    const T delta = calcres<T>(p.delta0, m.level[ib]);
    const T rdelta = (T)1.0 / delta;
    const T outer = rule_eval(outer_rule<T>(m.nbr, m.nblkmem, m.level, ib, s, t), Acc324<T>{zb});
    const Acc324<T> z{zb};
    int hx, hy;
    halo_xy(s, t, hx, hy);
    const size_t i = (size_t)ib * 324 + hi18(hx, hy);
    if (s == 0) gx[i] = div_by(minmod2(p.theta, outer, zb[i], z(ib, 0, t)), delta, rdelta);
    else if (s == 1) gx[i] = div_by(minmod2(p.theta, z(ib, BW - 1, t), zb[i], outer), delta, rdelta);
    else if (s == 2) gy[i] = div_by(minmod2(p.theta, outer, zb[i], z(ib, t, 0)), delta, rdelta);
    else gy[i] = div_by(minmod2(p.theta, z(ib, t, BW - 1), zb[i], outer), delta, rdelta);
}

// refine_linear on the bed (src/Halo.cu:1044-1394)
template <class T>
__global__ void __launch_bounds__(64) bed_refine_kernel(DevModel<T> m, StepParams<T> p, T* zb, const T* gx, const T* gy)
{
    const int ib = m.active[blockIdx.x];
    const int s = threadIdx.x >> 4, j = threadIdx.x & 15;
    int pb, px, py;
    if (!parent_cell(m.nbr, m.nblkmem, m.level, ib, s, j, pb, px, py)) return;
    int hx, hy;
    halo_xy(s, j, hx, hy);
    zb[(size_t)ib * 324 + hi18(hx, hy)] = refine_value<T>(Acc324<T>{zb}, Acc324<T>{gx}, Acc324<T>{gy}, s, j, pb, px, py,
                                                           m.level[ib], p.delta0, p.delta0_d);
}

// ---------------------------------------------------------------- launchers

template <class T> static size_t amr_smem() { return sizeof(Smem<T>); }

template <class T, int ENGINE> static cudaError_t amr_configure_engine()
{
    cudaError_t e = cudaFuncSetAttribute(amr_flux2_kernel<T, ENGINE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem2_pred<T>());
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(amr_update_kernel<T, ENGINE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)amr_smem<T>());
}

template <class T> cudaError_t configure_amr_kernels()
{
    cudaError_t e = amr_configure_engine<T, 1>();
    if (e != cudaSuccess) return e;
    return amr_configure_engine<T, 2>();
}

template <class T>
int launch_amr_stage(const DevModel<T>& m, const AmrDev<T>& a, const StepParams<T>& p, int engine, int parity, int stage,
                     int minlev, int maxlev, cudaStream_t st)
{
    const int n = m.nblk;
    int launches = 0;
    amr_halo_kernel<T><<<n, HALO_THREADS, 0, st>>>(m, a, p, parity, stage);
    amr_refine_kernel<T><<<n, 64, 0, st>>>(m, a, p, parity, stage);
    launches += 2;
    if (a.wetdryfix) {
        for (int l = minlev + 1; l <= maxlev; l++) {
            amr_wetdry_kernel<T><<<n, 64, 0, st>>>(m, a, p, parity, stage, l);
            launches++;
        }
    }
    amr_apply_kernel<T><<<n, 64, 0, st>>>(m, a, p, parity, stage);
    if (engine == 1) {
        amr_flux2_kernel<T, 1><<<n, NT2, smem2_pred<T>(), st>>>(m, a, p, parity, stage);
        amr_update_kernel<T, 1><<<n, NTHREADS, amr_smem<T>(), st>>>(m, a, p, parity, stage);
    } else {
        amr_flux2_kernel<T, 2><<<n, NT2, smem2_pred<T>(), st>>>(m, a, p, parity, stage);
        amr_update_kernel<T, 2><<<n, NTHREADS, amr_smem<T>(), st>>>(m, a, p, parity, stage);
    }
    return launches + 3;
}

template <class T>
int launch_bed_init(const DevModel<T>& m, const StepParams<T>& p, T* zb, T* gx, T* gy, cudaStream_t st)
{
    const int n = m.nblk;
    bed_halo_kernel<T><<<n, 64, 0, st>>>(m, zb);
    bed_grad_kernel<T><<<n, NTHREADS, 0, st>>>(m, p, zb, gx, gy);
    bed_grad_halo_kernel<T><<<n, 64, 0, st>>>(m, p, zb, gx, gy);
    bed_refine_kernel<T><<<n, 64, 0, st>>>(m, p, zb, gx, gy);
    bed_grad_halo_kernel<T><<<n, 64, 0, st>>>(m, p, zb, gx, gy);
    return 5;
}

template cudaError_t configure_amr_kernels<float>();
template cudaError_t configure_amr_kernels<double>();
template int launch_amr_stage<float>(const DevModel<float>&, const AmrDev<float>&, const StepParams<float>&, int, int,
                                     int, int, int, cudaStream_t);
template int launch_amr_stage<double>(const DevModel<double>&, const AmrDev<double>&, const StepParams<double>&, int,
                                      int, int, int, int, cudaStream_t);
template int launch_bed_init<float>(const DevModel<float>&, const StepParams<float>&, float*, float*, float*,
                                    cudaStream_t);
template int launch_bed_init<double>(const DevModel<double>&, const StepParams<double>&, double*, double*, double*,
                                     cudaStream_t);

}  // namespace BGF_VARIANT
}  // namespace bgf
