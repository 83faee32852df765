// Flow-step kernels (see bgf_flow.cuh for the design) and their launchers.
//
// This file is compiled twice: with BGF_VARIANT=exact (--fmad=false, IEEE
// division and square root: bit-identical to the reference CPU build) and with
// BGF_VARIANT=fast (FMA contraction, approximate division and square root,
// flush-to-zero).  Each build puts its kernels and launchers in its own namespace.
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdio.h>

#include "bgf_flow.cuh"
#include "bgf_internal.h"

#ifndef BGF_VARIANT
#define BGF_VARIANT exact
#endif

namespace bgf {
namespace BGF_VARIANT {

#include "bgf_stage.cuh"
#include "bgf_pair.cuh"
#include "bgf_flow2.cuh"
#include "bgf_flow3.cuh"

// ---------------------------------------------------------------- tile assembly

// zs of a tile cell: ring 1 and the interior use the block's own bed tile
// (RecalculateZs, src/Halo.cu:72-107); ring 2 uses the bed under its source cell,
// as the neighbour's own RecalculateZs does before gradientHalo reads it.  In split
// mode beds are deviations zb + D of the tile block's datum D.
// Read from global memory (the block's own tile for ring 1 and the interior), so
// that the state tile can be assembled in the same phase as the bed tile.
template <class T, bool SPLIT>
__device__ __forceinline__ T tile_zb(const DevModel<T>& m, int ib, int x, int y, int sb, int sx, int sy, T D)
{
    bool ring2 = x < -1 || x > BW || y < -1 || y > BW;
    const T z = ring2 ? m.zb[(size_t)sb * 324 + hi18(sx, sy)] : m.zb[(size_t)ib * 324 + hi18(x, y)];
    return SPLIT ? z + D : z;
}

// Depth of a source cell in the tile block's frame: split mode converts the source
// block's deviation to the tile block's datum (datums are whole metres, so the
// difference is exact).
template <class T, bool SPLIT>
__device__ __forceinline__ T to_tile_datum(const DevModel<T>& m, T hv, int sb, int ib, T D)
{
    return SPLIT && sb != ib ? hv + (m.datum[sb] - D) : hv;
}

// Source of ring position k (< 128) of block ib; a cross-level side raises the
// error word and falls back to the block's own clamped cell.
template <class T>
__device__ __forceinline__ void ring_source(const DevModel<T>& m, int ib, int k, int& x, int& y, int& sb, int& sx,
                                            int& sy)
{
    ring_pos(k, x, y);
    if (!tile_source(m.nbr, m.nblkmem, m.level, ib, x, y, sb, sx, sy, m.checklev != 0)) {
        atomicOr(m.err, 1);
        sb = ib; sx = min(max(x, 0), BW - 1); sy = min(max(y, 0), BW - 1);
    }
}

// Predictor tile: state n of the block and its two-cell ring.  Threads 0..127 also
// take one ring cell; its neighbour-table lookup is issued first, so that its
// latency overlaps the interior loads instead of following them.
template <class T, bool SPLIT>
__device__ __forceinline__ void load_state_tile(Smem<T>& s, const DevModel<T>& m, int ib, int cur, int tid, T D)
{
    static_assert(NTHREADS == 256, "one interior cell per thread, ring cells on threads 0..127");
    const T* H = m.h[cur];
    const T* U = m.u[cur];
    const T* V = m.v[cur];
    int rx = 0, ry = 0, sb = ib, sx = 0, sy = 0;
    const bool ring = tid < 128;
    if (ring) ring_source<T>(m, ib, tid, rx, ry, sb, sx, sy);
    {
        int x = tid & 15, y = tid >> 4;
        size_t g = (size_t)ib * 256 + tid;
        T hv = H[g], uv = U[g], vv = V[g];
        int c = ti(x, y);
        s.t[VH][c] = hv; s.t[VU][c] = uv; s.t[VV][c] = vv;
        const T zbv = m.zb[(size_t)ib * 324 + hi18(x, y)];
        s.t[VZS][c] = (SPLIT ? zbv + D : zbv) + hv;
        int c18 = si(x, y);
        s.h0[c18] = hv; s.u0[c18] = uv; s.v0[c18] = vv;
    }
    if (ring) {
        const int x = rx, y = ry;
        size_t g = (size_t)sb * 256 + sy * 16 + sx;
        T hv = to_tile_datum<T, SPLIT>(m, H[g], sb, ib, D), uv = U[g], vv = V[g];
        int c = ti(x, y);
        s.t[VH][c] = hv; s.t[VU][c] = uv; s.t[VV][c] = vv;
        s.t[VZS][c] = tile_zb<T, SPLIT>(m, ib, x, y, sb, sx, sy, D) + hv;
        if (x >= -1 && x <= BW && y >= -1 && y <= BW) {
            int c18 = si(x, y);
            s.h0[c18] = hv; s.u0[c18] = uv; s.v0[c18] = vv;
        }
    }
}

// One cell of the corrector tile: h* = Advance(state n, adv, dt/2) of source cell
// (sb, sx, sy) at tile position (x, y), and state n on the 18x18 tile.
template <class T, bool SPLIT>
__device__ __forceinline__ void half_tile_cell(Smem<T>& s, const DevModel<T>& m, const StepParams<T>& p, int ib,
                                               int cur, T halfdt, T D, double time, int x, int y, int sb, int sx,
                                               int sy)
{
    const T* H = m.h[cur];
    const T* U = m.u[cur];
    const T* V = m.v[cur];
    size_t g = (size_t)sb * 256 + sy * 16 + sx;
    T hv = H[g], uv = U[g], vv = V[g];
    // the predictor's river source (AddRiverForcing after updateEV) of the source cell
    const T dhs = add_rivers<T>(m, p, sb, sx, sy, m.dh[g], time);
    T ho, uo, vo;
    if (SPLIT) {
        const T Ds = sb == ib ? D : m.datum[sb];
        advance_split<T>(halfdt, p.eps, p.forcemass != 0, Ds, hv, uv, vv, dhs, m.dhu[g], m.dhv[g], ho, uo, vo);
        hv = to_tile_datum<T, SPLIT>(m, hv, sb, ib, D);
        ho = to_tile_datum<T, SPLIT>(m, ho, sb, ib, D);
    } else {
        advance<T>(halfdt, p.eps, p.eps_d, p.forcemass != 0, hv, uv, vv, dhs, m.dhu[g], m.dhv[g], ho, uo, vo);
    }
    int c = ti(x, y);
    s.t[VH][c] = ho; s.t[VU][c] = uo; s.t[VV][c] = vo;
    s.t[VZS][c] = tile_zb<T, SPLIT>(m, ib, x, y, sb, sx, sy, D) + ho;
    if (x >= -1 && x <= BW && y >= -1 && y <= BW) {
        int c18 = si(x, y);
        s.h0[c18] = hv; s.u0[c18] = uv; s.v0[c18] = vv;
    }
}

// Corrector tile: half-step state h* = Advance(state n, adv, dt/2) at every tile
// cell, evaluated from the source cell's state and flux divergence; state n is kept
// on the 18x18 tile for the boundary fluxes and the full-step advance.  Threads
// 128..255 take the ring cells (threads 0..67 load the bed entries beyond 256 in
// the same phase), looking up their source before the interior.
template <class T, bool SPLIT>
__device__ __forceinline__ void load_half_tile(Smem<T>& s, const DevModel<T>& m, const StepParams<T>& p, int ib,
                                               int cur, T halfdt, int tid, T D, double time)
{
    static_assert(NTHREADS == 256, "one interior cell per thread, ring cells on threads 128..255");
    int rx = 0, ry = 0, sb = ib, sx = 0, sy = 0;
    const bool ring = tid >= 128;
    if (ring) ring_source<T>(m, ib, tid - 128, rx, ry, sb, sx, sy);
    half_tile_cell<T, SPLIT>(s, m, p, ib, cur, halfdt, D, time, tid & 15, tid >> 4, ib, tid & 15, tid >> 4);
    if (ring) half_tile_cell<T, SPLIT>(s, m, p, ib, cur, halfdt, D, time, rx, ry, sb, sx, sy);
}

// ---------------------------------------------------------------- kernels

// Minimum resident CTAs per SM the register allocation must allow (launch
// bounds): both FP32 builds trade a few spilled registers for six CTAs per SM
// (the shared-memory limit), which hides the tile loads now that each phase's
// work is spread over the warps; FP64 instantiations keep more registers.
#if BGF_FAST
template <class T> struct Occ {
    static constexpr int flux = sizeof(T) == 4 ? 6 : 3, update = sizeof(T) == 4 ? 6 : 3;
};
#else
template <class T> struct Occ {
    static constexpr int flux = sizeof(T) == 4 ? 6 : 3, update = sizeof(T) == 4 ? 6 : 3;
};
#endif

// Both kernels walk the active list with a grid-stride loop: a launch of one CTA
// per block and a persistent launch of a few CTAs per SM give the same result.
// In a batched pool every block belongs to a scenario with its own parameters,
// time slot and dt minimum (the segmented CFL reduction).

template <class T, int ENGINE, bool SPLIT, bool POOL>
__global__ void __launch_bounds__(NTHREADS, Occ<T>::flux) flux_kernel(DevModel<T> m, StepParams<T> p0, int parity)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem<T>& s = *reinterpret_cast<Smem<T>*>(smem_raw);
    const int tid = threadIdx.x;
    for (int w = blockIdx.x; w < m.nblk; w += gridDim.x) {
        const int ib = m.active[w];
        const int sc = POOL ? m.scen[ib] : 0;
        const TimeState ts = m.time[2 * sc + parity];
        if (!step_live(ts)) continue;
        const StepParams<T>& p = params_ref<POOL>(m, p0, sc);
        const T delta = calcres<T>(p.delta0, m.level[ib]);
        const int cur = ts.cur;
        const T D = SPLIT ? m.datum[ib] : (T)0;

        // bed and state tiles in one phase (the state tile takes zs from global zb)
        load_bed<T, ENGINE, SPLIT, true>(s, m, ib, tid, D);
        load_state_tile<T, SPLIT>(s, m, ib, cur, tid, D);
        __syncthreads();
        T celldt = tile_fluxes<T, ENGINE, false, SPLIT>(s, p, delta, tid, nullptr, D);
        celldt = finite_state_dt<T>(s, tid, celldt);
        __syncthreads();
        // CFL minimum: the interior dtmax values reduced with the warp shuffle, then one
        // atomic per block on the float bit pattern (dt > 0, so integer order == float order).
        T v = celldt;
        for (int o = 16; o > 0; o >>= 1) {
            T q = __shfl_xor_sync(0xffffffffu, v, o);
            v = q < v ? q : v;
        }
        if ((tid & 31) == 0) s.red[tid >> 5] = v;
        // Boundary segments (FlowbndFlux) after the dt, at t + dt_prev/2 as FlowCPU does.
        apply_boundaries<T, SPLIT>(s, m, p, ib, ts.totaltime + ts.dt * 0.5, tid, D);
        __syncthreads();
        if (tid == 0) {
            T b = s.red[0];
            for (int k = 1; k < NTHREADS / 32; k++) b = s.red[k] < b ? s.red[k] : b;
            atomicMin(&m.dtmin[2 * sc + parity], dt_bits(b));
        }
        const int x = tid & 15, y = tid >> 4;
        const int c = ti(x, y);
        T dh, dhu, dhv;
        flux_divergence<T>(s, p, (T)1.0 / ((T)1.0 * delta), x, y, SPLIT ? D + s.t[VH][c] : s.t[VH][c], s.t[VU][c],
                           s.t[VV][c], dh, dhu, dhv);
        size_t g = (size_t)ib * 256 + tid;
        m.dh[g] = dh;
        m.dhu[g] = dhu;
        m.dhv[g] = dhv;
        if (w + (int)gridDim.x < m.nblk) __syncthreads();  // the tile is reused by the next block
    }
}

template <class T, int ENGINE, bool SPLIT, bool POOL>
__global__ void __launch_bounds__(NTHREADS, Occ<T>::update) update_kernel(DevModel<T> m, StepParams<T> p0, int parity)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem<T>& s = *reinterpret_cast<Smem<T>*>(smem_raw);
    const int tid = threadIdx.x;
    for (int w = blockIdx.x; w < m.nblk; w += gridDim.x) {
        const int ib = m.active[w];
        const int sc = POOL ? m.scen[ib] : 0;
        const TimeState ts = m.time[2 * sc + parity];
        const bool lead = POOL ? m.lead[ib] != 0 : w == 0;
        if (!step_live(ts)) {
            if (lead && tid == 0) {
                TimeState nt = ts;
                nt.done = 1;
                m.time[2 * sc + (parity ^ 1)] = nt;
            }
            continue;
        }
        const StepParams<T>& p = params_ref<POOL>(m, p0, sc);
        const T delta = calcres<T>(p.delta0, m.level[ib]);
        const int cur = ts.cur;
        const T dt = step_dt<T>(ts, m.dtmin[2 * sc + parity]);
        const double dtd = (double)dt;
        const T D = SPLIT ? m.datum[ib] : (T)0;

        load_half_tile<T, SPLIT>(s, m, p, ib, cur, dt * (T)0.5, tid, D, ts.totaltime);
        load_bed<T, ENGINE, SPLIT>(s, m, ib, tid, D);
        __syncthreads();
        (void)tile_fluxes<T, ENGINE, false, SPLIT>(s, p, delta, tid, nullptr, D);
        __syncthreads();
        if (block_has_segments<T>(m, ib)) {  // interior blocks skip the step and its barrier
            apply_boundaries<T, SPLIT>(s, m, p, ib, ts.totaltime + dtd, tid, D);
            __syncthreads();
        }
        const int x = tid & 15, y = tid >> 4;
        const int c = ti(x, y);
        T dh, dhu, dhv;
        flux_divergence<T>(s, p, (T)1.0 / ((T)1.0 * delta), x, y, SPLIT ? D + s.t[VH][c] : s.t[VH][c], s.t[VU][c],
                           s.t[VV][c], dh, dhu, dhv);
        dh = add_rivers<T>(m, p, ib, x, y, dh, ts.totaltime);
        // full step from state n (AdvkernelCPU with evolv), then friction on the result
        const int c18 = si(x, y);
        T hold = s.h0[c18], uold = s.u0[c18], vold = s.v0[c18];
        T ho, uo, vo;
        if (SPLIT) advance_split<T>(dt, p.eps, p.forcemass != 0, D, hold, uold, vold, dh, dhu, dhv, ho, uo, vo);
        else advance<T>(dt, p.eps, p.eps_d, p.forcemass != 0, hold, uold, vold, dh, dhu, dhv, ho, uo, vo);
        size_t g = (size_t)ib * 256 + tid;
        T cfv = p.has_cf ? m.cf[g] : p.cf;
        if (SPLIT) {
            // friction on the full depth; the deviation is not changed by it
            bottom_friction<T>(p.frictionmodel, p.g, p.eps, dt, cfv, D + ho, uo, vo);
        } else {
            bottom_friction<T>(p.frictionmodel, p.g, p.eps, dt, cfv, ho, uo, vo);
        }
        if (p.has_rain) {
            // AddrainforcingImplicitCPU (src/Updateforcing.cu:530-580): the rain rate at
            // the start of the step (updateforcing), uniform or gridded
            T Rainhh;
            if (p.rain_map) {
                // the cell position as AddrainforcingImplicitCPU forms it, in T
                const T xc = (T)p.xo_d + (T)m.bxo[ib] + (T)x * delta;
                const T yc = (T)p.yo_d + (T)m.byo[ib] + (T)y * delta;
                Rainhh = rain_map_at<T>(m.rmap, xc, yc, ts.totaltime);
            } else {
                Rainhh = (T)series_at(m.rain_t + p.rain_off, m.rain_r + p.rain_off, p.rain_n, ts.totaltime,
                                      p.rain_sorted != 0);
            }
            T mask = m.rainmask ? (T)m.rainmask[g] : (T)1;
            Rainhh = M<T>::fmax_(Rainhh / (T)1000.0 / (T)3600.0 * (T)dtd, (T)0.0) * mask;
            T hi = SPLIT ? D + ho : ho;
            T qvol = hi / (hi + Rainhh);
            ho = ho + Rainhh;
            if ((double)hi > p.eps_d) {
                uo = uo * qvol;
                vo = vo * qvol;
            }
        }
        const int nxt = cur ^ 1;
        m.h[nxt][g] = ho;
        m.u[nxt][g] = uo;
        m.v[nxt][g] = vo;
        if (m.hmax) {
            const T hf = SPLIT ? D + ho : ho;
            m.hmax[g] = hf > m.hmax[g] ? hf : m.hmax[g];
        }
        if (lead && tid == 0)
            m.time[2 * sc + (parity ^ 1)] = next_time_state<T>(ts, p, dtd, nxt, m.dtmin + 2 * sc, parity);
        if (w + (int)gridDim.x < m.nblk) __syncthreads();  // the tile is reused by the next block
    }
}

// initdt (src/Mainloop.cu:515-554): CalcInitdtCPU per cell, block minimum, atomic.
template <class T> __global__ void initdt_kernel(DevModel<T> m, StepParams<T> p0, int cur, unsigned long long* out)
{
    __shared__ T red[NTHREADS / 32];
    const int tid = threadIdx.x;
    const int ib = m.active[blockIdx.x];
    const int sc = scen_of(m, ib);
    const StepParams<T> p = params_of(m, p0, sc);
    const T delta = calcres<T>(p.delta0, m.level[ib]);
    T hv = m.h[cur][(size_t)ib * 256 + tid];
    if (m.datum) hv = m.datum[ib] + hv;
    T epsT = (T)p.eps_d;
    T hm = hv < epsT ? epsT : hv;
    T v = delta / M<T>::sqrt_(p.g * hm);
    for (int o = 16; o > 0; o >>= 1) {
        T w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w < v ? w : v;
    }
    if ((tid & 31) == 0) red[tid >> 5] = v;
    __syncthreads();
    if (tid == 0) {
        T b = red[0];
        for (int k = 1; k < NTHREADS / 32; k++) b = red[k] < b ? red[k] : b;
        atomicMin(out + sc, dt_bits(b));
    }
}

// Volume sum_h h * delta^2 over active interior cells in double.
template <class T> __global__ void volume_kernel(DevModel<T> m, T delta0, int cur, double* out)
{
    __shared__ double red[NTHREADS / 32];
    const int tid = threadIdx.x;
    const int ib = m.active[blockIdx.x];
    const int sc = scen_of(m, ib);
    double d = (double)calcres<T>(delta0, m.level[ib]);
    double v = ((double)m.h[cur][(size_t)ib * 256 + tid] + (m.datum ? (double)m.datum[ib] : 0.0)) * d * d;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((tid & 31) == 0) red[tid >> 5] = v;
    __syncthreads();
    if (tid == 0) {
        double b = 0;
        for (int k = 0; k < NTHREADS / 32; k++) b += red[k];
        atomicAdd(out + sc, b);
    }
}

// ---------------------------------------------------------------- launchers

template <class T> size_t smem_bytes() { return sizeof(Smem<T>); }

template <class T, int ENGINE, bool SPLIT, bool POOL> cudaError_t configure_one()
{
    const int sm = (int)smem_bytes<T>();
    cudaError_t e = cudaFuncSetAttribute(flux_kernel<T, ENGINE, SPLIT, POOL>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(update_kernel<T, ENGINE, SPLIT, POOL>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if (e != cudaSuccess) return e;
    // two cells per thread
    e = cudaFuncSetAttribute(flux2_kernel<T, ENGINE, POOL, SPLIT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem2_pred<T>());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(update2_kernel<T, ENGINE, POOL, SPLIT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem2_corr<T>());
    if (e != cudaSuccess || SPLIT) return e;  // (the staged layout has no split mode)
    // staged tiles (persistent CTAs with a producer warp)
    e = cudaFuncSetAttribute(flux3_kernel<T, ENGINE, POOL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem3_pred<T>());
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(update3_kernel<T, ENGINE, POOL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem3_corr<T>());
}

// Persistent grid of the staged kernels: CTAs resident on all SMs at once (from the
// occupancy of the kernel at its shared memory), at most one per block.
template <class KERN> static int resident_grid(KERN k, size_t smem, int nblk)
{
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
    }
    int per = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, NT3, smem) != cudaSuccess || per <= 0) per = 1;
    const int g = sms * per;
    return g < nblk ? g : nblk;
}

template <class T, int ENGINE> cudaError_t configure_engine()
{
    cudaError_t e = configure_one<T, ENGINE, false, false>();
    if (e == cudaSuccess) e = configure_one<T, ENGINE, false, true>();
    if constexpr (sizeof(T) == 4) {
        // split precision is an FP32 mode
        if (e == cudaSuccess) e = configure_one<T, ENGINE, true, false>();
        if (e == cudaSuccess) e = configure_one<T, ENGINE, true, true>();
    }
    return e;
}

template <class T> cudaError_t configure_kernels()
{
    cudaError_t e = configure_engine<T, 1>();
    if (e != cudaSuccess) return e;
    return configure_engine<T, 2>();
}

// grid: CTAs of the launch (0: one per active block); fewer CTAs loop over the blocks
template <class T, bool FLUX, int ENGINE>
static void launch_step_kernel(const DevModel<T>& m, const StepParams<T>& p, int parity, cudaStream_t st, int g)
{
    const size_t sm = smem_bytes<T>();
    const bool pool = m.scen != nullptr;
    bool split = false;
    if constexpr (sizeof(T) == 4) split = m.datum != nullptr;
    if (!split && m.gen == 3) {
        // staged tiles, persistent CTAs (the grid argument, when set, is the CTA count)
        if constexpr (FLUX) {
            auto k = pool ? flux3_kernel<T, ENGINE, true> : flux3_kernel<T, ENGINE, false>;
            const int gg = g < m.nblk ? g : resident_grid(k, smem3_pred<T>(), m.nblk);
            k<<<gg, NT3, smem3_pred<T>(), st>>>(m, p, parity);
        } else {
            auto k = pool ? update3_kernel<T, ENGINE, true> : update3_kernel<T, ENGINE, false>;
            const int gg = g < m.nblk ? g : resident_grid(k, smem3_corr<T>(), m.nblk);
            k<<<gg, NT3, smem3_corr<T>(), st>>>(m, p, parity);
        }
        return;
    }
    if (m.gen != 1) {
        // two cells per thread (split precision too; the staged layout falls back here)
        if constexpr (sizeof(T) == 4) {
            if (split) {
                if constexpr (FLUX) {
                    if (pool) flux2_kernel<T, ENGINE, true, true><<<g, NT2, smem2_pred<T>(), st>>>(m, p, parity);
                    else flux2_kernel<T, ENGINE, false, true><<<g, NT2, smem2_pred<T>(), st>>>(m, p, parity);
                } else {
                    if (pool) update2_kernel<T, ENGINE, true, true><<<g, NT2, smem2_corr<T>(), st>>>(m, p, parity);
                    else update2_kernel<T, ENGINE, false, true><<<g, NT2, smem2_corr<T>(), st>>>(m, p, parity);
                }
                return;
            }
        }
        if constexpr (FLUX) {
            if (pool) flux2_kernel<T, ENGINE, true><<<g, NT2, smem2_pred<T>(), st>>>(m, p, parity);
            else flux2_kernel<T, ENGINE, false><<<g, NT2, smem2_pred<T>(), st>>>(m, p, parity);
        } else {
            if (pool) update2_kernel<T, ENGINE, true><<<g, NT2, smem2_corr<T>(), st>>>(m, p, parity);
            else update2_kernel<T, ENGINE, false><<<g, NT2, smem2_corr<T>(), st>>>(m, p, parity);
        }
        return;
    }
    if constexpr (FLUX) {
        if constexpr (sizeof(T) == 4) {
            if (split) {
                if (pool) flux_kernel<T, ENGINE, true, true><<<g, NTHREADS, sm, st>>>(m, p, parity);
                else flux_kernel<T, ENGINE, true, false><<<g, NTHREADS, sm, st>>>(m, p, parity);
                return;
            }
        }
        if (pool) flux_kernel<T, ENGINE, false, true><<<g, NTHREADS, sm, st>>>(m, p, parity);
        else flux_kernel<T, ENGINE, false, false><<<g, NTHREADS, sm, st>>>(m, p, parity);
    } else {
        if constexpr (sizeof(T) == 4) {
            if (split) {
                if (pool) update_kernel<T, ENGINE, true, true><<<g, NTHREADS, sm, st>>>(m, p, parity);
                else update_kernel<T, ENGINE, true, false><<<g, NTHREADS, sm, st>>>(m, p, parity);
                return;
            }
        }
        if (pool) update_kernel<T, ENGINE, false, true><<<g, NTHREADS, sm, st>>>(m, p, parity);
        else update_kernel<T, ENGINE, false, false><<<g, NTHREADS, sm, st>>>(m, p, parity);
    }
}

template <class T>
void launch_flux(const DevModel<T>& m, const StepParams<T>& p, int engine, int parity, cudaStream_t st, int grid)
{
    const int g = grid > 0 && grid < m.nblk ? grid : m.nblk;
    if (engine == 1) launch_step_kernel<T, true, 1>(m, p, parity, st, g);
    else launch_step_kernel<T, true, 2>(m, p, parity, st, g);
}

template <class T>
void launch_update(const DevModel<T>& m, const StepParams<T>& p, int engine, int parity, cudaStream_t st, int grid)
{
    const int g = grid > 0 && grid < m.nblk ? grid : m.nblk;
    if (engine == 1) launch_step_kernel<T, false, 1>(m, p, parity, st, g);
    else launch_step_kernel<T, false, 2>(m, p, parity, st, g);
}

template <class T>
void launch_initdt(const DevModel<T>& m, const StepParams<T>& p, int cur, unsigned long long* out, cudaStream_t st)
{
    initdt_kernel<T><<<m.nblk, NTHREADS, 0, st>>>(m, p, cur, out);
}

template <class T> void launch_volume(const DevModel<T>& m, T delta0, int cur, double* out, cudaStream_t st)
{
    volume_kernel<T><<<m.nblk, NTHREADS, 0, st>>>(m, delta0, cur, out);
}

template cudaError_t configure_kernels<float>();
template cudaError_t configure_kernels<double>();
template void launch_flux<float>(const DevModel<float>&, const StepParams<float>&, int, int, cudaStream_t, int);
template void launch_flux<double>(const DevModel<double>&, const StepParams<double>&, int, int, cudaStream_t, int);
template void launch_update<float>(const DevModel<float>&, const StepParams<float>&, int, int, cudaStream_t, int);
template void launch_update<double>(const DevModel<double>&, const StepParams<double>&, int, int, cudaStream_t, int);
template void launch_initdt<float>(const DevModel<float>&, const StepParams<float>&, int, unsigned long long*, cudaStream_t);
template void launch_initdt<double>(const DevModel<double>&, const StepParams<double>&, int, unsigned long long*, cudaStream_t);
template void launch_volume<float>(const DevModel<float>&, float, int, double*, cudaStream_t);
template void launch_volume<double>(const DevModel<double>&, double, int, double*, cudaStream_t);

}  // namespace BGF_VARIANT
}  // namespace bgf
