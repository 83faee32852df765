// Third-generation single-level stage kernels: staged tiles.
//
// Same step and same arithmetic as flux2_kernel / update2_kernel (two cells per
// thread, bgf_flow2.cuh); what changes is how a block's inputs reach shared memory.
// Each CTA is persistent (it loops over blocks w = blockIdx.x, + gridDim.x, ...) and
// holds five warps:
//
//  * warp 4, the producer, stages the NEXT block of the CTA into a staging area
//    while warps 0..3 compute the current one.  Contiguous pieces go by bulk
//    asynchronous copies (cp.async.bulk, global -> shared, completing on an
//    mbarrier with a byte count): the 16x16 interior of every state array (1 KB in
//    FP32), the two rows of the lower and upper neighbours next to the block
//    (rows 14-15 and 0-1, 128 B each, 16-byte aligned) and the bed tile with its
//    halo (18x18, 1296 B).  The left and right neighbours' two columns are strided,
//    so each lane copies its cells with 4-byte (8-byte in FP64) cp.async operations
//    that arrive on the same mbarrier when they land; so do the 64 outer-ring bed
//    values of the neighbours.  At a domain edge (no neighbour) the copies read the
//    block's own edge cells, as the tile assembly of the other kernels does.
//  * warps 0..3 wait for the stage, unpack it into the pair layouts of the compute
//    phases (shared to shared), release the stage (the producer refills it with the
//    next block at once) and run gradients, faces, CFL, boundaries and divergence
//    exactly as the two-cell kernels do.  They synchronise among themselves with
//    named barrier 1 (128 threads), never with the producer.
//
// The neighbours must be on the block's level (single-level meshes and the blocks of
// a multi-level mesh whose eight neighbour entries share their level).
//
// Every wait on an mbarrier is bounded by the global timer; a wait that runs out
// sets bit 4 of the error word, the consumer warps agree on it with a barrier
// reduction and the CTA leaves after the producer has waited (bounded again) for
// the copies it issued.
//
// Included inside namespace bgf::BGF_VARIANT after bgf_flow2.cuh.
#pragma once

constexpr int NT3 = NT2 + 32;                 // four compute warps + the producer warp
constexpr unsigned long long WAIT_NS = 1000000000ull;  // 1 s bound on every wait
constexpr int ERR_STAGE_TIMEOUT = 16;

// ---------------------------------------------------------------- staging area
// Offsets (elements of T) of the pieces of one staged block; NV state-like arrays
// (3 for the predictor: h, u, v; 6 for the corrector: h, u, v, dh, dhu, dhv).
template <class T, int NV> struct StageLayout {
    static constexpr int in = 0;               // [NV][256] interiors
    static constexpr int rb = in + NV * 256;   // [NV][32] rows y = -2, -1 (neighbour rows 14, 15)
    static constexpr int rt = rb + NV * 32;    // [NV][32] rows y = 16, 17 (neighbour rows 0, 1)
    static constexpr int rl = rt + NV * 32;    // [NV][16][2] columns x = -2, -1
    static constexpr int rr = rl + NV * 32;    // [NV][16][2] columns x = 16, 17
    static constexpr int zb = rr + NV * 32;    // [324] bed tile with halo
    static constexpr int z2 = zb + 324;        // [64] outer-ring bed: side * 16 + t
    static constexpr int cf = z2 + 64;         // [256] friction (corrector)
    static constexpr int n_pred = cf;          // predictor: no friction, no rain mask
    static constexpr int n_corr = cf + 256;
    static constexpr size_t bytes_pred = (size_t)n_pred * sizeof(T);
    static constexpr size_t bytes_corr = (size_t)n_corr * sizeof(T) + 256;  // + rain mask bytes
};
static_assert((StageLayout<float, 3>::zb * 4) % 16 == 0 && (StageLayout<float, 6>::zb * 4) % 16 == 0,
              "bulk copy destinations are 16-byte aligned");
static_assert((StageLayout<float, 6>::cf * 4) % 16 == 0 && (StageLayout<float, 6>::n_corr * 4) % 16 == 0,
              "bulk copy destinations are 16-byte aligned");

// Dynamic shared memory: two mbarriers (full, empty; 16 bytes), the stage, Smem2.
template <class T, int NV, bool CORR> __host__ __device__ constexpr size_t stage_bytes()
{
    return CORR ? StageLayout<T, NV>::bytes_corr : StageLayout<T, NV>::bytes_pred;
}
template <class T, int NV, bool CORR> __host__ __device__ constexpr size_t smem3_off()
{ return (16 + stage_bytes<T, NV, CORR>() + 15) & ~(size_t)15; }
template <class T> constexpr size_t smem3_pred() { return smem3_off<T, 3, false>() + smem2_pred<T>(); }
// corrector: + each thread's friction and rain-mask pair, kept from the unpack to the
// end of the block (shared instead of registers)
template <class T> constexpr size_t smem3_corr() { return smem3_off<T, 6, true>() + smem2_corr<T>() + 256 * sizeof(T) + 256; }

// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t sh_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(sh_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(sh_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(sh_addr(bar)),
                 "r"(bytes)
                 : "memory");
}
// try_wait with a suspend-time hint: a waiting thread sleeps in hardware (up to
// about 20 us) instead of spinning through issue slots the compute warps need.
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\tselp.u32 %0, 1, 0, "
        "p;\n\t}"
        : "=r"(ok)
        : "r"(sh_addr(bar)), "r"(parity), "r"(20000u)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ unsigned long long gtimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Waits until the phase of the given parity completed, at most WAIT_NS.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity)
{
    if (mbar_test(bar, parity)) return true;
    const unsigned long long t0 = gtimer();
    while (!mbar_test(bar, parity))
        if (gtimer() - t0 > WAIT_NS) return false;
    return true;
}
// Bulk copy global -> shared, completion counted in bytes on bar.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     sh_addr(dst)),
                 "l"(src), "r"(bytes), "r"(sh_addr(bar))
                 : "memory");
}
// One 4- or 8-byte asynchronous copy global -> shared.
template <class T> __device__ __forceinline__ void cp_async_elem(T* dst, const T* src)
{
    if constexpr (sizeof(T) == 4)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(sh_addr(dst)), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sh_addr(dst)), "l"(src) : "memory");
}
// Arrive on bar once every cp.async this thread issued so far has landed.
__device__ __forceinline__ void cp_async_arrive(uint64_t* bar)
{
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(sh_addr(bar)) : "memory");
}
__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// Named barrier 1 over the 128 compute threads.
__device__ __forceinline__ void csync() { asm volatile("bar.sync 1, 128;" ::: "memory"); }
// Named barrier 1 with an AND over the 128 compute threads.
__device__ __forceinline__ bool csync_and(bool v)
{
    uint32_t r;
    asm volatile("{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.and.pred q, 1, 128, p;\n\tselp.u32 %0, 1, "
                 "0, q;\n\t}"
                 : "=r"(r)
                 : "r"(v ? 1u : 0u)
                 : "memory");
    return r != 0;
}

// ---------------------------------------------------------------- producer
// Stages block ib: NV arrays of src (h, u, v[, dh, dhu, dhv]) with their two-cell
// ring, the bed tile, the outer-ring bed and (corrector) friction and rain mask.
// Lane 0 posts the byte count and issues the bulk copies; every lane issues its
// cp.async cells and arrives when they land (the full barrier counts 1 + 32).
template <class T, int NV, bool CORR>
__device__ __forceinline__ void stage_block(const DevModel<T>& m, const T* const (&src)[6], unsigned char* stage,
                                            uint64_t* full, int ib, int lane, bool with_cf, bool with_mask)
{
    using L = StageLayout<T, NV>;
    T* S = reinterpret_cast<T*>(stage);
    const int nbm = m.nblkmem;
    const int lb = m.nbr[0 * nbm + ib], rb = m.nbr[2 * nbm + ib], bl = m.nbr[4 * nbm + ib], tl = m.nbr[6 * nbm + ib];
    constexpr uint32_t E = sizeof(T);
    if (lane == 0) {
        uint32_t bytes = NV * (256 + 32 + 32) * E + 324 * E;
        if (CORR && with_cf) bytes += 256 * E;
        if (CORR && with_mask) bytes += 256;
        mbar_arrive_expect_tx(full, bytes);
#pragma unroll
        for (int v = 0; v < NV; v++) {
            const T* a = src[v];
            bulk_g2s(S + L::in + v * 256, a + (size_t)ib * 256, 256 * E, full);
            if (bl != ib) {
                bulk_g2s(S + L::rb + v * 32, a + (size_t)bl * 256 + 14 * 16, 32 * E, full);
            } else {  // domain edge: both rows take the block's row 0
                bulk_g2s(S + L::rb + v * 32, a + (size_t)ib * 256, 16 * E, full);
                bulk_g2s(S + L::rb + v * 32 + 16, a + (size_t)ib * 256, 16 * E, full);
            }
            if (tl != ib) {
                bulk_g2s(S + L::rt + v * 32, a + (size_t)tl * 256, 32 * E, full);
            } else {  // domain edge: both rows take the block's row 15
                bulk_g2s(S + L::rt + v * 32, a + (size_t)ib * 256 + 15 * 16, 16 * E, full);
                bulk_g2s(S + L::rt + v * 32 + 16, a + (size_t)ib * 256 + 15 * 16, 16 * E, full);
            }
        }
        bulk_g2s(S + L::zb, m.zb + (size_t)ib * 324, 324 * E, full);
        if (CORR && with_cf) bulk_g2s(S + L::cf, m.cf + (size_t)ib * 256, 256 * E, full);
        if (CORR && with_mask)
            bulk_g2s(stage + L::n_corr * sizeof(T), m.rainmask + (size_t)ib * 256, 256, full);
    }
    // columns x = -2, -1 (left) and 16, 17 (right): lane = 2 y + j
    {
        const int y = lane >> 1, j = lane & 1;
        const size_t lo = lb != ib ? (size_t)lb * 256 + y * 16 + 14 + j : (size_t)ib * 256 + y * 16;
        const size_t ro = rb != ib ? (size_t)rb * 256 + y * 16 + j : (size_t)ib * 256 + y * 16 + 15;
#pragma unroll
        for (int v = 0; v < NV; v++) {
            cp_async_elem<T>(S + L::rl + v * 32 + lane, src[v] + lo);
            cp_async_elem<T>(S + L::rr + v * 32 + lane, src[v] + ro);
        }
    }
    // outer-ring bed (x = -2, 17 or y = -2, 17): k = side * 16 + t
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int k = lane + 32 * h, side = k >> 4, t = k & 15;
        int sb, sx, sy;
        if (side == 0) { sb = lb != ib ? lb : ib; sx = lb != ib ? 14 : 0; sy = t; }
        else if (side == 1) { sb = rb != ib ? rb : ib; sx = rb != ib ? 1 : 15; sy = t; }
        else if (side == 2) { sb = bl != ib ? bl : ib; sx = t; sy = bl != ib ? 14 : 0; }
        else { sb = tl != ib ? tl : ib; sx = t; sy = tl != ib ? 1 : 15; }
        cp_async_elem<T>(S + L::z2 + k, m.zb + (size_t)sb * 324 + hi18(sx, sy));
    }
    cp_async_arrive(full);
}

// The producer warp's loop: block k of this CTA goes to the stage once the compute
// warps released block k - 1 (empty barrier phase k - 1).
template <class T, int NV, bool CORR>
__device__ __forceinline__ void producer_loop(const DevModel<T>& m, int parity, unsigned char* stage, uint64_t* full,
                                              uint64_t* empty, int lane, bool with_cf, bool with_mask)
{
    int k = 0;
    for (int w = blockIdx.x; w < m.nblk; w += gridDim.x, k++) {
        // the state buffers of the block's scenario (pooled scenarios that finished
        // stop swapping theirs)
        const int ib = m.active[w];
        const int cur = m.time[2 * (m.scen ? m.scen[ib] : 0) + parity].cur;
        const T* const src[6] = {m.h[cur], m.u[cur], m.v[cur], m.dh, m.dhu, m.dhv};
        if (k > 0) {
            bool ok = true;
            if (lane == 0) ok = mbar_wait(empty, (uint32_t)((k - 1) & 1));
            ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
            if (!ok) {
                if (lane == 0) atomicOr(m.err, ERR_STAGE_TIMEOUT);
                break;
            }
            fence_async_shared();  // the compute warps' reads of the stage come before the new copies
        }
        stage_block<T, NV, CORR>(m, src, stage, full, ib, lane, with_cf, with_mask);
    }
    // leave only after the last issued copies landed (bounded)
    if (k > 0 && lane == 0) (void)mbar_wait(full, (uint32_t)((k - 1) & 1));
    __syncwarp();
}

// ---------------------------------------------------------------- consumers
// Ring cell r (0..127, as ring_pos) of variable v from the stage.
template <class T, int NV>
__device__ __forceinline__ T ring_val(const T* S, int v, int r)
{
    using L = StageLayout<T, NV>;
    const int side = r >> 5, ring = (r >> 4) & 1, t = r & 15;
    if (side == 0) return S[L::rl + v * 32 + t * 2 + (1 - ring)];
    if (side == 1) return S[L::rr + v * 32 + t * 2 + ring];
    if (side == 2) return S[L::rb + v * 32 + (1 - ring) * 16 + t];
    return S[L::rt + v * 32 + ring * 16 + t];
}

// the bed tile keeps its global (row-major, hi18) layout in Smem2
template <class T> __device__ __forceinline__ void unpack_bed(Smem2<T>& s, const T* zbt, int tid)
{
    for (int k = tid; k < 324; k += NT2) s.zb[k] = zbt[k];
}

template <class T, int ENGINE, bool POOL>
__global__ void __launch_bounds__(NT3, sizeof(T) == 4 ? 6 : 2) flux3_kernel(DevModel<T> m, StepParams<T> p0, int parity)
{
    using V = V2<T>;
    using L = StageLayout<T, 3>;
    extern __shared__ __align__(16) unsigned char smem_raw3[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw3);
    uint64_t* empty = full + 1;
    unsigned char* stage = smem_raw3 + 16;
    Smem2<T>& s = *reinterpret_cast<Smem2<T>*>(smem_raw3 + smem3_off<T, 3, false>());
    const int tid = threadIdx.x;
    if (tid == 0) {
        mbar_init(full, 33);
        mbar_init(empty, 1);
        mbar_init_fence();
    }
    __syncthreads();
    if (tid >= NT2) {
        producer_loop<T, 3, false>(m, parity, stage, full, empty, tid - NT2, false, false);
        return;
    }
    const T* S = reinterpret_cast<const T*>(stage);
    const int w4 = tid >> 5, lane = tid & 31;
    const int x = lane & 15;
    const int py = (w4 & 1) + 4 * (w4 >> 1) + 2 * (lane >> 4);
    const int y = 2 * py;
    int k = 0;
    for (int w = blockIdx.x; w < m.nblk; w += gridDim.x, k++) {
        const int ib = m.active[w];
        const int sc = POOL ? m.scen[ib] : 0;
        const TimeState ts = m.time[2 * sc + parity];
        const bool live = step_live(ts);
        const StepParams<T>& p = params_ref<POOL>(m, p0, sc);
        const T delta = calcres<T>(p.delta0, m.level[ib]);
        int rx, ry;
        ring_pos(tid, rx, ry);
        const BedGrad<T> bg = live ? load_bedgrad<T, ENGINE>(m, ib, tid, x, y) : BedGrad<T>{};
        if (!csync_and(mbar_wait(full, (uint32_t)(k & 1)))) {
            if (tid == 0) atomicOr(m.err, ERR_STAGE_TIMEOUT);
            return;
        }
        V c[4];
        if (live) {
            c[VH] = V{S[L::in + y * 16 + x], S[L::in + (y + 1) * 16 + x]};
            c[VU] = V{S[L::in + 256 + y * 16 + x], S[L::in + 256 + (y + 1) * 16 + x]};
            c[VV] = V{S[L::in + 512 + y * 16 + x], S[L::in + 512 + (y + 1) * 16 + x]};
            const V zbo{S[L::zb + hi18(x, y)], S[L::zb + hi18(x, y + 1)]};
            c[VZS] = add(zbo, c[VH]);
            const bool ring2 = rx < -1 || rx > BW || ry < -1 || ry > BW;
            const T hv = ring_val<T, 3>(S, 0, tid);
            const T zr = ring2 ? S[L::z2 + (tid >> 5) * 16 + (tid & 15)] : S[L::zb + hi18(rx, ry)];
            const int o = p2t(rx, ry);
            s.t[VH][o] = hv; s.t[VU][o] = ring_val<T, 3>(S, 1, tid); s.t[VV][o] = ring_val<T, 3>(S, 2, tid);
            s.t[VZS][o] = zr + hv;
            const int ct = p2t(x, y);
#pragma unroll
            for (int q = 0; q < 4; q++) st2<T>(s.t[q], ct, c[q]);
            unpack_bed<T>(s, S + L::zb, tid);
        }
        csync();
        if (tid == 0) mbar_arrive(empty);  // the stage is free for the next block
        if (!live) continue;
        V xm[4], gxo[4], gyo[4];
        T ym[4];
        gradients2<T, ENGINE>(s, bg, p.theta, delta, tid, x, py, c, xm, ym, gxo, gyo);
        csync();
        V cdt = faces2<T, ENGINE>(s, p, delta, tid, x, py, c, xm, ym, gxo, gyo);
        cdt = finite_dt2<T>(c[VH], c[VU], c[VV], cdt);
        T v = cdt.b < cdt.a ? cdt.b : cdt.a;
        for (int o = 16; o > 0; o >>= 1) {
            const T q = __shfl_xor_sync(0xffffffffu, v, o);
            v = q < v ? q : v;
        }
        if (lane == 0) s.red[w4] = v;
        csync();
        if (block_has_segments<T>(m, ib)) {
            boundaries2<T, false>(s, m, p, ib, ts.totaltime + ts.dt * 0.5, tid);
            csync();
        }
        if (tid == 0) {
            T b = s.red[0];
            for (int q = 1; q < NT2 / 32; q++) b = s.red[q] < b ? s.red[q] : b;
            atomicMin(&m.dtmin[2 * sc + parity], dt_bits(b));
        }
        V dh, dhu, dhv;
        divergence2<T>(s, p, (T)1.0 / ((T)1.0 * delta), x, py, c[VH], c[VU], c[VV], dh, dhu, dhv);
        const size_t g0 = (size_t)ib * 256 + y * 16 + x;
        m.dh[g0] = dh.a; m.dh[g0 + 16] = dh.b;
        m.dhu[g0] = dhu.a; m.dhu[g0 + 16] = dhu.b;
        m.dhv[g0] = dhv.a; m.dhv[g0 + 16] = dhv.b;
        csync();  // the working tiles are reused by the next block
    }
}

template <class T, int ENGINE, bool POOL>
__global__ void __launch_bounds__(NT3, sizeof(T) == 4 ? 5 : 2) update3_kernel(DevModel<T> m, StepParams<T> p0, int parity)
{
    using V = V2<T>;
    using L = StageLayout<T, 6>;
    extern __shared__ __align__(16) unsigned char smem_raw3[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw3);
    uint64_t* empty = full + 1;
    unsigned char* stage = smem_raw3 + 16;
    Smem2<T>& s = *reinterpret_cast<Smem2<T>*>(smem_raw3 + smem3_off<T, 6, true>());
    T* cfw = reinterpret_cast<T*>(smem_raw3 + smem3_off<T, 6, true>() + smem2_corr<T>());
    uint8_t* rmw = reinterpret_cast<uint8_t*>(cfw + 256);
    const int tid = threadIdx.x;
    if (tid == 0) {
        mbar_init(full, 33);
        mbar_init(empty, 1);
        mbar_init_fence();
    }
    __syncthreads();
    const bool with_mask = m.rainmask != nullptr;
    if (tid >= NT2) {
        producer_loop<T, 6, true>(m, parity, stage, full, empty, tid - NT2, m.cf != nullptr, with_mask);
        return;
    }
    const T* S = reinterpret_cast<const T*>(stage);
    const uint8_t* RM = stage + L::n_corr * sizeof(T);
    const int w4 = tid >> 5, lane = tid & 31;
    const int x = lane & 15;
    const int py = (w4 & 1) + 4 * (w4 >> 1) + 2 * (lane >> 4);
    const int y = 2 * py;
    int k = 0;
    for (int w = blockIdx.x; w < m.nblk; w += gridDim.x, k++) {
        const int ib = m.active[w];
        const int sc = POOL ? m.scen[ib] : 0;
        const TimeState ts = m.time[2 * sc + parity];
        const bool lead = POOL ? m.lead[ib] != 0 : w == 0;
        const bool live = step_live(ts);
        const StepParams<T>& p = params_ref<POOL>(m, p0, sc);
        if (live && tid == 0) s.dtv = step_dt<T>(ts, m.dtmin[2 * sc + parity]);
        const T delta = calcres<T>(p.delta0, m.level[ib]);
        const int cur = ts.cur;
        int rx, ry;
        ring_pos(tid, rx, ry);
        const BedGrad<T> bg = live ? load_bedgrad<T, ENGINE>(m, ib, tid, x, y) : BedGrad<T>{};
        if (!csync_and(mbar_wait(full, (uint32_t)(k & 1)))) {
            if (tid == 0) atomicOr(m.err, ERR_STAGE_TIMEOUT);
            return;
        }
        V hold, uold, vold, ddh, ddhu, ddhv, zbo;
        T rh = 0, ru = 0, rv = 0, rdh = 0, rdhu = 0, rdhv = 0, rzb = 0;
        const bool ring2 = rx < -1 || rx > BW || ry < -1 || ry > BW;
        if (live) {
            auto pair = [&](int v) { return V{S[L::in + v * 256 + y * 16 + x], S[L::in + v * 256 + (y + 1) * 16 + x]}; };
            hold = pair(0); uold = pair(1); vold = pair(2);
            ddh = pair(3); ddhu = pair(4); ddhv = pair(5);
            zbo = V{S[L::zb + hi18(x, y)], S[L::zb + hi18(x, y + 1)]};
            rh = ring_val<T, 6>(S, 0, tid); ru = ring_val<T, 6>(S, 1, tid); rv = ring_val<T, 6>(S, 2, tid);
            rdh = ring_val<T, 6>(S, 3, tid); rdhu = ring_val<T, 6>(S, 4, tid); rdhv = ring_val<T, 6>(S, 5, tid);
            rzb = ring2 ? S[L::z2 + (tid >> 5) * 16 + (tid & 15)] : S[L::zb + hi18(rx, ry)];
            if (p.has_cf) {  // m.cf is set (and staged) whenever a scenario has per-cell friction
                cfw[y * 16 + x] = S[L::cf + y * 16 + x];
                cfw[(y + 1) * 16 + x] = S[L::cf + (y + 1) * 16 + x];
            }
            if (with_mask) {
                rmw[y * 16 + x] = RM[y * 16 + x];
                rmw[(y + 1) * 16 + x] = RM[(y + 1) * 16 + x];
            }
            unpack_bed<T>(s, S + L::zb, tid);
        }
        csync();  // s.dtv, s.zb; the stage has been read
        if (tid == 0) mbar_arrive(empty);
        if (!live) {
            if (lead && tid == 0) {
                TimeState nt = ts;
                nt.done = 1;
                m.time[2 * sc + (parity ^ 1)] = nt;
            }
            continue;
        }
        const T dt = s.dtv;
        const double dtd = (double)dt;
        const T halfdt = dt * (T)0.5;
        if (p.nriver > 0) {
            // the predictor's river source of the source cells (AddRiverForcing after updateEV)
            int sb, sx, sy;
            ring_src2<T>(m, ib, tid, rx, ry, sb, sx, sy);
            ddh = V{add_rivers<T>(m, p, ib, x, y, ddh.a, ts.totaltime), add_rivers<T>(m, p, ib, x, y + 1, ddh.b, ts.totaltime)};
            rdh = add_rivers<T>(m, p, sb, sx, sy, rdh, ts.totaltime);
        }
        V c[4];
        advance_v<V>(halfdt, p.eps, p.eps_d, p.forcemass != 0, hold, uold, vold, ddh, ddhu, ddhv, c[VH], c[VU], c[VV]);
        c[VZS] = add(zbo, c[VH]);
        {
            T ho, uo, vo;
            advance_v<T>(halfdt, p.eps, p.eps_d, p.forcemass != 0, rh, ru, rv, rdh, rdhu, rdhv, ho, uo, vo);
            const int o = p2t(rx, ry);
            s.t[VH][o] = ho; s.t[VU][o] = uo; s.t[VV][o] = vo; s.t[VZS][o] = rzb + ho;
            if (!ring2) {
                const int o2 = p2z(rx, ry);
                s.h0[o2] = rh; s.u0[o2] = ru; s.v0[o2] = rv;
            }
        }
        const int ct = p2t(x, y);
#pragma unroll
        for (int q = 0; q < 4; q++) st2<T>(s.t[q], ct, c[q]);
        {
            const int o2 = p2z(x, y);
            st2<T>(s.h0, o2, hold); st2<T>(s.u0, o2, uold); st2<T>(s.v0, o2, vold);
        }
        csync();
        V xm[4], gxo[4], gyo[4];
        T ym[4];
        gradients2<T, ENGINE>(s, bg, p.theta, delta, tid, x, py, c, xm, ym, gxo, gyo);
        csync();
        (void)faces2<T, ENGINE>(s, p, delta, tid, x, py, c, xm, ym, gxo, gyo);
        csync();
        if (block_has_segments<T>(m, ib)) {
            boundaries2<T, true>(s, m, p, ib, ts.totaltime + dtd, tid);
            csync();
        }
        V dh, dhu, dhv;
        divergence2<T>(s, p, (T)1.0 / ((T)1.0 * delta), x, py, c[VH], c[VU], c[VV], dh, dhu, dhv);
        if (p.nriver > 0)
            dh = V{add_rivers<T>(m, p, ib, x, y, dh.a, ts.totaltime), add_rivers<T>(m, p, ib, x, y + 1, dh.b, ts.totaltime)};
        V ho, uo, vo;
        advance_v<V>(dt, p.eps, p.eps_d, p.forcemass != 0, hold, uold, vold, dh, dhu, dhv, ho, uo, vo);
        const V cfv = p.has_cf ? V{cfw[y * 16 + x], cfw[(y + 1) * 16 + x]} : V{p.cf, p.cf};
        friction_v<T>(p.frictionmodel, p.g, p.eps, dt, cfv, ho, uo, vo);
        if (p.has_rain) {
            // AddrainforcingImplicitCPU (src/Updateforcing.cu:530-580)
            V Rainhh;
            if (p.rain_map) {
                const T xc = (T)p.xo_d + (T)m.bxo[ib] + (T)x * delta;
                const T yc0 = (T)p.yo_d + (T)m.byo[ib] + (T)y * delta;
                const T yc1 = (T)p.yo_d + (T)m.byo[ib] + (T)(y + 1) * delta;
                Rainhh = V{rain_map_at<T>(m.rmap, xc, yc0, ts.totaltime), rain_map_at<T>(m.rmap, xc, yc1, ts.totaltime)};
            } else {
                const T r = (T)series_at(m.rain_t + p.rain_off, m.rain_r + p.rain_off, p.rain_n, ts.totaltime,
                                         p.rain_sorted != 0);
                Rainhh = V{r, r};
            }
            const T rs = (T)dtd;
            const V rr = dv(dv(Rainhh, V{(T)1000.0, (T)1000.0}), V{(T)3600.0, (T)3600.0});
            const V maskv = with_mask ? V{(T)rmw[y * 16 + x], (T)rmw[(y + 1) * 16 + x]} : V{(T)1, (T)1};
            Rainhh = mul(vmax(mul(rr, V{rs, rs}), V{(T)0.0, (T)0.0}), maskv);
            const V hi = ho;
            const V qvol = dv(hi, add(hi, Rainhh));
            ho = add(hi, Rainhh);
            const M2 wet{(double)hi.a > p.eps_d, (double)hi.b > p.eps_d};
            uo = sel(wet, mul(uo, qvol), uo);
            vo = sel(wet, mul(vo, qvol), vo);
        }
        const int nxt = cur ^ 1;
        const size_t g0 = (size_t)ib * 256 + y * 16 + x;
        m.h[nxt][g0] = ho.a; m.h[nxt][g0 + 16] = ho.b;
        m.u[nxt][g0] = uo.a; m.u[nxt][g0 + 16] = uo.b;
        m.v[nxt][g0] = vo.a; m.v[nxt][g0 + 16] = vo.b;
        if (m.hmax) {
            m.hmax[g0] = ho.a > m.hmax[g0] ? ho.a : m.hmax[g0];
            m.hmax[g0 + 16] = ho.b > m.hmax[g0 + 16] ? ho.b : m.hmax[g0 + 16];
        }
        if (lead && tid == 0)
            m.time[2 * sc + (parity ^ 1)] = next_time_state<T>(ts, p, dtd, nxt, m.dtmin + 2 * sc, parity);
        csync();  // the working tiles are reused by the next block
    }
}
