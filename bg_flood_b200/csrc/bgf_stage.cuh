// Device helpers shared by the fused single-level kernels (bgf_flow.cu) and the
// multi-level kernels (bgf_amr.cu): bed tile loads, boundary-segment fluxes, the
// flux divergence, and the step / dt bookkeeping of the device time loop.
//
// Included inside namespace bgf::BGF_VARIANT by each kernel file, so that every
// arithmetic variant (exact, fast) gets its own copy compiled with its own flags.
#pragma once

// Loads the bed halo tile and (engine 1) the bed-gradient rows/columns.
// Split mode stores the tile's bed as the deviation zb + D of the block's datum.
template <class T, int ENGINE, bool SPLIT = false, bool BALANCE = false>
__device__ __forceinline__ void load_bed(Smem<T>& s, const DevModel<T>& m, int ib, int tid, T D = (T)0)
{
    const T* zbt = m.zb + (size_t)ib * 324;
    const T* gx = m.dzbdx + (size_t)ib * 324;
    const T* gy = m.dzbdy + (size_t)ib * 324;
    if constexpr (BALANCE) {
        // one entry per thread, and the 68 (bed) and 32 (bed gradient) entries beyond
        // 256 on threads 128..195 and 224..255: threads 0..127 load a ring cell of the
        // state tile in the same phase.  (The corrector keeps the plain loops: there
        // the extra live values cost register spills.)
        static_assert(NTHREADS == 256, "entries 256.. go to threads 128..");
        {
            const int k = tid;
            const int x = k % 18 - 1, y = k / 18 - 1;
            s.zb[si(x, y)] = SPLIT ? zbt[k] + D : zbt[k];
        }
        if (tid >= 128 && tid < 128 + 324 - NTHREADS) {
            const int k = tid + (NTHREADS - 128);
            const int x = k % 18 - 1, y = k / 18 - 1;
            s.zb[si(x, y)] = SPLIT ? zbt[k] + D : zbt[k];
        }
        if (ENGINE == 1) {
            {
                const int k = tid;
                int x = k % 18 - 1, y = k / 18;
                s.dzbx[gxi(x, y)] = gx[hi18(x, y)];
                int xx = k % 16, yy = k / 16 - 1;
                s.dzby[k] = gy[hi18(xx, yy)];
            }
            if (tid >= NTHREADS - (18 * 16 - NTHREADS)) {
                const int k = tid + (18 * 16 - NTHREADS);
                int x = k % 18 - 1, y = k / 18;
                s.dzbx[gxi(x, y)] = gx[hi18(x, y)];
                int xx = k % 16, yy = k / 16 - 1;
                s.dzby[k] = gy[hi18(xx, yy)];
            }
        }
    } else {
        for (int k = tid; k < 324; k += NTHREADS) {
            const int x = k % 18 - 1, y = k / 18 - 1;
            s.zb[si(x, y)] = SPLIT ? zbt[k] + D : zbt[k];
        }
        if (ENGINE == 1) {
            for (int k = tid; k < 18 * 16; k += NTHREADS) {
                int x = k % 18 - 1, y = k / 18;
                s.dzbx[gxi(x, y)] = gx[hi18(x, y)];
                int xx = k % 16, yy = k / 16 - 1;
                s.dzby[k] = gy[hi18(xx, yy)];
            }
        }
    }
}

// interptime (src/Util_CPU.cu:107-110) over a uniform series, stepping as
// FlowbndFlux does (src/Boundary.cu:130-143).
// The sample index is the first st in [1, n-1) whose time is not before `time`, else
// n - 1.  For non-decreasing times that condition holds on a prefix, so bisection
// finds the same index in log2(n) dependent loads instead of up to n (late in a long
// series the scan dominated the boundary blocks); other series keep the scan.
__device__ __forceinline__ double series_at(const double* t, const double* v, int n, double time, bool sorted)
{
    int st = 1;
    if (sorted) {
        int hi = n - 1;
        while (st < hi) {
            const int mid = (st + hi) >> 1;
            if (t[mid] - time < 0.0) st = mid + 1;
            else hi = mid;
        }
    } else {
        while (st < n - 1 && t[st] - time < 0.0) st++;
    }
    return v[st - 1] + (time - t[st - 1]) / (t[st] - t[st - 1]) * (v[st] - v[st - 1]);
}

// Gridded rain rate (mm/h) at (x, y) and `time`: the two frames around `time`
// (Forcingthisstep, src/Updateforcing.cu:87-125: frame index clamped to
// [0, nt-2]) interpolated in time at the four grid nodes around the point, each
// rounded to float as the reference's "now" grid holds it, then the bilinear
// interpolation of interp2BUQ (src/GridManip.cu:540-575) in double.  Kept out of
// line: inlined, its live values push the update kernels into register spills even
// when no scenario has a rain map.
template <class T> __device__ __noinline__ T rain_map_at(const RainMapDev r, T x, T y, double time)
{
    int st = (int)floor((time - r.to) / r.dt);
    st = min(max(st, 0), r.nt - 2);
    const double tb = r.to + r.dt * st;
    const float* b = r.val + (size_t)st * r.nx * r.ny;
    const float* a = b + (size_t)r.nx * r.ny;
    const double xi = fmax(fmin((double)x, r.xmax), r.xo);
    const double yi = fmax(fmin((double)y, r.ymax), r.yo);
    const int cfi = min(max((int)floor((xi - r.xo) / r.dx), 0), r.nx - 2), cfip = cfi + 1;
    const int cfj = min(max((int)floor((yi - r.yo) / r.dy), 0), r.ny - 2), cfjp = cfj + 1;
    auto now = [&](int i, int j) -> double {
        const size_t k = (size_t)i + (size_t)j * r.nx;
        return (double)(float)((double)b[k] + (time - tb) * (double)(a[k] - b[k]) / r.dt);
    };
    const double q11 = now(cfi, cfj), q12 = now(cfi, cfjp), q21 = now(cfip, cfj), q22 = now(cfip, cfjp);
    const double x1 = r.xo + r.dx * cfi, x2 = r.xo + r.dx * cfip;
    const double y1 = r.yo + r.dy * cfj, y2 = r.yo + r.dy * cfjp;
    const double x2x1 = x2 - x1, y2y1 = y2 - y1, x2x = x2 - xi, y2y = y2 - yi, yy1 = yi - y1, xx1 = xi - x1;
    return (T)(1.0 / (x2x1 * y2y1) * (q11 * x2x * y2y + q21 * xx1 * y2y + q12 * x2x * yy1 + q22 * xx1 * yy1));
}

// River discharge of one river at `time` per unit area, as AddRiverForcing computes
// it (src/Updateforcing.cu:146-170): the first sample later than `time`, the
// interpolated discharge rounded to T, then divided by the discharge area.
template <class T> __device__ __forceinline__ T river_rate(const RiverDev& r, const double* t, const double* q, double time)
{
    // the first st in [0, n-1) whose time is after `time`, else n - 1, by bisection:
    // bgf_add_river takes strictly increasing times only, for which the reference's
    // forward scan finds the same index
    int st = 0;
    int hi = r.n - 1;
    while (st < hi) {
        const int mid = (st + hi) >> 1;
        if (t[r.off + mid] - time <= 0.0) st = mid + 1;
        else hi = mid;
    }
    const int pv = st > 0 ? st - 1 : 0;
    // before the first sample the reference divides by zero; the first value is used here
    const double qi = st == pv ? q[r.off + st]
                               : q[r.off + pv] + (time - t[r.off + pv]) / (t[r.off + st] - t[r.off + pv]) *
                                                     (q[r.off + st] - q[r.off + pv]);
    return (T)((double)(T)qi / r.area);
}

// InjectManyRiversGPU (src/Updateforcing.cu:245-300) for cell (x, y) of block ib:
// every river whose box overlaps the cell's box (OBBdetect in T) adds its rate to
// dh, in river order.  `time` is the start of the step (both stages).
template <class T>
__device__ __forceinline__ T add_rivers_cell(const RiverDev* rivers, const double* riv_t, const double* riv_q, int first,
                                          int nriver, T levdx, double xo, double yo, int x, int y, T dh, double time)
{
    const T xllo = (T)xo, yllo = (T)yo;
    const T half = (T)0.5 * levdx;
    const T xl = xllo + (T)x * levdx - half, xr = xllo + (T)x * levdx + half;
    const T yb = yllo + (T)y * levdx - half, yt = yllo + (T)y * levdx + half;
    for (int k = 0; k < nriver; k++) {
        const RiverDev r = rivers[first + k];
        const bool ox = (T)r.xs <= xr && (T)r.xe >= xl;
        const bool oy = (T)r.ys <= yt && (T)r.ye >= yb;
        if (ox && oy) dh = dh + river_rate<T>(r, riv_t, riv_q, time);
    }
    return dh;
}

template <class T>
__device__ __forceinline__ T add_rivers(const DevModel<T>& m, const StepParams<T>& p, int ib, int x, int y, T dh,
                                        double time)
{
    if (p.nriver == 0) return dh;
    return add_rivers_cell<T>(m.rivers, m.riv_t, m.riv_q, p.riv_first, p.nriver, calcres<T>(p.delta0, m.level[ib]),
                              p.xo_d + m.bxo[ib], p.yo_d + m.byo[ib], x, y, dh, time);
}

// bndFluxGPUSideCPU (src/Boundary.cu:587-745) for the four sides of one block.
// Face arrays in s are modified in place; state n comes from s.h0/u0/v0 and the
// bed tile (zs = zb + h, as RecalculateZs leaves it).
// True when some side of block ib carries a boundary segment (the same for every
// thread of the block, so a barrier may depend on it).
template <class T> __device__ __forceinline__ bool block_has_segments(const DevModel<T>& m, int ib)
{
    const int* b = m.bndseg + (size_t)ib * 4;
    return (b[0] & b[1] & b[2] & b[3]) >= 0;  // the sign bit survives only if all four are -1
}

template <class T, bool SPLIT = false>
__device__ __forceinline__ void apply_boundaries(Smem<T>& s, const DevModel<T>& m, const StepParams<T>& p, int ib,
                                                 double tbnd, int tid, T D = (T)0)
{
    if (tid >= 64) return;
    int side = tid >> 4, t = tid & 15;
    int k = m.bndseg[ib * 4 + side];
    if (k < 0) return;
    SegDev sg = m.segs[k];
    if (sg.type == 1) return;
    double zsbnd = 0.0;
    if (!isnan(p.zsinit)) zsbnd = p.zsinit;
    T taper = (T)1.0;
    if (sg.n > 0) {
        if (p.bndtaper > 0.0) taper = (T)fmin((tbnd - p.inittime) / p.bndtaper, 1.0);
        zsbnd = series_at(m.seg_t + sg.off, m.seg_wl + sg.off, sg.n, tbnd, sg.sorted != 0);
    }
    int isright = side == 0 ? -1 : side == 1 ? 1 : 0;
    int istop = side == 2 ? 1 : side == 3 ? -1 : 0;
    int ix, iy, inx, iny;
    if (isright == 0) { ix = t; iy = istop < 0 ? 0 : BW; }
    else { iy = t; ix = isright < 0 ? 0 : BW; }
    if (isright < 0) { inx = ix + 1; iny = iy; }
    else if (isright > 0) { inx = ix - 1; iny = iy; }
    else if (istop < 0) { inx = ix; iny = iy + 1; }
    else { inx = ix; iny = iy - 1; }
    T sign = (T)isright + (T)istop;
    float zsb = (float)zsbnd;
    zsb = (float)((double)zsb + p.zsoffset);
    int ci = si(ix, iy), cin = si(inx, iny);
    T zsi = s.zb[ci] + s.h0[ci];
    T zsinside = s.zb[cin] + s.h0[cin];
    // (split mode: the tile holds deviations; zs = zb' + h' is the surface either way)
    T hinside = SPLIT ? D + s.h0[cin] : s.h0[cin];
    T uninside = isright != 0 ? s.u0[cin] : s.v0[cin];
    T hface = SPLIT ? D + s.h0[ci] : s.h0[ci];
    T zsX = (T)(((double)((T)zsb + (T)0.0) - 0.5 * (double)(zsi + zsinside)) * (double)taper + 0.5 * (double)(zsi + zsinside));
    float* qm = m.qmean + ib * 64 + side * 16 + t;
    T qmean = (T)*qm;
    T *Fh, *Fq, *Ss;
    int fi, fin;
    if (isright != 0) {
        Fh = s.Fhu; Fq = s.Fqux; Ss = s.Su;
        fi = fxi(ix, iy); fin = fxi(inx, iny);
    } else {
        Fh = s.Fhv; Fq = s.Fqvy; Ss = s.Sv;
        fi = fyi(ix, iy); fin = fyi(inx, iny);
    }
    T F, G, S;
    bool lowside = isright < 0 || istop < 0;
    if (lowside) { F = Fh[fi]; G = Fq[fi]; S = Ss[fin]; }
    else { F = Fh[fi]; G = Ss[fi]; S = Fq[fin]; }
    T factime = M<T>::fmin_((T)(p.dtparam / p.bndfiltertime), (T)1.0);
    T facrel = (T)1.0 - M<T>::fmin_((T)(p.dtparam / p.bndrelaxtime), (T)1.0);
    if (sg.type == 0) {
        F = (T)0.0;
        S = G;
    } else if (sg.type == 3) {
        if ((double)hface > p.eps_d || zsX > zsi) {
            abs1dq<T>(p.g, sign, factime, facrel, zsi, zsX, hface, qmean, F);
        } else {
            F = (T)0.0; S = G; qmean = (T)0.0;
        }
        *qm = (float)qmean;
    } else if (sg.type == 2) {
        if ((double)hface > p.eps_d || zsX > zsi) {
            dirichlet1q<T>(p.g, sign, zsX, zsinside, hinside, uninside, F);
        } else {
            F = (T)0.0; S = G; qmean = (T)0.0;
        }
        *qm = (float)qmean;
    }
    if (lowside) { Fh[fi] = F; Fq[fi] = G; Ss[fin] = S; }
    else { Fh[fi] = F; Ss[fi] = G; Fq[fin] = S; }
}

// updateEVCPU (src/Advection.cu:160-254), Cartesian.  Returns dh, dhu, dhv of the
// thread's cell from the face arrays.
template <class T>
__device__ __forceinline__ void flux_divergence(const Smem<T>& s, const StepParams<T>& p, T cmdinv, int x, int y, T hi,
                                                T uui, T vvi, T& dh, T& dhu, T& dhv)
{
    // Cartesian grid: the metric terms dmdl, dmdt and fG of the reference are zero
    // and their products only add signed zeros.
    int fi = fxi(x, y), fr = fxi(x + 1, y);
    int gi = fyi(x, y), gt = gi + 16;
    dh = (T)-1.0 * (s.Fhu[fr] - s.Fhu[fi] + s.Fhv[gt] - s.Fhv[gi]) * cmdinv;
    dhu = (s.Fqux[fi] + s.Fquy[gi] - s.Su[fr] - s.Fquy[gt]) * cmdinv + p.fc * hi * vvi;
    dhv = (s.Fqvy[gi] + s.Fqvx[fi] - s.Sv[gt] - s.Fqvx[fr]) * cmdinv - p.fc * hi * uui;
}

// Scenario of block slot ib (0 unless the model is a batched pool), its
// parameters, and whether the block writes its scenario's next time slot (the
// first block of the scenario in the active list).
template <class T> __device__ __forceinline__ int scen_of(const DevModel<T>& m, int ib) { return m.scen ? m.scen[ib] : 0; }
template <class T>
__device__ __forceinline__ StepParams<T> params_of(const DevModel<T>& m, const StepParams<T>& p, int sc)
{
    return m.sparams ? m.sparams[sc] : p;
}
template <class T> __device__ __forceinline__ bool lead_of(const DevModel<T>& m, int ib, int w)
{
    return m.lead ? m.lead[ib] != 0 : w == 0;
}
// The step parameters of a block: the kernel argument for a single scenario, the
// scenario's entry of the pool's table otherwise (global memory, cached).
template <bool POOL, class T>
__device__ __forceinline__ const StepParams<T>& params_ref(const DevModel<T>& m, const StepParams<T>& p0, int sc)
{
    if constexpr (POOL) return m.sparams[sc];
    else return p0;
}

// Whether this step runs (the reference loop condition totaltime < endtime plus
// the step budget); identical in both kernels of a step.
__device__ __forceinline__ bool step_live(const TimeState& ts)
{
    return !ts.done && ts.totaltime < ts.endtime && ts.nstep < ts.maxsteps;
}

// A cell whose state (h, u, v on the assembled tile) is not finite contributes a dt
// of 0 to the CFL minimum: the step then ends its scenario with status BGF_ENAN (a
// finite state always gives dt > 0).  The reference has no such check; a NaN there
// propagates silently, since dry-face tests are false for it.
template <class T> __device__ __forceinline__ T finite_state_dt(const Smem<T>& s, int tid, T celldt)
{
    const int c = ti(tid & 15, tid >> 4);
    return isfinite(s.t[VH][c]) && isfinite(s.t[VU][c]) && isfinite(s.t[VV][c]) ? celldt : (T)0;
}

// dt of the step from the reduced minimum (CalctimestepGPU, src/Advection.cu:549-620
// and CalctimestepCPU, :511-535): clamp to 1.5 * the previous dt, then split the
// time to the next output into an integer number of equal steps.
template <class T> __device__ __forceinline__ T step_dt(const TimeState& ts, unsigned long long minbits)
{
    T dt = dt_from_bits<T>(minbits);
    if ((double)dt > (1.5 * ts.dtmax)) dt = (T)(1.5 * ts.dtmax);
    if (ceil((ts.nextoutputtime - ts.totaltime) / (double)dt) > 0.0)
        dt = (T)((ts.nextoutputtime - ts.totaltime) / ceil((ts.nextoutputtime - ts.totaltime) / (double)dt));
    return dt;
}


// Time slot of the next step (the Mainloop bookkeeping, src/Mainloop.cu:43-86 and
// the crash check :648-719), written by one thread once dt is known; re-arms the
// running dt minimum of the slot the next step reduces into.
template <class T>
__device__ __forceinline__ TimeState next_time_state(const TimeState& ts, const StepParams<T>& p, double dtd, int nxt,
                                                     unsigned long long* dtmin, int parity)
{
    TimeState nt = ts;
    nt.dt = dtd;
    nt.dtmax = dtd;
    nt.totaltime = ts.totaltime + dtd;
    nt.nstep = ts.nstep + 1;
    nt.cur = nxt;
    if (dtd < p.dtmin && nt.totaltime < ts.endtime) {
        nt.status = 4;  // BGF_EDT_UNDERFLOW
        nt.done = 1;
    }
    if (dtd == 0.0) {  // a non-finite state zeroed the dt minimum (finite_state_dt)
        nt.status = 5;  // BGF_ENAN
        nt.done = 1;
    }
    if (ts.outputtimestep > 0.0 && nt.nextoutputtime - nt.totaltime <= dtd * 0.00001) {
        nt.nextoutputtime = fmin(nt.nextoutputtime + ts.outputtimestep, ts.endtime);
    }
    dtmin[parity ^ 1] = dt_bits(inv_epsi<T>());
    return nt;
}
