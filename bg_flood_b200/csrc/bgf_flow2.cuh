// Second-generation single-level stage kernels: two cells per thread.
//
// Same step as flux_kernel / update_kernel (bgf_flow.cuh): the predictor assembles
// the block's 20x20 tile (block + two-cell ring from the neighbour tables),
// computes limited gradients, the wet-slope reset, every X and Y face, the CFL
// minimum, the boundary segments and the flux divergence; the corrector rebuilds
// the half-step tile, repeats the faces and applies the full-step advance,
// friction and rain.  What changes is how the work maps onto the SM:
//
//  * 128 threads per 16x16 block.  Thread (x, p) owns the vertically adjacent
//    cells (x, 2p) and (x, 2p+1) and evaluates both with one instruction stream on
//    pair values (bgf_pair.cuh): in the fast build FP32 sums and products are
//    paired .f32x2 instructions; in both builds the index arithmetic and the
//    shared-memory addressing are done once for both cells, and the Y face between
//    the two cells reuses registers.
//  * Shared arrays interleave each pair of rows (2p, 2p+1) column by column, so a
//    thread's two cells are one 64-bit word: loads and stores of a pair are single
//    64-bit shared accesses, and neighbours are at constant offsets.
//  * Branches of the Riemann solvers, the limiter and the wet/dry tests are
//    per-lane selects between values computed exactly as the scalar code computes
//    them; the exact build is bit-identical to the one-cell kernels.
//  * The dt of the step (time slot and clamps, in FP64) is evaluated once per block
//    and broadcast through shared memory; every global load of a block (tile, bed,
//    bed gradients) is issued before the first barrier.
//
// Warp w, half-warp h: pair p = (w & 1) + 4 (w >> 1) + 2 h, so the two half-warps
// of a warp are two pair rows apart (their 64-bit accesses fall in separate
// wavefronts without bank conflicts).
//
// Included inside namespace bgf::BGF_VARIANT after bgf_stage.cuh and bgf_pair.cuh.
#pragma once

constexpr int NT2 = 128;

// ---------------------------------------------------------------- layouts
// tile, x, y = -2..17: 10 pair rows of 20 columns x 2
__device__ __forceinline__ int p2t(int x, int y) { return ((y + 2) >> 1) * 40 + (x + 2) * 2 + ((y + 2) & 1); }
// x-gradients, x = -1..16, y = 0..15
__device__ __forceinline__ int p2gx(int x, int y) { return (y >> 1) * 36 + (x + 1) * 2 + (y & 1); }
// y-gradients, x = 0..15, y = -1..16
__device__ __forceinline__ int p2gy(int x, int y) { return ((y + 2) >> 1) * 32 + x * 2 + ((y + 2) & 1); }
// bed and state n on the 18x18 tile, x, y = -1..16
__device__ __forceinline__ int p2z(int x, int y) { return ((y + 2) >> 1) * 36 + (x + 1) * 2 + ((y + 2) & 1); }
// X faces, x = 0..16, y = 0..15
__device__ __forceinline__ int p2fx(int x, int y) { return (y >> 1) * 34 + x * 2 + (y & 1); }
// Y faces, x = 0..15, y = 0..16
__device__ __forceinline__ int p2fy(int x, int y) { return (y >> 1) * 32 + x * 2 + (y & 1); }

template <class T> struct Smem2 {
    T t[4][400];    // h, zs, u, v on the 20x20 tile
    T gx[4][288];   // x-gradients
    T gy[4][320];   // y-gradients
    T zb[360];      // bed, 18x18
    T fx[4][272];   // Fhu, Fqux, Su, Fqvx
    T fy[4][288];   // Fhv, Fqvy, Sv, Fquy
    T red[NT2 / 32];
    T dtv;          // dt of the step (corrector), evaluated once per block
    T rainv;        // uniform rain depth of the step (corrector), evaluated once per block
    // corrector only (the predictor's launch leaves these out of its shared memory)
    T h0[360], u0[360], v0[360];  // state n on the 18x18 tile (boundary fluxes)
};
template <class T> __host__ __device__ constexpr size_t smem2_pred() { return offsetof(Smem2<T>, h0); }
template <class T> __host__ __device__ constexpr size_t smem2_corr() { return sizeof(Smem2<T>); }

// 64-bit shared access of the pair of rows (2p, 2p+1) at index i (even).
template <class T> __device__ __forceinline__ V2<T> ld2(const T* a, int i)
{
    if constexpr (sizeof(T) == 4) {
        const float2 v = *reinterpret_cast<const float2*>(a + i);
        return V2<T>{v.x, v.y};
    } else {
        return V2<T>{a[i], a[i + 1]};
    }
}
template <class T> __device__ __forceinline__ void st2(T* a, int i, V2<T> v)
{
    if constexpr (sizeof(T) == 4) {
        *reinterpret_cast<float2*>(a + i) = make_float2(v.a, v.b);
    } else {
        a[i] = v.a;
        a[i + 1] = v.b;
    }
}

template <class V> __device__ __forceinline__ V cst(typename LaneOf<V>::T x)
{
    if constexpr (sizeof(V) == sizeof(typename LaneOf<V>::T)) return x;
    else return V{x, x};
}

// ---------------------------------------------------------------- numerics on pairs
// Each restates the scalar routine of bgf_numerics.cuh operation by operation.

// minmod2 (src/Util_CPU.cu:243-263).  In the increasing case all three candidates
// are >= +0 and the routine returns their minimum; in the decreasing case all are
// <= -0 and it returns their maximum.
template <class V> __device__ __forceinline__ V minmod_v(V theta, V s0, V s1, V s2)
{
    using T = typename LaneOf<V>::T;
#if BGF_FAST
    if constexpr (sizeof(T) == 4) {
        // Fast build: the same limiter as a sign test and one three-way minimum of
        // magnitudes.  s0 < s1 < s2 (or s0 > s1 > s2) holds exactly when the two
        // one-sided differences have the same strict sign, i.e. when their product is
        // positive (a product flushed to zero only drops a subnormal slope); the
        // result is then the candidate of least magnitude with that sign.
        const V a = sub(s1, s0), b = sub(s2, s1);
        const V d1 = mul(theta, a), d3 = mul(theta, b);
        const V d2 = mul(sub(s2, s0), cst<V>((T)0.5));
        const V m = vmin(vmin(vabs(d1), vabs(d2)), vabs(d3));
        return sel(gt(mul(a, b), cst<V>((T)0.0)), vcopysign(m, a), cst<V>((T)0.0));
    }
#endif
    const auto inc = lt(s0, s1) && lt(s1, s2);
    const auto dec = gt(s0, s1) && gt(s1, s2);
    const V d1 = mul(theta, sub(s1, s0));
    const V d2 = mul(sub(s2, s0), cst<V>((T)0.5));
    const V d3 = mul(theta, sub(s2, s1));
    const V lo = vmin(sel(lt(d2, d1), d2, d1), d3);
    const V hi = vmax(sel(gt(d2, d1), d2, d1), d3);
    return sel(inc, lo, sel(dec, hi, cst<V>((T)0.0)));
}

// x / delta for the block spacing (div_by): the fast build multiplies by the
// rounded reciprocal, the exact build takes Markstein's correctly rounded quotient.
template <class T> __device__ __forceinline__ T divd_v(T x, T d, T r) { return div_by<T>(x, d, r); }
template <class T> __device__ __forceinline__ V2<T> divd_v(V2<T> x, T d, T r)
{
#if BGF_FAST
    return mul(x, V2<T>{r, r});
#else
    return V2<T>{div_by<T>(x.a, d, r), div_by<T>(x.b, d, r)};
#endif
}

// Limited slope minmod2(theta, s0, s1, s2) / delta.  The fast build folds 1 / delta
// into the limiter's factors (theta / delta and 0.5 / delta) and evaluates the
// sign-test form of minmod_v, one product fewer per slope.
template <class V> __device__ __forceinline__ V slope_v(V th, V thr, V hr, V s0, V s1, V s2,
                                                        typename LaneOf<V>::T delta, typename LaneOf<V>::T rdelta)
{
    using T = typename LaneOf<V>::T;
#if BGF_FAST
    if constexpr (sizeof(T) == 4) {
        const V a = sub(s1, s0), b = sub(s2, s1);
        const V m = vmin(vmin(vabs(mul(thr, a)), vabs(mul(hr, sub(s2, s0)))), vabs(mul(thr, b)));
        return sel(gt(mul(a, b), cst<V>((T)0.0)), vcopysign(m, a), cst<V>((T)0.0));
    }
#endif
    (void)thr;
    (void)hr;
    return divd_v(minmod_v<V>(th, s0, s1, s2), delta, rdelta);
}

// Wet-slope reset (wetslope)
template <class V>
__device__ __forceinline__ V wetslope_v(V hdelta, V zsi, V hi, V zsm, V zsp, V dzs, V dh, V dzb)
{
    using T = typename LaneOf<V>::T;
    const V base = sub(zsi, hi);
    const V ddz = sub(dzs, dh);
    const V mzs = mad(mul(cst<V>((T)-1.0), hdelta), ddz, base);  // base - hdelta (dzs - dh)
    const V pzs = mad(hdelta, ddz, base);
    const auto reset = gt(mul(dzs, dzs), mul(dzb, dzb)) && (gt(mzs, zsm) || gt(pzs, zsp));
    return sel(reset, add(dh, dzb), dzs);
}

template <class V> struct FaceV {
    V hi, hn, zsi, zsn, uni, unn, uti, utn;
    V dhi, dhn, dzsi, dzsn, duni, dunn, duti, dutn;
    V zbi, zbn;
    // source-term depth and bed of each side: the cells' own (engine 1: zb; engine 2:
    // zs - h) except at a coarse/fine face, where the coarser side's cell is used
    V hsi, hsn, zri, zrn;
};
template <class V> struct FaceOutV {
    V Fh, Fq, S, Ft, dt;
    typename LaneOf<V>::Mask wet;
};

// hllc (src/Reimann.cu:838-877), Cartesian.
template <class V>
__device__ __forceinline__ V hllc_v(V g, V CFLdelta, V epsi, V hm, V hp, V um, V up, V& fh, V& fq)
{
    using T = typename LaneOf<V>::T;
    const V half = cst<V>((T)0.5), zero = cst<V>((T)0.0), two = cst<V>((T)2.0);
    const V cmo = vsqrt(mul(g, hm));
    const V cp = vsqrt(mul(g, hp));
    const V ustar = sub(mad(add(um, up), half, cmo), cp);
    const V cstar = mad(add(cmo, cp), half, mul(sub(um, up), cst<V>((T)0.25)));
    const V SL = sel(eq(hm, zero), mad(cst<V>((T)-2.0), cp, up), vmin(sub(um, cmo), sub(ustar, cstar)));
    const V SR = sel(eq(hp, zero), mad(two, cmo, um), vmax(add(up, cp), add(ustar, cstar)));
    const V fhm = mul(um, hm);
    const V fum = mul(hm, mad(um, um, mul(mul(g, hm), half)));
    const V fhp = mul(up, hp);
    const V fup = mul(hp, mad(up, up, mul(mul(g, hp), half)));
    const V SLSR = mul(SL, SR);
    const V den = sub(SR, SL);
    const V nSL = mul(cst<V>((T)-1.0), SL);
    const V nh = mad(SLSR, sub(hp, hm), mad(nSL, fhp, mul(SR, fhm)));
    const V nq = mad(SLSR, sub(mul(hp, up), mul(hm, um)), mad(nSL, fup, mul(SR, fum)));
#if BGF_FAST
    // one reciprocal of the wave-speed spread for both star-region fluxes
    const V rden = dv(cst<V>((T)1.0), den);
    const V fhM = mul(nh, rden);
    const V fqM = mul(nq, rden);
#else
    const V fhM = dv(nh, den);
    const V fqM = dv(nq, den);
#endif
    const auto caseL = le(zero, SL);
    const auto caseR = ge(zero, SR);
    fh = sel(caseL, fhm, sel(caseR, fhp, fhM));
    fq = sel(caseL, fum, sel(caseR, fup, fqM));
    // the reference forms max(|SL|, |SR|) in double; both conversions are exact
    const V a = vmax(vabs(SL), vabs(SR));
    return sel(gt(a, epsi), dv(CFLdelta, a), cst<V>(inv_epsi<T>()));
}

// KurgSolver (src/Kurganov.cu:1865-1911), Cartesian.
template <class V>
__device__ __forceinline__ V kurg_v(V g, V CFLdelta, V epsi, V hp, V hm, V up, V um, V& fh, V& fu)
{
    using T = typename LaneOf<V>::T;
    const V zero = cst<V>((T)0.0);
    const V cp = vsqrt(mul(g, hp));
    const V cmo = vsqrt(mul(g, hm));
    const V ap = vmax(vmax(add(up, cp), add(um, cmo)), zero);
    const V am = vmin(vmin(sub(up, cp), sub(um, cmo)), zero);
    const V a = vmax(ap, mul(cst<V>((T)-1.0), am));  // -am
    const auto live = gt(a, epsi);
    const V ad = dv(cst<V>((T)1.0), sub(ap, am));
    const V qm = mul(hm, um);
    const V qp = mul(hp, up);
    const V ga = mul(g, cst<V>((T)0.5));
    const V apm = mul(ap, am);
    const V fhl = mul(mad(apm, sub(hp, hm), sub(mul(ap, qm), mul(am, qp))), ad);
    const V ful = mul(mad(apm, sub(qp, qm),
                          sub(mul(ap, mad(qm, um, mul(ga, mul(hm, hm)))), mul(am, mad(qp, up, mul(ga, mul(hp, hp)))))),
                      ad);
    fh = sel(live, fhl, zero);
    fu = sel(live, ful, zero);
    return sel(live, dv(CFLdelta, a), cst<V>(inv_epsi<T>()));
}

// face_flux (bgf_numerics.cuh) without a coarse/fine substitution: the source-term
// depth and bed are the cells' own (engine 1: zb; engine 2: zs - h).
template <class V, int ENGINE>
__device__ __forceinline__ FaceOutV<V> face_v(const FaceV<V>& f, V g, V CFLdelta, V epsi, V eps, V dx, V ga)
{
    using T = typename LaneOf<V>::T;
    const V zero = cst<V>((T)0.0), one = cst<V>((T)1.0);
    FaceOutV<V> r;
    r.wet = gt(f.hi, eps) || gt(f.hn, eps);
    V fh, fu, fv, sl, sr;
    if constexpr (ENGINE == 2) {
        const V zi = sub(f.zsi, f.hi);
        const V ndx = mul(cst<V>((T)-1.0), dx);
        const V zl = mad(ndx, sub(f.dzsi, f.dhi), zi);
        const V zn = sub(f.zsn, f.hn);
        const V zr = mad(dx, sub(f.dzsn, f.dhn), zn);
        const V zlr = vmax(zl, zr);
        const V hl = mad(ndx, f.dhi, f.hi);
        const V up = mad(ndx, f.duni, f.uni);
        const V hp = vmax(zero, sub(add(hl, zl), zlr));
        const V hr = mad(dx, f.dhn, f.hn);
        const V um = mad(dx, f.dunn, f.unn);
        const V hm = vmax(zero, sub(add(hr, zr), zlr));
        r.dt = kurg_v<V>(g, CFLdelta, epsi, hp, hm, up, um, fh, fu);
        fv = mul(sel(gt(fh, zero), mad(dx, f.dutn, f.utn), mad(ndx, f.duti, f.uti)), fh);
        sl = mul(ga, mad(add(hl, f.hsi), sub(f.zri, zl), sub(mul(hp, hp), mul(hl, hl))));
        sr = mul(ga, mad(add(hr, f.hsn), sub(f.zrn, zr), sub(mul(hm, hm), mul(hr, hr))));
    } else {
        // products fused into the sums (exact build: separately rounded, the same values)
        const V ndx = mul(cst<V>((T)-1.0), dx);
        const V hr = mad(ndx, f.dhi, f.hi);
        const V hl = mad(dx, f.dhn, f.hn);
        const V etar = mad(ndx, f.dzsi, f.zsi);
        const V etal = mad(dx, f.dzsn, f.zsn);
        const V zr = sub(etar, hr);
        const V zl = sub(etal, hl);
        const V zA = vmax(zr, zl);
        const V zCN = vmin(zA, vmin(etal, etar));
        const V hCNr = vmax(zero, vmin(sub(etar, zCN), hr));
        const V hCNl = vmax(zero, vmin(sub(etal, zCN), hl));
        // Bouchut velocity reconstruction; a dry side keeps the plain slope
        // (nfr is -fr exactly)
        const V nfr = sel(gt(f.hi, eps), mul(add(one, dv(mul(dx, f.dhi), f.hi)), ndx), ndx);
        const V fl = sel(gt(f.hn, eps), mul(sub(one, dv(mul(dx, f.dhn), f.hn)), dx), dx);
        const V ur = mad(nfr, f.duni, f.uni);
        const V vr = mad(nfr, f.duti, f.uti);
        const V ul = mad(fl, f.dunn, f.unn);
        const V vl = mad(fl, f.dutn, f.utn);
        r.dt = hllc_v<V>(g, CFLdelta, epsi, hCNl, hCNr, ul, ur, fh, fu);
        fv = mul(sel(gt(fh, zero), vl, vr), fh);
        sl = mul(mul(ga, add(f.hsi, hCNr)), sub(f.zri, zCN));
        sr = mul(mul(ga, add(hCNl, f.hsn)), sub(f.zrn, zCN));
    }
    r.Fh = sel(r.wet, fh, zero);
    r.Fq = sel(r.wet, sub(fu, sl), zero);
    r.S = sel(r.wet, sub(fu, sr), zero);
    r.Ft = sel(r.wet, fv, zero);
    r.dt = sel(r.wet, r.dt, cst<V>(inv_epsi<T>()));
    return r;
}

// face_flux_split (bgf_split.cuh) on pairs: split precision, each operation in the
// scalar routine's order (the exact build reproduces it bit for bit).  The FaceV
// depths hi, hn are deviations from the block datum D; zsi, zsn surface elevations;
// zbi, zbn beds as deviations zb + D (engine 1).  Momentum fluxes carry the datum's
// hydrostatic shift -g D^2 / 2, which a dry face carries alone.
template <class V, int ENGINE>
__device__ __forceinline__ FaceOutV<V> face_v_split(const FaceV<V>& f, V D, V g, V CFLdelta, V epsi, V eps, V dx,
                                                    V ga)
{
    using T = typename LaneOf<V>::T;
    const V zero = cst<V>((T)0.0), one = cst<V>((T)1.0), two = cst<V>((T)2.0), mone = cst<V>((T)-1.0);
    const V half = cst<V>((T)0.5), quarter = cst<V>((T)0.25);
    const V nD = mul(mone, D), ndx = mul(mone, dx);
    const V shift = mul(mul(mul(mone, ga), D), D);  // -ga * D * D
    FaceOutV<V> r;
    const V Hi = add(D, f.hi), Hn = add(D, f.hn);  // full depths
    r.wet = gt(Hi, eps) || gt(Hn, eps);
    V fh, fu, fv, sl, sr;
    if constexpr (ENGINE == 2) {
        const V zi = sub(f.zsi, f.hi);  // bed deviations
        const V zl = mad(ndx, sub(f.dzsi, f.dhi), zi);
        const V zn = sub(f.zsn, f.hn);
        const V zr = mad(dx, sub(f.dzsn, f.dhn), zn);
        const V zlr = vmax(zl, zr);
        const V hl = mad(ndx, f.dhi, f.hi);
        const V up = mad(ndx, f.duni, f.uni);
        const V hp = vmax(nD, sub(add(hl, zl), zlr));
        const V hr = mad(dx, f.dhn, f.hn);
        const V um = mad(dx, f.dunn, f.unn);
        const V hm = vmax(nD, sub(add(hr, zr), zlr));
        const V Hp = add(D, hp), Hm = add(D, hm), Hl = add(D, hl), Hr = add(D, hr);
        const V cp = vsqrt(mul(g, Hp)), cmo = vsqrt(mul(g, Hm));
        const V ap = vmax(vmax(add(up, cp), add(um, cmo)), zero);
        const V am = vmin(vmin(sub(up, cp), sub(um, cmo)), zero);
        const V a = vmax(ap, mul(mone, am));
        const auto live = gt(a, epsi);
        const V ad = dv(one, sub(ap, am));
        const V qm = mul(Hm, um), qp = mul(Hp, up), apm = mul(ap, am);
        const V pm = mul(mul(ga, hm), mad(two, D, hm)), pp = mul(mul(ga, hp), mad(two, D, hp));
        const V fhl = mul(mad(apm, sub(hp, hm), sub(mul(ap, qm), mul(am, qp))), ad);
        const V ful = mul(mad(apm, sub(qp, qm), sub(mul(ap, mad(qm, um, pm)), mul(am, mad(qp, up, pp)))), ad);
        fh = sel(live, fhl, zero);
        fu = sel(live, ful, shift);
        r.dt = sel(live, dv(CFLdelta, a), cst<V>(inv_epsi<T>()));
        fv = sel(gt(fh, zero), mul(mad(dx, f.dutn, f.utn), fh), mul(mad(ndx, f.duti, f.uti), fh));
        sl = mul(ga, mad(sub(hp, hl), add(Hp, Hl), mul(add(Hl, Hi), sub(zi, zl))));
        sr = mul(ga, mad(sub(hm, hr), add(Hm, Hr), mul(add(Hr, Hn), sub(zn, zr))));
    } else {
        const V hr = mad(ndx, f.dhi, f.hi);
        const V hl = mad(dx, f.dhn, f.hn);
        const V etar = mad(ndx, f.dzsi, f.zsi);
        const V etal = mad(dx, f.dzsn, f.zsn);
        const V zr = sub(etar, hr);
        const V zl = sub(etal, hl);
        const V zA = vmax(zr, zl);
        const V zCN = vmin(zA, add(vmin(etal, etar), D));
        const V hCNr = vmax(nD, vmin(sub(etar, zCN), hr));
        const V hCNl = vmax(nD, vmin(sub(etal, zCN), hl));
        // Bouchut velocity reconstruction on the full depths (nfr is -fr exactly)
        const V nfr = sel(gt(Hi, eps), mul(add(one, dv(mul(dx, f.dhi), Hi)), ndx), ndx);
        const V fl = sel(gt(Hn, eps), mul(sub(one, dv(mul(dx, f.dhn), Hn)), dx), dx);
        const V ur = mad(nfr, f.duni, f.uni);
        const V vr = mad(nfr, f.duti, f.uti);
        const V ul = mad(fl, f.dunn, f.unn);
        const V vl = mad(fl, f.dutn, f.utn);
        // hllc on the reconstructed states, pressures shifted by the datum
        const V hm = add(D, hCNl), hp = add(D, hCNr), um = ul, up = ur;
        const V cmo = vsqrt(mul(g, hm)), cp = vsqrt(mul(g, hp));
        const V ustar = sub(mad(add(um, up), half, cmo), cp);
        const V cstar = mad(add(cmo, cp), half, mul(sub(um, up), quarter));
        const V SL = sel(eq(hm, zero), mad(cst<V>((T)-2.0), cp, up), vmin(sub(um, cmo), sub(ustar, cstar)));
        const V SR = sel(eq(hp, zero), mad(two, cmo, um), vmax(add(up, cp), add(ustar, cstar)));
        const V fum = mad(mul(hm, um), um, mul(mul(ga, hCNl), mad(two, D, hCNl)));
        const V fup = mad(mul(hp, up), up, mul(mul(ga, hCNr), mad(two, D, hCNr)));
        const V fhm = mul(um, hm), fhp = mul(up, hp);
        const V rs = dv(one, sub(SR, SL));
        const V SLSR = mul(SL, SR);
        const V nSL = mul(mone, SL);
        const V fhM = mul(mad(SLSR, sub(hCNr, hCNl), mad(nSL, fhp, mul(SR, fhm))), rs);
        const V fqM = mul(mad(SLSR, sub(mul(hp, up), mul(hm, um)), mad(nSL, fup, mul(SR, fum))), rs);
        const auto caseL = le(zero, SL);
        const auto caseR = ge(zero, SR);
        fh = sel(caseL, fhm, sel(caseR, fhp, fhM));
        fu = sel(caseL, fum, sel(caseR, fup, fqM));
        const V a = vmax(vabs(SL), vabs(SR));
        r.dt = sel(gt(a, epsi), dv(CFLdelta, a), cst<V>(inv_epsi<T>()));
        fv = mul(sel(gt(fh, zero), vl, vr), fh);
        sl = mul(mul(ga, add(Hi, add(D, hCNr))), sub(f.zbi, zCN));
        sr = mul(mul(ga, add(add(D, hCNl), Hn)), sub(f.zbn, zCN));
    }
    r.Fh = sel(r.wet, fh, zero);
    r.Fq = sel(r.wet, sub(fu, sl), shift);
    r.S = sel(r.wet, sub(fu, sr), shift);
    r.Ft = sel(r.wet, fv, zero);
    r.dt = sel(r.wet, r.dt, cst<V>(inv_epsi<T>()));
    return r;
}

// AdvkernelCPU / AdvkernelGPU (src/Advection.cu:272-385) on pairs.
template <class T>
__device__ __forceinline__ T edt_lane(T dt, double eps_d, bool forcemass, T hold, T dhi)
{
#if BGF_FAST
    return forcemass ? dt : dhi >= (T)0.0 ? dt : M<T>::fmin_(dt, dv(M<T>::fmax_(hold, (T)eps_d), M<T>::fabs_(dhi)));
#else
    return forcemass ? dt : dhi >= (T)0.0 ? dt : (T)fmin((double)dt, fmax((double)hold, eps_d) / (double)M<T>::fabs_(dhi));
#endif
}
template <class T> __device__ __forceinline__ T edt_v(T dt, double eps_d, bool fm, T hold, T dhi)
{
    return edt_lane<T>(dt, eps_d, fm, hold, dhi);
}
template <class T> __device__ __forceinline__ V2<T> edt_v(T dt, double eps_d, bool fm, V2<T> hold, V2<T> dhi)
{
    return V2<T>{edt_lane<T>(dt, eps_d, fm, hold.a, dhi.a), edt_lane<T>(dt, eps_d, fm, hold.b, dhi.b)};
}
template <class V>
__device__ __forceinline__ void advance_v(typename LaneOf<V>::T dt, typename LaneOf<V>::T eps, double eps_d,
                                          bool forcemass, V hold, V uold, V vold, V dhi, V dhui, V dhvi, V& ho, V& uo,
                                          V& vo)
{
    using T = typename LaneOf<V>::T;
    const V edt = edt_v(dt, eps_d, forcemass, hold, dhi);
    ho = mad(edt, dhi, hold);
    const auto wet = gt(ho, cst<V>(eps));
    uo = sel(wet, dv(mad(hold, uold, mul(edt, dhui)), ho), cst<V>((T)0.0));
    vo = sel(wet, dv(mad(hold, vold, mul(edt, dhvi)), ho), cst<V>((T)0.0));
}

template <class T> __device__ __forceinline__ V2<T> cbrt_v(V2<T> h)
{
#if BGF_FAST
    if constexpr (sizeof(T) == 4) return V2<T>{cbrta(h.a), cbrta(h.b)};
#endif
    return V2<T>{M<T>::cbrt_(h.a), M<T>::cbrt_(h.b)};
}

// advance_split (bgf_split.cuh) on pairs: depths as deviations from the datum D,
// full depths for the limiter and the velocities.
template <class T> __device__ __forceinline__ T edt_split_lane(T dt, T eps, bool forcemass, T Hold, T dhi)
{
    return forcemass ? dt : dhi >= (T)0.0 ? dt : M<T>::fmin_(dt, dv(M<T>::fmax_(Hold, eps), M<T>::fabs_(dhi)));
}
template <class T>
__device__ __forceinline__ void advance_split_v(T dt, T eps, bool forcemass, V2<T> D, V2<T> hold, V2<T> uold,
                                                V2<T> vold, V2<T> dhi, V2<T> dhui, V2<T> dhvi, V2<T>& ho, V2<T>& uo,
                                                V2<T>& vo)
{
    const V2<T> Hold = add(D, hold);
    const V2<T> edt{edt_split_lane<T>(dt, eps, forcemass, Hold.a, dhi.a), edt_split_lane<T>(dt, eps, forcemass, Hold.b, dhi.b)};
    ho = mad(edt, dhi, hold);
    const V2<T> Ho = add(D, ho);
    const M2 wet = gt(Ho, V2<T>{eps, eps});
    uo = sel(wet, dv(mad(Hold, uold, mul(edt, dhui)), Ho), V2<T>{(T)0.0, (T)0.0});
    vo = sel(wet, dv(mad(Hold, vold, mul(edt, dhvi)), Ho), V2<T>{(T)0.0, (T)0.0});
}

// bottomfriction (src/Friction.cu:17-143) on a pair; model is uniform.
template <class T>
__device__ __forceinline__ void friction_v(int model, T g, T eps, T dt, V2<T> cfv, V2<T> hi, V2<T>& ui, V2<T>& vi)
{
    const V2<T> normu = vsqrt(mad(ui, ui, mul(vi, vi)));
    V2<T> cfi;
    if (model == 0) cfi = cfv;
    else if (model == 1) cfi = V2<T>{smartfriction<T>(hi.a, cfv.a), smartfriction<T>(hi.b, cfv.b)};
    else if (model == -1) cfi = dv(mul(mul(V2<T>{g, g}, cfv), cfv), cbrt_v<T>(hi));
    else cfi = V2<T>{(T)0.0, (T)0.0};
    const V2<T> den = mad(dv(mul(cfi, normu), hi), V2<T>{dt, dt}, V2<T>{(T)1.0, (T)1.0});
    const M2 wet = gt(hi, V2<T>{eps, eps});
    ui = sel(wet, dv(ui, den), ui);
    vi = sel(wet, dv(vi, den), vi);
}

// ---------------------------------------------------------------- phases

// Ring cell r (0..127) of the tile: source block and cell, as ring_source.  On a
// regular grid of blocks the neighbour comes from the block's row and column (the
// same ids the tables hold) instead of a dependent table load.
template <class T>
__device__ __forceinline__ void ring_src2(const DevModel<T>& m, int ib, int r, int& x, int& y, int& sb, int& sx, int& sy)
{
    ring_pos(r, x, y);
    if (m.regular_nbx > 0) {
        const int nbx = m.regular_nbx, nby = m.regular_nby;
        const int by = m.regular_magic ? (int)__umulhi((unsigned)ib, m.regular_magic) : ib / nbx;
        const int bx = ib - by * nbx;
        sb = ib;
        sx = x;
        sy = y;
        if (x < 0) { if (bx > 0) { sb = ib - 1; sx = BW + x; } else sx = 0; }
        else if (x >= BW) { if (bx < nbx - 1) { sb = ib + 1; sx = x - BW; } else sx = BW - 1; }
        else if (y < 0) { if (by > 0) { sb = ib - nbx; sy = BW + y; } else sy = 0; }
        else if (y >= BW) { if (by < nby - 1) { sb = ib + nbx; sy = y - BW; } else sy = BW - 1; }
        return;
    }
    if (!tile_source(m.nbr, m.nblkmem, m.level, ib, x, y, sb, sx, sy, m.checklev != 0)) {
        atomicOr(m.err, 1);
        sb = ib; sx = min(max(x, 0), BW - 1); sy = min(max(y, 0), BW - 1);
    }
}

// The bed tile (18 x 18 values with the halo) is kept in shared memory as it lies in
// global memory, row-major (hi18): it arrives by 16-byte asynchronous copies
// (cp.async, no registers, no index arithmetic), which each thread waits for with
// bed_wait before the block's first barrier.  Both addresses are 16-byte aligned:
// block pieces of the bed are 1296 (FP32) or 2592 (FP64) bytes from a 256-byte
// aligned allocation, and s.zb starts on a 16-byte boundary of the CTA's shared memory.
template <class T> __device__ __forceinline__ void load_bed2(Smem2<T>& s, const T* zbt, int tid)
{
    static_assert(offsetof(Smem2<T>, zb) % 16 == 0 && (324 * sizeof(T)) % 16 == 0, "bed tile alignment");
    constexpr int n16 = (int)(324 * sizeof(T) / 16);  // 81 pieces in FP32, 162 in FP64
    for (int k = tid; k < n16; k += NT2) {
        const unsigned dst = (unsigned)__cvta_generic_to_shared(reinterpret_cast<char*>(s.zb) + 16 * k);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst),
                     "l"(reinterpret_cast<const char*>(zbt) + 16 * k)
                     : "memory");
    }
}
__device__ __forceinline__ void bed_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Bed gradients the engine-1 wet-slope reset reads: the own pair's x and y values
// and the one of this thread's ring cell, loaded with the tile (before the barrier).
template <class T> struct BedGrad {
    V2<T> gx, gy;
    T ring;
};
template <class T, int ENGINE>
__device__ __forceinline__ BedGrad<T> load_bedgrad(const DevModel<T>& m, int ib, int tid, int x, int y)
{
    BedGrad<T> b{};
    if (ENGINE == 1) {
        const size_t zo = (size_t)ib * 324;
        b.gx = V2<T>{m.dzbdx[zo + hi18(x, y)], m.dzbdx[zo + hi18(x, y + 1)]};
        b.gy = V2<T>{m.dzbdy[zo + hi18(x, y)], m.dzbdy[zo + hi18(x, y + 1)]};
        // ring cell tid / 2 at ring 1 of side r / 16: x-sides take dzbdx, y-sides dzbdy
        const int r = tid >> 1, side = r >> 4;
        int zx, zy;
        ring_pos(side * 32 + (r & 15), zx, zy);
        b.ring = side < 2 ? m.dzbdx[zo + hi18(zx, zy)] : m.dzbdy[zo + hi18(zx, zy)];
    }
    return b;
}

// Gradients of the own pair (registers and shared) and two ring gradients per thread,
// with the engine-1 wet-slope reset.  c holds the pair's h, zs, u, v; xm / ym the
// left and lower neighbours (kept for the faces).
template <class T, int ENGINE, bool SPLIT = false>
__device__ __forceinline__ void gradients2(Smem2<T>& s, const BedGrad<T>& bg, T theta, T delta, int tid, int x,
                                           int py, const V2<T> (&c)[4], V2<T> (&xm)[4], T (&ym)[4], V2<T> (&gxo)[4],
                                           V2<T> (&gyo)[4], T D = (T)0)
{
    using V = V2<T>;
    const T rdelta = (T)1.0 / delta;
    const V th = V{theta, theta};
    const T thr_s = theta * rdelta, hr_s = (T)0.5 * rdelta;
    const V thr{thr_s, thr_s}, hr{hr_s, hr_s};
    const int ct = p2t(x, 2 * py);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const T* a = s.t[k];
        xm[k] = ld2<T>(a, ct - 2);
        const V xp = ld2<T>(a, ct + 2);
        ym[k] = a[ct - 39];        // (x, 2p-1)
        const T yp = a[ct + 40];   // (x, 2p+2)
        gxo[k] = slope_v<V>(th, thr, hr, xm[k], c[k], xp, delta, rdelta);
        gyo[k] = slope_v<V>(th, thr, hr, V{ym[k], c[k].a}, c[k], V{c[k].b, yp}, delta, rdelta);
    }
    // ring gradients: ring cell r = tid / 2 (side r / 16, position r % 16), variables
    // h, zs (even tid) or u, v (odd tid); x-gradients on the left / right columns,
    // y-gradients on the bottom / top rows
    const int r = tid >> 1, side = r >> 4, q = r & 15, k0 = (tid & 1) * 2;
    int cm, cr, cp, o;
    const bool isx = side < 2;
    if (side == 0) { cm = p2t(-2, q); cr = p2t(-1, q); cp = p2t(0, q); o = p2gx(-1, q); }
    else if (side == 1) { cm = p2t(BW - 1, q); cr = p2t(BW, q); cp = p2t(BW + 1, q); o = p2gx(BW, q); }
    else if (side == 2) { cm = p2t(q, -2); cr = p2t(q, -1); cp = p2t(q, 0); o = p2gy(q, -1); }
    else { cm = p2t(q, BW - 1); cr = p2t(q, BW); cp = p2t(q, BW + 1); o = p2gy(q, BW); }
    T rg[2];
#pragma unroll
    for (int j = 0; j < 2; j++) {
        const T* a = s.t[k0 + j];
        rg[j] = slope_v<T>(theta, thr_s, hr_s, a[cm], a[cr], a[cp], delta, rdelta);
    }
    if (ENGINE == 1) {
        const T hd = delta * (T)0.5;
        // own pair: the x test compares with both x-neighbours, the y test with the
        // lower neighbour twice (WetsloperesetCPU)
        const V zsxp = ld2<T>(s.t[VZS], ct + 2);
        const V zsym{ym[VZS], c[VZS].a};
        // (split precision: the reset tests the full depth D + h')
        const V hc = SPLIT ? add(V{D, D}, c[VH]) : c[VH];
        gxo[VZS] = wetslope_v<V>(V{hd, hd}, c[VZS], hc, xm[VZS], zsxp, gxo[VZS], gxo[VH], bg.gx);
        gyo[VZS] = wetslope_v<V>(V{hd, hd}, c[VZS], hc, zsym, zsym, gyo[VZS], gyo[VH], bg.gy);
        if (k0 == 0) {
            // ring cell: rg[0] = h gradient, rg[1] = zs gradient
            const T* zs = s.t[VZS];
            const T zm = isx ? zs[cr - 2] : zs[cm];
            const T zp = isx ? zs[cr + 2] : zs[cp];
            const T hr = SPLIT ? D + s.t[VH][cr] : s.t[VH][cr];
            rg[1] = wetslope_v<T>(hd, zs[cr], hr, zm, zp, rg[1], rg[0], bg.ring);
        }
    }
    T* go = isx ? s.gx[0] : s.gy[0];
    const int stride = isx ? 288 : 320;
    go[k0 * stride + o] = rg[0];
    go[(k0 + 1) * stride + o] = rg[1];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        st2<T>(s.gx[k], p2gx(x, 2 * py), gxo[k]);
        st2<T>(s.gy[k], p2gy(x, 2 * py), gyo[k]);
    }
}

// The own pair's X faces (left of each cell) and Y faces (below each cell), and the
// 16 + 16 faces on the right column and the top row (warp 0, lanes 0..7 X, 8..15 Y).
// Returns the pair's cell dtmax as the one-cell kernels leave it.
// SUB: faces on a side whose neighbour is coarser take the neighbour's parent cell
// (subf, filled by the multi-level flux kernel) as their source-term depth and bed.
template <class T, int ENGINE, bool SPLIT = false, bool SUB = false>
__device__ __forceinline__ V2<T> faces2(Smem2<T>& s, const StepParams<T>& p, T delta, int tid, int x, int py,
                                        const V2<T> (&c)[4], const V2<T> (&xm)[4], const T (&ym)[4],
                                        const V2<T> (&gxo)[4], const V2<T> (&gyo)[4], T D = (T)0,
                                        const SubFaces<T>* subf = nullptr)
{
    using V = V2<T>;
    const V g{p.g, p.g}, epsi{p.epsi, p.epsi}, eps{p.epsface, p.epsface};
    const T cd = p.CFL * delta, dxs = delta * (T)0.5, gas = p.g * (T)0.5;
    const V CFLd{cd, cd}, dx{dxs, dxs}, ga{gas, gas};
    const int y = 2 * py;
    V zbc{(T)0, (T)0}, zbx{(T)0, (T)0};
    T zby = (T)0;
    if (ENGINE == 1) {
        zbc = V{s.zb[hi18(x, y)], s.zb[hi18(x, y + 1)]};
        zbx = V{s.zb[hi18(x - 1, y)], s.zb[hi18(x - 1, y + 1)]};
        zby = s.zb[hi18(x, y - 1)];
        if (SPLIT) {
            // split precision: beds as deviations zb + D of the block's datum
            zbc = add(zbc, V{D, D});
            zbx = add(zbx, V{D, D});
            zby = zby + D;
        }
    }
    const V Dv{D, D};
    // the cells' own source-term depth and bed
    auto own_sources = [&](FaceV<V>& ff) {
        ff.hsi = ff.hi;
        ff.hsn = ff.hn;
        if constexpr (ENGINE == 1) {
            ff.zri = ff.zbi;
            ff.zrn = ff.zbn;
        } else {
            ff.zri = sub(ff.zsi, ff.hi);
            ff.zrn = sub(ff.zsn, ff.hn);
        }
    };
    auto face = [&](const FaceV<V>& ff) {
        if constexpr (SPLIT) return face_v_split<V, ENGINE>(ff, Dv, g, CFLd, epsi, eps, dx, ga);
        else return face_v<V, ENGINE>(ff, g, CFLd, epsi, eps, dx, ga);
    };
    // X face pair (x-1 | x) at rows y, y+1
    FaceV<V> f;
    f.hi = c[VH]; f.zsi = c[VZS]; f.uni = c[VU]; f.uti = c[VV];
    f.hn = xm[VH]; f.zsn = xm[VZS]; f.unn = xm[VU]; f.utn = xm[VV];
    f.dhi = gxo[VH]; f.dzsi = gxo[VZS]; f.duni = gxo[VU]; f.duti = gxo[VV];
    {
        const int gn = p2gx(x - 1, y);
        f.dhn = ld2<T>(s.gx[VH], gn); f.dzsn = ld2<T>(s.gx[VZS], gn);
        f.dunn = ld2<T>(s.gx[VU], gn); f.dutn = ld2<T>(s.gx[VV], gn);
    }
    f.zbi = zbc; f.zbn = zbx;
    own_sources(f);
    if constexpr (SUB) {
        if (x == 0 && subf->on[0]) {  // left side coarser: the n-side sources
            f.hsn = V{subf->h[0][y], subf->h[0][y + 1]};
            f.zrn = V{subf->z[0][y], subf->z[0][y + 1]};
        }
    }
    const FaceOutV<V> fx = face(f);
    {
        const int o = p2fx(x, y);
        st2<T>(s.fx[0], o, fx.Fh); st2<T>(s.fx[1], o, fx.Fq); st2<T>(s.fx[2], o, fx.S); st2<T>(s.fx[3], o, fx.Ft);
    }
    // Y face pair (y-1 | y) and (y | y+1)
    f.hi = c[VH]; f.zsi = c[VZS]; f.uni = c[VV]; f.uti = c[VU];
    f.hn = V{ym[VH], c[VH].a}; f.zsn = V{ym[VZS], c[VZS].a}; f.unn = V{ym[VV], c[VV].a}; f.utn = V{ym[VU], c[VU].a};
    f.dhi = gyo[VH]; f.dzsi = gyo[VZS]; f.duni = gyo[VV]; f.duti = gyo[VU];
    {
        const int gn = p2gy(x, y - 1);
        f.dhn = V{s.gy[VH][gn], gyo[VH].a}; f.dzsn = V{s.gy[VZS][gn], gyo[VZS].a};
        f.dunn = V{s.gy[VV][gn], gyo[VV].a}; f.dutn = V{s.gy[VU][gn], gyo[VU].a};
    }
    f.zbi = zbc; f.zbn = V{zby, zbc.a};
    own_sources(f);
    if constexpr (SUB) {
        if (y == 0 && subf->on[2]) {  // bottom side coarser: the lower face's n-side sources
            f.hsn.a = subf->h[2][x];
            f.zrn.a = subf->z[2][x];
        }
    }
    const FaceOutV<V> fy = face(f);
    {
        const int o = p2fy(x, y);
        st2<T>(s.fy[0], o, fy.Fh); st2<T>(s.fy[1], o, fy.Fq); st2<T>(s.fy[2], o, fy.S); st2<T>(s.fy[3], o, fy.Ft);
    }
    // cell dtmax: the X sweep's value, then the Y sweep's where its face is wet
    const V cdt{fy.wet.a ? (fy.dt.a < fx.dt.a ? fy.dt.a : fx.dt.a) : fy.dt.a,
                fy.wet.b ? (fy.dt.b < fx.dt.b ? fy.dt.b : fx.dt.b) : fy.dt.b};
    // the right column's and the top row's faces
    if (tid < 16) {
        const bool isx = tid < 8;
        const int q = tid & 7;
        int ia, ib2, na, nb2, za, zb2, zna, znb, ga2, gb2, gna, gnb;
        const T* G[4];
        if (isx) {
            // faces x = 16 at rows 2q, 2q+1: i-side cells (16, .), n-side (15, .)
            ia = p2t(BW, 2 * q); ib2 = ia + 1; na = p2t(BW - 1, 2 * q); nb2 = na + 1;
            za = hi18(BW, 2 * q); zb2 = za + 18; zna = hi18(BW - 1, 2 * q); znb = zna + 18;
            ga2 = p2gx(BW, 2 * q); gb2 = ga2 + 1; gna = p2gx(BW - 1, 2 * q); gnb = gna + 1;
            G[0] = s.gx[VH]; G[1] = s.gx[VZS]; G[2] = s.gx[VU]; G[3] = s.gx[VV];
        } else {
            // faces y = 16 at columns 2q, 2q+1: i-side cells (., 16), n-side (., 15)
            ia = p2t(2 * q, BW); ib2 = p2t(2 * q + 1, BW); na = p2t(2 * q, BW - 1); nb2 = p2t(2 * q + 1, BW - 1);
            za = hi18(2 * q, BW); zb2 = za + 1; zna = hi18(2 * q, BW - 1); znb = zna + 1;
            ga2 = p2gy(2 * q, BW); gb2 = p2gy(2 * q + 1, BW); gna = p2gy(2 * q, BW - 1); gnb = p2gy(2 * q + 1, BW - 1);
            G[0] = s.gy[VH]; G[1] = s.gy[VZS]; G[2] = s.gy[VV]; G[3] = s.gy[VU];
        }
        const int nu = isx ? VU : VV, tu = isx ? VV : VU;
        FaceV<V> e;
        e.hi = V{s.t[VH][ia], s.t[VH][ib2]}; e.hn = V{s.t[VH][na], s.t[VH][nb2]};
        e.zsi = V{s.t[VZS][ia], s.t[VZS][ib2]}; e.zsn = V{s.t[VZS][na], s.t[VZS][nb2]};
        e.uni = V{s.t[nu][ia], s.t[nu][ib2]}; e.unn = V{s.t[nu][na], s.t[nu][nb2]};
        e.uti = V{s.t[tu][ia], s.t[tu][ib2]}; e.utn = V{s.t[tu][na], s.t[tu][nb2]};
        e.dhi = V{G[0][ga2], G[0][gb2]}; e.dhn = V{G[0][gna], G[0][gnb]};
        e.dzsi = V{G[1][ga2], G[1][gb2]}; e.dzsn = V{G[1][gna], G[1][gnb]};
        e.duni = V{G[2][ga2], G[2][gb2]}; e.dunn = V{G[2][gna], G[2][gnb]};
        e.duti = V{G[3][ga2], G[3][gb2]}; e.dutn = V{G[3][gna], G[3][gnb]};
        e.zbi = V{s.zb[za], s.zb[zb2]}; e.zbn = V{s.zb[zna], s.zb[znb]};
        if (SPLIT) {
            e.zbi = add(e.zbi, Dv);
            e.zbn = add(e.zbn, Dv);
        }
        own_sources(e);
        if constexpr (SUB) {
            const int sd = isx ? 1 : 3;  // right / top side coarser: the i-side sources
            if (subf->on[sd]) {
                e.hsi = V{subf->h[sd][2 * q], subf->h[sd][2 * q + 1]};
                e.zri = V{subf->z[sd][2 * q], subf->z[sd][2 * q + 1]};
            }
        }
        const FaceOutV<V> fe = face(e);
        if (isx) {
            const int o = p2fx(BW, 2 * q);
            st2<T>(s.fx[0], o, fe.Fh); st2<T>(s.fx[1], o, fe.Fq); st2<T>(s.fx[2], o, fe.S); st2<T>(s.fx[3], o, fe.Ft);
        } else {
            const int oa = p2fy(2 * q, BW), ob = p2fy(2 * q + 1, BW);
            s.fy[0][oa] = fe.Fh.a; s.fy[1][oa] = fe.Fq.a; s.fy[2][oa] = fe.S.a; s.fy[3][oa] = fe.Ft.a;
            s.fy[0][ob] = fe.Fh.b; s.fy[1][ob] = fe.Fq.b; s.fy[2][ob] = fe.S.b; s.fy[3][ob] = fe.Ft.b;
        }
    }
    return cdt;
}

// bndFluxGPUSideCPU (src/Boundary.cu:587-745) on the pair layouts; CORR: state n
// from the corrector's h0/u0/v0, else from the predictor's tile (which is state n).
template <class T, bool CORR, bool SPLIT = false>
__device__ __forceinline__ void boundaries2(Smem2<T>& s, const DevModel<T>& m, const StepParams<T>& p, int ib,
                                            double tbnd, int tid, T D = (T)0)
{
    if (tid >= 64) return;
    const int side = tid >> 4, t = tid & 15;
    const int k = m.bndseg[ib * 4 + side];
    if (k < 0) return;
    const SegDev sg = m.segs[k];
    if (sg.type == 1) return;
    double zsbnd = 0.0;
    if (!isnan(p.zsinit)) zsbnd = p.zsinit;
    T taper = (T)1.0;
    if (sg.n > 0) {
        if (p.bndtaper > 0.0) taper = (T)fmin((tbnd - p.inittime) / p.bndtaper, 1.0);
        zsbnd = series_at(m.seg_t + sg.off, m.seg_wl + sg.off, sg.n, tbnd, sg.sorted != 0);
    }
    const int isright = side == 0 ? -1 : side == 1 ? 1 : 0;
    const int istop = side == 2 ? 1 : side == 3 ? -1 : 0;
    int ix, iy, inx, iny;
    if (isright == 0) { ix = t; iy = istop < 0 ? 0 : BW; }
    else { iy = t; ix = isright < 0 ? 0 : BW; }
    if (isright < 0) { inx = ix + 1; iny = iy; }
    else if (isright > 0) { inx = ix - 1; iny = iy; }
    else if (istop < 0) { inx = ix; iny = iy + 1; }
    else { inx = ix; iny = iy - 1; }
    const T sign = (T)isright + (T)istop;
    float zsb = (float)zsbnd;
    zsb = (float)((double)zsb + p.zsoffset);
    auto H0 = [&](int xx, int yy) -> T { return CORR ? s.h0[p2z(xx, yy)] : s.t[VH][p2t(xx, yy)]; };
    auto U0 = [&](int xx, int yy) -> T { return CORR ? s.u0[p2z(xx, yy)] : s.t[VU][p2t(xx, yy)]; };
    auto W0 = [&](int xx, int yy) -> T { return CORR ? s.v0[p2z(xx, yy)] : s.t[VV][p2t(xx, yy)]; };
    // (split precision: beds zb + D and depths D + h'; zs is the surface either way)
    const T zsi = (SPLIT ? s.zb[hi18(ix, iy)] + D : s.zb[hi18(ix, iy)]) + H0(ix, iy);
    const T zsinside = (SPLIT ? s.zb[hi18(inx, iny)] + D : s.zb[hi18(inx, iny)]) + H0(inx, iny);
    const T hinside = SPLIT ? D + H0(inx, iny) : H0(inx, iny);
    const T uninside = isright != 0 ? U0(inx, iny) : W0(inx, iny);
    const T hface = SPLIT ? D + H0(ix, iy) : H0(ix, iy);
    const T zsX = (T)(((double)((T)zsb + (T)0.0) - 0.5 * (double)(zsi + zsinside)) * (double)taper +
                      0.5 * (double)(zsi + zsinside));
    float* qm = m.qmean + ib * 64 + side * 16 + t;
    T qmean = (T)*qm;
    T *Fh, *Fq, *Ss;
    int fi, fin;
    if (isright != 0) {
        Fh = s.fx[0]; Fq = s.fx[1]; Ss = s.fx[2];
        fi = p2fx(ix, iy); fin = p2fx(inx, iny);
    } else {
        Fh = s.fy[0]; Fq = s.fy[1]; Ss = s.fy[2];
        fi = p2fy(ix, iy); fin = p2fy(inx, iny);
    }
    T F, G, S;
    const bool lowside = isright < 0 || istop < 0;
    if (lowside) { F = Fh[fi]; G = Fq[fi]; S = Ss[fin]; }
    else { F = Fh[fi]; G = Ss[fi]; S = Fq[fin]; }
    const T factime = M<T>::fmin_((T)(p.dtparam / p.bndfiltertime), (T)1.0);
    const T facrel = (T)1.0 - M<T>::fmin_((T)(p.dtparam / p.bndrelaxtime), (T)1.0);
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

// updateEVCPU (src/Advection.cu:160-254), Cartesian, for the own pair.
template <class T>
__device__ __forceinline__ void divergence2(const Smem2<T>& s, const StepParams<T>& p, T cmdinv, int x, int py, V2<T> hi,
                                            V2<T> uui, V2<T> vvi, V2<T>& dh, V2<T>& dhu, V2<T>& dhv)
{
    using V = V2<T>;
    const int y = 2 * py;
    const int fi = p2fx(x, y), fr = fi + 2;
    const int gi = p2fy(x, y), gt2 = p2fy(x, y + 2);
    const V Fhu_i = ld2<T>(s.fx[0], fi), Fhu_r = ld2<T>(s.fx[0], fr);
    const V Fqux_i = ld2<T>(s.fx[1], fi), Su_r = ld2<T>(s.fx[2], fr);
    const V Fqvx_i = ld2<T>(s.fx[3], fi), Fqvx_r = ld2<T>(s.fx[3], fr);
    const V Fhv_i = ld2<T>(s.fy[0], gi), Fqvy_i = ld2<T>(s.fy[1], gi);
    const V Sv_i = ld2<T>(s.fy[2], gi), Fquy_i = ld2<T>(s.fy[3], gi);
    const V Fhv_t{Fhv_i.b, s.fy[0][gt2]};
    const V Sv_t{Sv_i.b, s.fy[2][gt2]};
    const V Fquy_t{Fquy_i.b, s.fy[3][gt2]};
    const V cm{cmdinv, cmdinv}, fc{p.fc, p.fc};
    dh = mul(mul(V{(T)-1.0, (T)-1.0}, sub(add(sub(Fhu_r, Fhu_i), Fhv_t), Fhv_i)), cm);
    // (the Coriolis products fused into the sums; -fc h u is -(fc h u) exactly)
    const V nfc{-p.fc, -p.fc};
    dhu = mad(sub(sub(add(Fqux_i, Fquy_i), Su_r), Fquy_t), cm, mul(mul(fc, hi), vvi));
    dhv = mad(sub(sub(add(Fqvy_i, Fqvx_i), Sv_t), Fqvx_r), cm, mul(mul(nfc, hi), uui));
}

template <class T> __device__ __forceinline__ V2<T> finite_dt2(V2<T> h, V2<T> u, V2<T> v, V2<T> cdt)
{
#if BGF_FAST
    if constexpr (sizeof(T) == 4) {
        // one test per cell: the sum is finite exactly when h, u and v are (a NaN or an
        // infinity carries through it; finite states are far below the float range)
        const V2<T> t = add(add(h, u), v);
        return V2<T>{isfinite(t.a) ? cdt.a : (T)0, isfinite(t.b) ? cdt.b : (T)0};
    }
#endif
    return V2<T>{isfinite(h.a) && isfinite(u.a) && isfinite(v.a) ? cdt.a : (T)0,
                 isfinite(h.b) && isfinite(u.b) && isfinite(v.b) ? cdt.b : (T)0};
}

// ---------------------------------------------------------------- kernels

template <class T, int ENGINE, bool POOL, bool SPLIT = false>
__global__ void __launch_bounds__(NT2, sizeof(T) == 4 ? 7 : 3) flux2_kernel(DevModel<T> m, StepParams<T> p0, int parity)
{
    using V = V2<T>;
    extern __shared__ __align__(16) unsigned char smem_raw2[];
    Smem2<T>& s = *reinterpret_cast<Smem2<T>*>(smem_raw2);
    const int tid = threadIdx.x;
    const int w4 = tid >> 5, lane = tid & 31;
    const int x = lane & 15;
    const int py = (w4 & 1) + 4 * (w4 >> 1) + 2 * (lane >> 4);
    const int y = 2 * py;
    for (int w = blockIdx.x; w < m.nblk; w += gridDim.x) {
        const int ib = m.regular_nbx > 0 ? w : m.active[w];
        // the bed tile, the own pair's bed and the bed gradients do not depend on the
        // time slot: their loads are in flight while it arrives
        const T* zbt = m.zb + (size_t)ib * 324;
        load_bed2<T>(s, zbt, tid);
        const BedGrad<T> bg = load_bedgrad<T, ENGINE>(m, ib, tid, x, y);
        const V zbo{zbt[hi18(x, y)], zbt[hi18(x, y + 1)]};
        // the ring cell's source lookup and its bed too
        int rx, ry, sb, sx, sy;
        ring_src2<T>(m, ib, tid, rx, ry, sb, sx, sy);
        const bool ring2 = rx < -1 || rx > BW || ry < -1 || ry > BW;
        const T zr = ring2 ? m.zb[(size_t)sb * 324 + hi18(sx, sy)] : zbt[hi18(rx, ry)];
        const int sc = POOL ? m.scen[ib] : 0;
        const TimeState ts = m.time[2 * sc + parity];
        if (!step_live(ts)) {
            bed_wait();  // the next block's copies go to the same shared words
            continue;
        }
        const StepParams<T>& p = params_ref<POOL>(m, p0, sc);
        const T delta = calcres<T>(p.delta0, m.level[ib]);
        const T D = SPLIT ? m.datum[ib] : (T)0;  // split precision: the block's datum
        const int cur = ts.cur;
        const T* H = m.h[cur];
        const T* U = m.u[cur];
        const T* Vv = m.v[cur];
        V c[4];
        const size_t g0 = (size_t)ib * 256 + y * 16 + x;
        c[VH] = V{H[g0], H[g0 + 16]};
        c[VU] = V{U[g0], U[g0 + 16]};
        c[VV] = V{Vv[g0], Vv[g0 + 16]};
        c[VZS] = SPLIT ? add(add(zbo, V{D, D}), c[VH]) : add(zbo, c[VH]);
        {
            const size_t gr = (size_t)sb * 256 + sy * 16 + sx;
            T hv = H[gr];
            // split precision: a neighbour's deviation in this block's datum (datums are
            // whole metres, so the difference is exact)
            if (SPLIT && sb != ib) hv = hv + (m.datum[sb] - D);
            const int o = p2t(rx, ry);
            s.t[VH][o] = hv; s.t[VU][o] = U[gr]; s.t[VV][o] = Vv[gr]; s.t[VZS][o] = (SPLIT ? zr + D : zr) + hv;
        }
        const int ct = p2t(x, y);
#pragma unroll
        for (int k = 0; k < 4; k++) st2<T>(s.t[k], ct, c[k]);
        bed_wait();
        __syncthreads();
        V xm[4], gxo[4], gyo[4];
        T ym[4];
        gradients2<T, ENGINE, SPLIT>(s, bg, p.theta, delta, tid, x, py, c, xm, ym, gxo, gyo, D);
        __syncthreads();
        V cdt = faces2<T, ENGINE, SPLIT>(s, p, delta, tid, x, py, c, xm, ym, gxo, gyo, D);
        cdt = finite_dt2<T>(c[VH], c[VU], c[VV], cdt);
        T v = cdt.b < cdt.a ? cdt.b : cdt.a;
        for (int o = 16; o > 0; o >>= 1) {
            const T q = __shfl_xor_sync(0xffffffffu, v, o);
            v = q < v ? q : v;
        }
        if (lane == 0) s.red[w4] = v;
        __syncthreads();
        // boundary segments (FlowbndFlux) after the dt, at t + dt_prev / 2 as FlowCPU does
        if (block_has_segments<T>(m, ib)) {
            boundaries2<T, false, SPLIT>(s, m, p, ib, ts.totaltime + ts.dt * 0.5, tid, D);
            __syncthreads();
        }
        if (tid == 0) {
            T b = s.red[0];
            for (int k = 1; k < NT2 / 32; k++) b = s.red[k] < b ? s.red[k] : b;
            atomicMin(&m.dtmin[2 * sc + parity], dt_bits(b));
        }
        V dh, dhu, dhv;
        divergence2<T>(s, p, (T)1.0 / ((T)1.0 * delta), x, py, SPLIT ? add(V{D, D}, c[VH]) : c[VH], c[VU], c[VV], dh,
                       dhu, dhv);
        m.dh[g0] = dh.a; m.dh[g0 + 16] = dh.b;
        m.dhu[g0] = dhu.a; m.dhu[g0 + 16] = dhu.b;
        m.dhv[g0] = dhv.a; m.dhv[g0 + 16] = dhv.b;
        if (w + (int)gridDim.x < m.nblk) __syncthreads();  // the tile is reused by the next block
    }
}

template <class T, int ENGINE, bool POOL, bool SPLIT = false>
__global__ void __launch_bounds__(NT2, sizeof(T) == 4 ? 7 : 3) update2_kernel(DevModel<T> m, StepParams<T> p0, int parity)
{
    using V = V2<T>;
    extern __shared__ __align__(16) unsigned char smem_raw2[];
    Smem2<T>& s = *reinterpret_cast<Smem2<T>*>(smem_raw2);
    const int tid = threadIdx.x;
    const int w4 = tid >> 5, lane = tid & 31;
    const int x = lane & 15;
    const int py = (w4 & 1) + 4 * (w4 >> 1) + 2 * (lane >> 4);
    const int y = 2 * py;
    for (int w = blockIdx.x; w < m.nblk; w += gridDim.x) {
        const int ib = m.regular_nbx > 0 ? w : m.active[w];
        // the bed, the predictor's tendencies and the ring cell's source do not depend
        // on the time slot (only the state buffer does): their loads are in flight
        // while it arrives
        const T* zbt = m.zb + (size_t)ib * 324;
        load_bed2<T>(s, zbt, tid);
        const BedGrad<T> bg = load_bedgrad<T, ENGINE>(m, ib, tid, x, y);
        const V zbo{zbt[hi18(x, y)], zbt[hi18(x, y + 1)]};
        int rx, ry, sb, sx, sy;
        ring_src2<T>(m, ib, tid, rx, ry, sb, sx, sy);
        const size_t g0 = (size_t)ib * 256 + y * 16 + x;
        V ddh{m.dh[g0], m.dh[g0 + 16]};
        const V ddhu{m.dhu[g0], m.dhu[g0 + 16]}, ddhv{m.dhv[g0], m.dhv[g0 + 16]};
        const size_t gr = (size_t)sb * 256 + sy * 16 + sx;
        T rdh = m.dh[gr];
        const T rdhu = m.dhu[gr], rdhv = m.dhv[gr];
        const bool ring2 = rx < -1 || rx > BW || ry < -1 || ry > BW;
        const T rzb = ring2 ? m.zb[(size_t)sb * 324 + hi18(sx, sy)] : zbt[hi18(rx, ry)];
        const int sc = POOL ? m.scen[ib] : 0;
        // the predictor's dt minimum (read by thread 0) does not depend on it either
        const unsigned long long dtbits = tid == 0 ? m.dtmin[2 * sc + parity] : 0ull;
        const TimeState ts = m.time[2 * sc + parity];
        const bool lead = POOL ? m.lead[ib] != 0 : w == 0;
        if (!step_live(ts)) {
            bed_wait();  // the next block's copies go to the same shared words
            if (lead && tid == 0) {
                TimeState nt = ts;
                nt.done = 1;
                m.time[2 * sc + (parity ^ 1)] = nt;
            }
            continue;
        }
        const StepParams<T>& p = params_ref<POOL>(m, p0, sc);
        if (tid == 0) {
            const T dt0 = step_dt<T>(ts, dtbits);
            s.dtv = dt0;
            if (p.has_rain && !p.rain_map) {
                // uniform rain (AddrainforcingImplicitCPU, src/Updateforcing.cu:530-580): the
                // rate at the start of the step and its depth over the step, the same for
                // every cell of the scenario, once per block instead of once per thread
                const T r = (T)series_at(m.rain_t + p.rain_off, m.rain_r + p.rain_off, p.rain_n, ts.totaltime,
                                         p.rain_sorted != 0);
                s.rainv = M<T>::fmax_(dv(dv(r, (T)1000.0), (T)3600.0) * dt0, (T)0.0);
            }
        }
        const T delta = calcres<T>(p.delta0, m.level[ib]);
        const T D = SPLIT ? m.datum[ib] : (T)0;  // split precision: the block's datum
        const V Dv{D, D};
        const int cur = ts.cur;
        const T* H = m.h[cur];
        const T* U = m.u[cur];
        const T* Vv = m.v[cur];
        const V hold{H[g0], H[g0 + 16]}, uold{U[g0], U[g0 + 16]}, vold{Vv[g0], Vv[g0 + 16]};
        const T rh = H[gr], ru = U[gr], rv = Vv[gr];
        bed_wait();
        __syncthreads();  // s.dtv, s.zb
        const T dt = s.dtv;
        const double dtd = (double)dt;
        const T halfdt = dt * (T)0.5;
        if (p.nriver > 0) {
            // the predictor's river source of the source cells (AddRiverForcing after updateEV)
            ddh = V{add_rivers<T>(m, p, ib, x, y, ddh.a, ts.totaltime), add_rivers<T>(m, p, ib, x, y + 1, ddh.b, ts.totaltime)};
            rdh = add_rivers<T>(m, p, sb, sx, sy, rdh, ts.totaltime);
        }
        V c[4];
        if constexpr (SPLIT) {
            advance_split_v<T>(halfdt, p.eps, p.forcemass != 0, Dv, hold, uold, vold, ddh, ddhu, ddhv, c[VH], c[VU],
                               c[VV]);
            c[VZS] = add(add(zbo, Dv), c[VH]);
        } else {
            advance_v<V>(halfdt, p.eps, p.eps_d, p.forcemass != 0, hold, uold, vold, ddh, ddhu, ddhv, c[VH], c[VU],
                         c[VV]);
            c[VZS] = add(zbo, c[VH]);
        }
        {
            T ho, uo, vo, rh0 = rh;
            if constexpr (SPLIT) {
                // the source cell's half step in its own datum, then both states in this
                // block's datum (whole metres: the difference is exact)
                const T Ds = sb == ib ? D : m.datum[sb];
                advance_split<T>(halfdt, p.eps, p.forcemass != 0, Ds, rh, ru, rv, rdh, rdhu, rdhv, ho, uo, vo);
                if (sb != ib) {
                    rh0 = rh + (m.datum[sb] - D);
                    ho = ho + (m.datum[sb] - D);
                }
            } else {
                advance_v<T>(halfdt, p.eps, p.eps_d, p.forcemass != 0, rh, ru, rv, rdh, rdhu, rdhv, ho, uo, vo);
            }
            const int o = p2t(rx, ry);
            s.t[VH][o] = ho; s.t[VU][o] = uo; s.t[VV][o] = vo; s.t[VZS][o] = (SPLIT ? rzb + D : rzb) + ho;
            if (!ring2) {
                const int o2 = p2z(rx, ry);
                s.h0[o2] = rh0; s.u0[o2] = ru; s.v0[o2] = rv;
            }
        }
        const int ct = p2t(x, y);
#pragma unroll
        for (int k = 0; k < 4; k++) st2<T>(s.t[k], ct, c[k]);
        {
            const int o2 = p2z(x, y);
            st2<T>(s.h0, o2, hold); st2<T>(s.u0, o2, uold); st2<T>(s.v0, o2, vold);
        }
        __syncthreads();
        V xm[4], gxo[4], gyo[4];
        T ym[4];
        gradients2<T, ENGINE, SPLIT>(s, bg, p.theta, delta, tid, x, py, c, xm, ym, gxo, gyo, D);
        __syncthreads();
        (void)faces2<T, ENGINE, SPLIT>(s, p, delta, tid, x, py, c, xm, ym, gxo, gyo, D);
        __syncthreads();
        if (block_has_segments<T>(m, ib)) {  // interior blocks skip the step and its barrier
            boundaries2<T, true, SPLIT>(s, m, p, ib, ts.totaltime + dtd, tid, D);
            __syncthreads();
        }
        V dh, dhu, dhv;
        divergence2<T>(s, p, (T)1.0 / ((T)1.0 * delta), x, py, SPLIT ? add(Dv, c[VH]) : c[VH], c[VU], c[VV], dh, dhu,
                       dhv);
        if (p.nriver > 0)
            dh = V{add_rivers<T>(m, p, ib, x, y, dh.a, ts.totaltime), add_rivers<T>(m, p, ib, x, y + 1, dh.b, ts.totaltime)};
        // full step from state n (AdvkernelCPU with evolv), then friction on the result;
        // state n comes back from its shared tile (fewer registers held over the faces)
        V ho, uo, vo;
        {
            const int o2 = p2z(x, y);
            const V hn = ld2<T>(s.h0, o2), un = ld2<T>(s.u0, o2), vn = ld2<T>(s.v0, o2);
            if constexpr (SPLIT) advance_split_v<T>(dt, p.eps, p.forcemass != 0, Dv, hn, un, vn, dh, dhu, dhv, ho, uo, vo);
            else advance_v<V>(dt, p.eps, p.eps_d, p.forcemass != 0, hn, un, vn, dh, dhu, dhv, ho, uo, vo);
        }
        const V cfv = p.has_cf ? V{m.cf[g0], m.cf[g0 + 16]} : V{p.cf, p.cf};
        // (split precision: friction on the full depth; the deviation is not changed by it)
        friction_v<T>(p.frictionmodel, p.g, p.eps, dt, cfv, SPLIT ? add(Dv, ho) : ho, uo, vo);
        if (p.has_rain) {
            // AddrainforcingImplicitCPU (src/Updateforcing.cu:530-580): the rain rate at
            // the start of the step, uniform or gridded
            V Rainhh;
            const V mask = m.rainmask ? V{(T)m.rainmask[g0], (T)m.rainmask[g0 + 16]} : V{(T)1, (T)1};
            if (p.rain_map) {
                const T xc = (T)p.xo_d + (T)m.bxo[ib] + (T)x * delta;
                const T yc0 = (T)p.yo_d + (T)m.byo[ib] + (T)y * delta;
                const T yc1 = (T)p.yo_d + (T)m.byo[ib] + (T)(y + 1) * delta;
                Rainhh = V{rain_map_at<T>(m.rmap, xc, yc0, ts.totaltime), rain_map_at<T>(m.rmap, xc, yc1, ts.totaltime)};
                const T rs = (T)dtd;
                const V rr = dv(dv(Rainhh, V{(T)1000.0, (T)1000.0}), V{(T)3600.0, (T)3600.0});
                Rainhh = mul(vmax(mul(rr, V{rs, rs}), V{(T)0.0, (T)0.0}), mask);
            } else {
                Rainhh = mul(V{s.rainv, s.rainv}, mask);  // (the block's uniform depth, above)
            }
            const V hi = SPLIT ? add(Dv, ho) : ho;
            const V qvol = dv(hi, add(hi, Rainhh));
            ho = add(ho, Rainhh);
            const M2 wet{(double)hi.a > p.eps_d, (double)hi.b > p.eps_d};
            uo = sel(wet, mul(uo, qvol), uo);
            vo = sel(wet, mul(vo, qvol), vo);
        }
        const int nxt = cur ^ 1;
        m.h[nxt][g0] = ho.a; m.h[nxt][g0 + 16] = ho.b;
        m.u[nxt][g0] = uo.a; m.u[nxt][g0 + 16] = uo.b;
        m.v[nxt][g0] = vo.a; m.v[nxt][g0 + 16] = vo.b;
        if (m.hmax) {
            const V hf = SPLIT ? add(Dv, ho) : ho;  // the full depth
            m.hmax[g0] = hf.a > m.hmax[g0] ? hf.a : m.hmax[g0];
            m.hmax[g0 + 16] = hf.b > m.hmax[g0 + 16] ? hf.b : m.hmax[g0 + 16];
        }
        if (lead && tid == 0)
            m.time[2 * sc + (parity ^ 1)] = next_time_state<T>(ts, p, dtd, nxt, m.dtmin + 2 * sc, parity);
        if (w + (int)gridDim.x < m.nblk) __syncthreads();  // the tile is reused by the next block
    }
}
