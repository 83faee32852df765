// Device numerics of the flow step: limiter, Riemann solvers, boundary fluxes,
// advance, friction.  Each function follows the reference routine named in its
// comment with the same floating-point operation order, so that a build with
// --fmad=false reproduces the reference CPU results bit for bit (float sqrt and
// division are IEEE-rounded on sm_100a).  T is float or double.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace bgf {

template <class T> struct M;  // math shims keyed on precision
template <> struct M<float> {
    static __device__ __forceinline__ float fmax_(float a, float b) { return fmaxf(a, b); }
    static __device__ __forceinline__ float fmin_(float a, float b) { return fminf(a, b); }
    static __device__ __forceinline__ float fabs_(float a) { return fabsf(a); }
    static __device__ __forceinline__ float sqrt_(float a) { return sqrtf(a); }
    static __device__ __forceinline__ float cbrt_(float a) { return cbrtf(a); }
    static __device__ __forceinline__ float log_(float a) { return logf(a); }
    static __device__ __forceinline__ float epsi() { return nextafterf(1.0f, 2.0f) - 1.0f; }
};
template <> struct M<double> {
    static __device__ __forceinline__ double fmax_(double a, double b) { return fmax(a, b); }
    static __device__ __forceinline__ double fmin_(double a, double b) { return fmin(a, b); }
    static __device__ __forceinline__ double fabs_(double a) { return fabs(a); }
    static __device__ __forceinline__ double sqrt_(double a) { return sqrt(a); }
    static __device__ __forceinline__ double cbrt_(double a) { return cbrt(a); }
    static __device__ __forceinline__ double log_(double a) { return log(a); }
    static __device__ __forceinline__ double epsi() { return nextafter(1.0, 2.0) - 1.0; }
};

// 1 / (nextafter(1, 2) - 1): the "dry" time step of the reference sweeps
template <class T> __device__ __forceinline__ T inv_epsi();
template <> __device__ __forceinline__ float inv_epsi<float>() { return 8388608.0f; }
template <> __device__ __forceinline__ double inv_epsi<double>() { return 4503599627370496.0; }

// calcres (src/Util_CPU.cu:193-198)
template <class T> __device__ __forceinline__ T calcres(T dx, int level)
{
    return level < 0 ? dx * (T)(1 << (-level)) : dx / (T)(1 << level);
}

// minmod2 (src/Util_CPU.cu:243-263)
template <class T> __device__ __forceinline__ T minmod2(T theta, T s0, T s1, T s2)
{
    if (s0 < s1 && s1 < s2) {
        T d1 = theta * (s1 - s0);
        T d2 = (s2 - s0) * (T)0.5;  // == (s2 - s0) / 2, exactly
        T d3 = theta * (s2 - s1);
        if (d2 < d1) d1 = d2;
        return M<T>::fmin_(d1, d3);
    }
    if (s0 > s1 && s1 > s2) {
        T d1 = theta * (s1 - s0), d2 = (s2 - s0) * (T)0.5, d3 = theta * (s2 - s1);
        if (d2 > d1) d1 = d2;
        return M<T>::fmax_(d1, d3);
    }
    return (T)0.0;
}

template <class T> __device__ __forceinline__ T sq(T a) { return a * a; }

// KurgSolver (src/Kurganov.cu:1865-1911), Cartesian metric (cm = fm = 1).
template <class T>
__device__ __forceinline__ T kurg_solver(T g, T delta, T epsi, T CFL, T hp, T hm, T up, T um, T& fh, T& fu)
{
    T cp = M<T>::sqrt_(g * hp);
    T cmo = M<T>::sqrt_(g * hm);
    T ap = M<T>::fmax_(M<T>::fmax_(up + cp, um + cmo), (T)0.0);
    T am = M<T>::fmin_(M<T>::fmin_(up - cp, um - cmo), (T)0.0);
    T a = M<T>::fmax_(ap, -am);
    if (a > epsi) {
        T ad = (T)1.0 / (ap - am);
        T qm = hm * um;
        T qp = hp * up;
        T ga = g * (T)0.5;
        T apm = ap * am;
        fh = (ap * qm - am * qp + apm * (hp - hm)) * ad;
        fu = (ap * (qm * um + ga * (hm * hm)) - am * (qp * up + ga * (hp * hp)) + apm * (qp - qm)) * ad;
        return CFL * delta / a;  // dlt = delta * cm / fm with cm = fm = 1
    }
    fh = (T)0.0;
    fu = (T)0.0;
    return inv_epsi<T>();
}

// hllc (src/Reimann.cu:838-877), Cartesian metric.
template <class T>
__device__ __forceinline__ T hllc(T g, T delta, T epsi, T CFL, T hm, T hp, T um, T up, T& fh, T& fq)
{
    T cmo = M<T>::sqrt_(g * hm);
    T cp = M<T>::sqrt_(g * hp);
    T ustar = (um + up) * (T)0.5 + cmo - cp;  // halving and quartering are exact
    T cstar = (cmo + cp) * (T)0.5 + (um - up) * (T)0.25;
    T SL = hm == (T)0. ? up - (T)2. * cp : M<T>::fmin_(um - cmo, ustar - cstar);
    T SR = hp == (T)0. ? um + (T)2. * cmo : M<T>::fmax_(up + cp, ustar + cstar);
    if ((T)0. <= SL) {
        fh = um * hm;
        fq = hm * (um * um + g * hm * (T)0.5);
    } else if ((T)0. >= SR) {
        fh = up * hp;
        fq = hp * (up * up + g * hp * (T)0.5);
    } else {
        T fhm = um * hm;
        T fum = hm * (um * um + g * hm * (T)0.5);
        T fhp = up * hp;
        T fup = hp * (up * up + g * hp * (T)0.5);
        fh = (SR * fhm - SL * fhp + SL * SR * (hp - hm)) / (SR - SL);
        fq = (SR * fum - SL * fup + SL * SR * (hp * up - hm * um)) / (SR - SL);
    }
    double a = (double)M<T>::fmax_(M<T>::fabs_(SL), M<T>::fabs_(SR));
    if (a > (double)epsi) {
        return CFL * delta / (T)a;
    }
    return inv_epsi<T>();
}

// Result of one face of the X or Y sweep (reference FluxP members for that face).
template <class T> struct Face {
    T Fh, Fq, S, Ft, dt;
    bool wet;
};

// One face between cell n (minus side) and cell i (plus side).  Arguments are the
// state and limited gradients along the sweep direction; ut/dut are the tangential
// velocity and its gradient.  Restates updateKurgXCPU/YCPU (src/Kurganov.cu:474-641,
// 1404-1547) for ENGINE 2 and UpdateButtingerXCPU/YCPU (src/Reimann.cu:223-426,
// 620-818) for ENGINE 1 on faces without a coarse/fine substitution.
template <class T, int ENGINE> struct FaceIn {
    T hi, hn, zsi, zsn, uni, unn, uti, utn;
    T dhi, dhn, dzsi, dzsn, duni, dunn, duti, dutn;
    T zbi, zbn;  // engine 1
    T hsi, zsrci, hsn, zsrcn;  // source-term depth/bed (substituted at coarse/fine faces)
};

template <class T, int ENGINE>
__device__ __forceinline__ Face<T> face_flux(const FaceIn<T, ENGINE>& f, T g, T CFL, T epsi, T eps, T delta)
{
    Face<T> r;
    if (f.hi > eps || f.hn > eps) {
        T dx = delta * (T)0.5;
        T ga = g * (T)0.5;
        T fh, fu, fv, sl, sr;
        if (ENGINE == 2) {
            T zi = f.zsi - f.hi;
            T zl = zi - dx * (f.dzsi - f.dhi);
            T zn = f.zsn - f.hn;
            T zr = zn + dx * (f.dzsn - f.dhn);
            T zlr = M<T>::fmax_(zl, zr);
            T hl = f.hi - dx * f.dhi;
            T up = f.uni - dx * f.duni;
            T hp = M<T>::fmax_((T)0.0, hl + zl - zlr);
            T hr = f.hn + dx * f.dhn;
            T um = f.unn + dx * f.dunn;
            T hm = M<T>::fmax_((T)0.0, hr + zr - zlr);
            r.dt = kurg_solver<T>(g, delta, epsi, CFL, hp, hm, up, um, fh, fu);
            if (fh > (T)0.0) fv = (f.utn + dx * f.dutn) * fh;
            else fv = (f.uti - dx * f.duti) * fh;
            // hsi/zsrci (hsn/zsrcn) are hi/zi (hn/zn) except at coarse/fine faces, where
            // the reference substitutes the finer neighbour's cell (src/Kurganov.cu:602-616)
            sl = ga * (sq(hp) - sq(hl) + (hl + f.hsi) * (f.zsrci - zl));
            sr = ga * (sq(hm) - sq(hr) + (hr + f.hsn) * (f.zsrcn - zr));
        } else {
            T hr = f.hi - dx * f.dhi;
            T hl = f.hn + dx * f.dhn;
            T etar = f.zsi - dx * f.dzsi;
            T etal = f.zsn + dx * f.dzsn;
            T zr = etar - hr;
            T zl = etal - hl;
            T zA = M<T>::fmax_(zr, zl);
            T zCN = M<T>::fmin_(zA, M<T>::fmin_(etal, etar));
            T hCNr = M<T>::fmax_((T)0.0, M<T>::fmin_(etar - zCN, hr));
            T hCNl = M<T>::fmax_((T)0.0, M<T>::fmin_(etal - zCN, hl));
            T ul, ur, vl, vr;
            if (f.hi > eps) {
                ur = f.uni - ((T)1.0 + dx * f.dhi / f.hi) * dx * f.duni;
                vr = f.uti - ((T)1.0 + dx * f.dhi / f.hi) * dx * f.duti;
            } else {
                ur = f.uni - dx * f.duni;
                vr = f.uti - dx * f.duti;
            }
            if (f.hn > eps) {
                ul = f.unn + ((T)1.0 - dx * f.dhn / f.hn) * dx * f.dunn;
                vl = f.utn + ((T)1.0 - dx * f.dhn / f.hn) * dx * f.dutn;
            } else {
                ul = f.unn + dx * f.dunn;
                vl = f.utn + dx * f.dutn;
            }
            r.dt = hllc<T>(g, delta, epsi, CFL, hCNl, hCNr, ul, ur, fh, fu);
            fv = (fh > (T)0. ? vl : vr) * fh;
            sl = ga * (f.hsi + hCNr) * (f.zsrci - zCN);
            sr = ga * (hCNl + f.hsn) * (f.zsrcn - zCN);
        }
        r.Fh = fh;
        r.Fq = fu - sl;
        r.S = fu - sr;
        r.Ft = fv;
        r.wet = true;
    } else {
        r.dt = inv_epsi<T>();
        r.Fh = (T)0.0;
        r.Fq = (T)0.0;
        r.S = (T)0.0;
        r.Ft = (T)0.0;
        r.wet = false;
    }
    return r;
}

// Wet-slope reset of one surface gradient (WetsloperesetCPU and the four halo
// variants, src/Gradients.cu:1067-1128, 1399-2580).
template <class T>
__device__ __forceinline__ T wetslope(T delta, T zsi, T hi, T zsm, T zsp, T dzs, T dh, T dzb)
{
    if (sq(dzs) > sq(dzb)) {
        T mzs = zsi - hi - delta * (T)0.5 * (dzs - dh);
        T pzs = zsi - hi + delta * (T)0.5 * (dzs - dh);
        if (mzs > zsm || pzs > zsp) return dh + dzb;
    }
    return dzs;
}

// AdvkernelCPU / AdvkernelGPU (src/Advection.cu:272-385).  The depth limiter is
// evaluated in double because max(float, double) / min(float, double) resolve to
// the double overloads in the reference build.
template <class T>
__device__ __forceinline__ void advance(T dt, T eps, double eps_d, bool forcemass, T hold, T uold, T vold, T dhi,
                                        T dhui, T dhvi, T& ho, T& uo, T& vo)
{
#if BGF_FAST
    // fast build: the limiter in the state precision
    T edt = forcemass ? dt : dhi >= (T)0.0 ? dt : M<T>::fmin_(dt, M<T>::fmax_(hold, (T)eps_d) / M<T>::fabs_(dhi));
#else
    T edt = forcemass ? dt : dhi >= (T)0.0 ? dt : (T)fmin((double)dt, fmax((double)hold, eps_d) / (double)M<T>::fabs_(dhi));
#endif
    ho = hold + edt * dhi;
    if (ho > eps) {
        uo = (hold * uold + edt * dhui) / ho;
        vo = (hold * vold + edt * dhvi) / ho;
    } else {
        uo = (T)0.0;
        vo = (T)0.0;
    }
}

// smartfriction (src/Friction.cu:317-334)
template <class T> __device__ __forceinline__ T smartfriction(T hi, T zo)
{
    T cfi;
    T ee = (T)2.71828182845905;
    T Hbar = hi / zo;
    if (Hbar <= ee) cfi = (T)1.0 / ((T)0.46 * Hbar);
    else cfi = (T)1.0 / ((T)2.5 * (M<T>::log_(Hbar) - (T)1.0 + (T)1.359 / Hbar));
    return cfi * cfi;
}

// bottomfrictionGPU / CPU (src/Friction.cu:17-143), manningfriction (:347-351)
template <class T>
__device__ __forceinline__ void bottom_friction(int model, T g, T eps, T dt, T cfv, T hi, T& ui, T& vi)
{
    if (hi > eps) {
        T normu = M<T>::sqrt_(ui * ui + vi * vi);
        T cfi = (T)0.0;
        if (model == 0) cfi = cfv;
        else if (model == 1) cfi = smartfriction<T>(hi, cfv);
        else if (model == -1) cfi = g * cfv * cfv / M<T>::cbrt_(hi);
        T tb = cfi * normu / hi * dt;
        ui = ui / ((T)1.0 + tb);
        vi = vi / ((T)1.0 + tb);
    }
}

// ABS1DQ / Dirichlet1Q (src/Boundary.cu:1943-2036)
template <class T>
__device__ __forceinline__ void abs1dq(T g, T sign, T factime, T facrel, T zs, T zsbnd, T h, T& qmean, T& q)
{
    qmean = h < (T)0.01 ? (T)0.0 : factime * q + facrel * ((T)1.0 - factime) * qmean;
    T zn = M<T>::fmax_(zsbnd, (zs - h));
    T hn = M<T>::fmax_(h, (T)0.0001);
    T un = sign * M<T>::sqrt_(g / hn) * (zs - zn);
    q = un * hn + qmean;
}

template <class T>
__device__ __forceinline__ void dirichlet1q(T g, T sign, T zsbnd, T zsinside, T hinside, T uninside, T& q)
{
    T zbinside = zsinside - hinside;
    T un = sign * (T)2.0 *
               (M<T>::sqrt_(g * M<T>::fmax_(hinside, (T)0.0)) - M<T>::sqrt_(g * M<T>::fmax_(zsbnd - zbinside, (T)0.0))) +
           uninside;
    q = un * hinside;
}

}  // namespace bgf
