// Split-precision face fluxes for deep water.
//
// In FP32, a 4000 m deep cell stores h with a resolution of 2.4e-4 m, and the
// free surface zs = zb + h, the hydrostatic reconstructions and the pressure
// terms g h^2 / 2 (about 8e7 m^3/s^2) all cancel catastrophically: tsunami
// amplitudes of centimetres drift by millimetres within a few hundred steps.
// In split mode every block carries a datum depth D (an integer number of metres,
// exact in FP32, kept in FP64 on the host) and the state stores the deviation
// h' = h - D.  Inside a block's tile all depths are deviations from that block's
// datum, so
//   * surface and bed reconstructions use zs (datum-free) and z' = zs - h'
//     (= zb + D), both small numbers;
//   * depth differences (gradients, hp - hm, hp^2 - hl^2 = (hp' - hl')(hp + hl))
//     are formed from deviations;
//   * the momentum fluxes are returned shifted by the datum's hydrostatic
//     pressure, F' = F - g D^2 / 2: the Riemann solvers combine the two states'
//     fluxes with weights that sum to one, so each state's pressure g h^2 / 2 is
//     replaced by g h' (2D + h') / 2.  The shift is the same for every face a
//     block evaluates (all with its own datum) and cancels exactly in its flux
//     divergence; a dry face carries the shift alone.
// Full depths D + h' (wave speeds, velocities, wet tests, friction) need only
// relative precision.  No counterpart in the reference.
#pragma once

#include "bgf_numerics.cuh"

namespace bgf {

// One face, split mode: the FaceIn depths hi, hn are deviations from D; zsi, zsn
// surface elevations; zbi, zbn beds as deviations z' = zb + D (engine 1).
template <class T, int ENGINE>
__device__ __forceinline__ Face<T> face_flux_split(const FaceIn<T, ENGINE>& f, T D, T g, T CFL, T epsi, T eps, T delta)
{
    Face<T> r;
    const T ga = g * (T)0.5;
    const T Hi = D + f.hi, Hn = D + f.hn;  // full depths
    if (Hi > eps || Hn > eps) {
        const T dx = delta * (T)0.5;
        T fh, fu, fv, sl, sr;
        if (ENGINE == 2) {
            const T zi = f.zsi - f.hi;  // bed deviations
            const T zl = zi - dx * (f.dzsi - f.dhi);
            const T zn = f.zsn - f.hn;
            const T zr = zn + dx * (f.dzsn - f.dhn);
            const T zlr = M<T>::fmax_(zl, zr);
            const T hl = f.hi - dx * f.dhi;
            const T up = f.uni - dx * f.duni;
            const T hp = M<T>::fmax_(-D, hl + zl - zlr);
            const T hr = f.hn + dx * f.dhn;
            const T um = f.unn + dx * f.dunn;
            const T hm = M<T>::fmax_(-D, hr + zr - zlr);
            const T Hp = D + hp, Hm = D + hm, Hl = D + hl, Hr = D + hr;
            const T cp = M<T>::sqrt_(g * Hp), cmo = M<T>::sqrt_(g * Hm);
            const T ap = M<T>::fmax_(M<T>::fmax_(up + cp, um + cmo), (T)0.0);
            const T am = M<T>::fmin_(M<T>::fmin_(up - cp, um - cmo), (T)0.0);
            const T a = M<T>::fmax_(ap, -am);
            if (a > epsi) {
                const T ad = (T)1.0 / (ap - am);
                const T qm = Hm * um, qp = Hp * up, apm = ap * am;
                const T pm = ga * hm * ((T)2.0 * D + hm), pp = ga * hp * ((T)2.0 * D + hp);
                fh = (ap * qm - am * qp + apm * (hp - hm)) * ad;
                fu = (ap * (qm * um + pm) - am * (qp * up + pp) + apm * (qp - qm)) * ad;
                r.dt = CFL * delta / a;
            } else {
                fh = (T)0.0;
                fu = -ga * D * D;
                r.dt = inv_epsi<T>();
            }
            if (fh > (T)0.0) fv = (f.utn + dx * f.dutn) * fh;
            else fv = (f.uti - dx * f.duti) * fh;
            sl = ga * ((hp - hl) * (Hp + Hl) + (Hl + Hi) * (zi - zl));
            sr = ga * ((hm - hr) * (Hm + Hr) + (Hr + Hn) * (zn - zr));
        } else {
            const T hr = f.hi - dx * f.dhi;
            const T hl = f.hn + dx * f.dhn;
            const T etar = f.zsi - dx * f.dzsi;
            const T etal = f.zsn + dx * f.dzsn;
            const T zr = etar - hr;
            const T zl = etal - hl;
            const T zA = M<T>::fmax_(zr, zl);
            const T zCN = M<T>::fmin_(zA, M<T>::fmin_(etal, etar) + D);
            const T hCNr = M<T>::fmax_(-D, M<T>::fmin_(etar - zCN, hr));
            const T hCNl = M<T>::fmax_(-D, M<T>::fmin_(etal - zCN, hl));
            T ul, ur, vl, vr;
            if (Hi > eps) {
                ur = f.uni - ((T)1.0 + dx * f.dhi / Hi) * dx * f.duni;
                vr = f.uti - ((T)1.0 + dx * f.dhi / Hi) * dx * f.duti;
            } else {
                ur = f.uni - dx * f.duni;
                vr = f.uti - dx * f.duti;
            }
            if (Hn > eps) {
                ul = f.unn + ((T)1.0 - dx * f.dhn / Hn) * dx * f.dunn;
                vl = f.utn + ((T)1.0 - dx * f.dhn / Hn) * dx * f.dutn;
            } else {
                ul = f.unn + dx * f.dunn;
                vl = f.utn + dx * f.dutn;
            }
            // hllc on the reconstructed states, pressures shifted by the datum
            const T hm = D + hCNl, hp = D + hCNr, um = ul, up = ur;
            const T cmo = M<T>::sqrt_(g * hm), cp = M<T>::sqrt_(g * hp);
            const T ustar = (um + up) * (T)0.5 + cmo - cp;
            const T cstar = (cmo + cp) * (T)0.5 + (um - up) * (T)0.25;
            const T SL = hm == (T)0. ? up - (T)2. * cp : M<T>::fmin_(um - cmo, ustar - cstar);
            const T SR = hp == (T)0. ? um + (T)2. * cmo : M<T>::fmax_(up + cp, ustar + cstar);
            const T fum = hm * um * um + ga * hCNl * ((T)2.0 * D + hCNl);
            const T fup = hp * up * up + ga * hCNr * ((T)2.0 * D + hCNr);
            if ((T)0. <= SL) {
                fh = um * hm;
                fu = fum;
            } else if ((T)0. >= SR) {
                fh = up * hp;
                fu = fup;
            } else {
                const T rs = (T)1.0 / (SR - SL);
                fh = (SR * (um * hm) - SL * (up * hp) + SL * SR * (hCNr - hCNl)) * rs;
                fu = (SR * fum - SL * fup + SL * SR * (hp * up - hm * um)) * rs;
            }
            const T a = M<T>::fmax_(M<T>::fabs_(SL), M<T>::fabs_(SR));
            r.dt = a > epsi ? CFL * delta / a : inv_epsi<T>();
            fv = (fh > (T)0. ? vl : vr) * fh;
            sl = ga * (Hi + (D + hCNr)) * (f.zbi - zCN);
            sr = ga * ((D + hCNl) + Hn) * (f.zbn - zCN);
        }
        r.Fh = fh;
        r.Fq = fu - sl;
        r.S = fu - sr;
        r.Ft = fv;
        r.wet = true;
    } else {
        r.dt = inv_epsi<T>();
        r.Fh = (T)0.0;
        r.Fq = -ga * D * D;
        r.S = -ga * D * D;
        r.Ft = (T)0.0;
        r.wet = false;
    }
    return r;
}

// AdvkernelCPU in split mode: depths as deviations, full depths for the limiter
// and the velocities.
template <class T>
__device__ __forceinline__ void advance_split(T dt, T eps, bool forcemass, T D, T hold, T uold, T vold, T dhi, T dhui,
                                              T dhvi, T& ho, T& uo, T& vo)
{
    const T Hold = D + hold;
    const T edt = forcemass ? dt : dhi >= (T)0.0 ? dt : M<T>::fmin_(dt, M<T>::fmax_(Hold, eps) / M<T>::fabs_(dhi));
    ho = hold + edt * dhi;
    const T Ho = D + ho;
    if (Ho > eps) {
        uo = (Hold * uold + edt * dhui) / Ho;
        vo = (Hold * vold + edt * dhvi) / Ho;
    } else {
        uo = (T)0.0;
        vo = (T)0.0;
    }
}

}  // namespace bgf
