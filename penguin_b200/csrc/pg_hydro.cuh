// FP64 hydrodynamics building blocks of the Godunov sweep: 4th-order PPM
// reconstruction, characteristic interface states, HLLC flux, conservative
// update.  Expression order follows the reference line by line wherever it is
// cited, so that results differ from it only at the rounding level; the one
// deliberate change is that the 4th-order edge slopes use per-index linear
// weights built once on the host instead of re-deriving 15 grid moments and 56
// divisions per call.
#pragma once

#include "pg_common.cuh"

namespace pg {

struct Par {
    double sL, a, sR;
};

// src/solver/recon/recon.cu:216-378 (slopes) + src/solver/recon/PPM.cu:64-91 (flattening,
// monotonicity).  w: {wL0,wL1,wL2, wR0,wR1,wR2} with sL = wL . (a[i-1]-a[i-2], a[i]-a[i-1],
// a[i+1]-a[i]) and sR = wR . (a[i]-a[i-1], a[i+1]-a[i], a[i+2]-a[i+1]).
__device__ __forceinline__ Par recon(const double* __restrict__ w, double am2, double am1, double a0,
                                     double ap1, double ap2, double flat) {
    const double d0 = am1 - am2, d1 = a0 - am1, d2 = ap1 - a0, d3 = ap2 - ap1;
    double sL = w[0] * d0 + w[1] * d1 + w[2] * d2;
    double sR = w[3] * d1 + w[4] * d2 + w[5] * d3;
    sL = copysign(fmin(fabs(sL), fabs(d1)), d1);
    sR = copysign(fmin(fabs(sR), fabs(d2)), d2);
    if (sR * sL <= 0.0) {
        sL = 0.0;
        sR = 0.0;
    }
    sR *= (1.0 - flat);
    sL *= (1.0 - flat);
    const double t3 = sR + sL;
    const double t2 = t3 * t3;
    const double t1 = t3 * 3.0 * (sL - sR);
    if (t2 < t1) sL = 2.0 * sR;
    else if (t2 < -t1) sR = 2.0 * sL;
    return {sL, a0, sR};
}

// Averages of the parabola over the fraction x of the cell touching its left /
// right edge (src/solver/recon/PPM.cu:95-113).  The x-only factors h = x/2 and
// g = 1 - x/1.5 are shared by every field averaged at the same x.
struct Frac {
    double x, h, g;
};
__device__ __forceinline__ Frac frac_left(double x) { return {x, x / 2.0, 1.0 - x / 1.5}; }
__device__ __forceinline__ Frac frac_right(double x) {
    const double y = 1.0 - x;
    return {y, y / 2.0, 1.0 - y / 1.5};
}
__device__ __forceinline__ double aveL(const Frac& f, const Par& p) {
    const double a6 = 3.0 * (p.sL - p.sR);
    const double aL = p.a - p.sL;
    const double S = p.sR + p.sL;
    return aL + f.h * (S + f.g * a6);
}
__device__ __forceinline__ double aveR(const Frac& f, const Par& p) {
    const double a6 = 3.0 * (p.sL - p.sR);
    const double aR = p.a + p.sR;
    const double S = p.sR + p.sL;
    return aR - f.h * (S - f.g * a6);
}

__device__ __forceinline__ double lim01(double a) { return fmin(fmax(a, 0.0), 1.0); }  // solve.cu:14
__device__ __forceinline__ double exp_lim(double x) { return fmax(1.0 + x, 1.0e-6); }    // solve.cu:29

// Shock flattening coefficient of the middle cell (src/solver/recon/PPM.cu:7-62);
// inv_cs = 1/sqrt(gam p0 / r0) is shared with the interface states.
__device__ __forceinline__ double flatten(double inv_cs, double p0, double pm2, double pm1, double pp1, double pp2,
                                          double um1, double u0, double up1) {
    const double dp1f = pp1 - p0, dp2f = pp2 - pm1;
    const double dp1b = p0 - pm1, dp2b = pp1 - pm2;
    const double Mf = (u0 - up1) * inv_cs;
    const double Mb = (um1 - u0) * inv_cs;
    double f = 0.0;
    if ((Mf > 0.0 || Mb > 0.0) && dp2f != 0.0 && dp2b != 0.0) {
        double ddp = 10.0 * fmax(0.0, fabs(dp1f / dp2f - 0.5) - 0.25);
        f = ddp;
        ddp = 10.0 * fmax(0.0, fabs(dp1b / dp2b - 0.5) - 0.25);
        f = fmax(f, ddp);
        f = fmin(0.5, f * fmax(fabs(dp1f), fabs(dp1b)) / p0);
    }
    return f;
}

struct Half {
    double r, p, u, v, w;
};

// Interface state on the LEFT edge of a cell = the right state of the face
// below it (src/solver/riemann/states.cu:151-206).  xl: left face, idx = 1/(xr-xl),
// sdt: dt/rad, cs0 = sqrt(gam p/r) of the cell averages r0c, p0c, u0c.
__device__ __forceinline__ Half state_at_left_edge(double gam, double xl, double idx, double sdt, double cs0,
                                                   double r0c, double p0c, double u0c, const Par& R, const Par& Pp,
                                                   const Par& U, const Par& V, const Par& W) {
    const double hdt = 0.5 * sdt;
    double tmp = fmin(u0c, 0.0);
    tmp = xl - tmp * sdt + cs0 * sdt;
    Frac q = frac_left(lim01((tmp - xl) * idx));
    const double rmin = r0c * 1.0e-10, pmin = p0c * 1.0e-10;
    const double ur = aveL(q, U);
    const double dis = fmin(ur, 0.0) * sdt;
    tmp = xl - dis;
    q = frac_left(lim01((tmp - xl) * idx));
    double r0 = aveL(q, R), p0 = aveL(q, Pp);
    const double u0 = aveL(q, U);
    r0 = fmax(r0, rmin);
    p0 = fmax(p0, pmin);
    const double ir0 = 1.0 / r0;
    const double cs = sqrt(gam * p0 * ir0);
    tmp = xl - dis + cs * sdt;
    q = frac_left(lim01((tmp - xl) * idx));
    double u_ = aveL(q, U), p_ = aveL(q, Pp);
    const double k = 2.0 / (cs * sdt);
    u_ = (u_ - u0) * k;
    p_ = (p_ - p0) * k;
    u_ *= -hdt;
    p_ *= -hdt;
    Half s;
    s.r = r0 * exp_lim(u_);
    s.p = p0 * exp_lim(gam * u_);
    s.u = u0 + p_ * ir0 + 0.0;
    s.v = aveL(q, V);
    s.w = aveL(q, W);
    return s;
}

// Interface state on the RIGHT edge of a cell = the left state of the face
// above it (src/solver/riemann/states.cu:210-264).
__device__ __forceinline__ Half state_at_right_edge(double gam, double xl, double xr, double idx, double sdt,
                                                    double cs0, double r0c, double p0c, double u0c, const Par& R,
                                                    const Par& Pp, const Par& U, const Par& V, const Par& W) {
    const double hdt = 0.5 * sdt;
    double tmp = fmax(u0c, 0.0);
    tmp = xr - tmp * sdt - cs0 * sdt;
    Frac q = frac_right(lim01((tmp - xl) * idx));
    const double rmin = r0c * 1.0e-10, pmin = p0c * 1.0e-10;
    const double ul = aveR(q, U);
    const double dis = fmax(ul, 0.0) * sdt;
    tmp = xr - dis;
    q = frac_right(lim01((tmp - xl) * idx));
    double r0 = aveR(q, R), p0 = aveR(q, Pp);
    const double u0 = aveR(q, U);
    r0 = fmax(r0, rmin);
    p0 = fmax(p0, pmin);
    const double ir0 = 1.0 / r0;
    const double cs = sqrt(gam * p0 * ir0);
    tmp = xr - dis - cs * sdt;
    q = frac_right(lim01((tmp - xl) * idx));
    double u_ = aveR(q, U), p_ = aveR(q, Pp);
    const double k = 2.0 / (cs * sdt);
    u_ = (u0 - u_) * k;
    p_ = (p0 - p_) * k;
    u_ *= -hdt;
    p_ *= -hdt;
    Half s;
    s.r = r0 * exp_lim(u_);
    s.p = p0 * exp_lim(gam * u_);
    s.u = u0 + p_ * ir0 + 0.0;
    s.v = aveR(q, V);
    s.w = aveR(q, W);
    return s;
}

// src/EOS/EOS.cu:4-18 (EOS 0: isothermal, 2: ideal gas; ie: internal_e_flag)
__device__ __forceinline__ double energy(int eos, int ie, double gam, double r, double p, double u, double v,
                                         double w) {
    if (eos == 2) {
        double e = p / ((gam - 1.0) * r);
        if (ie == 0) e += u * u / 2.0 + v * v / 2.0 + w * w / 2.0;
        return e;
    }
    return p / r;
}

__device__ __forceinline__ double pick(double FL, double F_L, double F_R, double FR, double sl, double sm,
                                       double sr) {  // src/solver/riemann/HLLC.cu:2-8
    if (signbit(sl) == 0) return FL;
    else if (signbit(sr) != 0) return FR;
    else if (signbit(sm) == 0) return F_L;
    return F_R;
}

struct Flux {
    double r, p, u, v, w, pres, uprs;
};

// Wave speeds (src/solver/riemann/wave_speeds.cu:24-35, 288-333) and the HLLC
// fluxes (src/solver/riemann/HLLC.cu:10-77) at one face, us = 0.  The reference
// forms all four candidate fluxes and picks one by the signs of sl, sr, sm
// (HLLC.cu:2-8); here the signs are tested first and only the selected
// candidate is formed.
__device__ __forceinline__ Flux hllc(int eos, int ie, double gam, const Half& L, const Half& R) {
    const double cl = sqrt(gam * L.p / L.r);
    const double cr = sqrt(gam * R.p / R.r);
    const double c_ = 0.5 * (cr + cl);
    const double p_ = 0.5 * (R.p + L.p);
    const double pm = p_ * exp_lim(0.5 * gam * (L.u - R.u) / c_);
    const double srl = sqrt(L.r), srr = sqrt(R.r);
    const double is = 1.0 / (srl + srr);
    const double u_ = (srl * L.u + srr * R.u) * is;
    const double n2 = 0.5 * srl * srr * (is * is);
    const double cc = sqrt((cl * cl * srl + cr * cr * srr) * is + n2 * (R.u - L.u) * (R.u - L.u));
    const double sl = u_ - cc, sr = u_ + cc;
    double sm = (L.r * L.u * cl + R.r * R.u * cr) / (L.r * cl + R.r * cr);
    sm += (L.p - R.p) / ((L.r + R.r) * (0.5 * (cl + cr)));

    // side of every upwinded quantity: left iff sl >= 0, or sr >= 0 and sm >= 0
    const bool left = (signbit(sl) == 0) || (signbit(sr) == 0 && signbit(sm) == 0);
    const Half& S = left ? L : R;
    Flux F;
    if (signbit(sl) == 0 || signbit(sr) != 0) {  // supersonic: the upwind state's own fluxes
        F.r = S.u * S.r;
        F.pres = S.p;
        F.uprs = (ie == 0) ? S.u * S.p : S.u;
    } else {  // star region on the side of the contact
        const double s_ = left ? sl : sr;
        const double inv = 1.0 / (s_ - sm);
        F.r = sm * S.r * (s_ - S.u) * inv;
        F.pres = (s_ * pm - sm * S.p) * inv;
        if (ie == 0) F.uprs = sm * (s_ * pm - S.u * S.p) * inv;
        else F.uprs = sm * (s_ * pm - S.u * S.p) / (s_ * pm - sm * S.p);
    }
    F.u = S.u * F.r;
    F.v = S.v * F.r;
    F.w = S.w * F.r;
    F.p = (eos > 0) ? energy(eos, ie, gam, S.r, S.p, S.u, 0.0, 0.0) * F.r : 0.0;
    if (eos != 2) F.uprs = 0.0;
    return F;
}

// Conservative update with floors (src/solver/sweeps.cu:218-261).  cs2: get_cs2
// at the cell.  For the isothermal EOS the energy slot is dead (it is
// overwritten by cs2 r), so it is not formed.
__device__ __forceinline__ Cell update_cell(int eos, int ie, double gam, double cs2, Cell Q, const Cell& D,
                                            int* floor_hits) {
    const double r_min = fmax(Q.r * 1.0e-10, SMALLR);
    const double p_min = fmax(Q.p * 1.0e-10, SMALLP);
    const double u_old = Q.u, v_old = Q.v, w_old = Q.w;
    if (eos == 2) {
        Q.p = energy(eos, ie, gam, Q.r, Q.p, Q.u, Q.v, Q.w);
        Q.p *= Q.r;
    }
    Q.u *= Q.r;
    Q.v *= Q.r;
    Q.w *= Q.r;
    Q.r += D.r;
    Q.p += D.p;
    Q.u += D.u;
    Q.v += D.v;
    Q.w += D.w;
    const double ir = 1.0 / Q.r;
    Q.u *= ir;
    Q.v *= ir;
    Q.w *= ir;
    if (Q.r < r_min) {
        Q.r = r_min;
        Q.p = p_min;
        Q.u = u_old;
        Q.v = v_old;
        Q.w = w_old;
        if (floor_hits) atomicAdd(floor_hits, 1);
    } else if (eos == 2) {
        const double gamm = gam - 1.0;
        if (ie == 0) Q.p = fmax(Q.p * gamm - gamm * Q.r * (Q.u * Q.u + Q.v * Q.v + Q.w * Q.w) / 2.0, p_min);
        else Q.p = fmax(Q.p * gamm, p_min);
    } else {
        Q.p = cs2 * Q.r;
    }
    return Q;
}

}  // namespace pg
