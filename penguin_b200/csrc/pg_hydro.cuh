// FP64 hydrodynamics building blocks of the Godunov sweep: 4th-order PPM
// reconstruction, characteristic interface states, HLLC flux, conservative
// update.  Expression order follows the reference line by line wherever it is
// cited, so that results differ from it only at the rounding level; the one
// deliberate change is that the 4th-order edge slopes use per-index linear
// weights built once on the host instead of re-deriving 15 grid moments and 56
// divisions per call.
//
// The functions are templates on the scalar type T: the sweeps instantiate
// them with double, the adjoint kernels with dual numbers (pg_dual.cuh).
#pragma once

#include "pg_common.cuh"

namespace pg {

template <class T>
struct ParT {
    T sL, a, sR;
};
using Par = ParT<double>;

// src/solver/recon/recon.cu:216-378 (slopes) + src/solver/recon/PPM.cu:64-91 (flattening,
// monotonicity).  w: {wL0,wL1,wL2, wR0,wR1,wR2} with sL = wL . (a[i-1]-a[i-2], a[i]-a[i-1],
// a[i+1]-a[i]) and sR = wR . (a[i]-a[i-1], a[i+1]-a[i], a[i+2]-a[i+1]).
template <class T>
__device__ __forceinline__ ParT<T> recon(const double* __restrict__ w, T am2, T am1, T a0, T ap1, T ap2, T flat) {
    const T d0 = am1 - am2, d1 = a0 - am1, d2 = ap1 - a0, d3 = ap2 - ap1;
    T sL = w[0] * d0 + w[1] * d1 + w[2] * d2;
    T sR = w[3] * d1 + w[4] * d2 + w[5] * d3;
    sL = copysign(fmin(fabs(sL), fabs(d1)), d1);
    sR = copysign(fmin(fabs(sR), fabs(d2)), d2);
    if (sR * sL <= 0.0) {
        sL = 0.0;
        sR = 0.0;
    }
    sR *= (1.0 - flat);
    sL *= (1.0 - flat);
    const T t3 = sR + sL;
    const T t2 = t3 * t3;
    const T t1 = t3 * 3.0 * (sL - sR);
    if (t2 < t1) sL = 2.0 * sR;
    else if (t2 < -t1) sR = 2.0 * sL;
    return {sL, a0, sR};
}

// Averages of the parabola over the fraction x of the cell touching its left /
// right edge (src/solver/recon/PPM.cu:95-113).  The x-only factors h = x/2 and
// g = 1 - x/1.5 are shared by every field averaged at the same x.
template <class T>
struct FracT {
    T x, h, g;
};
using Frac = FracT<double>;
// x / 1.5 correctly rounded without a division: with y = RN(1/1.5) = RN(2/3),
// q = RN(x y) lies within an ulp of x / 1.5 and the remainder x - 1.5 q is
// exact in one FMA, so RN(q + (x - 1.5 q) y) is the correctly rounded quotient
// (Markstein, IBM J. Res. Dev. 34 (1990) 111-119); 2x/3 is never a midpoint of
// two doubles.  Bit for bit the IEEE quotient the reference computes
// (src/solver/recon/PPM.cu:100,111), three FP64 instructions.
template <class T>
__device__ __forceinline__ T div_1p5(T x) { return x / 1.5; }
template <>
__device__ __forceinline__ double div_1p5<double>(double x) {
    constexpr double y = 2.0 / 3.0;
    const double q = x * y;
    const double r = fma(-q, 1.5, x);
    return copysign(fma(r, y, q), x);  // the quotient of a positive divisor keeps x's sign (-0 / 1.5 = -0)
}
template <class T>
__device__ __forceinline__ FracT<T> frac_left(T x) { return {x, x / 2.0, 1.0 - div_1p5(x)}; }
template <class T>
__device__ __forceinline__ FracT<T> frac_right(T x) {
    const T y = 1.0 - x;
    return {y, y / 2.0, 1.0 - div_1p5(y)};
}
template <class T>
__device__ __forceinline__ T aveL(const FracT<T>& f, const ParT<T>& p) {
    const T a6 = 3.0 * (p.sL - p.sR);
    const T aL = p.a - p.sL;
    const T S = p.sR + p.sL;
    return aL + f.h * (S + f.g * a6);
}
template <class T>
__device__ __forceinline__ T aveR(const FracT<T>& f, const ParT<T>& p) {
    const T a6 = 3.0 * (p.sL - p.sR);
    const T aR = p.a + p.sR;
    const T S = p.sR + p.sL;
    return aR - f.h * (S - f.g * a6);
}

template <class T>
__device__ __forceinline__ T lim01(T a) { return fmin(fmax(a, T(0.0)), T(1.0)); }  // solve.cu:14
template <class T>
__device__ __forceinline__ T exp_lim(T x) { return fmax(1.0 + x, T(1.0e-6)); }  // solve.cu:29

// Shock flattening coefficient of the middle cell (src/solver/recon/PPM.cu:7-62).
// The reference forms the Mach numbers (u0 - up1) / cs and (um1 - u0) / cs only
// to test their signs; with cs > 0 those are the signs of the differences, so
// the differences are tested (the quotient would differ only by underflowing a
// difference below cs 2^-1074 to zero).  inv_cs (1 / cs) is not needed.
template <class T>
__device__ __forceinline__ T flatten(T inv_cs, T p0, T pm2, T pm1, T pp1, T pp2, T um1, T u0, T up1) {
    (void)inv_cs;
    const T dp1f = pp1 - p0, dp2f = pp2 - pm1;
    const T dp1b = p0 - pm1, dp2b = pp1 - pm2;
    const T Mf = u0 - up1;
    const T Mb = um1 - u0;
    T f = 0.0;
    if ((Mf > 0.0 || Mb > 0.0) && dp2f != 0.0 && dp2b != 0.0) {
        T ddp = 10.0 * fmax(T(0.0), fabs(dp1f / dp2f - 0.5) - 0.25);
        f = ddp;
        ddp = 10.0 * fmax(T(0.0), fabs(dp1b / dp2b - 0.5) - 0.25);
        f = fmax(f, ddp);
        f = fmin(T(0.5), f * fmax(fabs(dp1f), fabs(dp1b)) / p0);
    }
    return f;
}

template <class T>
struct HalfT {
    T r, p, u, v, w;
};
using Half = HalfT<double>;

// Interface state on the LEFT edge of a cell = the right state of the face
// below it (src/solver/riemann/states.cu:151-206).  xl: left face, idx = 1/(xr-xl),
// sdt: dt/rad, cs0 = sqrt(gam p/r) of the cell averages r0c, p0c, u0c.
template <class T>
__device__ __forceinline__ HalfT<T> state_at_left_edge(double gam, double xl, double idx, double sdt, T cs0, T r0c,
                                                       T p0c, T u0c, const ParT<T>& R, const ParT<T>& Pp,
                                                       const ParT<T>& U, const ParT<T>& V, const ParT<T>& W) {
    const double hdt = 0.5 * sdt;
    T tmp = fmin(u0c, T(0.0));
    tmp = xl - tmp * sdt + cs0 * sdt;
    FracT<T> q = frac_left(lim01((tmp - xl) * idx));
    const T rmin = r0c * 1.0e-10, pmin = p0c * 1.0e-10;
    const T ur = aveL(q, U);
    const T dis = fmin(ur, T(0.0)) * sdt;
    tmp = xl - dis;
    q = frac_left(lim01((tmp - xl) * idx));
    T r0 = aveL(q, R), p0 = aveL(q, Pp);
    const T u0 = aveL(q, U);
    r0 = fmax(r0, rmin);
    p0 = fmax(p0, pmin);
    const T ir0 = 1.0 / r0;
    const T cs = sqrt(gam * p0 * ir0);
    tmp = xl - dis + cs * sdt;
    q = frac_left(lim01((tmp - xl) * idx));
    T u_ = aveL(q, U), p_ = aveL(q, Pp);
    const T k = 2.0 / (cs * sdt);
    u_ = (u_ - u0) * k;
    p_ = (p_ - p0) * k;
    u_ *= -hdt;
    p_ *= -hdt;
    HalfT<T> s;
    s.r = r0 * exp_lim(u_);
    s.p = p0 * exp_lim(gam * u_);
    s.u = u0 + p_ * ir0 + 0.0;
    s.v = aveL(q, V);
    s.w = aveL(q, W);
    return s;
}

// Interface state on the RIGHT edge of a cell = the left state of the face
// above it (src/solver/riemann/states.cu:210-264).
template <class T>
__device__ __forceinline__ HalfT<T> state_at_right_edge(double gam, double xl, double xr, double idx, double sdt, T cs0,
                                                        T r0c, T p0c, T u0c, const ParT<T>& R, const ParT<T>& Pp,
                                                        const ParT<T>& U, const ParT<T>& V, const ParT<T>& W) {
    const double hdt = 0.5 * sdt;
    T tmp = fmax(u0c, T(0.0));
    tmp = xr - tmp * sdt - cs0 * sdt;
    FracT<T> q = frac_right(lim01((tmp - xl) * idx));
    const T rmin = r0c * 1.0e-10, pmin = p0c * 1.0e-10;
    const T ul = aveR(q, U);
    const T dis = fmax(ul, T(0.0)) * sdt;
    tmp = xr - dis;
    q = frac_right(lim01((tmp - xl) * idx));
    T r0 = aveR(q, R), p0 = aveR(q, Pp);
    const T u0 = aveR(q, U);
    r0 = fmax(r0, rmin);
    p0 = fmax(p0, pmin);
    const T ir0 = 1.0 / r0;
    const T cs = sqrt(gam * p0 * ir0);
    tmp = xr - dis - cs * sdt;
    q = frac_right(lim01((tmp - xl) * idx));
    T u_ = aveR(q, U), p_ = aveR(q, Pp);
    const T k = 2.0 / (cs * sdt);
    u_ = (u0 - u_) * k;
    p_ = (p0 - p_) * k;
    u_ *= -hdt;
    p_ *= -hdt;
    HalfT<T> s;
    s.r = r0 * exp_lim(u_);
    s.p = p0 * exp_lim(gam * u_);
    s.u = u0 + p_ * ir0 + 0.0;
    s.v = aveR(q, V);
    s.w = aveR(q, W);
    return s;
}

// src/EOS/EOS.cu:4-18 (EOS 0: isothermal, 2: ideal gas; ie: internal_e_flag)
template <class T>
__device__ __forceinline__ T energy(int eos, int ie, double gam, T r, T p, T u, T v, T w) {
    if (eos == 2) {
        T e = p / ((gam - 1.0) * r);
        if (ie == 0) e += u * u / 2.0 + v * v / 2.0 + w * w / 2.0;
        return e;
    }
    return p / r;
}

template <class T>
struct FluxT {
    T r, p, u, v, w, pres, uprs;
};
using Flux = FluxT<double>;

// Wave speeds (src/solver/riemann/wave_speeds.cu:24-35, 288-333) and the HLLC
// fluxes (src/solver/riemann/HLLC.cu:10-77) at one face, us = 0.  The reference
// forms all four candidate fluxes and picks one by the signs of sl, sr, sm
// (HLLC.cu:2-8); here the signs are tested first and only the selected
// candidate is formed.
template <class T>
__device__ __forceinline__ FluxT<T> hllc(int eos, int ie, double gam, const HalfT<T>& L, const HalfT<T>& R) {
    const T cl = sqrt(gam * L.p / L.r);
    const T cr = sqrt(gam * R.p / R.r);
    const T c_ = 0.5 * (cr + cl);
    const T p_ = 0.5 * (R.p + L.p);
    const T pm = p_ * exp_lim(0.5 * gam * (L.u - R.u) / c_);
    const T srl = sqrt(L.r), srr = sqrt(R.r);
    const T is = 1.0 / (srl + srr);
    const T u_ = (srl * L.u + srr * R.u) * is;
    const T n2 = 0.5 * srl * srr * (is * is);
    const T cc = sqrt((cl * cl * srl + cr * cr * srr) * is + n2 * (R.u - L.u) * (R.u - L.u));
    const T sl = u_ - cc, sr = u_ + cc;
    T sm = (L.r * L.u * cl + R.r * R.u * cr) / (L.r * cl + R.r * cr);
    sm += (L.p - R.p) / ((L.r + R.r) * (0.5 * (cl + cr)));

    // side of every upwinded quantity: left iff sl >= 0, or sr >= 0 and sm >= 0
    const bool left = (signbit(sl) == 0) || (signbit(sr) == 0 && signbit(sm) == 0);
    const HalfT<T>& S = left ? L : R;
    FluxT<T> F;
    if (signbit(sl) == 0 || signbit(sr) != 0) {  // supersonic: the upwind state's own fluxes
        F.r = S.u * S.r;
        F.pres = S.p;
        F.uprs = (ie == 0) ? S.u * S.p : S.u;
    } else {  // star region on the side of the contact
        const T s_ = left ? sl : sr;
        const T inv = 1.0 / (s_ - sm);
        F.r = sm * S.r * (s_ - S.u) * inv;
        F.pres = (s_ * pm - sm * S.p) * inv;
        if (ie == 0) F.uprs = sm * (s_ * pm - S.u * S.p) * inv;
        else F.uprs = sm * (s_ * pm - S.u * S.p) / (s_ * pm - sm * S.p);
    }
    F.u = S.u * F.r;
    F.v = S.v * F.r;
    F.w = S.w * F.r;
    F.p = (eos > 0) ? energy<T>(eos, ie, gam, S.r, S.p, S.u, T(0.0), T(0.0)) * F.r : T(0.0);
    if (eos != 2) F.uprs = 0.0;
    return F;
}

// Viscous force density of the middle cell of a 3x3 stencil
// (src/viscosity/viscosity.cu:9-22, 84-194, ndim 2).  Stencil order: n<3 row j,
// 3..5 row j-1, 6..8 row j+1, columns i-1..i+1.  The grid spacings enter as
// per-index reciprocals: X = {1/(r2-r0), 1/(r2-r1), 1/(r1-r0), 1/(0.5(r2-r0)), 1/r1},
// Y = {1/(t2-t0), 1/(t2-t1), 1/(t1-t0), 1/(0.5(t2-t0))}.
template <class T>
__device__ __forceinline__ void viscous(const double* __restrict__ X, const double* __restrict__ Y, const T* u,
                                        const T* v, const T* nr, T& fx_out, T& fy_out) {
    const double i_r20 = X[0], i_r21 = X[1], i_r10 = X[2], i_hr20 = X[3], i_r1 = X[4];
    const double i_t20 = Y[0], i_t21 = Y[1], i_t10 = Y[2], i_ht20 = Y[3];
    const T dudx = (u[2] - u[0]) * i_r20;
    const T d2udx2 = ((u[2] - u[1]) * i_r21 - (u[1] - u[0]) * i_r10) * i_hr20;
    const T dndx = (nr[2] - nr[0]) * i_r20;
    const T dvdx = (v[2] - v[0]) * i_r20;
    const T d2vdx2 = ((v[2] - v[1]) * i_r21 - (v[1] - v[0]) * i_r10) * i_hr20;
    const T dvdy = (v[7] - v[4]) * i_t20 * i_r1;
    const T d2vdy2 = ((v[7] - v[1]) * i_t21 - (v[1] - v[4]) * i_t10) * i_ht20 * i_r1 * i_r1;
    const T d2vdxy = (v[8] - v[6] - v[5] + v[3]) * i_r20 * i_t20 * i_r1;
    const T dudy = (u[7] - u[4]) * i_t20 * i_r1;
    const T d2udy2 = ((u[7] - u[1]) * i_t21 - (u[1] - u[4]) * i_t10) * i_ht20 * i_r1 * i_r1;
    const T d2udxy = (u[8] - u[6] - u[5] + u[3]) * i_r20 * i_t20 * i_r1;
    const T dndy = (nr[7] - nr[4]) * i_t20 * i_r1;

    const T sxx = 2.0 * nr[1] * dudx;
    T fx = 2.0 * dndx * dudx + 2.0 * nr[1] * d2udx2 + sxx * i_r1;
    const T syy = 2.0 * nr[1] * (dvdy + u[1] * i_r1);
    const T sxy = nr[1] * (dudy + dvdx - v[1] * i_r1);
    T fy = 2.0 * dndy * dvdy + 2.0 * nr[1] * d2vdy2 + 2.0 * nr[1] * dudy * i_r1 + 2.0 * dndy * u[1] * i_r1;
    fx += dndy * (dudy + dvdx) + nr[1] * (d2udy2 + d2vdxy) - dndy * v[1] * i_r1 - nr[1] * dvdy * i_r1 - syy * i_r1;
    fy += dndx * (dudy + dvdx) + nr[1] * (d2udxy + d2vdx2) - dndx * v[1] * i_r1 - nr[1] * dvdx * i_r1 +
          nr[1] * v[1] * i_r1 * i_r1 + 2.0 * sxy * i_r1;
    fx_out = fx;
    fy_out = fy;
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
