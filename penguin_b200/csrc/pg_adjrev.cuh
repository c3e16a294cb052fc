// Hand-written reverse mode of the sweep's face function for the adjoint
// (isothermal EOS, the configuration the adjoint covers).
//
// Each function replays the FP64 building block of pg_hydro.cuh with the
// same expressions, keeping the intermediates it needs on a small tape (a
// struct), and then propagates adjoints backwards through the branch the
// replay took: limiter selections, clamps of the swept fraction, floors,
// HLLC wave signs.  The result equals the dual-number derivative of the
// same blocks (pg_dual.cuh) contracted with the output adjoint; the dual
// kernels check it.  Adjoints accumulate into the caller's variables (+=).
#pragma once

#include <cmath>

#include "pg_hydro.cuh"

namespace pg {
namespace rev {

// adjoint of sqrt(a) at s = sqrt(a) (zero at a = 0, like the dual sqrt)
__device__ __forceinline__ double dsqrt(double s, double bs) { return s == 0.0 ? 0.0 : 0.5 * bs / s; }

// ------------------------------------------------------------- HLLC (EOS 0)
// Adjoint of hllc(0, ie, gam, L, R) for the flux components r, u, v, w and pres
// (the energy fluxes vanish for EOS 0).  bF: {r, u, v, w, pres}.
__device__ __forceinline__ void hllc_rev(double gam, const Half& L, const Half& R, const double* bF, Half& bL,
                                         Half& bR) {
    const double cl = sqrt(gam * L.p / L.r);
    const double cr = sqrt(gam * R.p / R.r);
    const double c_ = 0.5 * (cr + cl);
    const double p_ = 0.5 * (R.p + L.p);
    const double xe = 0.5 * gam * (L.u - R.u) / c_;
    const double el = exp_lim(xe);
    const double pm = p_ * el;
    const double srl = sqrt(L.r), srr = sqrt(R.r);
    const double is = 1.0 / (srl + srr);
    const double u_ = (srl * L.u + srr * R.u) * is;
    const double n2 = 0.5 * srl * srr * (is * is);
    const double du = R.u - L.u;
    const double H = cl * cl * srl + cr * cr * srr;
    const double cc = sqrt(H * is + n2 * du * du);
    const double sl = u_ - cc, sr = u_ + cc;
    const double num = L.r * L.u * cl + R.r * R.u * cr;
    const double den = L.r * cl + R.r * cr;
    const double q1 = num / den;
    const double E = (L.r + R.r) * (0.5 * (cl + cr));
    const double q2 = (L.p - R.p) / E;
    const double sm = q1 + q2;
    const bool left = (std::signbit(sl) == 0) || (std::signbit(sr) == 0 && std::signbit(sm) == 0);
    const Half& S = left ? L : R;
    Half& bS = left ? bL : bR;
    const bool super = (std::signbit(sl) == 0 || std::signbit(sr) != 0);
    double Fr;
    double b_sl = 0.0, b_sr = 0.0, b_sm = 0.0, b_pm = 0.0;
    double s_ = 0.0, inv = 0.0, A = 0.0, B = 0.0;
    if (super) {
        Fr = S.u * S.r;
    } else {
        s_ = left ? sl : sr;
        inv = 1.0 / (s_ - sm);
        A = sm * S.r * (s_ - S.u);
        B = s_ * pm - sm * S.p;
        Fr = A * inv;
    }
    // F.u = S.u F.r, F.v = S.v F.r, F.w = S.w F.r
    const double bFr = bF[0] + bF[1] * S.u + bF[2] * S.v + bF[3] * S.w;
    bS.u += bF[1] * Fr;
    bS.v += bF[2] * Fr;
    bS.w += bF[3] * Fr;
    if (super) {
        bS.u += bFr * S.r;
        bS.r += bFr * S.u;
        bS.p += bF[4];
    } else {
        const double b_inv = bFr * A + bF[4] * B;
        const double bA = bFr * inv, bB = bF[4] * inv;
        double b_s = -inv * inv * b_inv;
        b_sm += inv * inv * b_inv;
        b_sm += bA * S.r * (s_ - S.u);
        bS.r += bA * sm * (s_ - S.u);
        b_s += bA * sm * S.r;
        bS.u -= bA * sm * S.r;
        b_s += bB * pm;
        b_pm += bB * s_;
        b_sm -= bB * S.p;
        bS.p -= bB * sm;
        if (left) b_sl += b_s;
        else b_sr += b_s;
    }
    double b_cl = 0.0, b_cr = 0.0, b_srl = 0.0, b_srr = 0.0, b_is = 0.0;
    // sl = u_ - cc, sr = u_ + cc
    const double b_u = b_sl + b_sr;
    const double b_cc = b_sr - b_sl;
    // sm = num / den + (L.p - R.p) / E
    {
        const double b_num = b_sm / den, b_den = -b_sm * q1 / den;
        bL.r += b_num * L.u * cl;
        bL.u += b_num * L.r * cl;
        b_cl += b_num * L.r * L.u;
        bR.r += b_num * R.u * cr;
        bR.u += b_num * R.r * cr;
        b_cr += b_num * R.r * R.u;
        bL.r += b_den * cl;
        b_cl += b_den * L.r;
        bR.r += b_den * cr;
        b_cr += b_den * R.r;
        const double b_dp = b_sm / E, b_E = -b_sm * q2 / E;
        bL.p += b_dp;
        bR.p -= b_dp;
        const double b_LR = b_E * (0.5 * (cl + cr)), b_ch = b_E * (L.r + R.r);
        bL.r += b_LR;
        bR.r += b_LR;
        b_cl += 0.5 * b_ch;
        b_cr += 0.5 * b_ch;
    }
    // cc = sqrt(H is + n2 du^2)
    {
        const double b_G = dsqrt(cc, b_cc);
        const double b_H = b_G * is;
        b_is += b_G * H;
        b_cl += b_H * 2.0 * cl * srl;
        b_srl += b_H * cl * cl;
        b_cr += b_H * 2.0 * cr * srr;
        b_srr += b_H * cr * cr;
        const double b_n2 = b_G * du * du;
        const double b_du = b_G * 2.0 * n2 * du;
        bR.u += b_du;
        bL.u -= b_du;
        // n2 = 0.5 srl srr is^2
        b_srl += b_n2 * 0.5 * srr * (is * is);
        b_srr += b_n2 * 0.5 * srl * (is * is);
        b_is += b_n2 * 0.5 * srl * srr * 2.0 * is;
    }
    // u_ = (srl L.u + srr R.u) is
    {
        const double K = srl * L.u + srr * R.u;
        const double b_K = b_u * is;
        b_is += b_u * K;
        b_srl += b_K * L.u;
        bL.u += b_K * srl;
        b_srr += b_K * R.u;
        bR.u += b_K * srr;
    }
    // is = 1 / (srl + srr)
    b_srl -= b_is * is * is;
    b_srr -= b_is * is * is;
    bL.r += dsqrt(srl, b_srl);
    bR.r += dsqrt(srr, b_srr);
    // pm = p_ exp_lim(xe), xe = 0.5 gam (L.u - R.u) / c_
    {
        const double b_p = b_pm * el;
        const double b_el = b_pm * p_;
        const double b_xe = (1.0e-6 > 1.0 + xe) ? 0.0 : b_el;
        const double g = 0.5 * gam / c_;
        bL.u += b_xe * g;
        bR.u -= b_xe * g;
        const double b_c = -b_xe * xe / c_;
        bR.p += 0.5 * b_p;
        bL.p += 0.5 * b_p;
        b_cr += 0.5 * b_c;
        b_cl += 0.5 * b_c;
    }
    // cl = sqrt(gam L.p / L.r)
    {
        const double ba = dsqrt(cl, b_cl);
        bL.p += ba * gam / L.r;
        bL.r -= ba * gam * L.p / (L.r * L.r);
        const double bb = dsqrt(cr, b_cr);
        bR.p += bb * gam / R.r;
        bR.r -= bb * gam * R.p / (R.r * R.r);
    }
}

// ---------------------------------------------------------- reconstruction
// Tape of recon(): the slope selections, the zeroing and monotonicity branches.
struct ReconTape {
    double sL2, sR2;   // slopes after the extremum zeroing, before flattening
    signed char selL, selR;  // fmin picked |d1| / |d2| (1) or the 4th-order slope (0)
    signed char cfL, cfR;    // copysign factor
    signed char fsL, fsR;    // fabs factor of the chosen operand
    signed char zero, mono;  // extremum zeroing; monotonicity branch (0 none, 1 sL = 2 sR, 2 sR = 2 sL)
};

__device__ __forceinline__ double fabs_factor(double x) { return std::signbit(x) ? -1.0 : 1.0; }

__device__ __forceinline__ Par recon_tape(const double* __restrict__ w, double am2, double am1, double a0, double ap1,
                                          double ap2, double flat, ReconTape& t) {
    const double d0 = am1 - am2, d1 = a0 - am1, d2 = ap1 - a0, d3 = ap2 - ap1;
    const double sL0 = w[0] * d0 + w[1] * d1 + w[2] * d2;
    const double sR0 = w[3] * d1 + w[4] * d2 + w[5] * d3;
    const double aL = fabs(sL0), bL = fabs(d1);
    const double mL = (bL < aL) ? bL : aL;
    t.selL = (bL < aL) ? 1 : 0;
    t.fsL = (signed char)fabs_factor(t.selL ? d1 : sL0);
    double sL = copysign(mL, d1);
    t.cfL = (std::signbit(sL) == std::signbit(mL)) ? 1 : -1;
    const double aR = fabs(sR0), bR = fabs(d2);
    const double mR = (bR < aR) ? bR : aR;
    t.selR = (bR < aR) ? 1 : 0;
    t.fsR = (signed char)fabs_factor(t.selR ? d2 : sR0);
    double sR = copysign(mR, d2);
    t.cfR = (std::signbit(sR) == std::signbit(mR)) ? 1 : -1;
    t.zero = (sR * sL <= 0.0) ? 1 : 0;
    if (t.zero) {
        sL = 0.0;
        sR = 0.0;
    }
    t.sL2 = sL;
    t.sR2 = sR;
    sR *= (1.0 - flat);
    sL *= (1.0 - flat);
    const double t3 = sR + sL;
    const double t2 = t3 * t3;
    const double t1 = t3 * 3.0 * (sL - sR);
    t.mono = 0;
    if (t2 < t1) {
        sL = 2.0 * sR;
        t.mono = 1;
    } else if (t2 < -t1) {
        sR = 2.0 * sL;
        t.mono = 2;
    }
    return {sL, a0, sR};
}

// bP: adjoint of {sL, a, sR}; accumulates into ba[5] (am2..ap2) and bflat
__device__ __forceinline__ void recon_rev(const double* __restrict__ w, const ReconTape& t, double flat,
                                          const Par& bP, double* ba, double& bflat) {
    double bsL3 = bP.sL, bsR3 = bP.sR;
    if (t.mono == 1) {
        bsR3 += 2.0 * bsL3;
        bsL3 = 0.0;
    } else if (t.mono == 2) {
        bsL3 += 2.0 * bsR3;
        bsR3 = 0.0;
    }
    bflat -= bsR3 * t.sR2 + bsL3 * t.sL2;
    double bsL = bsL3 * (1.0 - flat), bsR = bsR3 * (1.0 - flat);
    if (t.zero) {
        bsL = 0.0;
        bsR = 0.0;
    }
    double bd0 = 0.0, bd1 = 0.0, bd2 = 0.0, bd3 = 0.0;
    const double gL = bsL * t.cfL * t.fsL;
    if (t.selL) {
        bd1 += gL;
    } else {
        bd0 += w[0] * gL;
        bd1 += w[1] * gL;
        bd2 += w[2] * gL;
    }
    const double gR = bsR * t.cfR * t.fsR;
    if (t.selR) {
        bd2 += gR;
    } else {
        bd1 += w[3] * gR;
        bd2 += w[4] * gR;
        bd3 += w[5] * gR;
    }
    // d0 = am1 - am2, d1 = a0 - am1, d2 = ap1 - a0, d3 = ap2 - ap1
    ba[0] -= bd0;
    ba[1] += bd0 - bd1;
    ba[2] += bd1 - bd2 + bP.a;
    ba[3] += bd2 - bd3;
    ba[4] += bd3;
}

// ---------------------------------------------------------------- flattening
struct FlatTape {
    double p0, dp1f, dp2f, dp1b, dp2b, rf, rb, fpre, mx, g;
    signed char active, pf, pb, selpre, selmx, cap, sgf, sgb, smf, smb;
};

__device__ __forceinline__ double flatten_tape(double inv_cs, double p0, double pm2, double pm1, double pp1,
                                               double pp2, double um1, double u0, double up1, FlatTape& t) {
    t.p0 = p0;
    t.dp1f = pp1 - p0;
    t.dp2f = pp2 - pm1;
    t.dp1b = p0 - pm1;
    t.dp2b = pp1 - pm2;
    (void)inv_cs;  // the branch of flatten (pg_hydro.cuh): signs of the velocity differences
    const double Mf = u0 - up1;
    const double Mb = um1 - u0;
    double f = 0.0;
    t.active = ((Mf > 0.0 || Mb > 0.0) && t.dp2f != 0.0 && t.dp2b != 0.0) ? 1 : 0;
    if (t.active) {
        t.rf = t.dp1f / t.dp2f;
        const double xf = fabs(t.rf - 0.5) - 0.25;
        t.sgf = (signed char)fabs_factor(t.rf - 0.5);
        t.pf = (xf > 0.0) ? 1 : 0;
        const double ddpf = 10.0 * (t.pf ? xf : 0.0);
        t.rb = t.dp1b / t.dp2b;
        const double xb = fabs(t.rb - 0.5) - 0.25;
        t.sgb = (signed char)fabs_factor(t.rb - 0.5);
        t.pb = (xb > 0.0) ? 1 : 0;
        const double ddpb = 10.0 * (t.pb ? xb : 0.0);
        t.selpre = (ddpb > ddpf) ? 1 : 0;
        t.fpre = t.selpre ? ddpb : ddpf;
        const double af = fabs(t.dp1f), ab = fabs(t.dp1b);
        t.smf = (signed char)fabs_factor(t.dp1f);
        t.smb = (signed char)fabs_factor(t.dp1b);
        t.selmx = (ab > af) ? 1 : 0;
        t.mx = t.selmx ? ab : af;
        t.g = t.fpre * t.mx / p0;
        t.cap = (t.g < 0.5) ? 0 : 1;
        f = t.cap ? 0.5 : t.g;
    }
    return f;
}

// accumulates into bp[5] = (pm2, pm1, p0, pp1, pp2)
__device__ __forceinline__ void flatten_rev(const FlatTape& t, double bf, double* bp) {
    if (!t.active || t.cap) return;
    const double b_fpre = bf * t.mx / t.p0;
    const double b_mx = bf * t.fpre / t.p0;
    bp[2] -= bf * t.g / t.p0;
    double b_dp1f = 0.0, b_dp1b = 0.0, b_dp2f = 0.0, b_dp2b = 0.0;
    if (t.selmx) b_dp1b += b_mx * t.smb;
    else b_dp1f += b_mx * t.smf;
    if (t.selpre) {
        if (t.pb) {
            const double b_r = 10.0 * b_fpre * t.sgb;
            b_dp1b += b_r / t.dp2b;
            b_dp2b -= b_r * t.rb / t.dp2b;
        }
    } else if (t.pf) {
        const double b_r = 10.0 * b_fpre * t.sgf;
        b_dp1f += b_r / t.dp2f;
        b_dp2f -= b_r * t.rf / t.dp2f;
    }
    // dp1f = pp1 - p0, dp2f = pp2 - pm1, dp1b = p0 - pm1, dp2b = pp1 - pm2
    bp[3] += b_dp1f + b_dp2b;
    bp[2] += b_dp1b - b_dp1f;
    bp[4] += b_dp2f;
    bp[1] -= b_dp2f + b_dp1b;
    bp[0] -= b_dp2b;
}

// --------------------------------------------------- parabola averages
// Adjoints of aveL / aveR at fraction x (frac_left / frac_right): accumulate the
// Par adjoint and return d(ave)/dx.
__device__ __forceinline__ double aveL_rev(double x, const Par& p, double b, Par& bp) {
    const double h = x / 2.0, g = 1.0 - div_1p5(x);
    const double a6 = 3.0 * (p.sL - p.sR);
    const double S = p.sR + p.sL;
    // aL + h (S + g a6), aL = a - sL
    bp.a += b;
    bp.sL += b * (-1.0 + h * (1.0 + 3.0 * g));
    bp.sR += b * (h * (1.0 - 3.0 * g));
    return b * ((S + g * a6) / 2.0 + h * a6 * (-1.0 / 1.5));
}
__device__ __forceinline__ double aveR_rev(double x, const Par& p, double b, Par& bp) {
    const double y = 1.0 - x;
    const double h = y / 2.0, g = 1.0 - div_1p5(y);
    const double a6 = 3.0 * (p.sL - p.sR);
    const double S = p.sR + p.sL;
    // aR - h (S - g a6), aR = a + sR
    bp.a += b;
    bp.sL += b * (-h * (1.0 - 3.0 * g));
    bp.sR += b * (1.0 - h * (1.0 + 3.0 * g));
    const double dy = -(S - g * a6) / 2.0 + h * a6 * (-1.0 / 1.5);  // d/dy
    return -b * dy;
}

// ------------------------------------------------------- interface states
// lim01 passes the derivative iff 0 <= a <= 1 (the dual fmax/fmin selections)
__device__ __forceinline__ bool lim_pass(double a) { return !(0.0 > a) && !(1.0 < a); }

// Adjoint of state_at_left_edge (states.cu:151-206) given bs, the adjoint of the
// returned state.  Accumulates into bcs0, br0c, bp0c, bu0c and the Par adjoints.
__device__ __forceinline__ void state_left_rev(double gam, double xl, double idx, double sdt, double cs0, double r0c,
                                               double p0c, double u0c, const Par& R, const Par& Pp, const Par& U,
                                               const Par& V, const Par& W, const Half& bs, double& bcs0,
                                               double& br0c, double& bp0c, double& bu0c, Par& bR, Par& bP, Par& bU,
                                               Par& bV, Par& bW) {
    const double hdt = 0.5 * sdt;
    // forward replay (the expressions of state_at_left_edge)
    const bool t0pass = !(0.0 < u0c);
    double tmp = fmin(u0c, 0.0);
    tmp = xl - tmp * sdt + cs0 * sdt;
    const double a1 = (tmp - xl) * idx;
    const double x1 = lim01(a1);
    const double rmin = r0c * 1.0e-10, pmin = p0c * 1.0e-10;
    const double ur = aveL(frac_left(x1), U);
    const bool dpass = !(0.0 < ur);
    const double dis = fmin(ur, 0.0) * sdt;
    tmp = xl - dis;
    const double a2 = (tmp - xl) * idx;
    const double x2 = lim01(a2);
    const Frac q2 = frac_left(x2);
    const double r0r = aveL(q2, R), p0r = aveL(q2, Pp);
    const double u0 = aveL(q2, U);
    const bool rsel = rmin > r0r, psel = pmin > p0r;
    const double r0 = fmax(r0r, rmin);
    const double p0 = fmax(p0r, pmin);
    const double ir0 = 1.0 / r0;
    const double cs = sqrt(gam * p0 * ir0);
    tmp = xl - dis + cs * sdt;
    const double a3 = (tmp - xl) * idx;
    const double x3 = lim01(a3);
    const Frac q3 = frac_left(x3);
    const double uA = aveL(q3, U), pA = aveL(q3, Pp);
    const double k = 2.0 / (cs * sdt);
    const double u2 = ((uA - u0) * k) * -hdt;
    const double p2 = ((pA - p0) * k) * -hdt;
    const double E1 = exp_lim(u2), E2 = exp_lim(gam * u2);
    // reverse
    double bx3 = aveL_rev(x3, V, bs.v, bV) + aveL_rev(x3, W, bs.w, bW);
    double b_u0 = bs.u, b_ir0 = bs.u * p2;
    const double b_p2 = bs.u * ir0;
    double b_p0 = bs.p * E2, b_r0 = bs.r * E1;
    double b_u2 = 0.0;
    if (!(1.0e-6 > 1.0 + gam * u2)) b_u2 += bs.p * p0 * gam;
    if (!(1.0e-6 > 1.0 + u2)) b_u2 += bs.r * r0;
    const double b_u1 = b_u2 * -hdt, b_pp1 = b_p2 * -hdt;
    const double b_uA = b_u1 * k, b_pA = b_pp1 * k;
    b_u0 -= b_u1 * k;
    b_p0 -= b_pp1 * k;
    const double b_k = b_u1 * (uA - u0) + b_pp1 * (pA - p0);
    double b_cs = -b_k * k / cs;
    bx3 += aveL_rev(x3, U, b_uA, bU) + aveL_rev(x3, Pp, b_pA, bP);
    double b_dis = 0.0;
    if (lim_pass(a3)) {
        const double bt = bx3 * idx;
        b_dis -= bt;
        b_cs += bt * sdt;
    }
    const double b_arg = dsqrt(cs, b_cs);
    b_p0 += b_arg * gam * ir0;
    b_ir0 += b_arg * gam * p0;
    b_r0 -= b_ir0 * ir0 * ir0;
    double b_r0r = 0.0, b_p0r = 0.0;
    if (rsel) br0c += b_r0 * 1.0e-10;
    else b_r0r = b_r0;
    if (psel) bp0c += b_p0 * 1.0e-10;
    else b_p0r = b_p0;
    double bx2 = aveL_rev(x2, R, b_r0r, bR) + aveL_rev(x2, Pp, b_p0r, bP) + aveL_rev(x2, U, b_u0, bU);
    if (lim_pass(a2)) b_dis -= bx2 * idx;
    const double b_ur = dpass ? b_dis * sdt : 0.0;
    const double bx1 = aveL_rev(x1, U, b_ur, bU);
    if (lim_pass(a1)) {
        const double bt = bx1 * idx;
        if (t0pass) bu0c -= bt * sdt;
        bcs0 += bt * sdt;
    }
}

// Adjoint of state_at_right_edge (states.cu:210-264).
__device__ __forceinline__ void state_right_rev(double gam, double xl, double xr, double idx, double sdt, double cs0,
                                                double r0c, double p0c, double u0c, const Par& R, const Par& Pp,
                                                const Par& U, const Par& V, const Par& W, const Half& bs,
                                                double& bcs0, double& br0c, double& bp0c, double& bu0c, Par& bR,
                                                Par& bP, Par& bU, Par& bV, Par& bW) {
    const double hdt = 0.5 * sdt;
    const bool t0pass = !(0.0 > u0c);
    double tmp = fmax(u0c, 0.0);
    tmp = xr - tmp * sdt - cs0 * sdt;
    const double a1 = (tmp - xl) * idx;
    const double x1 = lim01(a1);
    const double rmin = r0c * 1.0e-10, pmin = p0c * 1.0e-10;
    const double ul = aveR(frac_right(x1), U);
    const bool dpass = !(0.0 > ul);
    const double dis = fmax(ul, 0.0) * sdt;
    tmp = xr - dis;
    const double a2 = (tmp - xl) * idx;
    const double x2 = lim01(a2);
    const Frac q2 = frac_right(x2);
    const double r0r = aveR(q2, R), p0r = aveR(q2, Pp);
    const double u0 = aveR(q2, U);
    const bool rsel = rmin > r0r, psel = pmin > p0r;
    const double r0 = fmax(r0r, rmin);
    const double p0 = fmax(p0r, pmin);
    const double ir0 = 1.0 / r0;
    const double cs = sqrt(gam * p0 * ir0);
    tmp = xr - dis - cs * sdt;
    const double a3 = (tmp - xl) * idx;
    const double x3 = lim01(a3);
    const Frac q3 = frac_right(x3);
    const double uA = aveR(q3, U), pA = aveR(q3, Pp);
    const double k = 2.0 / (cs * sdt);
    const double u2 = ((u0 - uA) * k) * -hdt;
    const double p2 = ((p0 - pA) * k) * -hdt;
    const double E1 = exp_lim(u2), E2 = exp_lim(gam * u2);
    double bx3 = aveR_rev(x3, V, bs.v, bV) + aveR_rev(x3, W, bs.w, bW);
    double b_u0 = bs.u, b_ir0 = bs.u * p2;
    const double b_p2 = bs.u * ir0;
    double b_p0 = bs.p * E2, b_r0 = bs.r * E1;
    double b_u2 = 0.0;
    if (!(1.0e-6 > 1.0 + gam * u2)) b_u2 += bs.p * p0 * gam;
    if (!(1.0e-6 > 1.0 + u2)) b_u2 += bs.r * r0;
    const double b_u1 = b_u2 * -hdt, b_pp1 = b_p2 * -hdt;
    const double b_uA = -b_u1 * k, b_pA = -b_pp1 * k;
    b_u0 += b_u1 * k;
    b_p0 += b_pp1 * k;
    const double b_k = b_u1 * (u0 - uA) + b_pp1 * (p0 - pA);
    double b_cs = -b_k * k / cs;
    bx3 += aveR_rev(x3, U, b_uA, bU) + aveR_rev(x3, Pp, b_pA, bP);
    double b_dis = 0.0;
    if (lim_pass(a3)) {
        const double bt = bx3 * idx;
        b_dis -= bt;
        b_cs -= bt * sdt;
    }
    const double b_arg = dsqrt(cs, b_cs);
    b_p0 += b_arg * gam * ir0;
    b_ir0 += b_arg * gam * p0;
    b_r0 -= b_ir0 * ir0 * ir0;
    double b_r0r = 0.0, b_p0r = 0.0;
    if (rsel) br0c += b_r0 * 1.0e-10;
    else b_r0r = b_r0;
    if (psel) bp0c += b_p0 * 1.0e-10;
    else b_p0r = b_p0;
    double bx2 = aveR_rev(x2, R, b_r0r, bR) + aveR_rev(x2, Pp, b_p0r, bP) + aveR_rev(x2, U, b_u0, bU);
    if (lim_pass(a2)) b_dis -= bx2 * idx;
    const double b_ul = dpass ? b_dis * sdt : 0.0;
    const double bx1 = aveR_rev(x1, U, b_ul, bU);
    if (lim_pass(a1)) {
        const double bt = bx1 * idx;
        if (t0pass) bu0c -= bt * sdt;
        bcs0 -= bt * sdt;
    }
}

// ------------------------------------------------------------ viscosity
// Adjoint of viscous() (viscosity.cu:84-194, 2D polar): the force is bilinear
// in nr = Sigma nu and the velocity derivatives.  Accumulates into bu[9],
// bv[9], bnr[9] (stencil order of viscous()).
__device__ __forceinline__ void viscous_rev(const double* __restrict__ X, const double* __restrict__ Y, const double* u,
                                            const double* v, const double* nr, double bfx, double bfy, double* bu,
                                            double* bv, double* bnr) {
    const double i_r20 = X[0], i_r21 = X[1], i_r10 = X[2], i_hr20 = X[3], i_r1 = X[4];
    const double i_t20 = Y[0], i_t21 = Y[1], i_t10 = Y[2], i_ht20 = Y[3];
    const double dudx = (u[2] - u[0]) * i_r20;
    const double d2udx2 = ((u[2] - u[1]) * i_r21 - (u[1] - u[0]) * i_r10) * i_hr20;
    const double dndx = (nr[2] - nr[0]) * i_r20;
    const double dvdx = (v[2] - v[0]) * i_r20;
    const double d2vdx2 = ((v[2] - v[1]) * i_r21 - (v[1] - v[0]) * i_r10) * i_hr20;
    const double dvdy = (v[7] - v[4]) * i_t20 * i_r1;
    const double d2vdy2 = ((v[7] - v[1]) * i_t21 - (v[1] - v[4]) * i_t10) * i_ht20 * i_r1 * i_r1;
    const double d2vdxy = (v[8] - v[6] - v[5] + v[3]) * i_r20 * i_t20 * i_r1;
    const double dudy = (u[7] - u[4]) * i_t20 * i_r1;
    const double d2udy2 = ((u[7] - u[1]) * i_t21 - (u[1] - u[4]) * i_t10) * i_ht20 * i_r1 * i_r1;
    const double d2udxy = (u[8] - u[6] - u[5] + u[3]) * i_r20 * i_t20 * i_r1;
    const double dndy = (nr[7] - nr[4]) * i_t20 * i_r1;
    const double n1 = nr[1], u1 = u[1], v1 = v[1];
    const double a = bfx, b = bfy;
    // adjoints of the derivatives and of the middle values
    const double b_dndx = a * 2.0 * dudx + b * ((dudy + dvdx) - v1 * i_r1);
    const double b_dudx = a * (2.0 * dndx + 2.0 * n1 * i_r1);
    const double b_d2udx2 = a * 2.0 * n1;
    const double b_dndy = a * ((dudy + dvdx) - v1 * i_r1) + b * (2.0 * dvdy + 2.0 * u1 * i_r1);
    const double b_dudy = a * dndy + b * (dndx + 4.0 * n1 * i_r1);
    const double b_dvdx = a * dndy + b * (dndx + n1 * i_r1);
    const double b_d2udy2 = a * n1, b_d2vdxy = a * n1;
    const double b_dvdy = -3.0 * a * n1 * i_r1 + 2.0 * b * dndy;
    const double b_d2vdy2 = b * 2.0 * n1;
    const double b_d2udxy = b * n1, b_d2vdx2 = b * n1;
    bnr[1] += a * (2.0 * d2udx2 + 2.0 * dudx * i_r1 + (d2udy2 + d2vdxy) - dvdy * i_r1 -
                   2.0 * (dvdy + u1 * i_r1) * i_r1) +
              b * (2.0 * d2vdy2 + 2.0 * dudy * i_r1 + (d2udxy + d2vdx2) - dvdx * i_r1 + v1 * i_r1 * i_r1 +
                   2.0 * (dudy + dvdx - v1 * i_r1) * i_r1);
    bu[1] += -a * 2.0 * n1 * i_r1 * i_r1 + b * 2.0 * dndy * i_r1;
    bv[1] += -a * dndy * i_r1 + b * (-dndx * i_r1 - n1 * i_r1 * i_r1);
    // the difference stencils
    const double K = i_ht20 * i_r1 * i_r1, L = i_r20 * i_t20 * i_r1, M = i_t20 * i_r1;
    bu[2] += b_dudx * i_r20 + b_d2udx2 * i_r21 * i_hr20;
    bu[0] += -b_dudx * i_r20 + b_d2udx2 * i_r10 * i_hr20;
    bu[1] += -b_d2udx2 * (i_r21 + i_r10) * i_hr20 - b_d2udy2 * (i_t21 + i_t10) * K;
    bu[7] += b_dudy * M + b_d2udy2 * i_t21 * K;
    bu[4] += -b_dudy * M + b_d2udy2 * i_t10 * K;
    bu[8] += b_d2udxy * L;
    bu[6] -= b_d2udxy * L;
    bu[5] -= b_d2udxy * L;
    bu[3] += b_d2udxy * L;
    bv[2] += b_dvdx * i_r20 + b_d2vdx2 * i_r21 * i_hr20;
    bv[0] += -b_dvdx * i_r20 + b_d2vdx2 * i_r10 * i_hr20;
    bv[1] += -b_d2vdx2 * (i_r21 + i_r10) * i_hr20 - b_d2vdy2 * (i_t21 + i_t10) * K;
    bv[7] += b_dvdy * M + b_d2vdy2 * i_t21 * K;
    bv[4] += -b_dvdy * M + b_d2vdy2 * i_t10 * K;
    bv[8] += b_d2vdxy * L;
    bv[6] -= b_d2vdxy * L;
    bv[5] -= b_d2vdxy * L;
    bv[3] += b_d2vdxy * L;
    bnr[2] += b_dndx * i_r20;
    bnr[0] -= b_dndx * i_r20;
    bnr[7] += b_dndy * M;
    bnr[4] -= b_dndy * M;
}

}  // namespace rev
}  // namespace pg
