// FP32-mixed form of the Godunov step for 2D polar planet-disks (geomx 1,
// geomy 3, isothermal, analytic radial boundaries).
//
// State: three FP32 planes per disk holding residuals against the disk's FP64
// axisymmetric initial state init_C(r) (src/init/init.cu:431-442):
//     dS = Sigma - Sigma_0(r),  du = v_r - v_r0(r),  dv = v_phi - v_phi0(r)
// (p = cs^2(r) Sigma is not stored).  Because v_phi0 - orb_rot - r Omega_frame
// vanishes, the azimuthal sweep's velocity residual (src/solver/sweeps.cu:398-403)
// is dv itself; the radial ghosts of boundary 0 hold init_C, i.e. zero residuals.
//
// Reconstruction and HLLC run in FP32 in "deviation form": every field enters
// as its difference from a reference value (the cell average of the stencil
// centre, or the face's left cell), formed from the FP32 residuals plus FP64
// table differences of the background.  PPM (recon.cu, PPM.cu) and the interface
// states (states.cu) are invariant under adding a constant to a field, so this
// is the reference's algorithm with its rounding measured against local
// variations rather than against O(1) magnitudes.  The conservative updates are
// written as residual increments, e.g. v_new - v = (D(Sigma v) - v D Sigma) /
// Sigma_new, with the large background terms cancelled analytically.  FP64 is
// kept for the orbital-advection shift and residual speed, the background
// tables, the CFL rate and dt, and conserved totals.
#pragma once

#include "pg_common.cuh"

namespace pg {
namespace f32 {

constexpr int NPL = 3;  // planes: dS, du, dv

// Per-radius FP32 tables, each slot xn = xarr + 1 floats; a table with several
// values per index takes consecutive slots (slot + m), so that threads of
// neighbouring radii read neighbouring words.
enum XSlot {
    X_SBG = 0,    // Sigma_0
    X_PBG = 1,    // p_0 = cs2 Sigma_0
    X_UBG = 2,    // v_r0
    X_CS2 = 3,    // cs^2
    X_RAD = 4,    // r
    X_IRAD = 5,   // 1/r
    X_IDX = 6,    // 1/(xa[i+1]-xa[i])
    X_IXV = 7,    // 1/xv[i]
    X_XA = 8,     // faces xa[i], i <= xarr
    X_NU = 9,     // viscosity nu
    X_ABG = 10,   // v_phi0^2/r + star gravity (the background's radial acceleration)
    X_V2R = 11,   // 2 v_phi0 / r
    X_EPS = 12,   // v_phi0 - orb_rot - r Omega_frame (zero up to FP64 rounding)
    X_CS0 = 13,   // sqrt(gam cs2)
    X_DBG = 14,   // 16 per i: background differences at stencil offsets -2,-1,+1,+2 of Sigma, p, v_r, r v_phi
    X_WX = 30,    // 6 reconstruction weights per i
    X_VISX = 36,  // 5 viscous-stencil reciprocals per i
    X_VBG = 41,   // 7 per i: background viscous force coefficients Ax Bx Cx Ay By Cy, and d(Sigma_0 nu) across i
    X_KILL = 48,  // 4 per i: damping ramp and 1/tau, inner then outer (1/tau = 0: no damping)
    // dust (dust_flag): the background is init_CD (src/init/init.cu:351-454)
    X_DSBG = 52,  // Sigma_d0
    X_DUBG = 53,  // v_r,d0 (the drift)
    X_DVBG = 54,  // v_phi,d0
    X_DEPS = 55,  // v_phi,d0 - orb_rot - r Omega_frame
    X_DABG = 56,  // v_phi,d0^2/r + star gravity
    X_DV2R = 57,  // 2 v_phi,d0 / r
    X_DGU = 58,   // v_r0 - v_r,d0 (gas minus dust background)
    X_DGV = 59,   // v_phi0 - v_phi,d0
    X_DDBG = 60,  // 12 per i: background differences at offsets -2,-1,+1,+2 of Sigma_d0, v_r,d0, r v_phi,d0
    X_NSLOT = 72
};
enum YSlot {
    Y_IDY = 0,   // 1/(ya[j+1]-ya[j])
    Y_IYV = 1,   // 1/yv[j]
    Y_WY = 2,    // 6 reconstruction weights per j
    Y_VISY = 8,  // 4 viscous-stencil reciprocals per j
    Y_NSLOT = 12
};
// Per-step planet table (k32_trig): rows [yn][6] = {sin, cos, 1-cos} of (phi - phi_p) for the
// planet of the first half-kick, then of the planet at t+dt; columns [xn][2] = r - x_p for both;
// then 8 scalars {m, x_p, rs^2, 1/x_p^2} x {first, second}.
constexpr int TRIG_ROW = 6;

// Everything one FP32 kernel needs about one disk; an array of these lives in
// device memory, one per ensemble member.
struct View32 {
    int xres, yres, xarr, yarr, pitch, xn, yn;
    int visc, orbadv, kill, nplanet, pad0;
    int ntx[3];  // tiles along the fast index: 0 radial sweep, 1 azimuthal sweep / advection, 2 stencil
    int pad1;
    float gam, pad2;
    float* buf[2];            // two state buffers, NPL planes of pitch * yarr floats each
    float* vis;               // viscous force density of kick1 (2 planes)
    const CUtensorMap* maps;  // buf0 {X, Y, S}, buf1 {X, Y, S}, vis
    const float* tx;
    const float* ty;
    float* trig;
    const double* cs64;       // sqrt(gam cs2) per radius, FP64 (CFL rate)
    DiskView d64;             // FP64 grid, tables, orbital-advection arrays, scalars
    // dust_flag: residual planes {dSigma_d, dv_r,d, dv_phi,d} against init_CD, no ghost
    // images (radial ghosts: zero residuals; rows wrap), and face-flux scratch
    float* dbuf[2];
    float* dflux;             // 3 planes of (xres + 1) * (yres + 1) faces
    int dust;
    float st_h;               // Stokes number times h/r: t_s = st_h / (c_s Sigma) (dust.cu:1-4)
    float dust_rmin;          // D_G_ratio * smallr
    __device__ __forceinline__ const float* x(int slot) const { return tx + (size_t)slot * xn; }
    __device__ __forceinline__ const float* y(int slot) const { return ty + (size_t)slot * yn; }
    __device__ __forceinline__ size_t plane() const { return (size_t)pitch * yarr; }
    __device__ __forceinline__ const float* trow(int j) const { return trig + (size_t)TRIG_ROW * j; }
    __device__ __forceinline__ const float* tcol() const { return trig + (size_t)TRIG_ROW * yn; }
    __device__ __forceinline__ const float* tscal() const { return trig + (size_t)TRIG_ROW * yn + 2 * (size_t)xn; }
};
inline size_t trig_floats(int xn, int yn) { return (size_t)TRIG_ROW * yn + 2 * (size_t)xn + 8; }

// ------------------------------------------------------------ FP32 hydro
struct Par32 {
    float sL, sR;  // parabola of one cell relative to its average
};

// recon.cu:216-378 + PPM.cu:64-91 with the centre value subtracted: am2..ap2 are
// the neighbours' differences from the centre.
__device__ __forceinline__ Par32 recon32(const float* __restrict__ w, float am2, float am1, float ap1, float ap2,
                                         float flat) {
    const float d0 = am1 - am2, d1 = -am1, d2 = ap1, d3 = ap2 - ap1;
    float sL = w[0] * d0 + w[1] * d1 + w[2] * d2;
    float sR = w[3] * d1 + w[4] * d2 + w[5] * d3;
    sL = copysignf(fminf(fabsf(sL), fabsf(d1)), d1);
    sR = copysignf(fminf(fabsf(sR), fabsf(d2)), d2);
    if (sR * sL <= 0.0f) {
        sL = 0.0f;
        sR = 0.0f;
    }
    sR *= (1.0f - flat);
    sL *= (1.0f - flat);
    const float t3 = sR + sL;
    const float t2 = t3 * t3;
    const float t1 = t3 * 3.0f * (sL - sR);
    if (t2 < t1) sL = 2.0f * sR;
    else if (t2 < -t1) sR = 2.0f * sL;
    return {sL, sR};
}

struct Frac32 {
    float h, g;  // x/2, 1 - x/1.5 for the swept fraction x (PPM.cu:95-113)
};
__device__ __forceinline__ Frac32 frac32(float x) { return {0.5f * x, 1.0f - x * (2.0f / 3.0f)}; }
__device__ __forceinline__ float lim01f(float a) { return fminf(fmaxf(a, 0.0f), 1.0f); }
__device__ __forceinline__ float aveL32(const Frac32& f, const Par32& p) {
    const float a6 = 3.0f * (p.sL - p.sR);
    return -p.sL + f.h * ((p.sR + p.sL) + f.g * a6);
}
__device__ __forceinline__ float aveR32(const Frac32& f, const Par32& p) {
    const float a6 = 3.0f * (p.sL - p.sR);
    return p.sR - f.h * ((p.sR + p.sL) - f.g * a6);
}

// PPM.cu:7-62 on deviations: pm2..pp2 are p differences from the centre, p0 its
// absolute value; um1/up1 the velocity differences.
__device__ __forceinline__ float flatten32(float inv_cs, float p0, float pm2, float pm1, float pp1, float pp2,
                                           float um1, float up1) {
    const float dp1f = pp1, dp2f = pp2 - pm1;
    const float dp1b = -pm1, dp2b = pp1 - pm2;
    (void)inv_cs;  // the signs of the Mach numbers are those of the velocity differences (flatten, pg_hydro.cuh)
    const float Mf = -up1;
    const float Mb = um1;
    float f = 0.0f;
    if ((Mf > 0.0f || Mb > 0.0f) && dp2f != 0.0f && dp2b != 0.0f) {
        f = 10.0f * fmaxf(0.0f, fabsf(dp1f / dp2f - 0.5f) - 0.25f);
        f = fmaxf(f, 10.0f * fmaxf(0.0f, fabsf(dp1b / dp2b - 0.5f) - 0.25f));
        f = fminf(0.5f, f * fmaxf(fabsf(dp1f), fabsf(dp1b)) / p0);
    }
    return f;
}

struct HS {
    float rd, pd;  // density and pressure: deviation from a reference value
    float u;       // normal velocity (absolute; a residual in the azimuthal sweep)
    float v;       // transported field (deviation from a reference value)
};

// states.cu:151-206 (left edge of a cell) in deviation form.  rc, pc, uc: the
// cell's absolute average density, pressure, normal velocity; R, P, U, V its
// parabolas relative to the averages.  The result's rd, pd, v are relative to
// the cell's averages.  The factor -hdt * 2/(cs sdt) of the reference is -1/cs.
__device__ __forceinline__ HS left_edge32(float gam, float idx, float sdt, float cs0, float rc, float pc, float uc,
                                          const Par32& R, const Par32& P, const Par32& U, const Par32& V) {
    Frac32 q = frac32(lim01f((cs0 - fminf(uc, 0.0f)) * sdt * idx));
    const float ur = uc + aveL32(q, U);
    const float dis = fminf(ur, 0.0f) * sdt;
    q = frac32(lim01f(-dis * idx));
    float r0d = aveL32(q, R), p0d = aveL32(q, P);
    const float u0d = aveL32(q, U);
    float r0 = rc + r0d, p0 = pc + p0d;
    const float rmin = rc * 1.0e-10f, pmin = pc * 1.0e-10f;
    if (r0 < rmin) {
        r0 = rmin;
        r0d = rmin - rc;
    }
    if (p0 < pmin) {
        p0 = pmin;
        p0d = pmin - pc;
    }
    const float ir0 = 1.0f / r0;
    const float cs = sqrtf(gam * p0 * ir0);
    const float ics = 1.0f / cs;
    q = frac32(lim01f((cs * sdt - dis) * idx));
    const float u_ = (u0d - aveL32(q, U)) * ics;
    const float p_ = (p0d - aveL32(q, P)) * ics;
    HS s;
    s.rd = (1.0f + u_ > 1.0e-6f) ? r0d + r0 * u_ : r0 * 1.0e-6f - rc;
    const float gu = gam * u_;
    s.pd = (1.0f + gu > 1.0e-6f) ? p0d + p0 * gu : p0 * 1.0e-6f - pc;
    s.u = uc + u0d + p_ * ir0;
    s.v = aveL32(q, V);
    return s;
}

// states.cu:210-264 (right edge of a cell) in deviation form.
__device__ __forceinline__ HS right_edge32(float gam, float idx, float sdt, float cs0, float rc, float pc, float uc,
                                           const Par32& R, const Par32& P, const Par32& U, const Par32& V) {
    Frac32 q = frac32(lim01f((cs0 + fmaxf(uc, 0.0f)) * sdt * idx));
    const float ul = uc + aveR32(q, U);
    const float dis = fmaxf(ul, 0.0f) * sdt;
    q = frac32(lim01f(dis * idx));
    float r0d = aveR32(q, R), p0d = aveR32(q, P);
    const float u0d = aveR32(q, U);
    float r0 = rc + r0d, p0 = pc + p0d;
    const float rmin = rc * 1.0e-10f, pmin = pc * 1.0e-10f;
    if (r0 < rmin) {
        r0 = rmin;
        r0d = rmin - rc;
    }
    if (p0 < pmin) {
        p0 = pmin;
        p0d = pmin - pc;
    }
    const float ir0 = 1.0f / r0;
    const float cs = sqrtf(gam * p0 * ir0);
    const float ics = 1.0f / cs;
    q = frac32(lim01f((dis + cs * sdt) * idx));
    const float u_ = (aveR32(q, U) - u0d) * ics;
    const float p_ = (aveR32(q, P) - p0d) * ics;
    HS s;
    s.rd = (1.0f + u_ > 1.0e-6f) ? r0d + r0 * u_ : r0 * 1.0e-6f - rc;
    const float gu = gam * u_;
    s.pd = (1.0f + gu > 1.0e-6f) ? p0d + p0 * gu : p0 * 1.0e-6f - pc;
    s.u = uc + u0d + p_ * ir0;
    s.v = aveR32(q, V);
    return s;
}

struct FX {
    float r;   // mass flux
    float u;   // normal momentum flux without pressure (S.u * F.r)
    float v;   // upwind transported deviation: the field's flux is F.r * (v_ref + v)
    float pd;  // interface pressure minus the face's reference pressure
};

// wave_speeds.cu:24-35, 288-333 + HLLC.cu:10-77 (isothermal: no energy flux) with
// densities and pressures as deviations from rref, pref; the pressure jump
// L.p - R.p and the star pressure enter only through deviations.
__device__ __forceinline__ FX hllc32(float gam, float rref, float pref, const HS& L, const HS& R) {
    const float Lr = rref + L.rd, Rr = rref + R.rd;
    const float Lp = pref + L.pd, Rp = pref + R.pd;
    const float cl = sqrtf(gam * Lp / Lr);
    const float cr = sqrtf(gam * Rp / Rr);
    const float c_ = 0.5f * (cr + cl);
    const float pbd = 0.5f * (R.pd + L.pd);
    const float pb = pref + pbd;
    const float x = 0.5f * gam * (L.u - R.u) / c_;
    const float pmd = (1.0f + x > 1.0e-6f) ? pbd + pb * x : pb * 1.0e-6f - pref;
    const float srl = sqrtf(Lr), srr = sqrtf(Rr);
    const float is = 1.0f / (srl + srr);
    const float u_ = (srl * L.u + srr * R.u) * is;
    const float n2 = 0.5f * srl * srr * (is * is);
    const float du = R.u - L.u;
    const float cc = sqrtf((cl * cl * srl + cr * cr * srr) * is + n2 * du * du);
    const float sl = u_ - cc, sr = u_ + cc;
    float sm = (Lr * L.u * cl + Rr * R.u * cr) / (Lr * cl + Rr * cr);
    sm += (L.pd - R.pd) / ((Lr + Rr) * (0.5f * (cl + cr)));
    const bool left = (signbit(sl) == 0) || (signbit(sr) == 0 && signbit(sm) == 0);
    const HS& S = left ? L : R;
    const float Sr = left ? Lr : Rr;
    FX F;
    if (signbit(sl) == 0 || signbit(sr) != 0) {
        F.r = S.u * Sr;
        F.pd = S.pd;
    } else {
        const float s_ = left ? sl : sr;
        const float inv = 1.0f / (s_ - sm);
        F.r = sm * Sr * (s_ - S.u) * inv;
        F.pd = (s_ * pmd - sm * S.pd) * inv;
    }
    F.u = S.u * F.r;
    F.v = S.v;
    return F;
}

// Viscous force density (src/viscosity/viscosity.cu:84-194, ndim 2) of a velocity
// field u, v given on the 3x3 stencil (order as gather9: row j, row j-1, row j+1),
// with rho*nu entering through its centre value nr1 and its differences dndx, dndy.
// Linear in (u, v): the disk's force is this on the residuals plus the background
// part A nr1 + B dndx + C dndy from per-radius coefficients.
__device__ __forceinline__ void viscous32(const float* __restrict__ X, const float* __restrict__ Y, const float* u,
                                          const float* v, float nr1, float dndx, float dndy, float& fx_out,
                                          float& fy_out) {
    const float i_r20 = X[0], i_r21 = X[1], i_r10 = X[2], i_hr20 = X[3], i_r1 = X[4];
    const float i_t20 = Y[0], i_t21 = Y[1], i_t10 = Y[2], i_ht20 = Y[3];
    const float dudx = (u[2] - u[0]) * i_r20;
    const float d2udx2 = ((u[2] - u[1]) * i_r21 - (u[1] - u[0]) * i_r10) * i_hr20;
    const float dvdx = (v[2] - v[0]) * i_r20;
    const float d2vdx2 = ((v[2] - v[1]) * i_r21 - (v[1] - v[0]) * i_r10) * i_hr20;
    const float dvdy = (v[7] - v[4]) * i_t20 * i_r1;
    const float d2vdy2 = ((v[7] - v[1]) * i_t21 - (v[1] - v[4]) * i_t10) * i_ht20 * i_r1 * i_r1;
    const float d2vdxy = (v[8] - v[6] - v[5] + v[3]) * i_r20 * i_t20 * i_r1;
    const float dudy = (u[7] - u[4]) * i_t20 * i_r1;
    const float d2udy2 = ((u[7] - u[1]) * i_t21 - (u[1] - u[4]) * i_t10) * i_ht20 * i_r1 * i_r1;
    const float d2udxy = (u[8] - u[6] - u[5] + u[3]) * i_r20 * i_t20 * i_r1;
    const float sxx = 2.0f * nr1 * dudx;
    float fx = 2.0f * dndx * dudx + 2.0f * nr1 * d2udx2 + sxx * i_r1;
    const float syy = 2.0f * nr1 * (dvdy + u[1] * i_r1);
    const float sxy = nr1 * (dudy + dvdx - v[1] * i_r1);
    float fy = 2.0f * dndy * dvdy + 2.0f * nr1 * d2vdy2 + 2.0f * nr1 * dudy * i_r1 + 2.0f * dndy * u[1] * i_r1;
    fx += dndy * (dudy + dvdx) + nr1 * (d2udy2 + d2vdxy) - dndy * v[1] * i_r1 - nr1 * dvdy * i_r1 - syy * i_r1;
    fy += dndx * (dudy + dvdx) + nr1 * (d2udxy + d2vdx2) - dndx * v[1] * i_r1 - nr1 * dvdx * i_r1 +
          nr1 * v[1] * i_r1 * i_r1 + 2.0f * sxy * i_r1;
    fx_out = fx;
    fy_out = fy;
}

}  // namespace f32
}  // namespace pg
